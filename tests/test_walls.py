"""Physical walls and reservoirs without a GPU: parameter handling (the deck keys
of boundaryStag.cpp round-trip through to_inputs / parse_inputs), fhd_create's
validation of wall settings before it touches a device, the entry points that
refuse walls, and the reference's own wall and reservoir steps (oracle/_ref) on
the cases the GPU tests compare against: mass conserved, wall faces at rest,
ghost cells at the wall and reservoir values."""
import ctypes as C

import pytest
import torch

from fhdex_b200 import capi
from fhdex_b200.params import argon, mixture4, parse_inputs, stable_dt, with_walls


def _walled():
    return with_walls(mixture4((6, 7, 8), dx=8e-6), x=dict(vel=2, therm=2, mass=1, t=(263.0, 293.0)),
                      z=dict(vel=1, therm=1, mass=2, Yk=((0.4, 0.2, 0.3, 0.1), (0.1, 0.3, 0.2, 0.4))))


def test_wall_parameters_round_trip_through_the_deck():
    p = _walled()
    q = parse_inputs(p.to_inputs())
    for key in ("walls", "bc_vel_lo", "bc_vel_hi", "bc_mass_lo", "bc_mass_hi", "bc_therm_lo", "bc_therm_hi",
                "t_lo", "t_hi", "p_lo", "p_hi", "rho_lo", "rho_hi"):
        assert tuple(getattr(q, key)) == tuple(getattr(p, key)) if key != "walls" else q.walls == 1, key
    assert q.bc_Yk_lo[2] == p.bc_Yk_lo[2] and q.bc_Yk_hi[2] == p.bc_Yk_hi[2]
    with pytest.raises(ValueError):
        parse_inputs(p.to_inputs().replace("bc_mass_lo = 1 -1 2", "bc_mass_lo = 1 -1 5"))
    r = parse_inputs(p.to_inputs().replace("bc_mass_lo = 1 -1 2", "bc_mass_lo = 1 -1 3"))
    assert r.bc_mass_lo == (1, -1, 3) and r.p_lo == p.p_lo and r.rho_lo == p.rho_lo


def _create_rc(p, **raw):
    cp = p.to_c()
    for k, v in raw.items():
        arr, d = k.rsplit("_", 1)
        getattr(cp, arr)[int(d)] = v
    h = C.c_void_p()
    rc = capi.load().fhd_create(C.byref(h), C.byref(cp), 0)
    assert not h.value or rc == 0
    return rc


@pytest.mark.parametrize("change,code", [
    (dict(bc_vel_lo_1=2), "FHD_ERR_BAD_ARG"),            # one side periodic, the other a wall
    (dict(bc_mass_lo_0=3), "FHD_ERR_BAD_ARG"),           # a reservoir without a composition
    (dict(bc_mass_hi_0=5), "FHD_ERR_UNSUPPORTED"),       # no such boundary
    (dict(bc_vel_hi_0=3), "FHD_ERR_BAD_ARG"),
    (dict(bc_therm_lo_2=0), "FHD_ERR_BAD_ARG"),
    (dict(t_hi_0=0.0), "FHD_ERR_BAD_ARG"),               # isothermal wall without a temperature
])
def test_create_rejects_bad_walls_without_gpu(change, code):
    assert _create_rc(_walled(), **change) == getattr(capi, code)


def test_create_checks_wall_composition_and_precision_without_gpu():
    p = _walled()
    bad = p.replace(bc_Yk_lo=((), (), (0.5, 0.2, 0.2, 0.2)))   # neither Y nor X sums to 1
    assert _create_rc(bad) == capi.FHD_ERR_BAD_ARG
    assert _create_rc(p.replace(precision=1)) == capi.FHD_ERR_UNSUPPORTED
    # valid settings pass validation and only then need a device
    rc = _create_rc(p)
    assert rc not in (capi.FHD_ERR_BAD_ARG, capi.FHD_ERR_UNSUPPORTED)


def test_noalloc_and_batch_refuse_walls_without_gpu():
    lib = capi.load()
    p = _walled().replace(nspecies=4)
    cp = p.to_c()
    nf = capi.FhdFab()
    f3 = (capi.FhdFab * 3)()
    st = C.c_int()
    assert lib.fhd_rk3_step_stag_noalloc(C.byref(cp), nf, f3, nf, f3, 1e-13, 0, None, C.byref(st)) == \
        capi.FHD_ERR_UNSUPPORTED


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R
    if not R.available():
        pytest.skip("oracle/_ref was not built")
    return R


def test_reference_wall_step_keeps_walls(ref):
    """The reference's own step with isothermal no-slip x walls and concentration
    slip z walls: total mass unchanged, x wall faces at rest, x ghost temperature
    at the wall temperature, z ghost composition at the wall composition."""
    p = _walled()
    st = ref.state_from_reference(p, seed=3)
    dt = stable_dt(p)
    m0 = st.cu.valid()[0].sum().item()
    for s in range(3):
        ref.rk3_step(st, ref.step_noise(p, seed=20 + s), dt, s)
    assert abs(st.cu.valid()[0].sum().item() - m0) <= 1e-13 * m0
    g = p.ngc
    mx = st.cumom[0].valid(0)
    assert torch.all(mx[..., 0] == 0) and torch.all(mx[..., -1] == 0)
    T = st.prim.arr[4]
    assert torch.all(T[g:-g, g:-g, :g] == 263.0) and torch.all(T[g:-g, g:-g, -g:] == 293.0)
    yk, _ = ref.wall_composition(p, 4)
    for n in range(p.nspecies):
        assert torch.all(st.prim.arr[6 + n, :g, g:-g, g:-g] == yk[n])
    for m in st.state_mfs():
        assert torch.isfinite(m.valid()).all()


def test_reference_single_wall_direction_is_mirror_symmetric(ref):
    """Slip adiabatic z walls on a state symmetric under z -> -z (no noise): the
    reference's step keeps the symmetry (a check that the harness drives the
    reference's wall branches, not the periodic ones)."""
    p = with_walls(argon((4, 4, 6), dx=8e-6, stoch_stress_form=0), z=dict(vel=1, therm=1, mass=1))
    st = ref.state_from_reference(p, seed=4)
    g = p.ngc
    v = st.cu.valid()
    v.copy_(0.5 * (v + v.flip(1)))
    for d in range(2):
        mv = st.cumom[d].valid(0)
        mv.copy_(0.5 * (mv + mv.flip(0)))
    mz = st.cumom[2].valid(0)
    mz.copy_(0.5 * (mz - mz.flip(0)))
    ref.fill_boundary(p, st.cu)
    for m in st.cumom:
        ref.fill_boundary(p, m, override_sync=True)
    ref.conserved_to_primitive(st)
    for m in [st.cu, st.prim] + st.vel:
        ref.fill_boundary(p, m)
    ref.set_bc(st)
    from fhdex_b200.state import StepNoise
    ref.rk3_step(st, StepNoise(p), stable_dt(p), 0)
    rho = st.cu.valid(0)
    assert torch.allclose(rho, rho.flip(0), rtol=1e-13, atol=0)
    assert g == 2


def test_reference_reservoir_step_holds_the_reservoir_state(ref):
    """The reference's own step with reservoirs (bc_mass 3) across x: the ghost
    cells hold the reservoir's temperature, pressure, density and composition
    after every step, the interface faces carry flow (non-zero momentum), and
    the reservoir pressure defaults to the initial state's."""
    p = with_walls(mixture4((8, 6, 6), dx=8e-6), x=dict(vel=2, therm=2, mass=3, t=(263.0, 283.0),
                                                         Yk=((0.4, 0.2, 0.3, 0.1), (0.1, 0.3, 0.2, 0.4))))
    st = ref.state_from_reference(p, seed=6)
    for s in range(2):
        ref.rk3_step(st, ref.step_noise(p, 30 + s), stable_dt(p), s)
    g = p.ngc
    t, pr, rho = ref.wall_state(p, 0)
    yk, _ = ref.wall_composition(p, 0)
    assert t == 263.0 and pr == pytest.approx(p.rho0 * 8.314462175e7 * p.T_init * sum(
        b / m for b, m in zip(p.rhobar, p.molmass)), rel=1e-12)
    P = st.prim.arr
    assert torch.all(P[4, g:-g, g:-g, :g] == t) and torch.all(P[5, g:-g, g:-g, :g] == pr)
    assert torch.all(P[0, g:-g, g:-g, :g] == rho)
    for n in range(p.nspecies):
        assert torch.all(P[6 + n, g:-g, g:-g, :g] == yk[n])
    assert st.cumom[0].valid(0)[..., 0].abs().max() > 0
