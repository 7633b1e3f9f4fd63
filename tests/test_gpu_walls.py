"""Physical walls (boundaryStag.cpp): the CUDA step of a box with walls against
the reference's own code (oracle/_ref: RK3stepStag, setBCStag, calculateFluxStag
with their wall branches, compiled unmodified), bit for bit (tolerance 0) on the
whole storage of the state and of the stage-3 coefficients and fluxes, with
injected noise and with the in-kernel noise materialised for the reference.

Cases: isothermal no-slip walls at two temperatures (a temperature gradient),
slip adiabatic walls, concentration walls of a 4-species mixture, walls in two
directions with different conditions (wall-wall edges), walls in all three
directions (corners), gravity along a wall normal, and reservoirs (bc_mass 3:
ghost cells at a reservoir state, flow through the interface) alone, on all
sides and beside a wall direction, and the chemistry source with concentration
walls."""
import pytest
import torch

from fhdex_b200.context import Context
from fhdex_b200.params import Params, argon, isomerization, mixture4, no2_dimerization, stable_dt, with_walls
from fhdex_b200.state import StagState, StepNoise
from tests.helpers import compare_named

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R
    if not R.available():
        pytest.skip("oracle/_ref was not built")
    return R


ISO = dict(vel=2, therm=2, mass=1)
RES_Y = (0.22, 0.24, 0.26, 0.28)
CASES = {
    "tempgrad_x": lambda: with_walls(argon((12, 9, 10), dx=8e-6, seed=101), x=dict(ISO, t=(263.0, 293.0))),
    "slip_adiabatic_z": lambda: with_walls(argon((9, 10, 12), dx=8e-6, seed=102), z=dict(vel=1, therm=1, mass=1)),
    "concentration_y": lambda: with_walls(
        mixture4((8, 10, 7), dx=8e-6, seed=103),
        y=dict(vel=2, therm=2, mass=2, t=(273.0, 283.0), Yk=((0.4, 0.2, 0.3, 0.1), (0.1, 0.3, 0.2, 0.4)))),
    "mixed_xz": lambda: with_walls(argon((10, 8, 11), dx=8e-6, advection_type=1, seed=104),
                                   x=dict(vel=1, therm=1, mass=1), z=dict(ISO, t=(280.0, 270.0))),
    "box_xyz": lambda: with_walls(
        mixture4((7, 8, 9), dx=8e-6, visc_type=3, zeta_ratio=0.5, seed=105),
        x=dict(vel=2, therm=1, mass=1), y=dict(vel=1, therm=2, mass=2, t=(268.0, 278.0),
                                               Xk=((0.25, 0.25, 0.25, 0.25), (0.4, 0.3, 0.2, 0.1))),
        z=dict(ISO, t=(273.0, 290.0))),
    "adv0_grav_y": lambda: with_walls(argon((9, 11, 8), dx=8e-6, advection_type=0, grav=(0.0, -981.0, 0.0),
                                            seed=106), y=dict(ISO, t=(273.0, 273.0))),
    # the boundary set-up of the reference's 3-D temperature-gradient regression
    # run: 80 x 10 x 10 cells of 4 identical argon species at 400 K, no-slip
    # isothermal x walls at 280.8 / 508.5 K, slip adiabatic y and z walls, all
    # impermeable, dt 1e-12 s
    "tempgrad_3d": lambda: with_walls(
        Params(nspecies=4, n_cells=(80, 10, 10), prob_hi=(1.6e-4, 2e-5, 2e-5), molmass=(39.948,) * 4,
               diameter=(3.66e-8,) * 4, dof=(3.0,) * 4, e0=(0.0,) * 4, hcv=(-1.0,) * 4, hcp=(-1.0,) * 4,
               rhobar=(0.25,) * 4, T_init=400.0, rho0=1.78e-3, seed=1),
        x=dict(vel=2, therm=2, mass=1, t=(280.8, 508.5)), y=dict(vel=1, therm=1, mass=1),
        z=dict(vel=1, therm=1, mass=1)),
    # reservoirs (bc_mass 3): the boundary set-up of the reference's 3-D reservoir
    # regression run (reservoirs on all six sides, no-slip, 390 / 410 K, 4 species
    # of argon at a reservoir composition) on a smaller box; a reservoir pair
    # facing each other across x with different compositions; a reservoir
    # direction beside a wall direction
    "reservoir_3d": lambda: with_walls(
        Params(nspecies=4, n_cells=(8, 8, 8), prob_hi=(2.5e-5,) * 3, molmass=(39.948,) * 4,
               diameter=(3.66e-8,) * 4, dof=(3.0,) * 4, e0=(0.0,) * 4, hcv=(-1.0,) * 4, hcp=(-1.0,) * 4,
               rhobar=(0.25,) * 4, T_init=400.0, rho0=1.78e-3, seed=2),
        **{ax: dict(vel=2, therm=2, mass=3, t=(390.0, 410.0), Yk=(RES_Y, RES_Y)) for ax in "xyz"}),
    "reservoir_x": lambda: with_walls(
        mixture4((12, 6, 6), dx=8e-6, seed=3),
        x=dict(vel=2, therm=2, mass=3, t=(263.0, 283.0), Yk=((0.4, 0.2, 0.3, 0.1), (0.1, 0.3, 0.2, 0.4)))),
    "reservoir_wall": lambda: with_walls(
        argon((10, 9, 8), dx=8e-6, seed=4), x=dict(vel=2, therm=2, mass=3, t=(270.0, 276.0), Yk=((0.5, 0.5),) * 2,
                                                   p=(1.0e6, 1.02e6)),
        z=dict(vel=1, therm=1, mass=1)),
    # the chemistry source of the compressible step (first-order A <-> B on the NO2 /
    # N2O4 gas) with concentration walls in y
    "chem_walls_y": lambda: with_walls(
        isomerization(no2_dimerization((6, 8, 5), dx=8e-6, seed=5)),
        y=dict(vel=2, therm=2, mass=2, t=(340.0, 360.0), Yk=((0.6, 0.4), (0.3, 0.7)))),
}
DT = {"tempgrad_3d": 1e-12, "reservoir_3d": 1e-12}
RESERVOIRS = ["reservoir_3d", "reservoir_x", "reservoir_wall"]


@pytest.mark.parametrize("name", list(CASES))
def test_wall_steps_equal_the_reference_injected_noise(ref, name):
    p = CASES[name]()
    st = ref.state_from_reference(p, seed=7)
    d = st.clone(device="cuda")
    ctx = Context(p)
    dt = DT.get(name, stable_dt(p))
    for s in range(3):
        nz = ref.step_noise(p, seed=50 + s)
        ctx.rk3_step(d, dt, s, noise=nz.to("cuda"), aux=True)
        torch.cuda.synchronize()
        ref.rk3_step(st, nz, dt, s)
        bad, _ = compare_named(d.named(aux=True), st.named(aux=True))
        assert not bad, (s, bad[:6])
    assert ctx.status() == 0
    ctx.close()


@pytest.mark.parametrize("name", ["tempgrad_x", "concentration_y", "box_xyz", "reservoir_x", "reservoir_wall",
                                  "chem_walls_y"])
def test_wall_steps_equal_the_reference_in_kernel_noise(ref, name):
    """In-kernel Philox noise (wall directions draw their ghost centres' own
    values), materialised by fhd_fill_step_noise for the reference."""
    p = CASES[name]()
    st = ref.state_from_reference(p, seed=8)
    d = st.clone(device="cuda")
    ctx = Context(p)
    dt = DT.get(name, stable_dt(p))
    nz = StepNoise(p, "cuda")
    for s in range(3):
        ctx.fill_step_noise(nz, s)
        ctx.rk3_step(d, dt, s, noise=None, aux=True)
        nzc = nz.to("cpu")
        torch.cuda.synchronize()
        ref.rk3_step(st, nzc, dt, s)
        bad, _ = compare_named(d.named(aux=True), st.named(aux=True))
        assert not bad, (s, bad[:6])
    assert ctx.status() == 0
    ctx.close()


def test_wall_graph_replay_equals_single_steps(ref):
    p = CASES["mixed_xz"]()
    st = ref.state_from_reference(p, seed=9)
    a = st.clone(device="cuda")
    b = st.clone(device="cuda")
    ctx = Context(p)
    dt = stable_dt(p)
    for s in range(4):
        ctx.rk3_step(a, dt, s, aux=False)
    ctx.rk3_steps(b, dt, 0, 4)
    torch.cuda.synchronize()
    bad, _ = compare_named(b.named(), a.named())
    assert not bad, bad[:4]
    assert ctx.status() == 0


@pytest.mark.parametrize("name", ["concentration_y", "box_xyz", "slip_adiabatic_z"] + RESERVOIRS)
def test_set_bc_and_init_equal_the_reference(ref, name):
    """fhd_set_bc_stag against setBCStag on a state whose ghosts hold garbage, the
    wall compositions after SetupCWallStag, and the main_driver init."""
    p = CASES[name]()
    st = ref.state_from_reference(p, seed=10)
    g = torch.Generator().manual_seed(11)
    for m in st.state_mfs():
        noise = torch.randn(m.arr.shape, generator=g, dtype=torch.float64)
        keep = torch.zeros_like(m.arr, dtype=torch.bool)
        keep[(slice(None),) + tuple(slice(m.ngrow, m.arr.shape[1 + q] - m.ngrow) for q in range(3))] = True
        m.arr.copy_(torch.where(keep, m.arr, m.arr + noise))
    d = st.clone(device="cuda")
    ref.set_bc(st)
    ctx = Context(p)
    ctx.set_bc(d)
    torch.cuda.synchronize()
    bad, _ = compare_named(d.named(), st.named())
    assert not bad, bad[:6]
    eff = ctx.effective_params()
    for side in range(6):
        dd, hi = divmod(side, 2)
        if (p.bc_mass_hi if hi else p.bc_mass_lo)[dd] not in (2, 3):
            continue
        yk, xk = ref.wall_composition(p, side)
        ey = (eff.bc_Yk_hi if hi else eff.bc_Yk_lo)[dd]
        ex = (eff.bc_Xk_hi if hi else eff.bc_Xk_lo)[dd]
        assert [ey[n] for n in range(p.nspecies)] == yk
        assert [ex[n] for n in range(p.nspecies)] == xk
        if (p.bc_mass_hi if hi else p.bc_mass_lo)[dd] == 3:
            t, pr, rho = ref.wall_state(p, side)
            assert (eff.t_hi if hi else eff.t_lo)[dd] == t
            assert (eff.p_hi if hi else eff.p_lo)[dd] == pr
            assert (eff.rho_hi if hi else eff.rho_lo)[dd] == rho
    # main_driver init (InitConsVarStag, conversion, FillBoundary, setBCStag)
    gi = StagState(p, "cuda", aux=False)
    ctx.init_state(gi)
    h = StagState(p)
    ref.init_cons_var_stag(h)
    ref.fill_boundary(p, h.cu)
    for m in h.cumom:
        ref.fill_boundary(p, m, override_sync=True)
    ref.conserved_to_primitive(h)
    for m in [h.cu, h.prim] + h.vel:
        ref.fill_boundary(p, m)
    ref.set_bc(h)
    torch.cuda.synchronize()
    bad, _ = compare_named(gi.named(), h.named())
    assert not bad, bad[:6]
    ctx.close()


def test_walls_conserve_mass_and_hold_the_wall_faces(ref):
    """50 steps with in-kernel noise: total mass unchanged to round-off (no flux
    through impermeable walls), wall-face normal momentum exactly 0."""
    p = CASES["tempgrad_x"]()
    st = ref.state_from_reference(p, seed=12)
    d = st.clone(device="cuda")
    ctx = Context(p)
    dt = stable_dt(p)
    m0 = d.cu.valid()[0].sum().item()
    ctx.rk3_steps(d, dt, 0, 50)
    torch.cuda.synchronize()
    assert ctx.status() == 0
    m1 = d.cu.valid()[0].sum().item()
    assert abs(m1 - m0) <= 1e-12 * abs(m0)
    mx = d.cumom[0].valid(0)  # (z, y, x): the x wall faces are x = 0 and x = n
    assert torch.all(mx[..., 0] == 0) and torch.all(mx[..., -1] == 0)
    ctx.close()


# the particle reservoir (bc_mass 4): the interface fluxes and momenta come from the
# particles crossing it (ComputeFluxMomReservoir, ResetReservoirFluxes / Mom)
PARTICLE = {
    "particle_reservoir_x": lambda: with_walls(
        argon((8, 4, 4), dx=8e-6, seed=13), x=dict(vel=2, therm=2, mass=4, t=(273.0, 280.0), Yk=((0.5, 0.5),) * 2)),
    "particle_reservoir_wall": lambda: with_walls(
        mixture4((6, 5, 4), dx=8e-6, seed=14),
        y=dict(vel=2, therm=2, mass=4, t=(270.0, 276.0), Yk=((0.4, 0.2, 0.3, 0.1), (0.1, 0.3, 0.2, 0.4))),
        z=dict(vel=1, therm=1, mass=1)),
}


def reservoir_faces(p):
    n = p.n_cells
    tot = 0
    for d in range(3):
        for m in (p.bc_mass_lo[d], p.bc_mass_hi[d]):
            if m == 4:
                e = [q for q in range(3) if q != d]
                tot += n[e[0]] * n[e[1]]
    return tot


@pytest.mark.parametrize("name", list(PARTICLE))
def test_particle_reservoir_steps_match_the_reference(ref, name):
    """The GPU records every random number its reservoir processes draw; the
    reference, fed the same numbers in its own call order, gives the same step.
    The processes' rates and velocities go through exp, erf and log, which CUDA and
    the host's libm may round differently in the last bit, so the state and the
    stage-3 by-products agree within 1e-12 of each field's norm (everything away
    from the interface is bit-identical)."""
    p = PARTICLE[name]()
    st = ref.state_from_reference(p, seed=7)
    d = st.clone(device="cuda")
    ctx = Context(p)
    dt = stable_dt(p)
    cap = 32768
    rec = torch.full((3 * reservoir_faces(p) * cap,), float("nan"), dtype=torch.float64, device="cuda")
    ctx.set_reservoir_record(rec, cap)
    for s in range(2):
        nz = ref.step_noise(p, seed=70 + s)
        ctx.rk3_step(d, dt, s, noise=nz.to("cuda"), aux=True)
        torch.cuda.synchronize()
        assert ctx.status() == 0
        drawn = rec.cpu().contiguous()
        ref.set_reservoir_draws(drawn, cap)
        try:
            ref.rk3_step(st, nz, dt, s)
        finally:
            ref.set_reservoir_draws(None, 0)
        bad, worst = compare_named(d.named(aux=True), st.named(aux=True), tol=1e-12)
        assert not bad, (s, bad[:6])
    # the interface carries flow: its normal momentum is the particles' (non-zero)
    dd = [q for q in range(3) if 4 in (p.bc_mass_lo[q], p.bc_mass_hi[q])][0]
    mv = d.cumom[dd].valid(0)
    face = mv[..., 0] if dd == 0 else (mv[:, 0, :] if dd == 1 else mv[0])
    assert face.abs().max() > 0
    ctx.set_reservoir_record(None)
    ctx.close()
