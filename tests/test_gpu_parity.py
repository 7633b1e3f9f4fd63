"""GPU parity: the sm_100a kernels through the C ABI against the CPU oracle.

FP64 path: bit-for-bit (tolerance 0) — the kernels keep the reference's
operation order and are built without FMA contraction; FP64 division and sqrt
are correctly rounded on both sides.  Mixed path: norm-relative error per field
against the FP64 oracle, bound stated in the test.
"""
import pytest
import torch

from fhdex_b200.context import Context
from fhdex_b200.params import argon, mixture4, stable_dt
from fhdex_b200.state import StagState, StepNoise
from tests.helpers import compare_named, max_rel, perturbed_state, seeded_noise

pytestmark = pytest.mark.gpu

CASES = [("argon12", lambda **k: argon(12, dx=8e-6, **k)),
         ("mix4_10x12x8", lambda **k: mixture4((10, 12, 8), dx=8e-6, **k))]


def gpu_copy(st):
    return st.clone(device="cuda")


@pytest.mark.parametrize("name,make", CASES)
def test_conversion_and_transport_bitwise(oracle, name, make):
    p = make()
    st = perturbed_state(oracle, p, seed=1)
    d = gpu_copy(st)
    ctx = Context(p)
    ctx.conserved_to_primitive(d)
    assert oracle.conserved_to_primitive(st) == 0
    ctx.transport_coeffs(d)
    assert oracle.transport_coeffs(st) == 0
    torch.cuda.synchronize()
    assert ctx.status() == 0
    names = ["cu", "prim", "vel0", "vel1", "vel2", "eta", "zeta", "kappa", "chi", "D"]
    bad, _ = compare_named(d.named(aux=True), {n: st.named(aux=True)[n] for n in names})
    assert not bad, bad


@pytest.mark.parametrize("name,make", CASES)
def test_flux_operator_bitwise(oracle, name, make):
    p = make()
    st = perturbed_state(oracle, p, seed=2)
    assert oracle.transport_coeffs(st) == 0
    nz = seeded_noise(oracle, p, 3, 0)
    d = gpu_copy(st)
    ndev = nz.to("cuda")
    dt = stable_dt(p)
    assert oracle.flux_stag(st, nz.face[0], nz.edge[0], nz.cen[0], dt) == 0
    ctx = Context(p)
    ctx.flux_stag(d, ndev.face[0], ndev.edge[0], ndev.cen[0], dt)
    torch.cuda.synchronize()
    ref = st.named(aux=True)
    names = [f"faceflux{q}" for q in range(3)] + [f"edgeflux{e}" for e in range(6)] + [f"cenflux{q}" for q in range(3)]
    bad, _ = compare_named(d.named(aux=True), {n: ref[n] for n in names})
    assert not bad, bad


@pytest.mark.parametrize("name,make,nsteps", [(CASES[0][0], CASES[0][1], 10), (CASES[1][0], CASES[1][1], 3)])
def test_rk3_step_injected_noise_bitwise(oracle, name, make, nsteps):
    """RK3stepStag with identical injected A/B noise: state, transport
    coefficients and stage-3 fluxes equal the oracle bit for bit after every step."""
    p = make()
    st = perturbed_state(oracle, p, seed=4)
    d = gpu_copy(st)
    ctx = Context(p)
    dt = stable_dt(p)
    for s in range(nsteps):
        nz = seeded_noise(oracle, p, 9, s)
        assert oracle.rk3_step(st, nz, dt) == 0
        ctx.rk3_step(d, dt, s, noise=nz.to("cuda"), aux=True)
        torch.cuda.synchronize()
        bad, _ = compare_named(d.named(aux=(s == nsteps - 1)), st.named(aux=(s == nsteps - 1)))
        assert not bad, (s, bad[:8])
    assert ctx.status() == 0


@pytest.mark.parametrize("opt", [dict(advection_type=0), dict(advection_type=1),
                                 dict(visc_type=3, zeta_ratio=0.7), dict(stoch_stress_form=0),
                                 dict(grav=(0.0, 0.0, -981.0))])
def test_rk3_step_options_bitwise(oracle, opt):
    p = argon(8, dx=8e-6, **opt)
    st = perturbed_state(oracle, p, seed=5)
    d = gpu_copy(st)
    ctx = Context(p)
    dt = stable_dt(p)
    for s in range(2):
        nz = seeded_noise(oracle, p, 13, s)
        assert oracle.rk3_step(st, nz, dt) == 0
        ctx.rk3_step(d, dt, s, noise=nz.to("cuda"), aux=True)
    torch.cuda.synchronize()
    bad, _ = compare_named(d.named(aux=True), st.named(aux=True))
    assert not bad, bad[:8]


def test_in_kernel_philox_equals_injected_replay(oracle):
    """The fused step's in-kernel Philox noise is exactly what fhd_fill_step_noise
    materialises: replaying those arrays through the injected path (GPU) and through
    the oracle gives the same trajectory bit for bit."""
    p = argon(12, dx=8e-6, seed=2024)
    st = perturbed_state(oracle, p, seed=6)
    a = gpu_copy(st)
    b = gpu_copy(st)
    ctx = Context(p)
    dt = stable_dt(p)
    nz = StepNoise(p, "cuda")
    for s in range(3):
        ctx.rk3_step(a, dt, s, noise=None, aux=False)
        ctx.fill_step_noise(nz, s)
        ctx.rk3_step(b, dt, s, noise=nz, aux=False)
        torch.cuda.synchronize()
        assert oracle.rk3_step(st, nz.to("cpu"), dt) == 0
        bad, _ = compare_named(a.named(), b.named())
        assert not bad, (s, bad[:4])
        bad, _ = compare_named(a.named(), st.named())
        assert not bad, (s, bad[:4])


def test_large_ragged_box_in_kernel_noise_bitwise(oracle):
    """A box large enough for every stage kernel's grid-stride loop to wrap (more
    work items than the 4736 x 128 threads of a launch) with unequal, non-power-of-
    two extents: one in-kernel-noise RK3 step equals the oracle fed the materialised
    noise, bit for bit, including the stage-3 fluxes and transport coefficients."""
    p = argon((100, 96, 90), dx=8e-6, seed=515)
    st = perturbed_state(oracle, p, seed=8)
    d = gpu_copy(st)
    ctx = Context(p)
    dt = stable_dt(p)
    nz = StepNoise(p, "cuda")
    ctx.fill_step_noise(nz, 0)
    ctx.rk3_step(d, dt, 0, noise=None, aux=True)
    torch.cuda.synchronize()
    assert ctx.status() == 0
    assert oracle.rk3_step(st, nz.to("cpu"), dt) == 0
    bad, _ = compare_named(d.named(aux=True), st.named(aux=True))
    assert not bad, bad[:8]


def test_all_tile_shapes_identical(oracle):
    p = argon((12, 10, 9), dx=8e-6)
    st = perturbed_state(oracle, p, seed=7)
    dt = stable_dt(p)
    outs = []
    for t, name in enumerate(Context.tiles()):
        d = gpu_copy(st)
        ctx = Context(p)
        ctx.set_tile(t)
        for s in range(2):
            ctx.rk3_step(d, dt, s, aux=False)
        torch.cuda.synchronize()
        outs.append((name, d))
    for name, d in outs[1:]:
        bad, _ = compare_named(d.named(), outs[0][1].named())
        assert not bad, (name, bad[:4])


@pytest.mark.parametrize("make", [lambda **k: argon(16, dx=8e-6, **k), lambda **k: mixture4(12, dx=8e-6, **k)])
def test_mixed_precision_against_fp64_oracle(oracle, make):
    """Mixed path (FP32 coefficients/stresses/dissipative fluxes, FP64 state and
    hyperbolic terms) vs the FP64 oracle with identical noise: per-field
    norm-relative error after 5 steps below 1e-4 (conserved state) / 1e-3
    (face velocities, which are O(noise))."""
    p = make(precision=1)
    st = perturbed_state(oracle, p.replace(precision=0), seed=8)
    st.p = p.replace(precision=0)
    d = gpu_copy(st)
    d.p = p
    ctx = Context(p)
    dt = stable_dt(p)
    for s in range(5):
        nz = seeded_noise(oracle, p, 17, s)
        assert oracle.rk3_step(st, nz, dt) == 0
        ctx.rk3_step(d, dt, s, noise=nz.to("cuda"), aux=False)
    torch.cuda.synchronize()
    errs = {}
    for n, m in st.named().items():
        g = d.named()[n]
        for c in range(m.ncomp):
            errs[f"{n}[{c}]"] = max_rel(g.valid(c), m.valid(c))
    print({k: f"{v:.2e}" for k, v in errs.items()})
    for k, v in errs.items():
        lim = 1e-3 if (k.startswith("vel") or k.startswith("cumom") or k[:6] in ("prim[1", "prim[2", "prim[3", "cu[1]", "cu[2]", "cu[3]")) else 1e-4
        assert v < lim, (k, v)


def test_conservation_philox_64(oracle):
    p = argon(64, dx=8e-6)
    st = StagState(p, "cuda")
    ctx = Context(p)
    ctx.init_state(st)
    dt = stable_dt(p)
    N = 64

    def totals():
        t = [st.cu.valid(n).sum().item() for n in (0, 4, 5, 6)]
        t += [m.arr[0, 2:2 + N, 2:2 + N, 2:2 + N].sum().item() for m in st.cumom]
        return t

    t0 = totals()
    for s in range(20):
        ctx.rk3_step(st, dt, s, aux=False)
    torch.cuda.synchronize()
    t1 = totals()
    assert ctx.status() == 0
    scale = [abs(x) for x in t0[:4]] + [p.rho0 * p.sound_speed() * N ** 3] * 3
    for a, b, sc in zip(t0, t1, scale):
        assert abs(a - b) <= 1e-12 * sc


def test_massfrac_status_is_reported_not_fatal(oracle):
    p = argon(8, dx=8e-6)
    st = perturbed_state(oracle, p, seed=9)
    d = gpu_copy(st)
    d.cu[2, 3, 4, 5] = 0.0          # rho*Y_0 = 0 -> Y_0 = 0 at one cell
    d.cu[2, 3, 4, 6] = d.cu[2, 3, 4, 0]
    ctx = Context(p)
    ctx.rk3_step(d, stable_dt(p), 0, aux=False)
    assert ctx.status() == 2        # FHD_ERR_MASSFRAC
    # the context stays usable
    ctx.rk3_step(gpu_copy(st), stable_dt(p), 0, aux=False)
    assert ctx.status() == 0


@pytest.mark.parametrize("opt", [dict(), dict(advection_type=0), dict(advection_type=1),
                                 dict(visc_type=3, zeta_ratio=0.7), dict(precision=1), dict(ns4=True)])
def test_step_does_not_read_input_prim_and_vel(oracle, opt):
    """The step derives prim and vel from cu and mom itself (its first conversion
    overwrites every point it later reads), so their input contents are dead: a
    step whose input prim and vel are NaN everywhere gives the same result, bit for
    bit, as one with consistent inputs.  The host-buffer step relies on this to
    upload only cu and mom."""
    opt = dict(opt)
    make = mixture4 if opt.pop("ns4", False) else argon
    p = make(10, dx=8e-6, seed=31, **opt)
    st = perturbed_state(oracle, p.replace(precision=0), seed=9)
    a = gpu_copy(st)
    b = gpu_copy(st)
    b.prim.arr.fill_(float("nan"))
    for v in b.vel:
        v.arr.fill_(float("nan"))
    ctx = Context(p)
    dt = stable_dt(p)
    aux = p.precision == 0          # the coefficient/flux by-products are FP64-only
    for s in range(2):
        ctx.rk3_step(a, dt, s, aux=aux)
        ctx.rk3_step(b, dt, s, aux=aux)
    torch.cuda.synchronize()
    assert ctx.status() == 0
    bad = [n for n, m in a.named(aux=aux).items() if not torch.equal(m.arr, b.named(aux=aux)[n].arr)]
    assert not bad, bad


def test_host_buffer_step_equals_device_step(oracle):
    """fhd_rk3_step_stag_host (pinned host fabs, copies inside the call) gives the
    device step's result bit for bit, uploads only cu and mom (prim and vel on
    entry may be anything), and downloads cu, mom, prim and vel."""
    p = argon(12, dx=8e-6, seed=77)
    st = perturbed_state(oracle, p, seed=4)
    dev = gpu_copy(st)
    host = st.clone(device="cpu", pin_memory=True)
    host.prim.arr.fill_(float("nan"))
    for v in host.vel:
        v.arr.fill_(float("nan"))
    ctx = Context(p)
    dt = stable_dt(p)
    for s in range(2):
        ctx.rk3_step(dev, dt, s, aux=False)
        h2d, d2h = ctx.rk3_step_host(host, dt, s)
    torch.cuda.synchronize()
    assert ctx.status() == 0
    bad = [n for n, m in dev.named().items() if not torch.equal(m.arr.cpu(), host.named()[n].arr)]
    assert not bad, bad
    up = host.cu.arr.numel() * 8 + sum(m.arr.numel() * 8 for m in host.cumom)
    assert h2d == up
    assert d2h == sum(m.arr.numel() * 8 for m in host.state_mfs())


@pytest.mark.parametrize("precision,stoch", [(0, 1), (1, 1), (0, 0)])
def test_graph_replayed_steps_equal_single_steps(oracle, precision, stoch):
    """fhd_rk3_steps_stag (one captured step replayed from a CUDA graph, the step
    number read from a device counter) gives bitwise the state of the same steps
    launched one by one, across a second call that continues the step count and
    after a change of fabs that forces a new capture."""
    p = argon((12, 10, 9), dx=8e-6, seed=4321, precision=precision)
    p.stoch_stress_form = stoch
    st = perturbed_state(oracle, p, seed=12)
    a = gpu_copy(st)
    b = gpu_copy(st)
    ctx = Context(p)
    dt = stable_dt(p)
    for s in range(7):
        ctx.rk3_step(a, dt, s, aux=False)
    ctx.rk3_steps(b, dt, 0, 4)
    ctx.rk3_steps(b, dt, 4, 3)
    torch.cuda.synchronize()
    bad, _ = compare_named(b.named(), a.named())
    assert not bad, bad[:4]
    c = gpu_copy(st)
    ctx.rk3_steps(c, dt, 0, 7)   # other fabs: captured anew
    torch.cuda.synchronize()
    bad, _ = compare_named(c.named(), a.named())
    assert not bad, bad[:4]
    assert ctx.status() == 0
    ctx.close()
