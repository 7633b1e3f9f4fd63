"""Quasi-1-D and quasi-2-D runs (do_1D / do_2D) on the GPU against the reference's
own code (oracle/_ref: RK3stepStag, calculateFluxStag and calculateTransportCoeffs
with their do_1D / do_2D branches, compiled unmodified), bit for bit (tolerance 0)
on the whole storage of the state and of the stage-3 coefficients and fluxes,
with injected noise and with the in-kernel noise materialised for the reference.

Cases: fully periodic boxes in both modes (argon and the 4-species mixture), the
boundary set-up of the reference's 1-D temperature-gradient regression run
(80 x 10 x 10 cells, isothermal no-slip x walls at 280.8 / 508.5 K), the set-up
of its 1-D reservoir regression run on a smaller box (bc_mass 3 reservoirs across
x at different compositions), and a 2-D run with slip walls in y."""
import pytest
import torch

from fhdex_b200.context import Context
from fhdex_b200.params import Params, argon, mixture4, stable_dt, with_walls
from fhdex_b200.state import StepNoise
from tests.helpers import compare_named

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R
    if not R.available():
        pytest.skip("oracle/_ref was not built")
    return R


CASES = {
    "periodic_1d": lambda: argon((16, 5, 4), dx=8e-6, seed=201).replace(do_1D=1),
    "periodic_1d_mix": lambda: mixture4((12, 4, 5), dx=8e-6, advection_type=1, seed=202).replace(do_1D=1),
    "periodic_2d": lambda: mixture4((9, 10, 4), dx=8e-6, seed=203).replace(do_2D=1),
    "periodic_2d_adv0": lambda: argon((10, 8, 3), dx=8e-6, advection_type=0, seed=204).replace(do_2D=1),
    # the boundary set-up of the reference's 1-D temperature-gradient regression run
    "tempgrad_1d": lambda: with_walls(
        Params(nspecies=4, n_cells=(80, 10, 10), prob_hi=(1.6e-4, 2e-5, 2e-5), molmass=(39.948,) * 4,
               diameter=(3.66e-8,) * 4, dof=(3.0,) * 4, e0=(0.0,) * 4, hcv=(-1.0,) * 4, hcp=(-1.0,) * 4,
               rhobar=(0.25,) * 4, T_init=400.0, rho0=1.78e-3, seed=1),
        x=dict(vel=2, therm=2, mass=1, t=(280.8, 508.5))).replace(do_1D=1),
    # the set-up of its 1-D reservoir regression run (two species of one molar mass
    # and different diameters, reservoirs across x) on a 24 x 6 x 6 box
    "reservoir_1d": lambda: with_walls(
        Params(nspecies=2, n_cells=(24, 6, 6), prob_hi=(1.44e-4, 3.6e-5, 3.6e-5), molmass=(20.17417748454183,) * 2,
               diameter=(2.58e-8, 4.16e-8), dof=(3.0,) * 2, e0=(0.0,) * 2, hcv=(-1.0,) * 2, hcp=(-1.0,) * 2,
               rhobar=(0.5, 0.5), T_init=300.0, rho0=0.0008168866420349571, seed=1),
        x=dict(vel=2, therm=2, mass=3, t=(300.0, 300.0), Yk=((0.1, 0.9), (0.9, 0.1)))).replace(do_1D=1),
    "walls_2d_y": lambda: with_walls(mixture4((8, 9, 4), dx=8e-6, seed=205),
                                     y=dict(vel=1, therm=1, mass=1)).replace(do_2D=1),
    # one-cell-thick boxes, the shapes the reference's driver runs these modes on
    "slab_2d": lambda: mixture4((10, 8, 1), dx=8e-6, seed=206).replace(do_2D=1),
    "pencil_1d": lambda: argon((24, 1, 1), dx=8e-6, seed=207).replace(do_1D=1),
    "pencil_1d_walls": lambda: with_walls(mixture4((20, 1, 1), dx=8e-6, seed=208),
                                          x=dict(vel=2, therm=2, mass=1, t=(280.0, 300.0))).replace(do_1D=1),
}
DT = {"tempgrad_1d": 1e-12, "reservoir_1d": 1e-12}


@pytest.mark.parametrize("name", list(CASES))
def test_lowdim_steps_equal_the_reference_injected_noise(ref, name):
    p = CASES[name]()
    st = ref.state_from_reference(p, seed=7)
    d = st.clone(device="cuda")
    ctx = Context(p)
    dt = DT.get(name, stable_dt(p))
    for s in range(3):
        nz = ref.step_noise(p, seed=70 + s)
        ctx.rk3_step(d, dt, s, noise=nz.to("cuda"), aux=True)
        torch.cuda.synchronize()
        ref.rk3_step(st, nz, dt, s)
        bad, _ = compare_named(d.named(aux=True), st.named(aux=True))
        assert not bad, (s, bad[:6])
    assert ctx.status() == 0
    ctx.close()


@pytest.mark.parametrize("name", ["periodic_1d_mix", "periodic_2d", "tempgrad_1d", "walls_2d_y", "slab_2d",
                                  "pencil_1d_walls"])
def test_lowdim_steps_equal_the_reference_in_kernel_noise(ref, name):
    """In-kernel Philox noise (the 1-D x centre noise at variance 1), materialised
    by fhd_fill_step_noise for the reference."""
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
    c = nzc.cen[0][0].valid(0)
    if p.do_1D and c.numel() >= 1000:
        assert 0.8 < float(c.var()) < 1.25          # the 1-D x centre noise has variance 1
    assert ctx.status() == 0
    ctx.close()


def test_lowdim_graph_replay_equals_single_steps(ref):
    p = CASES["periodic_2d"]()
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


def test_lowdim_transport_operator_equals_the_reference(ref):
    """calculateTransportCoeffs with do_1D: the coefficients on the box grown by one;
    the second ghost layer keeps what the caller held."""
    p = CASES["periodic_1d_mix"]()
    st = ref.state_from_reference(p, seed=12)
    for m in (st.eta, st.zeta, st.kappa, st.chi, st.D):
        m.arr.fill_(-7.0)
    d = st.clone(device="cuda")
    ref.transport(st)
    ctx = Context(p)
    ctx.transport_coeffs(d)
    torch.cuda.synchronize()
    for name in ("eta", "zeta", "kappa", "chi", "D"):
        assert torch.equal(getattr(d, name).arr.cpu(), getattr(st, name).arr), name
    assert (st.eta.arr[0, 0] == -7.0).all() and (st.eta.arr[0, 2, 2, 2] != -7.0)


@pytest.mark.parametrize("name,all_correl", [("periodic_1d_mix", 0), ("periodic_1d", 1), ("tempgrad_1d", 0),
                                             ("periodic_2d", 0), ("pencil_1d_walls", 1), ("slab_2d", 0)])
def test_lowdim_statistics_equal_the_reference(ref, name, all_correl):
    """fhd_stats_stag with every flag and FHD_STATS_CROSS in a quasi-1-D run (the
    per-pencil correlations with x* = cross_cell, or the five x* of all_correl) and
    in a quasi-2-D run (no correlations), after steps of the run, bit for bit
    against the reference's evaluateStatsStag1D / 2D."""
    from fhdex_b200 import capi
    from fhdex_b200.stats import StatsState
    p = CASES[name]().replace(cross_cell=3, all_correl=all_correl)
    st = ref.state_from_reference(p, seed=13)
    d = st.clone(device="cuda")
    ctx = Context(p)
    dt = DT.get(name, stable_dt(p))
    host = StatsState(p, cross=True)
    dev = StatsState(p, "cuda", cross=True)
    flags = 15 | capi.STATS_CROSS
    for s in range(3):
        nz = ref.step_noise(p, seed=90 + s)
        ctx.rk3_step(d, dt, s, noise=nz.to("cuda"), aux=False)
        ref.rk3_step(st, nz, dt, s)
        ctx.stats_stag(d, dev, s + 1, flags)
        ref.eval_stats(st, host, s + 1, flags)
    torch.cuda.synchronize()
    bad = [n for n, m in dev.named().items() if not torch.equal(m.arr.cpu(), host.named()[n].arr)]
    assert not bad, bad
    assert torch.equal(dev.spatialCross.cpu(), host.spatialCross)
    if p.do_1D:
        assert host.spatialCross.abs().max() > 0
    else:
        assert not host.spatialCross.any()
    assert ctx.status() == 0
