"""Running statistics on the GPU (fhd_stats_stag): bit for bit against the CPU
oracle on random states, and, accumulated after every step of an equilibrium
run, the box-averaged running variances against the fluctuation theory the
reference checks its runs with (tests/theory.py), within 3 %."""
import pytest
import torch

from fhdex_b200 import capi
from fhdex_b200.context import Context
from fhdex_b200.params import argon, mixture4, stable_dt
from fhdex_b200.state import StagState
from fhdex_b200.stats import StatsState
from tests.helpers import perturbed_state
from fhdex_b200.equilibrium import equilibrium_variances

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("flags", [15, capi.STATS_MEANS, capi.STATS_MEANS | capi.STATS_VARS])
@pytest.mark.parametrize("make", [lambda: argon((6, 5, 4), dx=8e-6), lambda: mixture4((5, 4, 6), dx=8e-6)])
def test_stats_bitwise_against_oracle(oracle, make, flags):
    p = make()
    host = StatsState(p)
    dev = StatsState(p, "cuda")
    ctx = Context(p)
    for s in range(1, 5):
        st = perturbed_state(oracle, p, seed=200 + s, amp=0.05)
        assert oracle.stats_stag(st, host, s, flags) == 0
        ctx.stats_stag(st.clone(device="cuda"), dev, s, flags)
    torch.cuda.synchronize()
    bad = [n for n, m in dev.named().items() if not torch.equal(m.arr.cpu(), host.named()[n].arr)]
    assert not bad, bad
    # the state moved the statistics away from zero
    assert host.cuVars.valid(0).abs().max() > 0 or flags == capi.STATS_MEANS


def test_stats_reject_bad_shapes():
    p = argon(6, dx=8e-6)
    ctx = Context(p)
    st = StagState(p, "cuda", aux=False)
    ctx.init_state(st)
    stats = StatsState(p, "cuda")
    with pytest.raises(capi.FhdError):
        ctx.stats_stag(st, stats, 1, capi.STATS_VARS)          # variances without means
    with pytest.raises(capi.FhdError):
        ctx.stats_stag(st, stats, 0, 15)                        # sample count < 1
    bad = StatsState(argon(7, dx=8e-6), "cuda")
    with pytest.raises(capi.FhdError):
        ctx.stats_stag(st, bad, 1, 15)                          # wrong box


def test_running_variances_match_theory_in_equilibrium():
    n = 32
    p = argon(n, dx=8e-6, seed=99)
    st = StagState(p, "cuda", aux=False)
    ctx = Context(p)
    ctx.init_state(st)
    dt = stable_dt(p)
    for s in range(1000):
        ctx.rk3_step(st, dt, s, aux=False)
    stats = StatsState(p, "cuda", mom34=False)
    nsamp = 1500
    for s in range(1, nsamp + 1):
        ctx.rk3_step(st, dt, 1000 + s, aux=False)
        ctx.stats_stag(st, stats, s, capi.STATS_MEANS | capi.STATS_VARS)
    torch.cuda.synchronize()
    assert ctx.status() == 0
    th = equilibrium_variances(p)
    got = {"rho": stats.cuVars.valid(0).mean().item(), "rho0": stats.cuVars.valid(5).mean().item(),
           "rhoE": stats.cuVars.valid(4).mean().item(), "T": stats.primVars.valid(4).mean().item(),
           "jx": stats.cumomVars[0].valid(0).mean().item(), "jy": stats.cumomVars[1].valid(0).mean().item(),
           "jz": stats.cumomVars[2].valid(0).mean().item()}
    ratios = {k: v / th[k] for k, v in got.items()}
    print({k: f"{v:.4f}" for k, v in ratios.items()})
    for k, r in ratios.items():
        assert r == pytest.approx(1.0, abs=0.03), (k, r)


@pytest.mark.parametrize("make,cc", [(lambda: argon((40, 7, 5), dx=8e-6), 17),
                                     (lambda: mixture4((33, 6, 6), dx=8e-6), 32),
                                     (lambda: argon((64, 48, 40), dx=8e-6), 0)])
def test_spatial_cross_bitwise_against_oracle_and_reference(oracle, make, cc):
    """FHD_STATS_CROSS (k_sum_to_line + k_spatial_cross after the per-cell passes):
    spatialCross and dataSliceMeans_xcross bit for bit against the oracle over
    four samples, and against the reference's own evaluateStatsStag3D where
    oracle/_ref is built.  The sizes give x lines that are not a multiple of the
    warp and y-z planes that are not a multiple of the kernel's load depth."""
    from oracle import ref as R
    p = make().replace(cross_cell=cc)
    flags = 15 | capi.STATS_CROSS
    host = StatsState(p, cross=True)
    theirs = StatsState(p, cross=True) if R.available() else None
    dev = StatsState(p, "cuda", cross=True)
    ctx = Context(p)
    for s in range(1, 5):
        st = perturbed_state(oracle, p, seed=400 + s, amp=0.05)
        assert oracle.stats_stag(st, host, s, flags) == 0
        if theirs is not None:
            R.eval_stats(st, theirs, s, flags)
        ctx.stats_stag(st.clone(device="cuda"), dev, s, flags)
    torch.cuda.synchronize()
    assert ctx.status() == 0
    assert torch.equal(dev.spatialCross.cpu(), host.spatialCross)
    assert torch.equal(dev.dataSliceMeans_xcross.cpu(), host.dataSliceMeans_xcross)
    bad = [n for n, m in dev.named().items() if not torch.equal(m.arr.cpu(), host.named()[n].arr)]
    assert not bad, bad
    if theirs is not None:
        assert torch.equal(host.spatialCross, theirs.spatialCross)
        assert torch.equal(host.dataSliceMeans_xcross, theirs.dataSliceMeans_xcross)
    assert host.spatialCross[:, 0].abs().max() > 0


def test_spatial_cross_rejects_bad_arguments():
    p = argon((6, 5, 4), dx=8e-6).replace(cross_cell=6)
    ctx = Context(p)
    st = StagState(p, "cuda", aux=False)
    ctx.init_state(st)
    with pytest.raises(capi.FhdError):
        ctx.stats_stag(st, StatsState(p, "cuda", cross=True), 1, 1 | capi.STATS_CROSS)   # x* outside the box
    q = p.replace(cross_cell=2)
    ctx = Context(q)
    with pytest.raises(capi.FhdError):
        ctx.stats_stag(st, StatsState(q, "cuda"), 1, 1 | capi.STATS_CROSS)              # no spatialCross buffers
