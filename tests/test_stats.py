"""Running statistics (evaluateStatsStag3D's per-cell part) in the oracle,
against an independent NumPy restatement of its recurrences
(statsStag.cpp:228-256, :281-317, :416-613):
mean_s = (mean_{s-1} (s-1) + x_s) / s and var_s = (var_{s-1} (s-1) + (x_s - mean_s)^2) / s,
with the fluctuation of the current sample taken about the current mean."""
import numpy as np
import pytest
import torch

from fhdex_b200 import capi
from fhdex_b200.params import argon, mixture4
from fhdex_b200.stats import StatsState
from tests.helpers import perturbed_state


def run_samples(O, p, nsamp, flags=15):
    stats = StatsState(p)
    samples = []
    for s in range(1, nsamp + 1):
        st = perturbed_state(O, p, seed=100 + s, amp=0.05)
        assert O.stats_stag(st, stats, s, flags) == 0
        samples.append(st)
    return stats, samples


def recur(xs):
    """mean and variance recurrences of the reference, in the same operation order."""
    mean = np.zeros_like(xs[0])
    var = np.zeros_like(xs[0])
    for s, x in enumerate(xs, start=1):
        sm1, sinv = s - 1.0, 1.0 / s
        mean = (mean * sm1 + x) * sinv
        d = x - mean
        var = (var * sm1 + d * d) * sinv
    return mean, var


@pytest.mark.parametrize("make", [lambda: argon((5, 4, 3), dx=8e-6), lambda: mixture4((4, 3, 5), dx=8e-6)])
def test_oracle_statistics_follow_the_recurrences(oracle, make):
    p = make()
    stats, samples = run_samples(oracle, p, 5)
    ns = p.nspecies
    cu = [s.cu.valid().numpy() for s in samples]
    # conserved means and variances: rho, rhoE, rhoY_k
    for c in [0, 4] + [5 + k for k in range(ns)]:
        m, v = recur([x[c] for x in cu])
        np.testing.assert_array_equal(stats.cuMeans.valid(c).numpy(), m)
        np.testing.assert_array_equal(stats.cuVars.valid(c).numpy(), v)
    # face momenta
    for d in range(3):
        m, v = recur([s.cumom[d].valid(0).numpy() for s in samples])
        np.testing.assert_array_equal(stats.cumomMeans[d].valid(0).numpy(), m)
        np.testing.assert_array_equal(stats.cumomVars[d].valid(0).numpy(), v)
    # temperature: direct variance about the running mean (statsStag.cpp:553-555)
    m, v = recur([s.prim.valid(4).numpy() for s in samples])
    np.testing.assert_array_equal(stats.primMeans.valid(4).numpy(), m)
    np.testing.assert_array_equal(stats.primVars.valid(4).numpy(), v)
    # covariance <rho rhoE> (coVars component 6) with both fluctuations about the current means
    rm = np.zeros_like(cu[0][0])
    em = np.zeros_like(cu[0][0])
    cov = np.zeros_like(cu[0][0])
    for s, x in enumerate(cu, start=1):
        sm1, sinv = s - 1.0, 1.0 / s
        rm = (rm * sm1 + x[0]) * sinv
        em = (em * sm1 + x[4]) * sinv
        cov = (cov * sm1 + (x[0] - rm) * (x[4] - em)) * sinv
    np.testing.assert_array_equal(stats.coVars.valid(6).numpy(), cov)
    # ghosts of the cell means are periodic images (FillBoundary)
    a = stats.cuMeans.arr.numpy()
    g = p.ngc
    np.testing.assert_array_equal(a[:, :, :, :g], a[:, :, :, -2 * g:-g])


def test_constant_samples_give_exact_means_and_zero_variances(oracle):
    p = argon(4, dx=8e-6)
    st = perturbed_state(oracle, p, seed=3)
    stats = StatsState(p)
    for s in range(1, 4):
        assert oracle.stats_stag(st, stats, s) == 0
    np.testing.assert_allclose(stats.cuMeans.valid(0).numpy(), st.cu.valid(0).numpy(), rtol=1e-15)
    # the running mean of a constant is the constant up to rounding (1/3 is inexact), so
    # the variances are rounding-sized: below (1e-15 x)^2 per component
    for c in (0, 4, 5, 6):
        scale = np.abs(st.cu.valid(c).numpy()).max() ** 2
        assert np.abs(stats.cuVars.valid(c).numpy()).max() <= 1e-30 * scale, c


def test_variances_without_means_are_rejected(oracle):
    p = argon(4, dx=8e-6)
    st = perturbed_state(oracle, p, seed=3)
    assert oracle.stats_stag(st, StatsState(p), 1, capi.STATS_VARS) == capi.FHD_ERR_BAD_ARG


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R
    if not R.available():
        pytest.skip("oracle/_ref was not built")
    return R


@pytest.mark.parametrize("flags", [15 | capi.STATS_CROSS, capi.STATS_MEANS | capi.STATS_CROSS, 15])
@pytest.mark.parametrize("make,cc", [(lambda: argon((7, 5, 4), dx=8e-6), 3),
                                     (lambda: mixture4((6, 4, 5), dx=8e-6), 0),
                                     (lambda: mixture4((5, 3, 4), dx=8e-6), 4)])
def test_oracle_statistics_equal_the_reference(oracle, ref, make, cc, flags):
    """The oracle's evaluateStatsStag3D (per-cell statistics and, with
    FHD_STATS_CROSS, the yz-averaged spatial cross-correlations at x* = cross_cell)
    bit for bit against the reference's own statsStag.cpp over five samples."""
    p = make().replace(cross_cell=cc)
    mine, theirs = StatsState(p, cross=True), StatsState(p, cross=True)
    for s in range(1, 6):
        st = perturbed_state(oracle, p, seed=300 + s, amp=0.05)
        assert oracle.stats_stag(st, mine, s, flags) == 0
        ref.eval_stats(st, theirs, s, flags)
    bad = [n for n, m in mine.named().items() if not torch.equal(m.arr, theirs.named()[n].arr)]
    assert not bad, bad
    if flags & capi.STATS_CROSS:
        assert torch.equal(mine.spatialCross, theirs.spatialCross)
        assert torch.equal(mine.dataSliceMeans_xcross, theirs.dataSliceMeans_xcross)
        assert mine.spatialCross[:, 0].abs().max() > 0 and torch.isfinite(mine.spatialCross).all()
    else:
        assert not mine.spatialCross.any()


def test_spatial_cross_line_averages(oracle):
    """dataSliceMeans_xcross holds the y-z averages at x* of rho, rhoE, the
    cell-centred momenta, the velocities, T and, per species, rhoY_k and the prim
    component 5 + k (the reference's lines read pressure as the first "Y_k")."""
    p = mixture4((6, 4, 5), dx=8e-6).replace(cross_cell=2)
    stats = StatsState(p, cross=True)
    st = perturbed_state(oracle, p, seed=7, amp=0.05)
    assert oracle.stats_stag(st, stats, 1, capi.STATS_MEANS | capi.STATS_CROSS) == 0
    x = stats.dataSliceMeans_xcross.numpy()
    cu, pr = st.cu.valid().numpy()[:, :, :, 2], st.prim.valid().numpy()[:, :, :, 2]
    np.testing.assert_allclose(x[0], cu[0].mean(), rtol=1e-14)
    np.testing.assert_allclose(x[2], cu[4].mean(), rtol=1e-14)
    np.testing.assert_allclose(x[4], cu[1].mean(), rtol=1e-12, atol=1e-30)
    np.testing.assert_allclose(x[16], pr[4].mean(), rtol=1e-14)
    for k in range(p.nspecies):
        np.testing.assert_allclose(x[18 + 4 * k], cu[5 + k].mean(), rtol=1e-14)
        np.testing.assert_allclose(x[18 + 4 * k + 2], pr[5 + k].mean(), rtol=1e-14)
    # one sample: the running means of rho, rhoE, the momenta and T equal the
    # sample (the velocity means are derived from the momentum and density means),
    # so the conserved-variable correlations are zero
    for q in (0, 2, 4, 6, 8, 16):
        assert x[q] == x[q + 1], q
    assert not stats.spatialCross[:, :19].any()


def test_spatial_cross_rejects_a_cross_cell_outside_the_box(oracle):
    p = argon((4, 3, 3), dx=8e-6).replace(cross_cell=4)
    stats = StatsState(p, cross=True)
    st = perturbed_state(oracle, p, seed=1)
    assert oracle.stats_stag(st, stats, 1, capi.STATS_MEANS | capi.STATS_CROSS) == capi.FHD_ERR_BAD_ARG
