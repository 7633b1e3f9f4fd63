"""Running statistics (evaluateStatsStag3D's per-cell part) in the oracle,
against an independent NumPy restatement of its recurrences
(statsStag.cpp:228-256, :281-317, :416-613):
mean_s = (mean_{s-1} (s-1) + x_s) / s and var_s = (var_{s-1} (s-1) + (x_s - mean_s)^2) / s,
with the fluctuation of the current sample taken about the current mean."""
import numpy as np
import pytest

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
