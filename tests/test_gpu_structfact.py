"""The device structure factor (fhd_sf_*, cuFFT + fused accumulation) against
the NumPy restatement of StructFact: norm-relative error below 1e-12 (the two
FFT libraries round differently; everything after the FFT is in the reference's
operation order), for default and chosen pairs, reset semantics, fabs with and
without ghosts, and odd box sizes."""
import numpy as np
import pytest
import torch

from fhdex_b200.fab import CELL, MultiFab
from fhdex_b200.structfact import StructFact
from oracle.structfact import StructFactOracle

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("shape_xyz,ng,pairs", [((8, 6, 4), 0, None), ((7, 5, 6), 2, None),
                                                ((16, 16, 16), 1, ([2, 0, 1], [0, 2, 1]))])
def test_structure_factor_matches_oracle(shape_xyz, ng, pairs):
    nvar = 3
    rng = np.random.default_rng(5)
    ncov = len(pairs[0]) if pairs else nvar * (nvar + 1) // 2
    scaling = list(rng.uniform(0.5, 2.0, ncov))
    sf = StructFact(shape_xyz, ["a", "b", "c"], scaling, pairs=pairs)
    zyx = shape_xyz[::-1]
    ora = StructFactOracle(zyx, nvar, scaling, pairs=pairs)
    mf = MultiFab(shape_xyz, CELL, nvar, ng, device="cuda")
    for s in range(4):
        v = rng.standard_normal((nvar,) + zyx)
        v[1] = 0.5 * v[0] + 0.2 * v[1]            # correlated pair
        mf.valid().copy_(torch.from_numpy(v))
        reset = 1 if s == 2 else 0                 # restart after two samples
        sf.fort_structure(mf, reset=reset)
        ora.fort_structure(v, reset=reset)
    assert sf.nsamples == ora.nsamples == 2
    for zero_avg in (0, 1):
        got = [m.valid().cpu().numpy() for m in sf.finalize(zero_avg)]
        ref = ora.finalize(zero_avg)
        for g, r, name in zip(got, ref, ("real", "imag", "mag")):
            assert rel(g, r) < 1e-12, (name, zero_avg, rel(g, r))
    torch.cuda.synchronize()
    sf.close()


def test_density_structure_factor_of_the_step_is_flat():
    """S(k) of density from the equilibrium step, accumulated by the library,
    flat at the theory variance (k-average within 3 %)."""
    from fhdex_b200.context import Context
    from fhdex_b200.params import argon, stable_dt
    from fhdex_b200.state import StagState
    from fhdex_b200.equilibrium import equilibrium_variances
    n = 32
    p = argon(n, dx=8e-6, seed=7)
    st = StagState(p, "cuda", aux=False)
    ctx = Context(p)
    ctx.init_state(st)
    dt = stable_dt(p)
    for s in range(1000):
        ctx.rk3_step(st, dt, s, aux=False)
    sf = StructFact(p.n_cells, ["rho"], [1.0])
    var = MultiFab(p.n_cells, CELL, 1, 0, device="cuda")
    for s in range(150):
        for q in range(5):
            ctx.rk3_step(st, dt, 1000 + 5 * s + q, aux=False)
        var.valid(0).copy_(st.cu.valid(0))
        sf.fort_structure(var)
    re, _, _ = sf.finalize(zero_avg=1)
    s = re.valid(0).cpu().numpy()
    th = equilibrium_variances(p)["rho"]
    assert s.sum() / (s.size - 1) / th == pytest.approx(1.0, abs=0.03)
    sf.close()


@pytest.mark.parametrize("stack,shape_xyz,ng,pairs", [("z_slices", (8, 6, 5), 0, None),
                                                      ("z_slices", (7, 4, 3), 2, ([2, 0], [1, 1])),
                                                      ("x_pencils", (16, 3, 3), 1, None),
                                                      ("x_pencils", (9, 4, 4), 0, ([1, 2, 0], [0, 2, 1]))])
def test_structure_factor_stacks_match_oracle(stack, shape_xyz, ng, pairs):
    """The quasi-2-D per-slice and quasi-1-D per-pencil structure factors (one
    batched cuFFT over the members) and the reference's averaged output of them
    against the NumPy restatement (one StructFact per member, AddToExternal in
    member order, 1/members): norm-relative error below 1e-12, with a reset."""
    from oracle.structfact import StructFactStackOracle
    nvar = 3
    rng = np.random.default_rng(11)
    ncov = len(pairs[0]) if pairs else nvar * (nvar + 1) // 2
    scaling = list(rng.uniform(0.5, 2.0, ncov))
    sf = StructFact(shape_xyz, ["a", "b", "c"], scaling, pairs=pairs, stack=stack)
    zyx = shape_xyz[::-1]
    ora = StructFactStackOracle(zyx, stack, nvar, scaling, pairs=pairs)
    mf = MultiFab(shape_xyz, CELL, nvar, ng, device="cuda")
    for s in range(4):
        v = rng.standard_normal((nvar,) + zyx)
        v[1] = 0.5 * v[0] + 0.2 * v[1]
        v[2] += np.linspace(0.0, 1.0, zyx[0])[:, None, None]   # members differ
        mf.valid().copy_(torch.from_numpy(v))
        reset = 1 if s == 1 else 0
        sf.fort_structure(mf, reset=reset)
        ora.fort_structure(v, reset=reset)
    assert sf.nsamples == ora.nsamples == 3
    for zero_avg in (0, 1):
        mag, ri = sf.stack_average(zero_avg)
        rmag, rri = ora.stack_average(zero_avg)
        assert mag.valid().shape[1:] == rmag.shape[1:]
        assert rel(mag.valid().cpu().numpy(), rmag) < 1e-12
        assert rel(ri.valid().cpu().numpy(), rri) < 1e-12
    from fhdex_b200.capi import FhdError
    with pytest.raises(FhdError):
        sf.finalize()
    torch.cuda.synchronize()
    sf.close()
