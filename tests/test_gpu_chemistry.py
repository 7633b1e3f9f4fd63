"""GPU chemistry source (compute_compressible_chemistry_source_CLE,
chemistry_functions.cpp:128-193) through the C ABI, against the CPU oracle.

Tolerances.  Where every power and exponential of the rate is exact (first-order
reactions, no activation energy, no temperature power: exp(+-0) = 1,
pow(x, 0) = 1, pow(x, 1) = x on both sides) the GPU source and a step with it are
bitwise the oracle's.  Otherwise the CUDA library's exp and pow and the host C
library's may round the last ulp differently (and c*c, correctly rounded, stands
for the reference's pow(c, 2)), so each rate carries a few ulps of relative
difference: the source is held to 1e-14 of the sum of the magnitudes of its
terms, and three RK3 steps to 1e-13 of each field's norm.
"""
import math

import pytest
import torch

from fhdex_b200.context import Context
from fhdex_b200.fab import CELL, MultiFab
from fhdex_b200.params import exchange_network, isomerization, mixture4, no2_dimerization, stable_dt
from fhdex_b200.state import StagState, StepNoise
from tests.helpers import compare_named, perturbed_state, seeded_noise

pytestmark = pytest.mark.gpu


def cell_volume(p):
    dx = p.dx
    return dx[0] * dx[1] * dx[2]


def on_gpu(mf):
    return MultiFab(mf.n_cells, mf.nodal, mf.ncomp, mf.ngrow, tensor=mf.arr.to("cuda"))


def chem_inputs(oracle, p, seed):
    st = perturbed_state(oracle, p, seed=seed)
    W = MultiFab(p.n_cells, CELL, p.nreaction, 0)
    g = torch.Generator().manual_seed(seed + 100)
    W.valid().copy_(torch.randn(W.valid().shape, generator=g, dtype=torch.float64))
    src = MultiFab(p.n_cells, CELL, p.nprimvars, 0)
    return st, W, src


def term_scale(p, prim, W, dt, dV):
    """Per species and cell, the sum of |terms| of the source (numpy restatement of
    the rates; only a scale for the tolerance)."""
    pv = prim.valid()
    T, pres = pv[4], pv[5]
    ctot = pres / p.Runiv / T
    ns = p.nspecies
    navo = p.Runiv / p.k_B
    out = torch.zeros((ns,) + tuple(T.shape), dtype=torch.float64)
    for m in range(p.nreaction):
        a = p.rate_const[m] * torch.exp(-p.alpha_param[m] / p.Runiv * (1 / T - 1 / p.T0_chem))
        a = a * (T / p.T0_chem) ** p.beta_param[m]
        for n in range(ns):
            a = a * (pv[6 + ns + n] * ctot) ** p.stoich_R[m][n]
        a = a.clamp(min=0)
        fl = torch.sqrt(a / navo) * W.valid()[m].abs() / math.sqrt(dt * dV)
        for n in range(ns):
            nu = abs(p.stoich_P[m][n] - p.stoich_R[m][n])
            out[n] += p.molmass[n] * nu * (a + fl)
    return out


@pytest.mark.parametrize("exact", [True, False])
def test_chemistry_operator_against_oracle(oracle, exact):
    p = no2_dimerization((9, 7, 6))
    if exact:
        p = isomerization(p)
    st, W, src = chem_inputs(oracle, p, seed=1)
    dt, dV = 1e-12, cell_volume(p)
    assert oracle.chemistry_source_cle(p, dt, dV, st.prim, src, W) == 0
    ctx = Context(p)
    dsrc = on_gpu(MultiFab(p.n_cells, CELL, p.nprimvars, 0))
    ctx.chemistry_source_cle(on_gpu(st.prim), dsrc, on_gpu(W), dt, dV)
    torch.cuda.synchronize()
    got = dsrc.arr.cpu()
    if exact:
        assert torch.equal(got, src.arr)
    else:
        diff = (got - src.arr).abs()
        scale = term_scale(p, st.prim, W, dt, dV)
        d = diff[5:5 + p.nspecies]
        assert torch.count_nonzero(diff[:5]) == 0
        assert (d <= 1e-14 * scale).all(), (d / scale).max().item()
    ctx.close()


@pytest.mark.parametrize("exact,nsteps", [(True, 4), (False, 3)])
def test_rk3_step_with_chemistry_injected_noise(oracle, exact, nsteps):
    """RK3stepStag with the chemistry source and identical injected A/B noise (the
    stress noises and ranchem_A / ranchem_B): the state and the last stage's
    source equal the oracle's."""
    p = no2_dimerization((8, 6, 7))
    if exact:
        p = isomerization(p)
    st = perturbed_state(oracle, p, seed=4)
    d = st.clone(device="cuda")
    ctx = Context(p)
    dt = stable_dt(p)
    for s in range(nsteps):
        nz = seeded_noise(oracle, p, 9, s)
        assert nz.chem[0] is not None
        assert oracle.rk3_step(st, nz, dt) == 0
        ctx.rk3_step(d, dt, s, noise=nz.to("cuda"), aux=True)
        torch.cuda.synchronize()
        got = dict(d.named(), source=d.source)
        ref = dict(st.named(), source=st.source)
        bad, worst = compare_named(got, ref, tol=0.0 if exact else 1e-13)
        assert not bad, (s, bad[:8])
    assert ctx.status() == 0
    # the chemistry moved the composition: the species source is not zero
    assert d.source.arr[5:5 + p.nspecies].abs().max().item() > 0
    ctx.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_in_kernel_reaction_noise_is_the_filled_noise(oracle, precision):
    """A step with in-kernel Philox noise equals the same step replayed through the
    injected path with fhd_fill_step_noise's A/B fields (stress and reaction), in
    both precisions (the chemistry source is FP64 in both)."""
    p = no2_dimerization((10, 8, 9), precision=precision)
    ctx = Context(p)
    st = perturbed_state(oracle, p, seed=6)
    d1 = st.clone(device="cuda")
    d2 = st.clone(device="cuda")
    dt = stable_dt(p)
    aux = precision == 0  # the by-products are FP64-path outputs
    for s in range(3):
        ctx.rk3_step(d1, dt, 40 + s, aux=aux)
        nz = StepNoise(p, device="cuda")
        ctx.fill_step_noise(nz, 40 + s)
        ctx.rk3_step(d2, dt, 40 + s, noise=nz, aux=aux)
    torch.cuda.synchronize()
    bad, _ = compare_named(dict(d1.named(), source=d1.source), dict(d2.named(), source=d2.source))
    assert not bad, bad[:8]
    assert ctx.status() == 0
    ctx.close()


def test_graph_replayed_steps_with_chemistry_equal_single_steps(oracle):
    p = no2_dimerization((12, 10, 8))
    st = perturbed_state(oracle, p, seed=7)
    dt = stable_dt(p)
    ctx = Context(p)
    d1 = st.clone(device="cuda")
    d2 = st.clone(device="cuda")
    for s in range(5):
        ctx.rk3_step(d1, dt, 3 + s, aux=False)
    ctx.rk3_steps(d2, dt, 3, 5)
    torch.cuda.synchronize()
    bad, _ = compare_named(d1.named(), d2.named())
    assert not bad, bad[:8]
    ctx.close()


def test_chemical_langevin_noise_has_the_theoretical_variance(oracle):
    """Uniform NO2 state, W ~ N(0, 1) per reaction and cell: the fluctuating part of
    S_n has variance sum_m (M_n nu_mn)^2 a_m / (N_A dt dV) over the cells."""
    p = no2_dimerization((48, 48, 48))
    st = StagState(p)
    oracle.init_state(st, p)
    ctx = Context(p)
    prim = on_gpu(st.prim)
    W = on_gpu(MultiFab(p.n_cells, CELL, p.nreaction, 0))
    ctx.fill_random_normal(W, 0, p.nreaction, 0.0, 1.0, overridesync=False, fillboundary=False, stream_id=11)
    Z = on_gpu(MultiFab(p.n_cells, CELL, p.nreaction, 0))
    s1 = on_gpu(MultiFab(p.n_cells, CELL, p.nprimvars, 0))
    s0 = on_gpu(MultiFab(p.n_cells, CELL, p.nprimvars, 0))
    dt, dV = 1e-12, cell_volume(p)
    ctx.chemistry_source_cle(prim, s1, W, dt, dV)
    ctx.chemistry_source_cle(prim, s0, Z, dt, dV)
    torch.cuda.synchronize()
    pv = st.prim.valid()
    T, pres = pv[4, 0, 0, 0].item(), pv[5, 0, 0, 0].item()
    ctot = pres / p.Runiv / T
    ck = [pv[8 + n, 0, 0, 0].item() * ctot for n in range(2)]
    a = []
    for m in range(2):
        r = p.rate_const[m] * math.exp(-p.alpha_param[m] / p.Runiv * (1 / T - 1 / p.T0_chem))
        r *= (T / p.T0_chem) ** p.beta_param[m]
        for n in range(2):
            r *= ck[n] ** p.stoich_R[m][n]
        a.append(r)
    navo = p.Runiv / p.k_B
    for n in range(2):
        fl = (s1.valid()[5 + n] - s0.valid()[5 + n]).flatten().cpu()
        theory = sum((p.molmass[n] * (p.stoich_P[m][n] - p.stoich_R[m][n])) ** 2 * a[m] / (navo * dt * dV)
                     for m in range(2))
        ratio = fl.var().item() / theory
        assert abs(ratio - 1.0) < 0.03, (n, ratio)
        assert abs(fl.mean().item()) < 5 * math.sqrt(theory / fl.numel())
    ctx.close()


def test_four_species_network_bitwise(oracle):
    """A + B <-> C + D and A <-> C on four species (the NS = 4 kernel): the operator
    and three RK3 steps with injected noise equal the oracle bit for bit."""
    p = exchange_network(mixture4((7, 6, 5), dx=8e-6))
    st, W, src = chem_inputs(oracle, p, seed=12)
    dt, dV = 1e-12, cell_volume(p)
    assert oracle.chemistry_source_cle(p, dt, dV, st.prim, src, W) == 0
    ctx = Context(p)
    dsrc = on_gpu(MultiFab(p.n_cells, CELL, p.nprimvars, 0))
    ctx.chemistry_source_cle(on_gpu(st.prim), dsrc, on_gpu(W), dt, dV)
    torch.cuda.synchronize()
    assert torch.equal(dsrc.arr.cpu(), src.arr)
    assert src.arr[5:9].abs().max().item() > 0
    d = st.clone(device="cuda")
    dt = stable_dt(p)
    for s in range(3):
        nz = seeded_noise(oracle, p, 21, s)
        assert oracle.rk3_step(st, nz, dt) == 0
        ctx.rk3_step(d, dt, s, noise=nz.to("cuda"), aux=True)
        torch.cuda.synchronize()
        bad, _ = compare_named(dict(d.named(), source=d.source), dict(st.named(), source=st.source))
        assert not bad, (s, bad[:8])
    assert ctx.status() == 0
    ctx.close()
