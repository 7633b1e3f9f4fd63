"""The fused stage kernel (k_stage_zm: stresses, face fluxes and the RK3 update of
one stage in a single z-marching launch, intermediates in shared memory) against
the CPU oracle, bit for bit in FP64, for every fused launch shape, on boxes that
cut the 16 x 8 tiles and the z-chunks unevenly, with in-kernel, injected and no
noise, and across the reference's options; the mixed path against the split
mixed pipeline (FMA contraction may differ between the two kernels' code, so
within 1e-5 of each field's norm)."""
import pytest
import torch

from fhdex_b200.context import Context
from fhdex_b200.params import argon, argon_single, isomerization, mixture4, no2_dimerization, stable_dt
from fhdex_b200.state import StagState, StepNoise
from tests.helpers import compare_named, max_rel, perturbed_state

pytestmark = pytest.mark.gpu


def fused_tiles():
    return [t for t, name in enumerate(Context.tiles()) if name.startswith("fused")]


CASES = {
    "argon_20x19x35": lambda: argon((20, 19, 35), dx=8e-6, seed=81),
    "mix4_10x12x8": lambda: mixture4((10, 12, 8), dx=8e-6, seed=82),
    "argon_adv0_grav": lambda: argon((17, 9, 18), dx=8e-6, advection_type=0, grav=(0.0, -300.0, -981.0), seed=83),
    "argon_adv1_visc3": lambda: argon((16, 8, 33), dx=8e-6, advection_type=1, visc_type=3, zeta_ratio=0.5, seed=84),
    "argon_nostoch": lambda: argon((9, 10, 11), dx=8e-6, stoch_stress_form=0, seed=85),
    "iso_no2": lambda: isomerization(no2_dimerization((9, 17, 10), dx=8e-6, seed=87)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_fused_stage_equals_oracle_bitwise(oracle, name):
    """Three steps with in-kernel noise through every fused launch shape: the state
    and the stage-3 coefficients and fluxes equal the oracle fed the materialised
    noise, bit for bit."""
    p = CASES[name]()
    st0 = perturbed_state(oracle, p, seed=88)
    dt = stable_dt(p)
    for t in fused_tiles():
        st = st0.clone()
        d = st0.clone(device="cuda")
        ctx = Context(p)
        ctx.set_tile(t)
        nz = StepNoise(p, "cuda")
        for s in range(3):
            ctx.fill_step_noise(nz, s)
            ctx.rk3_step(d, dt, s, noise=None, aux=(s == 2))
            nzc = nz.to("cpu")
            torch.cuda.synchronize()
            assert oracle.rk3_step(st, nzc, dt) == 0
        assert ctx.status() == 0
        bad, _ = compare_named(d.named(aux=True), st.named(aux=True))
        assert not bad, (Context.tiles()[t], bad[:6])
        ctx.close()


def test_fused_injected_noise_and_large_box_bitwise(oracle):
    """Injected A/B noise through the fused kernel, on a box with several tiles
    and z-chunks in every direction (100 x 96 x 90)."""
    p = argon((100, 96, 90), dx=8e-6, seed=89)
    st = perturbed_state(oracle, p, seed=90)
    d = st.clone(device="cuda")
    ctx = Context(p)
    ctx.set_tile(fused_tiles()[0])
    dt = stable_dt(p)
    nz = StepNoise(p)
    oracle.fill_noise_mt64(nz, 91)
    ctx.rk3_step(d, dt, 0, noise=nz.to("cuda"), aux=True)
    torch.cuda.synchronize()
    assert ctx.status() == 0
    assert oracle.rk3_step(st, nz, dt) == 0
    bad, _ = compare_named(d.named(aux=True), st.named(aux=True))
    assert not bad, bad[:6]


@pytest.mark.parametrize("name", ["argon_20x19x35", "mix4_10x12x8", "argon_single"])
def test_fused_mixed_and_single_gas_match_the_split_pipeline(oracle, name):
    """The mixed path (and the one-species fast path) through the fused kernel
    against the split kernels with the same in-kernel noise: FP64 runs bit for
    bit, mixed runs within 1e-5 of each field's norm after 3 steps."""
    base = argon_single((12, 11, 10), dx=8e-6, seed=86) if name == "argon_single" else CASES[name]()
    for prec in (0, 1):
        p = base.replace(precision=prec)
        if p.nspecies == 1:
            st0 = StagState(p, "cuda", aux=False)
            ctx0 = Context(p)
            ctx0.init_state(st0)
            g = torch.Generator(device="cuda").manual_seed(3)
            for m in st0.cumom:
                m.arr.add_(1e-3 * p.rho0 * p.sound_speed() * torch.randn(m.arr.shape, generator=g, device="cuda",
                                                                         dtype=torch.float64))
                ctx0.override_sync(m)
                ctx0.fill_boundary(m)
        else:
            st0 = perturbed_state(oracle, p.replace(precision=0), seed=92).clone(device="cuda")
            st0.p = p
        dt = stable_dt(p)
        outs = []
        for t in (0, fused_tiles()[1]):
            d = st0.clone(device="cuda")
            ctx = Context(p)
            ctx.set_tile(t)
            for s in range(3):
                ctx.rk3_step(d, dt, s, aux=False)
            torch.cuda.synchronize()
            assert ctx.status() == 0
            outs.append(d)
        if prec == 0:
            bad, _ = compare_named(outs[1].named(), outs[0].named())
            assert not bad, (prec, bad[:6])
        else:
            for k, m in outs[0].named().items():
                e = max_rel(outs[1].named()[k].arr, m.arr)
                assert e < 1e-5, (k, e)


def test_fused_graph_replay_equals_single_steps(oracle):
    p = argon((24, 20, 18), dx=8e-6, seed=93)
    st = perturbed_state(oracle, p, seed=94)
    a = st.clone(device="cuda")
    b = st.clone(device="cuda")
    ctx = Context(p)
    ctx.set_tile(fused_tiles()[0])
    dt = stable_dt(p)
    for s in range(5):
        ctx.rk3_step(a, dt, s, aux=False)
    ctx.rk3_steps(b, dt, 0, 5)
    torch.cuda.synchronize()
    bad, _ = compare_named(b.named(), a.named())
    assert not bad, bad[:4]
    assert ctx.status() == 0
