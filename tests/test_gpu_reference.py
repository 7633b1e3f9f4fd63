"""The CUDA path against the reference's own code (oracle/_ref: FHDeX's hot-path
sources compiled unmodified against the host-only AMReX stand-in), with no
restatement in between: InitConsVarStag + conservedToPrimitiveStag, and whole
RK3stepStag steps with the same injected noise, bit for bit (tolerance 0) on the
whole storage of the state and the stage-3 coefficients and fluxes."""
import pytest
import torch

from fhdex_b200.context import Context
from fhdex_b200.params import argon, isomerization, mixture4, no2_dimerization, stable_dt
from fhdex_b200.state import StagState, StepNoise
from tests.helpers import compare_named, perturbed_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R
    if not R.available():
        pytest.skip("oracle/_ref was not built")
    return R


CASES = {
    "argon12": lambda: argon(12, dx=8e-6, seed=71),
    "mix4_10x12x8_visc3": lambda: mixture4((10, 12, 8), dx=8e-6, visc_type=3, zeta_ratio=0.7, seed=72),
    "argon_adv0_grav": lambda: argon((9, 8, 7), dx=8e-6, advection_type=0, grav=(0.0, 0.0, -981.0), seed=73),
    "iso_no2": lambda: isomerization(no2_dimerization((6, 5, 7), dx=8e-6, seed=74)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_init_and_conversion_equal_the_reference(ref, name):
    """fhd_init_cons_var_stag + fhd_conserved_to_primitive_stag + FillBoundary (the
    main_driver init) on the GPU against the reference's InitConsVarStag +
    conservedToPrimitiveStag + FillBoundary."""
    p = CASES[name]()
    g = StagState(p, "cuda", aux=False)
    Context(p).init_state(g)
    h = StagState(p)
    ref.init_cons_var_stag(h)
    ref.conserved_to_primitive(h)
    from oracle import oracle as O
    for m in [h.cu, h.prim] + h.cumom + h.vel:
        O.fill_boundary(m)
    torch.cuda.synchronize()
    bad, _ = compare_named(g.named(), h.named())
    assert not bad, bad[:6]


@pytest.mark.parametrize("name", list(CASES))
def test_rk3_steps_equal_the_reference(oracle, ref, name):
    p = CASES[name]()
    st = perturbed_state(oracle, p, seed=75)
    d = st.clone(device="cuda")
    ctx = Context(p)
    dt = stable_dt(p)
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
