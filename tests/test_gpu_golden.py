"""The CUDA step against the golden fixtures (tests/golden), without running
the oracle: FP64 bit for bit, by-products included; mixed precision within the
per-field norm-relative bounds of the mixed path (1e-4 density, energy, species
and primitives; 1e-3 momenta and velocities, which are O(noise))."""
import pytest
import torch

from fhdex_b200.context import Context
from tests.golden.make_golden import CASES, load_case, params_from_json
from tests.helpers import max_rel
from tests.test_golden import noise_from, state_from

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(CASES))
def test_cuda_step_reproduces_fixture_bitwise(name):
    meta, arrays = load_case(name)
    p = params_from_json(meta["params"])
    dt = float.fromhex(meta["dt"])
    st = state_from(p, arrays, "in").clone(device="cuda")
    ctx = Context(p)
    for step in range(meta["steps"]):
        last = step == meta["steps"] - 1
        ctx.rk3_step(st, dt, step, noise=noise_from(p, arrays, step).to("cuda"), aux=True)
        torch.cuda.synchronize()
        bad = [k for k, m in st.named(aux=last).items()
               if not torch.equal(m.arr.cpu(), torch.from_numpy(arrays[f"out{step}/{k}"]))]
        assert not bad, (step, bad)
    assert ctx.status() == 0


@pytest.mark.parametrize("name", list(CASES))
def test_mixed_step_within_bounds_of_fixture(name):
    meta, arrays = load_case(name)
    p = params_from_json(meta["params"]).replace(precision=1)
    dt = float.fromhex(meta["dt"])
    st = state_from(p, arrays, "in").clone(device="cuda")
    ctx = Context(p)
    for step in range(meta["steps"]):
        ctx.rk3_step(st, dt, step, noise=noise_from(p, arrays, step).to("cuda"), aux=False)
    torch.cuda.synchronize()
    assert ctx.status() == 0
    last = meta["steps"] - 1
    for k, m in st.named().items():
        ref = torch.from_numpy(arrays[f"out{last}/{k}"])
        for c in range(m.ncomp):
            e = max_rel(m.arr[c].cpu(), ref[c])
            loose = k.startswith(("vel", "cumom")) or (k in ("cu", "prim") and c in (1, 2, 3))
            assert e < (1e-3 if loose else 1e-4), (k, c, e)
