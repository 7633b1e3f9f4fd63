"""Golden fixtures of the injected-noise RK3 step (tests/golden): the files
match their manifest, the host noise generator reproduces the stored noise
(with the OverrideSync invariant), and the oracle reproduces the stored states
bit for bit."""
import pytest
import torch

from fhdex_b200.state import StagState, StepNoise
from tests.golden.make_golden import CASES, load_case, load_manifest, noise_arrays, params_from_json, sha


def state_from(p, arrays, prefix, aux=False):
    st = StagState(p)
    for k, m in st.named(aux=aux).items():
        m.arr.copy_(torch.from_numpy(arrays[f"{prefix}/{k}"]))
    return st


def noise_from(p, arrays, step):
    nz = StepNoise(p)
    for k, a in noise_arrays(nz).items():
        a.copy_(torch.from_numpy(arrays[f"noise{step}/{k}"]))
    return nz


@pytest.mark.parametrize("name", list(CASES))
def test_fixture_matches_manifest(name):
    _, arrays = load_case(name)
    man = load_manifest()[name]
    assert sorted(man) == sorted(arrays)
    bad = [k for k, a in arrays.items() if sha(a) != man[k]]
    assert not bad, bad


@pytest.mark.parametrize("name", list(CASES))
def test_host_noise_generator_reproduces_fixture(oracle, name):
    meta, arrays = load_case(name)
    p = params_from_json(meta["params"])
    for step, seed in enumerate(meta["noise_seeds"]):
        nz = StepNoise(p)
        oracle.fill_noise_mt64(nz, seed=seed)
        for k, a in noise_arrays(nz).items():
            assert torch.equal(a, torch.from_numpy(arrays[f"noise{step}/{k}"])), (step, k)
        # OverrideSync invariant: the periodic duplicate face n_cells equals face 0
        for d in range(3):
            f = nz.face[0][d].valid()
            assert torch.equal(f.select(3 - d, 0), f.select(3 - d, p.n_cells[d]))


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_reproduces_fixture_bitwise(oracle, name):
    meta, arrays = load_case(name)
    p = params_from_json(meta["params"])
    dt = float.fromhex(meta["dt"])
    st = state_from(p, arrays, "in")
    for step in range(meta["steps"]):
        assert oracle.rk3_step(st, noise_from(p, arrays, step), dt) == 0
        last = step == meta["steps"] - 1
        bad = [k for k, m in st.named(aux=last).items()
               if not torch.equal(m.arr, torch.from_numpy(arrays[f"out{step}/{k}"]))]
        assert not bad, (step, bad)
