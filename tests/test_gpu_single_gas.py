"""The single-gas fast path (nspecies = 1, no species flux) against the
reference's parity form of a single gas (two identical species, which is bit
for bit the CPU oracle's trajectory): with the same seed the energy and
momentum noise are the same Philox numbers, and the parity form's species
terms cancel to rounding for identical species, so density, momenta, energy,
temperature and pressure agree within a measured norm-relative bound after 10
steps.  The single gas's rhoY stays bitwise equal to rho."""
import pytest
import torch

from fhdex_b200.context import Context
from fhdex_b200.params import argon, argon_single, stable_dt
from fhdex_b200.state import StagState
from tests.helpers import max_rel, perturbed_state

pytestmark = pytest.mark.gpu

# measured on B200 after 10 steps (norm-relative, worst field): FP64 2.3e-9 on the
# momenta (1e-10 to 4e-10 on rho, rhoE, T, p), mixed 5.2e-5; bounds with margin.  The
# parity form's Soret/Dufour terms do not cancel exactly for identical species.
TOL = {0: 1e-8, 1: 2e-4}


@pytest.mark.parametrize("precision", [0, 1])
def test_single_gas_matches_two_identical_species(oracle, precision):
    p2 = argon(16, dx=8e-6, seed=11, precision=precision)
    p1 = argon_single(16, dx=8e-6, seed=11, precision=precision)
    st2h = perturbed_state(oracle, p2.replace(precision=0), seed=5)
    st1h = StagState(p1)
    st1h.cu.arr[:5].copy_(st2h.cu.arr[:5])
    st1h.cu.arr[5].copy_(st2h.cu.arr[0])            # rhoY = rho
    for d in range(3):
        st1h.cumom[d].arr.copy_(st2h.cumom[d].arr)
    st2 = st2h.clone(device="cuda")
    st1 = st1h.clone(device="cuda")
    dt = stable_dt(p2)
    assert dt == stable_dt(p1)
    c1, c2 = Context(p1), Context(p2)
    for s in range(10):
        c1.rk3_step(st1, dt, s, aux=False)
        c2.rk3_step(st2, dt, s, aux=False)
    torch.cuda.synchronize()
    assert c1.status() == 0 and c2.status() == 0
    assert torch.equal(st1.cu.arr[5], st1.cu.arr[0])
    errs = {"rho": max_rel(st1.cu.valid(0), st2.cu.valid(0)), "rhoE": max_rel(st1.cu.valid(4), st2.cu.valid(4)),
            "T": max_rel(st1.prim.valid(4), st2.prim.valid(4)), "p": max_rel(st1.prim.valid(5), st2.prim.valid(5))}
    for d in range(3):
        errs[f"mom{d}"] = max_rel(st1.cumom[d].valid(0), st2.cumom[d].valid(0))
    print(precision, {k: f"{v:.2e}" for k, v in errs.items()})
    assert max(errs.values()) < TOL[precision], errs
    # the fields moved (the comparison is not of two initial states)
    assert not torch.equal(st1.cu.arr[0].cpu(), st1h.cu.arr[0])
