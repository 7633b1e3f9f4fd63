"""bench.py's host-side pieces that every bench line goes through, checked on the
CPU: the workload description of each gas and species form, and the parameters
each command line selects."""
import importlib.util
import os

import pytest

from fhdex_b200.params import argon, argon_single, mixture4, no2_dimerization

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class Args:
    precision = "fp64"
    gpus = 1
    n = 8
    dx = 8e-6
    seed = 1
    gas = "argon"
    ns = 2


@pytest.mark.parametrize("p,word", [(argon(8), "argon (2 identical species)"), (argon_single(8), "single gas"),
                                    (mixture4(8), "4-species mixture"), (no2_dimerization(8), "NO2")])
def test_workload_description(p, word):
    b = load_bench()
    cfg = b.config_dict(Args, p, 1e-12, "b128-min8")
    assert word in cfg["workload"] and "8^3" in cfg["workload"]
    assert cfg["n_cells"] == [8, 8, 8] and cfg["nspecies"] == p.nspecies


@pytest.mark.parametrize("gas,ns,nreaction", [("argon", 1, 0), ("argon", 2, 0), ("argon", 4, 0), ("no2", 2, 2)])
def test_make_params(gas, ns, nreaction):
    b = load_bench()

    class A(Args):
        pass
    A.gas, A.ns = gas, ns
    p = b.make_params(A)
    assert p.nspecies == ns and p.nreaction == nreaction and p.n_cells == (8, 8, 8)
