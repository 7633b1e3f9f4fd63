"""Generates the golden fixtures of the injected-noise RK3 step (run from the
repository root: ``python -m tests.golden.make_golden [case ...]``).

The reference holds no stored outputs for this path (its regression decks have
no golden files), so the fixtures freeze the CPU oracle's results on small
boxes, with noise drawn on the host from
std::mt19937_64 and Box-Muller (``oracle.fill_noise_mt64``):

  * ``<case>.npz``: parameters and dt (``meta``, JSON), the input state
    (``in/<field>``, ghost-inclusive arrays), the A/B noise of each step
    (``noise<step>/<f|e|c><s><d>``) and the state after each step
    (``out<step>/<field>``; the last step also carries the transport
    coefficients and fluxes the step writes as by-products);
  * ``MANIFEST.json``: SHA-256 of every array, so a changed fixture or a
    drifted oracle is caught.

The reference's own hot-path sources, compiled unmodified into oracle/_ref,
reproduce every fixture bit for bit (tests/test_reference_pin.py); the oracle
is also checked against the reference's known answers (closed-form GIO
coefficients, equilibrium variances, conservation) in tests/test_oracle.py.  The
fixtures let the GPU tests check the CUDA path without running the oracle and
guard the oracle against silent drift.
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import os

import numpy as np

import sys

from fhdex_b200.params import Params, argon, isomerization, mixture4, no2_dimerization, stable_dt
from fhdex_b200.state import StepNoise

HERE = os.path.dirname(os.path.abspath(__file__))
STEPS = 2

# name -> (params, state seed, noise seed)
CASES = {
    "argon_4x4x4": (lambda: argon(4, dx=8e-6), 11, 1),
    "mix4_5x4x3_visc3_adv1": (lambda: mixture4((5, 4, 3), dx=8e-6, visc_type=3, zeta_ratio=0.7,
                                                advection_type=1), 12, 2),
    "argon_6x4x5_adv0_grav": (lambda: argon((6, 4, 5), dx=8e-6, advection_type=0,
                                            grav=(0.0, 0.0, -981.0)), 13, 3),
    # NO2 / N2O4 gas with a first-order CLE reaction pair: the chemistry source inside
    # every stage, its reaction noises stored with the rest (h<s>)
    "iso_no2_5x4x4_chem": (lambda: isomerization(no2_dimerization((5, 4, 4), dx=8e-6)), 14, 4),
}


def noise_arrays(nz: StepNoise):
    out = {}
    for s in range(2):
        for d in range(3):
            out[f"f{s}{d}"] = nz.face[s][d].arr
            out[f"e{s}{d}"] = nz.edge[s][d].arr
            out[f"c{s}{d}"] = nz.cen[s][d].arr
        if nz.chem[s] is not None:
            out[f"h{s}"] = nz.chem[s].arr
    return out


def params_from_json(d: dict) -> Params:
    def tup(v):
        return tuple(tup(x) for x in v) if isinstance(v, list) else v
    return Params(**{k: tup(v) for k, v in d.items()})


def make_case(O, name):
    from tests.helpers import perturbed_state
    make, sseed, nseed = CASES[name]
    p = make()
    st = perturbed_state(O, p, seed=sseed)
    dt = stable_dt(p)
    arrays = {f"in/{k}": m.arr.numpy().copy() for k, m in st.named().items()}
    seeds = [nseed * 1000 + s for s in range(STEPS)]
    for step in range(STEPS):
        nz = StepNoise(p)
        O.fill_noise_mt64(nz, seed=seeds[step])
        for k, a in noise_arrays(nz).items():
            arrays[f"noise{step}/{k}"] = a.numpy().copy()
        assert O.rk3_step(st, nz, dt) == 0
        for k, m in st.named(aux=step == STEPS - 1).items():
            arrays[f"out{step}/{k}"] = m.arr.numpy().copy()
    meta = {"params": dataclasses.asdict(p), "dt": dt.hex(), "steps": STEPS, "state_seed": sseed,
            "noise_seeds": seeds}
    return meta, arrays


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def load_case(name):
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    meta = json.loads(str(z["meta"]))
    return meta, {k: z[k] for k in z.files if k != "meta"}


def load_manifest():
    with open(os.path.join(HERE, "MANIFEST.json")) as f:
        return json.load(f)


def main(names=None):
    """Writes the fixtures of `names` (all cases when None) and their manifest
    entries, keeping the other cases' entries."""
    from oracle import oracle as O
    O.build()
    manifest = load_manifest() if os.path.exists(os.path.join(HERE, "MANIFEST.json")) else {}
    for name in names or CASES:
        meta, arrays = make_case(O, name)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=np.array(json.dumps(meta)), **arrays)
        manifest[name] = {k: sha(a) for k, a in sorted(arrays.items())}
        print(name, sum(a.nbytes for a in arrays.values()), "bytes")
    with open(os.path.join(HERE, "MANIFEST.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
