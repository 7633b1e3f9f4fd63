"""The restated oracle pinned to the reference's own code.

``oracle/_ref/libfhd_ref.so`` is FHDeX's hot-path sources compiled unmodified
(timeStepStag.cpp, fluxStag.cpp, conservedPrimitiveConversionsStag.cpp,
transCoeffs.cpp, compressible_functions*.cpp, boundaryStag.cpp,
MultiFabFillRandom.cpp, chemistry_functions.cpp, common_functions.cpp, ...)
against a host-only AMReX stand-in (``oracle/amrex_host``).  Fed the same
states and the same injected noise, it and ``oracle/fhd_oracle.cpp`` must agree
bit for bit (tolerance 0) on every operator and on whole RK3 steps, state and
by-products; the golden fixtures must be what the reference computes; and the
reference's parameter initialisers must derive what the host layer derives.
Since the GPU tests hold the CUDA path bitwise to the oracle, this chain pins
the CUDA path to the reference.  What stays unpinned is the AMReX layer itself
(FillBoundary / OverrideSync / LinComb semantics, restated in the stand-in) and
the random generator (the noise is injected on both sides)."""
import math

import pytest
import torch

from fhdex_b200.params import argon, exchange_network, isomerization, mixture4, no2_dimerization, stable_dt
from fhdex_b200.state import StepNoise
from tests.golden.make_golden import CASES, load_case, params_from_json
from tests.helpers import compare_named, perturbed_state


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R
    if not R.available():
        R.build()
    if not R.available():
        pytest.skip("oracle/_ref was not built (the reference tree is absent and no prebuilt library travelled)")
    return R


GASES = {
    "argon12": lambda: argon(12, dx=8e-6),
    "mix4_10x12x8": lambda: mixture4((10, 12, 8), dx=8e-6),
    "mix4_visc3": lambda: mixture4((6, 5, 7), dx=8e-6, visc_type=3, zeta_ratio=0.7),
    "argon_visc1_adv0": lambda: argon((7, 6, 5), dx=8e-6, visc_type=1, advection_type=0),
    "argon_adv1_grav": lambda: argon((6, 7, 5), dx=8e-6, advection_type=1, grav=(0.0, -500.0, -981.0)),
    "argon_nostoch": lambda: argon(6, dx=8e-6, stoch_stress_form=0),
    "no2": lambda: no2_dimerization((5, 6, 4), dx=8e-6),
    "iso_no2": lambda: isomerization(no2_dimerization((5, 4, 6), dx=8e-6)),
    "exchange_mix4": lambda: exchange_network(mixture4((5, 6, 4), dx=8e-6)),
}


def test_reference_parameter_initialisers_match_the_host_layer(ref):
    """InitializeCommonNamespace / GetHcGas read the deck that Params writes and
    derive the same counts and heat capacities (compressible_functions.cpp:91-100)."""
    for make in GASES.values():
        p = make()
        ns, nv, npv, ng, hcv, hcp, nr = ref.globals_(p)
        assert (ns, nv, npv, ng, nr) == (p.nspecies, p.nvars, p.nprimvars, p.ngc, p.nreaction)
        hv, hp = p.hc()
        assert hcv == hv[:ns] and hcp == hp[:ns]


@pytest.mark.parametrize("name", list(GASES))
def test_reference_init_conversion_transport_bitwise(oracle, ref, name):
    p = GASES[name]()
    a = perturbed_state(oracle, p, seed=31)
    b = a.clone()
    assert oracle.conserved_to_primitive(a) == 0
    ref.conserved_to_primitive(b)
    bad, _ = compare_named(b.named(), a.named())
    assert not bad, bad[:6]
    assert oracle.transport_coeffs(a) == 0
    ref.transport(b)
    names = ("eta", "zeta", "kappa", "chi", "D")
    bad, _ = compare_named(b.named(aux=True), {k: v for k, v in a.named(aux=True).items() if k in names})
    assert not bad, bad[:6]
    # InitConsVarStag (prob_type 1) and the acoustic CFL diagnostic
    c = a.clone()
    d = a.clone()
    oracle.init_cons_var_stag(c, p)
    ref.init_cons_var_stag(d)
    assert torch.equal(c.cu.valid(), d.cu.valid())
    for q in range(3):
        assert torch.equal(c.cumom[q].valid(), d.cumom[q].valid())
    dt = stable_dt(p)
    assert oracle.max_acoustic_cfl(a, dt) == ref.max_acoustic_cfl(a, dt)


@pytest.mark.parametrize("name", ["argon12", "mix4_10x12x8", "mix4_visc3", "argon_visc1_adv0"])
def test_reference_flux_operator_bitwise(oracle, ref, name):
    p = GASES[name]()
    st = perturbed_state(oracle, p, seed=32)
    assert oracle.transport_coeffs(st) == 0
    nz = StepNoise(p)
    oracle.fill_noise_mt64(nz, 77)
    dt = stable_dt(p)
    a = st.clone()
    b = st.clone()
    assert oracle.flux_stag(a, nz.face[0], nz.edge[0], nz.cen[0], dt) == 0
    ref.flux(b, nz.face[0], nz.edge[0], nz.cen[0], dt)
    fluxes = [f"faceflux{q}" for q in range(3)] + [f"edgeflux{e}" for e in range(6)] + [f"cenflux{q}" for q in range(3)]
    ra = a.named(aux=True)
    bad, _ = compare_named(b.named(aux=True), {k: ra[k] for k in fluxes})
    assert not bad, bad[:6]


@pytest.mark.parametrize("name", list(GASES))
def test_reference_rk3_steps_bitwise(oracle, ref, name):
    """Three RK3stepStag calls with the same injected A/B noise (and reaction
    noise): the whole storage of the state and the stage-3 coefficients and
    fluxes after every step, bit for bit.  The reference's noise fills request
    mean 0 and variance 1 (faces, edges) or 2 (centres), as the oracle assumes."""
    p = GASES[name]()
    a = perturbed_state(oracle, p, seed=33)
    b = a.clone()
    dt = stable_dt(p)
    for s in range(3):
        nz = StepNoise(p)
        oracle.fill_noise_mt64(nz, 100 + s)
        assert oracle.rk3_step(a, nz, dt) == 0
        log = ref.rk3_step(b, nz, dt, s)
        bad, _ = compare_named(b.named(aux=True), a.named(aux=True))
        assert not bad, (s, bad[:6])
    assert len(log) == 24
    for q, rec in enumerate(log):
        assert rec["mean"] == 0.0
        assert rec["stddev"] == (math.sqrt(2.0) if q >= 18 else 1.0), q
        assert rec["ncomp"] == (p.nspecies + 1 if q < 6 else 1)
        assert rec["scomp"] == (4 if q < 6 else 0)


@pytest.mark.parametrize("name", list(CASES))
def test_reference_reproduces_golden_fixtures(ref, name):
    """The stored fixtures are the reference's results, not only the oracle's."""
    from tests.test_golden import noise_from, state_from
    meta, arrays = load_case(name)
    p = params_from_json(meta["params"])
    dt = float.fromhex(meta["dt"])
    st = state_from(p, arrays, "in")
    for step in range(meta["steps"]):
        ref.rk3_step(st, noise_from(p, arrays, step), dt, step)
        last = step == meta["steps"] - 1
        bad = [k for k, m in st.named(aux=last).items()
               if not torch.equal(m.arr, torch.from_numpy(arrays[f"out{step}/{k}"]))]
        assert not bad, (step, bad)


@pytest.mark.parametrize("name", ["no2", "exchange_mix4"])
def test_reference_chemistry_source_bitwise(oracle, ref, name):
    """compute_compressible_chemistry_source_CLE on a perturbed state with given
    reaction noise."""
    p = GASES[name]()
    st = perturbed_state(oracle, p, seed=34)
    from fhdex_b200.fab import CELL, MultiFab
    ranchem = MultiFab(p.n_cells, CELL, p.nreaction, p.ngc)
    g = torch.Generator().manual_seed(5)
    ranchem.arr.copy_(torch.randn(ranchem.arr.shape, generator=g, dtype=torch.float64))
    dt = stable_dt(p)
    dV = p.dx[0] * p.dx[1] * p.dx[2]
    sa = MultiFab(p.n_cells, CELL, p.nprimvars, p.ngc)
    sb = MultiFab(p.n_cells, CELL, p.nprimvars, p.ngc)
    assert oracle.chemistry_source_cle(p, dt, dV, st.prim, sa, ranchem) == 0
    ref.chemistry_source(p, dt, dV, st.prim, sb, ranchem)
    assert torch.equal(sa.valid(), sb.valid())
