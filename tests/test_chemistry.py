"""Chemistry source of the compressible step in the CPU oracle
(compute_compressible_chemistry_source_CLE, chemistry_functions.cpp:128-193).

The oracle is checked against (1) a line-by-line Python transcription evaluated
with the same C library (math.exp / math.pow): bitwise; (2) exact mass
conservation of every reaction; (3) the known answer of the reference's NO2
dimerization deck, whose initial state is at chemical equilibrium: forward and
backward rates agree to the deck's six significant digits, so the deterministic
source vanishes to that precision; (4) the linearity of the Langevin term in the
noise.  Inputs-deck parsing of the chemistry keys is checked against the keys the
reference reads (chemistry_functions.cpp:45-124).
"""
import math

import pytest
import torch

from fhdex_b200.fab import CELL, MultiFab
from fhdex_b200.params import exchange_network, isomerization, mixture4, no2_dimerization, parse_inputs
from tests.helpers import perturbed_state


def py_source(p, prim, W, dt, dV):
    """chemistry_functions.cpp:147-190 transcribed, per valid cell."""
    ns, nr = p.nspecies, p.nreaction
    pv = prim.valid().reshape(prim.ncomp, -1)
    Wv = W.valid().reshape(W.ncomp, -1) if W is not None else None
    navo = p.avogadro if p.avogadro > 0 else p.Runiv / p.k_B
    out = torch.zeros(ns, pv.shape[1], dtype=torch.float64)
    for c in range(pv.shape[1]):
        pres, T = pv[5, c].item(), pv[4, c].item()
        T0 = p.T0_chem
        ctot = pres / p.Runiv / T
        ck = [pv[6 + ns + n, c].item() * ctot for n in range(ns)]
        a = []
        for m in range(nr):
            r = p.rate_const[m]
            r *= math.exp(-p.alpha_param[m] / p.Runiv * (1 / T - 1 / T0))
            r *= math.pow(T / T0, p.beta_param[m])
            for n in range(ns):
                r *= math.pow(ck[n], p.stoich_R[m][n])
            a.append(r)
        S = [0.0] * ns
        for m in range(nr):
            a[m] = max(0.0, a[m])
            w = (Wv[m, c].item() if p.reaction_type == 1 else 0.0) / math.sqrt(dt * dV)
            for n in range(ns):
                pr = p.stoich_P[m][n] - p.stoich_R[m][n]
                S[n] += p.molmass[n] * pr * a[m]
                if p.reaction_type == 1:
                    S[n] += p.molmass[n] * pr * math.sqrt(a[m] / navo) * w
        for n in range(ns):
            out[n, c] = S[n]
    return out


def chem_inputs(oracle, p, seed):
    st = perturbed_state(oracle, p, seed=seed)
    W = MultiFab(p.n_cells, CELL, p.nreaction, 0)
    g = torch.Generator().manual_seed(seed + 100)
    W.valid().copy_(torch.randn(W.valid().shape, generator=g, dtype=torch.float64))
    src = MultiFab(p.n_cells, CELL, p.nprimvars, 0)
    return st, W, src


def cell_volume(p):
    dx = p.dx
    return dx[0] * dx[1] * dx[2]


@pytest.mark.parametrize("make", [lambda: no2_dimerization((5, 4, 3)),
                                  lambda: isomerization(no2_dimerization((4, 3, 5))),
                                  lambda: no2_dimerization((3, 4, 4), reaction_type=0),
                                  lambda: exchange_network(mixture4((4, 3, 3), dx=8e-6))])
def test_oracle_matches_python_transcription_bitwise(oracle, make):
    p = make()
    st, W, src = chem_inputs(oracle, p, seed=3)
    dt, dV = 1e-12, cell_volume(p)
    assert oracle.chemistry_source_cle(p, dt, dV, st.prim, src, W) == 0
    ref = py_source(p, st.prim, W, dt, dV)
    got = src.valid()[5:5 + p.nspecies].reshape(p.nspecies, -1)
    assert torch.equal(got, ref)
    # components other than the species are left as they were (zero here)
    assert torch.count_nonzero(src.valid()[:5]) == 0


def test_every_reaction_conserves_mass(oracle):
    """sum_n M_n (P_mn - R_mn) = 0 for 2 NO2 <-> N2O4, so the species sources sum to
    zero up to rounding of the individual terms."""
    p = no2_dimerization((4, 4, 4))
    st, W, src = chem_inputs(oracle, p, seed=5)
    assert oracle.chemistry_source_cle(p, 1e-12, cell_volume(p), st.prim, src, W) == 0
    S = src.valid()[5:7]
    total = S.sum(0).abs()
    scale = S.abs().sum(0)
    assert (total <= 1e-14 * scale).all()


def test_no2_deck_initial_state_is_at_chemical_equilibrium(oracle):
    """The deck's uniform state (rho0, T_init = T0_chem, rhobar): 2 NO2 -> N2O4 and
    N2O4 -> 2 NO2 run at the same rate to ~1.6e-6 (the deck's constants carry six
    digits), so the deterministic source is ~1e-6 of either reaction's mass rate."""
    p = no2_dimerization((2, 2, 2), reaction_type=0)
    st, _, src = chem_inputs(oracle, p, seed=0)
    oracle.init_state(st, p)
    assert oracle.conserved_to_primitive(st) == 0
    assert oracle.chemistry_source_cle(p, 1e-12, cell_volume(p), st.prim, src, None) == 0
    prim = st.prim.valid()
    ctot = prim[5] / p.Runiv / prim[4]
    a1 = p.rate_const[0] * (prim[6 + 2] * ctot) ** 2
    S = src.valid()[5:7]
    assert float(a1.min()) > 300.0
    rel = (S[0].abs() / (2 * p.molmass[0] * a1)).max().item()
    assert rel < 5e-6, rel


def test_langevin_term_is_linear_in_the_noise(oracle):
    """S(W) - S(0) = sum_m M_n nu_mn sqrt(a_m / N_A) W_m / sqrt(dt dV): doubling W
    doubles the fluctuation (up to rounding)."""
    p = no2_dimerization((4, 3, 3))
    st, W, src = chem_inputs(oracle, p, seed=9)
    dt, dV = 2e-12, cell_volume(p)
    src0 = MultiFab(p.n_cells, CELL, p.nprimvars, 0)
    src2 = MultiFab(p.n_cells, CELL, p.nprimvars, 0)
    Z = MultiFab(p.n_cells, CELL, p.nreaction, 0)
    W2 = MultiFab(p.n_cells, CELL, p.nreaction, 0)
    W2.valid().copy_(2.0 * W.valid())
    for s, w in ((src, W), (src0, Z), (src2, W2)):
        assert oracle.chemistry_source_cle(p, dt, dV, st.prim, s, w) == 0
    f1 = src.valid()[5:7] - src0.valid()[5:7]
    f2 = src2.valid()[5:7] - src0.valid()[5:7]
    assert f1.abs().max() > 0
    assert torch.allclose(f2, 2 * f1, rtol=1e-9, atol=1e-12 * src0.valid()[5:7].abs().max().item())


def test_parse_inputs_reads_the_chemistry_keys():
    deck = """
      nspecies = 2
      n_cells = 16 16 16
      prob_hi = 1.6e-4 1.6e-4 1.6e-4
      molmass = 46.0055 92.0110
      nreaction = 2
      T0_chem = 350
      rate_const = 4.065753e+11 6.236899e+07
      alpha_param = -5.337990e+10 5.370000e+11
      beta_param  = 0.644950 -1.100000
      stoich_1R = 2 0
      stoich_1P = 0 1
      stoich_2R = 0 1
      stoich_2P = 2 0
      reaction_type = 1
    """
    p = parse_inputs(deck)
    assert p.nreaction == 2 and p.reaction_type == 1
    assert p.stoich_R == ((2, 0), (0, 1)) and p.stoich_P == ((0, 1), (2, 0))
    assert p.rate_const == (4.065753e+11, 6.236899e+07)
    assert p.beta_param == (0.644950, -1.100000) and p.T0_chem == 350.0
    c = p.to_c()
    assert c.nreaction == 2 and c.stoich_R[0][0] == 2 and c.stoich_P[1][0] == 2
    # avogadro given: Runiv = k_B * avogadro (common_functions.cpp:776-777)
    q = parse_inputs(deck + "\navogadro = 6.0e23\n")
    assert q.avogadro == 6.0e23 and q.Runiv == q.k_B * 6.0e23
