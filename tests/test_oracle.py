"""CPU tests of the oracle against the reference's known-answer formulas.

No golden vectors exist in the reference (it has no test suite; CI only builds),
so the oracle is pinned by: the closed-form hard-sphere transport the
Giovangigli formulas reduce to for one gas, exact discrete conservation under
periodic boundaries, the equilibrium fluctuation variances of the reference's
own analysis scripts, and AMReX FillBoundary/OverrideSync semantics.
"""
import math

import pytest
import torch

from fhdex_b200.params import argon, hard_sphere_single_gas, mixture4, parse_inputs, stable_dt
from fhdex_b200.state import StagState, StepNoise
from tests.helpers import perturbed_state, seeded_noise
from fhdex_b200.equilibrium import equilibrium_variances


def test_gio_reduces_to_closed_form_hard_sphere(oracle):
    """compressible_functions.H:1218-1326 for two identical species must give the
    pure-gas Chapman-Enskog values eta = 5/(16 d^2) sqrt(m k T / pi),
    kappa = 75/64 k/d^2 sqrt(kT/(pi m))."""
    for T in (150.0, 273.0, 500.0):
        p = argon(8, T_init=T)
        st = StagState(p)
        oracle.init_state(st, p)
        assert oracle.transport_coeffs(st) == 0
        eta, kappa = hard_sphere_single_gas(p, T)
        assert st.eta[3, 4, 5].item() == pytest.approx(eta, rel=1e-13)
        assert st.kappa[3, 4, 5].item() == pytest.approx(kappa, rel=1e-13)
        assert st.zeta[3, 4, 5].item() == 0.0
        # identical species: no thermal diffusion
        assert abs(st.chi[3, 4, 5, 0].item()) < 1e-12


def test_gethcgas_and_eos_roundtrip(oracle):
    p = mixture4(8)
    oracle.set_params(p)
    hcv, hcp = oracle.hc()
    for i in range(4):
        assert hcv[i] == 0.5 * 3.0 * p.Runiv / p.molmass[i]
        assert hcp[i] == 0.5 * 5.0 * p.Runiv / p.molmass[i]
    st = StagState(p)
    oracle.init_state(st, p)
    # uniform state: T and p recovered exactly up to round-off
    T = st.prim.valid(4)
    assert torch.allclose(T, torch.full_like(T, p.T_init), rtol=1e-14, atol=0)
    molmix = 1.0 / sum(p.rhobar[k] / p.molmass[k] for k in range(4))
    pres = p.rho0 * p.Runiv / molmix * p.T_init
    assert torch.allclose(st.prim.valid(5), torch.full_like(T, pres), rtol=1e-13, atol=0)
    for k in range(4):
        X = p.rhobar[k] * molmix / p.molmass[k]
        assert torch.allclose(st.prim.valid(6 + 4 + k), torch.full_like(T, X), rtol=1e-14, atol=0)


@pytest.mark.parametrize("factory,ns", [(argon, 2), (mixture4, 4)])
def test_conservation_roundoff(oracle, factory, ns):
    """Flux form + periodic boundaries: total mass, species mass, momentum and
    energy change only by round-off."""
    p = factory(8, dx=8e-6)
    st = perturbed_state(oracle, p, seed=3)
    dt = stable_dt(p)
    N = p.n_cells[0]

    def totals():
        t = [st.cu.valid(n).sum().item() for n in [0, 4] + [5 + k for k in range(ns)]]
        t += [m.arr[0, 2:2 + N, 2:2 + N, 2:2 + N].sum().item() for m in st.cumom]
        return t

    t0 = totals()
    for s in range(4):
        nz = seeded_noise(oracle, p, 11, s)
        assert oracle.rk3_step(st, nz, dt) == 0
    t1 = totals()
    scale = [abs(x) for x in t0[:2 + ns]] + [p.rho0 * p.sound_speed() * N ** 3] * 3
    for a, b, s in zip(t0, t1, scale):
        assert abs(a - b) <= 1e-13 * s


def test_fill_boundary_and_override_sync_semantics(oracle):
    p = argon(6)
    oracle.set_params(p)
    from fhdex_b200.fab import MultiFab, NODAL_X, NODAL_XY, CELL
    g = torch.Generator().manual_seed(0)
    for nodal in (CELL, NODAL_X, NODAL_XY):
        m = MultiFab(p.n_cells, nodal, 2, 2)
        m.arr.copy_(torch.rand(m.arr.shape, generator=g, dtype=torch.float64))
        valid_before = m.valid().clone()
        oracle.override_sync(m)
        v = m.valid()
        # duplicated nodal points now equal their low-side owner
        if nodal[0]:
            assert torch.equal(v[..., 6], v[..., 0])
        if nodal[1]:
            assert torch.equal(v[:, :, 6, :], v[:, :, 0, :])
        oracle.fill_boundary(m)
        # ghosts are periodic images of valid points; valid points unchanged
        assert torch.equal(m.valid(), v)
        for (i, j, k) in [(-1, 0, 0), (-2, -1, 3), (6 + nodal[0], 2, -2), (1, 6 + nodal[1] + 1, 0)]:
            n0 = 6
            si = i % n0 if not (0 <= i <= 5 + nodal[0]) else i
            sj = j % n0 if not (0 <= j <= 5 + nodal[1]) else j
            sk = k % n0 if not (0 <= k <= 5) else k
            assert m[i, j, k, 1].item() == m[si, sj, sk, 1].item()
        if not any(nodal):
            assert torch.equal(valid_before, m.valid())


def test_noise_fill_statistics_and_sync(oracle):
    p = argon(16)
    nz = seeded_noise(oracle, p, 5, 0)
    a = nz.face[0][0].valid()
    assert abs(a.mean().item()) < 0.02
    assert a.var().item() == pytest.approx(1.0, rel=0.03)
    c = nz.cen[1][2].valid()
    assert c.var().item() == pytest.approx(2.0, rel=0.03)
    assert torch.equal(a[..., 16], a[..., 0])


def test_philox_is_deterministic_and_key_sensitive(oracle):
    o1 = oracle.philox4x32_10((1, 2, 3, 4), (5, 6))
    o2 = oracle.philox4x32_10((1, 2, 3, 4), (5, 6))
    o3 = oracle.philox4x32_10((1, 2, 3, 4), (5, 7))
    assert o1 == o2 and o1 != o3


def test_massfrac_guard_reports_instead_of_abort(oracle):
    """transCoeffs.cpp:45-46 aborts on Y <= 0 or Y >= 1; the oracle returns the
    status code instead."""
    p = argon(4)
    st = StagState(p)
    oracle.init_state(st, p)
    st.prim[1, 1, 1, 6] = 0.0
    assert oracle.transport_coeffs(st) == 2


def test_parse_inputs_reference_keys():
    deck = """
      n_cells = 16 16 16
      prob_hi = 1.28e-4 1.28e-4 1.28e-4   # comment
      nspecies = 2
      molmass = 39.948 39.948
      diameter = 3.66e-8 3.66e-8
      rhobar = 0.5 0.5
      dof = 3 3
      T_init = 273
      rho0 = 1.7775e-3
      visc_type = 2
      advection_type = 2
      algorithm_type = 2
      seed = 7
      bc_vel_lo = -1 -1 -1
      plot_int = 10
    """
    p = parse_inputs(deck)
    assert p.n_cells == (16, 16, 16) and p.nspecies == 2 and p.seed == 7
    assert p.dx[0] == pytest.approx(8e-6)
    assert p.hcv == (-1.0, -1.0)
    # walls and reservoirs are read; bc_mass above 4 is refused
    w = parse_inputs(deck + "\nbc_vel_lo = 1 -1 -1\nbc_vel_hi = 1 -1 -1\nbc_mass_lo = 1 -1 -1\n")
    assert w.walls == 1 and w.bc_vel_lo == (1, -1, -1) and w.bc_mass_lo == (1, -1, -1)
    with pytest.raises(ValueError):
        parse_inputs(deck + "\nbc_vel_lo = 1 -1 -1\nbc_mass_lo = 5 -1 -1\n")


def test_dt_rule_respects_diffusive_limit():
    p = argon(32, dx=1e-6)
    dt = stable_dt(p)
    eta, kappa = hard_sphere_single_gas(p)
    hcv, _ = p.hc()
    chi = kappa / (p.rho0 * hcv[0])
    assert chi * dt / 1e-12 <= 0.1 + 1e-12
    assert dt < 0.2 * 1e-6 / p.sound_speed()


@pytest.mark.slow
def test_equilibrium_variances_match_theory(oracle):
    """Equilibrium variances of density, species density, momentum, energy and
    temperature against the reference's theory formulas (16^3 argon, dx = 8e-6 cm)."""
    p = argon(16, dx=8e-6)
    st = StagState(p)
    oracle.init_state(st, p)
    dt = stable_dt(p)
    nz = StepNoise(p)
    keys = {"rho": lambda: st.cu.valid(0), "rho0": lambda: st.cu.valid(5), "rhoE": lambda: st.cu.valid(4),
            "T": lambda: st.prim.valid(4), "jx": lambda: st.cumom[0].valid(0)[:, :, :16]}
    samples = {k: [] for k in keys}
    nwarm, nsamp, every = 300, 60, 5
    for s in range(nwarm + nsamp * every):
        oracle.fill_step_noise(nz, 7, s)
        assert oracle.rk3_step(st, nz, dt) == 0
        if s >= nwarm and (s - nwarm) % every == 0:
            for k, f in keys.items():
                samples[k].append(f().clone())
    th = equilibrium_variances(p)
    for k, lst in samples.items():
        x = torch.stack(lst)
        var = ((x - x.mean()) ** 2).mean().item()
        assert var / th[k] == pytest.approx(1.0, abs=0.03), k
