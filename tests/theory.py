"""Equilibrium fluctuation theory used as the statistical oracle.

Formulas of the reference's own equilibrium checks
(exec/compressible/chemistry_inputs_files/params_RBtest_eq_SF.py:94-104,
exec/compressible_stag/test_MFsurfchem_COAr_eq/params_COAr_eq.py:204-210):
  <d rho_k^2> = rho_k^2 / N_k            (N_k molecules of species k in dV)
  <d j^2>     = rho k_B T / dV           (each momentum component)
  <d (rhoE)^2> = (k_B T)^2/dV * sum_k (dof_k/2)(dof_k/2+1) n_k
  <d T^2>     = k_B T^2 / (rho c_v dV)
"""
from __future__ import annotations

from fhdex_b200.params import Params


def equilibrium_variances(p: Params, T=None):
    T = p.T_init if T is None else T
    kB = p.k_B
    dV = p.dx[0] * p.dx[1] * p.dx[2]
    rho = p.rho0
    hcv, _ = p.hc()
    out = {}
    drho = 0.0
    dE = 0.0
    for k in range(p.nspecies):
        rk = rho * p.rhobar[k]
        mk = p.molmass[k] * kB / p.Runiv
        nk = rk / mk
        Nk = nk * dV
        v = rk * rk / Nk
        out[f"rho{k}"] = v
        drho += v
        dE += (0.5 * p.dof[k]) * (0.5 * p.dof[k] + 1.0) * nk
    out["rho"] = drho
    out["jx"] = out["jy"] = out["jz"] = rho * kB * T / dV
    out["rhoE"] = (kB * T) ** 2 / dV * dE
    cv = sum(p.rhobar[k] * hcv[k] for k in range(p.nspecies))
    out["T"] = kB * T * T / (rho * cv * dV)
    return out
