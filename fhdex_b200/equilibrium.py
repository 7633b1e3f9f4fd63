"""Equilibrium fluctuation theory (the reference's statistical checks) and the
equilibrium check of the batched step.

Formulas of the reference's own equilibrium checks
(exec/compressible/chemistry_inputs_files/params_RBtest_eq_SF.py:94-104,
exec/compressible_stag/test_MFsurfchem_COAr_eq/params_COAr_eq.py:204-210):
  <d rho_k^2> = rho_k^2 / N_k            (N_k molecules of species k in dV)
  <d j^2>     = rho k_B T / dV           (each momentum component)
  <d (rhoE)^2> = (k_B T)^2/dV * sum_k (dof_k/2)(dof_k/2+1) n_k
  <d T^2>     = k_B T^2 / (rho c_v dV)
"""
from __future__ import annotations

import torch

from .params import Params, argon, stable_dt
from .state import StagState


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


# cell-centred conserved fields, temperature and face momenta (valid regions)
FIELDS = ("rho", "rho0", "rhoE", "T", "jx", "jy", "jz")


def field_views(st: StagState, n: int):
    return {"rho": st.cu.valid(0), "rho0": st.cu.valid(5), "rhoE": st.cu.valid(4), "T": st.prim.valid(4),
            "jx": st.cumom[0].valid(0)[:, :, :n], "jy": st.cumom[1].valid(0)[:, :n, :],
            "jz": st.cumom[2].valid(0)[:n, :, :]}


def batch_variance_ratios(members: int = 16, n: int = 32, precision: int = 1, warm: int = 1000,
                          samples: int = 150, every: int = 5, seed: int = 7, device: int = 0,
                          dt_scale: float = 1.0):
    """Equilibrium check of the batched step (fhd_batch_*, in-kernel Philox noise):
    `members` independent n^3 argon runs (dx = 8e-6 cm, T0 = 273 K, rho0 = 1.78e-3)
    advanced together; after `warm` steps the variances over cells, members and
    `samples` snapshots `every` steps apart, divided by equilibrium_variances.
    dt = dt_scale * stable_dt.  Returns ({field: measured/theory}, samples per field)."""
    from .batch import Batch
    b = Batch(2, precision, device)
    sts = []
    p = None
    for q in range(members):
        p = argon(n, dx=8e-6, precision=precision, seed=(seed << 16) + q + 1)
        st = StagState(p, f"cuda:{device}", aux=False)
        b.add(p, st, dt_scale * stable_dt(p))
        sts.append(st)
    acc = {k: torch.zeros(2, dtype=torch.float64, device=f"cuda:{device}") for k in FIELDS}
    b.step(warm)
    for _ in range(samples):
        b.step(every)
        b.synchronize()
        for st in sts:
            for k, x in field_views(st, n).items():
                acc[k][0] += x.sum()
                acc[k][1] += (x * x).sum()
    bad = sum(1 for mid in list(b.members) if b.status(mid) != 0)
    b.close()
    if bad:
        raise RuntimeError(f"{bad} members reported a device status")
    th = equilibrium_variances(p)
    m = n ** 3 * members * samples
    ratios = {}
    for k, a in acc.items():
        mean = a[0].item() / m
        ratios[k] = (a[1].item() / m - mean * mean) / th[k]
    return ratios, m
