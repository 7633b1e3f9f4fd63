"""Shared test helpers: perturbed physical states, noise, comparisons."""
from __future__ import annotations

import torch

from fhdex_b200.params import Params
from fhdex_b200.state import StagState, StepNoise


def perturbed_state(O, p: Params, seed=0, amp=0.02, vel_amp=0.05):
    """A random but physical state: the uniform rest state of InitConsVarStag with
    density, composition, energy and face momenta perturbed, then converted to
    primitives and ghost-filled by the oracle (the main_driver init sequence)."""
    st = StagState(p)
    O.init_state(st, p)
    g = torch.Generator().manual_seed(seed)
    ns = p.nspecies
    vc = st.cu.valid()
    shp = vc.shape[1:]
    rho = vc[0]
    frac = torch.stack([vc[5 + s] / rho for s in range(ns)])
    frac = frac * (1.0 + amp * (2 * torch.rand((ns,) + shp, generator=g, dtype=torch.float64) - 1))
    frac = frac / frac.sum(0)
    rho_new = rho * (1.0 + amp * (2 * torch.rand(shp, generator=g, dtype=torch.float64) - 1))
    vc[0] = rho_new
    for s in range(ns):
        vc[5 + s] = rho_new * frac[s]
    vc[4] = vc[4] * (1.0 + 0.5 * amp * (2 * torch.rand(shp, generator=g, dtype=torch.float64) - 1))
    c = p.sound_speed()
    for d in range(3):
        mv = st.cumom[d].valid(0)
        mv.copy_(p.rho0 * vel_amp * c * (2 * torch.rand(mv.shape, generator=g, dtype=torch.float64) - 1))
        O.override_sync(st.cumom[d])
        O.fill_boundary(st.cumom[d])
    O.fill_boundary(st.cu)
    rc = O.conserved_to_primitive(st)
    assert rc == 0
    for m in [st.cu, st.prim] + st.vel:
        O.fill_boundary(m)
    return st


def seeded_noise(O, p: Params, seed, step):
    nz = StepNoise(p)
    O.fill_step_noise(nz, seed, step)
    return nz


def max_rel(a: torch.Tensor, b: torch.Tensor):
    """max|a-b| / max|b| over the whole array (norm-relative error of a field)."""
    a = a.double().cpu()
    b = b.double().cpu()
    den = b.abs().max().item()
    num = (a - b).abs().max().item()
    return num / den if den > 0 else num


def compare_named(got: dict, ref: dict, tol: float = 0.0, per_comp=True):
    """Compare MultiFabs by name (whole storage, ghosts included).  tol = 0:
    bitwise equality (== semantics); else norm-relative error per component."""
    bad = []
    worst = 0.0
    for name, r in ref.items():
        gm = got[name].arr.cpu()
        rm = r.arr.cpu()
        for n in range(rm.shape[0]) if per_comp else [None]:
            ga = gm[n] if n is not None else gm
            ra = rm[n] if n is not None else rm
            if tol == 0.0:
                if not torch.equal(ga, ra):
                    d = (ga - ra).abs().max().item()
                    bad.append(f"{name}[{n}] max|diff|={d:.3e} rel={max_rel(ga, ra):.3e}")
            else:
                e = max_rel(ga, ra)
                worst = max(worst, e)
                if not (e <= tol):
                    bad.append(f"{name}[{n}] rel={e:.3e} > {tol:.1e}")
    return bad, worst
