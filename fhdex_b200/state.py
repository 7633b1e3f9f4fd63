"""The MultiFabs the reference's driver allocates for the staggered step
(main_driver.cpp:596-640, 995-1050), as single-box mirrors.

``StagState`` holds the evolving state (cu, cumom, prim, vel) and the per-step
by-products the reference's ``RK3stepStag`` writes (transport coefficients and
fluxes).  ``StepNoise`` holds the A/B white-noise fields of one step in the
layout ``fhd_noise`` documents.
"""
from __future__ import annotations

import torch

from .capi import FabArr3, FabArr6, FhdNoise
from .fab import CELL, EDGE, FACE, NODAL_XY, NODAL_XZ, NODAL_YZ, MultiFab, fab_array
from .params import Params


class StagState:
    def __init__(self, p: Params, device="cpu", *, aux=True, pin_memory=False,
                 dtype=torch.float64):
        N, ng, ns = p.n_cells, p.ngc, p.nspecies
        kw = dict(dtype=dtype, device=device, pin_memory=pin_memory)
        self.p = p
        self.cu = MultiFab(N, CELL, p.nvars, ng, **kw)
        self.cumom = [MultiFab(N, FACE[d], 1, ng, **kw) for d in range(3)]
        self.prim = MultiFab(N, CELL, p.nprimvars, ng, **kw)
        self.vel = [MultiFab(N, FACE[d], 1, ng, **kw) for d in range(3)]
        self.aux = aux
        if aux:
            self.source = MultiFab(N, CELL, p.nprimvars, ng, **kw)
            self.eta = MultiFab(N, CELL, 1, ng, **kw)
            self.zeta = MultiFab(N, CELL, 1, ng, **kw)
            self.kappa = MultiFab(N, CELL, 1, ng, **kw)
            self.chi = MultiFab(N, CELL, ns, ng, **kw)
            self.D = MultiFab(N, CELL, ns * ns, ng, **kw)
            self.faceflux = [MultiFab(N, FACE[d], p.nvars + 4, 0, **kw) for d in range(3)]
            # edgeflux_x = {xy, xz}, edgeflux_y = {xy, yz}, edgeflux_z = {xz, yz}
            en = (NODAL_XY, NODAL_XZ, NODAL_XY, NODAL_YZ, NODAL_XZ, NODAL_YZ)
            self.edgeflux = [MultiFab(N, en[e], 1, 0, **kw) for e in range(6)]
            self.cenflux = [MultiFab(N, CELL, 1, 1, **kw) for d in range(3)]

    # state MultiFabs in a fixed order (for copies / comparisons)
    def state_mfs(self):
        return [self.cu] + self.cumom + [self.prim] + self.vel

    def aux_mfs(self):
        return ([self.eta, self.zeta, self.kappa, self.chi, self.D] + self.faceflux
                + self.edgeflux + self.cenflux)

    def named(self, aux=False):
        d = {"cu": self.cu, "prim": self.prim}
        for q in range(3):
            d[f"cumom{q}"] = self.cumom[q]
            d[f"vel{q}"] = self.vel[q]
        if aux and self.aux:
            for n in ("eta", "zeta", "kappa", "chi", "D"):
                d[n] = getattr(self, n)
            for q in range(3):
                d[f"faceflux{q}"] = self.faceflux[q]
                d[f"cenflux{q}"] = self.cenflux[q]
            for e in range(6):
                d[f"edgeflux{e}"] = self.edgeflux[e]
        return d

    def copy_from(self, other: "StagState", aux=False):
        for a, b in zip(self.state_mfs(), other.state_mfs()):
            a.arr.copy_(b.arr)
        if aux and self.aux and other.aux:
            for a, b in zip(self.aux_mfs(), other.aux_mfs()):
                a.arr.copy_(b.arr)

    def clone(self, device=None, pin_memory=False):
        s = StagState(self.p, device or self.cu.arr.device, aux=self.aux, pin_memory=pin_memory)
        s.copy_from(self, aux=True)
        return s

    def state_bytes(self):
        return sum(m.nbytes() for m in self.state_mfs())

    # C views
    def mom_fabs(self):
        return fab_array(self.cumom, FabArr3)

    def vel_fabs(self):
        return fab_array(self.vel, FabArr3)

    def faceflux_fabs(self):
        return fab_array(self.faceflux, FabArr3)

    def edgeflux_fabs(self):
        return fab_array(self.edgeflux, FabArr6)

    def cenflux_fabs(self):
        return fab_array(self.cenflux, FabArr3)


class StepNoise:
    """A/B noise of one step: face[s][d] (nspecies+1 comps: energy then species),
    edge[s][e] (xy, xz, yz), cen[s][d] (1 ghost).  s = 0 (A) or 1 (B)."""

    def __init__(self, p: Params, device="cpu", dtype=torch.float64):
        N, ns = p.n_cells, p.nspecies
        kw = dict(dtype=dtype, device=device)
        self.p = p
        self.face = [[MultiFab(N, FACE[d], ns + 1, 0, **kw) for d in range(3)] for _ in range(2)]
        self.edge = [[MultiFab(N, EDGE[e], 1, 0, **kw) for e in range(3)] for _ in range(2)]
        self.cen = [[MultiFab(N, CELL, 1, 1, **kw) for d in range(3)] for _ in range(2)]
        # ranchem_A / ranchem_B (nreaction comps) when the run has reactions
        nr = getattr(p, "nreaction", 0)
        self.chem = [MultiFab(N, CELL, nr, 0, **kw) if nr > 0 else None for _ in range(2)]

    def mfs(self):
        out = []
        for s in range(2):
            out += self.face[s] + self.edge[s] + self.cen[s]
        out += [c for c in self.chem if c is not None]
        return out

    def c_struct(self) -> FhdNoise:
        n = FhdNoise()
        for s in range(2):
            for d in range(3):
                n.face[s][d] = self.face[s][d].fab()
                n.edge[s][d] = self.edge[s][d].fab()
                n.cen[s][d] = self.cen[s][d].fab()
            if self.chem[s] is not None:
                n.chem[s] = self.chem[s].fab()
        return n

    def to(self, device):
        q = StepNoise(self.p, device)
        for a, b in zip(q.mfs(), self.mfs()):
            a.arr.copy_(b.arr)
        return q
