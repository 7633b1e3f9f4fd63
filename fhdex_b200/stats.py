"""Running statistics of the staggered state: the MultiFabs of the reference's
evaluateStatsStag3D (main_driver.cpp:646-714 shapes) and their update through
``fhd_stats_stag`` (``Context.stats_stag``).

Component maps (statsStag.cpp:200-691):
  cuMeans / cuVars   nvars: rho, jx, jy, jz (cell-centred), rhoE, rhoY_k
  primMeans          nprimvars + 3: rho, vx, vy, vz, T, p, Y_k, X_k, then the
                     running mean of the cell-centred velocity (3)
  primVars           nprimvars + 5: rho, vx, vy, vz, T (direct), (p unused),
                     Y_k, X_k (unused), then gvar, kgcross, krcross, rgcross and
                     <T T> from the energy/momentum fluctuations
  coVars             26 covariances (<rho jx> ... <rhoY_heaviest vx>)
  mom3 / mom4        nvars + 1 third / fourth moments (rho, vx, vy, vz, rhoE, Y_k, T)
  velMeans/velVars/cumomMeans/cumomVars   face-centred, one per direction
"""
from __future__ import annotations

import torch

from .capi import FhdStats, STATS_MEANS, STATS_MOM3, STATS_MOM4, STATS_VARS
from .fab import CELL, FACE, MultiFab
from .params import Params

ALL = STATS_MEANS | STATS_VARS | STATS_MOM3 | STATS_MOM4


class StatsState:
    def __init__(self, p: Params, device="cpu", mom34: bool = True):
        N, ng = p.n_cells, p.ngc
        kw = dict(device=device, dtype=torch.float64)
        self.p = p
        self.cuMeans = MultiFab(N, CELL, p.nvars, ng, **kw)
        self.cuVars = MultiFab(N, CELL, p.nvars, ng, **kw)
        self.primMeans = MultiFab(N, CELL, p.nprimvars + 3, ng, **kw)
        self.primVars = MultiFab(N, CELL, p.nprimvars + 5, ng, **kw)
        self.coVars = MultiFab(N, CELL, 26, 0, **kw)
        self.mom3 = MultiFab(N, CELL, p.nvars + 1, 0, **kw) if mom34 else None
        self.mom4 = MultiFab(N, CELL, p.nvars + 1, 0, **kw) if mom34 else None
        self.velMeans = [MultiFab(N, FACE[d], 1, 0, **kw) for d in range(3)]
        self.velVars = [MultiFab(N, FACE[d], 1, 0, **kw) for d in range(3)]
        self.cumomMeans = [MultiFab(N, FACE[d], 1, 0, **kw) for d in range(3)]
        self.cumomVars = [MultiFab(N, FACE[d], 1, 0, **kw) for d in range(3)]

    def named(self):
        d = {n: getattr(self, n) for n in ("cuMeans", "cuVars", "primMeans", "primVars", "coVars")}
        if self.mom3 is not None:
            d["mom3"], d["mom4"] = self.mom3, self.mom4
        for q in range(3):
            d[f"velMeans{q}"] = self.velMeans[q]
            d[f"velVars{q}"] = self.velVars[q]
            d[f"cumomMeans{q}"] = self.cumomMeans[q]
            d[f"cumomVars{q}"] = self.cumomVars[q]
        return d

    def reset(self):
        """setVal(0) of every statistic (main_driver.cpp:1183-1203)."""
        for m in self.named().values():
            m.arr.zero_()

    def clone(self, device=None):
        s = StatsState(self.p, device or self.cuMeans.arr.device, mom34=self.mom3 is not None)
        for a, b in zip(s.named().values(), self.named().values()):
            a.arr.copy_(b.arr)
        return s

    def c_struct(self) -> FhdStats:
        s = FhdStats()
        for n in ("cuMeans", "cuVars", "primMeans", "primVars", "coVars"):
            setattr(s, n, getattr(self, n).fab())
        if self.mom3 is not None:
            s.mom3 = self.mom3.fab()
            s.mom4 = self.mom4.fab()
        for q in range(3):
            s.velMeans[q] = self.velMeans[q].fab()
            s.velVars[q] = self.velVars[q].fab()
            s.cumomMeans[q] = self.cumomMeans[q].fab()
            s.cumomVars[q] = self.cumomVars[q].fab()
        return s
