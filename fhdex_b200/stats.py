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
  spatialCross       (cross=True) n_cells[0] x ncross yz-averaged spatial
                     cross-correlations at x* = Params.cross_cell, ncross =
                     37 + nspecies + 3 (statsStag.cpp:868-1105; main_driver.cpp:283);
                     in a quasi-1-D run the per-pencil correlations, spatialCrossMF
                     (ncross or 5 ncross comps, nz, ny, nx; statsStag.cpp:1311-1557);
                     in a quasi-2-D run an ncross-component field left at zero
  dataSliceMeans_xcross  (cross=True) the 2*nvars + 8 + 2*nspecies line
                     averages at x* (the reference's crossMeans file rows)
"""
from __future__ import annotations

import torch

from .capi import FhdStats, STATS_CROSS, STATS_MEANS, STATS_MOM3, STATS_MOM4, STATS_VARS
from .fab import CELL, FACE, MultiFab
from .params import Params

ALL = STATS_MEANS | STATS_VARS | STATS_MOM3 | STATS_MOM4


def ncross(nspecies: int) -> int:
    """Entries per x cell of spatialCross (main_driver.cpp:283)."""
    return 37 + nspecies + 3


def nstats(nspecies: int) -> int:
    """Entries of dataSliceMeans_xcross (main_driver.cpp:279)."""
    return 2 * (5 + nspecies) + 8 + 2 * nspecies


class StatsState:
    def __init__(self, p: Params, device="cpu", mom34: bool = True, cross: bool = False):
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
        if cross and p.do_1D:
            # evaluateStatsStag1D's spatialCrossMF: cell-centred, no ghosts, ncross comps per x*
            nst = 5 if p.all_correl == 1 else 1
            self.spatialCross = torch.zeros(nst * ncross(p.nspecies), N[2], N[1], N[0], **kw)
        elif cross and p.do_2D:
            self.spatialCross = torch.zeros(ncross(p.nspecies), N[2], N[1], N[0], **kw)
        else:
            self.spatialCross = torch.zeros(N[0], ncross(p.nspecies), **kw) if cross else None
        self.dataSliceMeans_xcross = torch.zeros(nstats(p.nspecies), **kw) if cross else None

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
        """setVal(0) of every statistic and spatialCrossVec.assign(0)
        (main_driver.cpp:1183-1213)."""
        for m in self.named().values():
            m.arr.zero_()
        if self.spatialCross is not None:
            self.spatialCross.zero_()

    def clone(self, device=None):
        s = StatsState(self.p, device or self.cuMeans.arr.device, mom34=self.mom3 is not None,
                       cross=self.spatialCross is not None)
        for a, b in zip(s.named().values(), self.named().values()):
            a.arr.copy_(b.arr)
        if self.spatialCross is not None:
            s.spatialCross.copy_(self.spatialCross)
            s.dataSliceMeans_xcross.copy_(self.dataSliceMeans_xcross)
        return s

    def write_spatial_cross(self, step: int, dir: str = ""):
        """WriteSpatialCross3D / WriteSpatialCross1D (writePlotFileStag.cpp:528-563):
        the reference's file names (spatialCross<step, 9 digits>, or
        [<s>_]spatialCross1D_<step> in a quasi-1-D run) prefixed by ``dir``."""
        from . import capi
        cp = self.p.to_c()
        capi.check(capi.load().fhd_write_spatial_cross(cp, dir.encode(), step, self.spatialCross.data_ptr()),
                   "fhd_write_spatial_cross")

    def append_cross_means(self, path: str, step: int):
        """One row of the reference's crossMeans file (main_driver.cpp:1284-1288):
        the step, then dataSliceMeans_xcross at the stream's default 6 significant
        digits, each followed by a space."""
        vals = self.dataSliceMeans_xcross.cpu().tolist()
        with open(path, "a") as f:
            f.write(f"{step} " + "".join(f"{v:g} " for v in vals) + "\n")

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
        if self.spatialCross is not None:
            s.spatialCross = self.spatialCross.data_ptr()
            s.dataSliceMeans_xcross = self.dataSliceMeans_xcross.data_ptr()
        return s
