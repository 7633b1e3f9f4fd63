"""Test helper: reads back the plotfiles fhd_write_plotfile_stag /
fhd_plotfile_write_host produce, and restates WritePlotFileStag's composition.

``read_header`` consumes the Header's whitespace-separated tokens in the order
the reference's own post-processing reads them (exec/compressible_stag/TURB_PDFS/
main.cpp:66-115: version string, component count, names, dimension, time,
finest level, prob_lo, prob_hi), then the rest of the single-level layout.
``read_cell_data`` parses Level_0/Cell_D_00000 (a one-line FAB descriptor, then
the doubles) and ``read_cell_h`` the per-component minima / maxima of Cell_H.
"""
from __future__ import annotations

import os
import re

import numpy as np


def read_header(path):
    toks = open(os.path.join(path, "Header")).read().split()
    it = iter(toks)
    h = {"version": next(it)}
    nc = int(next(it))
    h["names"] = [next(it) for _ in range(nc)]
    h["dim"] = int(next(it))
    h["time"] = float(next(it))
    h["finest_level"] = int(next(it))
    h["prob_lo"] = [float(next(it)) for _ in range(3)]
    h["prob_hi"] = [float(next(it)) for _ in range(3)]
    h["domain"] = next(it) + next(it) + next(it)   # ((lo) (hi) (type)), no refinement ratios at level 0
    h["step"] = int(next(it))
    h["dx"] = [float(next(it)) for _ in range(3)]
    h["coord_sys"] = int(next(it))
    h["bwidth"] = int(next(it))
    h["level"], h["nboxes"] = int(next(it)), int(next(it))
    h["level_time"] = float(next(it))
    h["level_step"] = int(next(it))
    h["box_phys"] = [(float(next(it)), float(next(it))) for _ in range(3)]
    h["cell_path"] = next(it)
    return h


def read_cell_data(path):
    raw = open(os.path.join(path, "Level_0", "Cell_D_00000"), "rb").read()
    nl = raw.index(b"\n")
    line = raw[:nl].decode()
    m = re.match(r"FAB \(\(8, \(64 11 52 0 1 12 0 1023\)\),\(8, \(1 2 3 4 5 6 7 8\)\)\)"
                 r"\(\((\d+),(\d+),(\d+)\) \((\d+),(\d+),(\d+)\) \(0,0,0\)\) (\d+)$", line)
    assert m, line
    lo = [int(m.group(i)) for i in (1, 2, 3)]
    hi = [int(m.group(i)) for i in (4, 5, 6)]
    nc = int(m.group(7))
    n = [hi[d] - lo[d] + 1 for d in range(3)]
    data = np.frombuffer(raw[nl + 1:], dtype="<f8")
    assert data.size == nc * n[0] * n[1] * n[2]
    return data.reshape(nc, n[2], n[1], n[0])


def read_cell_h(path):
    lines = open(os.path.join(path, "Level_0", "Cell_H")).read().split("\n")
    nc = int(lines[2])
    i = lines.index(f"1,{nc}")
    mins = [float(x) for x in lines[i + 1].split(",") if x]
    j = lines.index(f"1,{nc}", i + 1)
    maxs = [float(x) for x in lines[j + 1].split(",") if x]
    return nc, mins, maxs


def reference_names(p, means=False, varz=False, covars=False, mom3=False, mom4=False, deltay=-1):
    """writePlotFileStag.cpp:313-447, as the reference builds its varNames."""
    ns = p.nspecies
    sp = lambda base: [base + chr(48 + i) for i in range(ns)]
    v = ["rhoInstant", "jxInstantCC", "jyInstantCC", "jzInstantCC", "rhoEInstant"] + sp("rhoYkInstant_")
    v += ["jxInstantFACE", "jyInstantFACE", "jzInstantFACE", "uxInstantCC", "uyInstantCC", "uzInstantCC",
          "tInstant", "pInstant"] + sp("YkInstant_") + sp("XkInstant_")
    v += ["uxInstantFACE", "uyInstantFACE", "uzInstantFACE", "eta", "kappa"]
    if abs(p.visc_type) == 3:
        v += ["zeta"]
    if means:
        v += ["rhoMean", "jxMeanCC", "jyMeanCC", "jzMeanCC", "rhoEMean"] + sp("rhoYkMean_")
        v += ["jxMeanFACE", "jyMeanFACE", "jzMeanFACE", "uxMeanCC", "uyMeanCC", "uzMeanCC", "tMean", "pMean"]
        v += sp("YkMean_") + sp("XkMean_")
        v += ["uxMeanFACE", "uyMeanFACE", "uzMeanFACE", "uxMeanCOM", "uyMeanCOM", "uzMeanCOM"]
    if varz:
        v += ["rhoVar", "jxVarCC", "jyVarCC", "jzVarCC", "rhoEVar"] + sp("rhoYkVar_")
        v += ["jxVarFACE", "jyVarFACE", "jzVarFACE", "uxVarCC", "uyVarCC", "uzVarCC", "TVarDirect"] + sp("YkVar_")
        v += ["g-g", "g-energy", "rho-energy", "rho-g", "TVar", "uxVarFACE", "uyVarFACE", "uzVarFACE"]
    if covars:
        v += ["rho-jx", "rho-jy", "rho-jz", "jx-jy", "jy-jz", "jx-jz", "rho-rhoE", "rhoE-jx", "rhoE-jy",
              "rhoE-jz", "rhoL-rhoH", "rho-vx", "rho-vy", "rho-vz", "vx-vy", "vy-vz", "vx-vz", "rho-T", "vx-T",
              "vy-T", "vz-T", "YkL-YkH", "YkL-vx", "YkH-vx", "rhoYkL-vx", "rhoYkH-vx"]
    for on, sfx in ((mom3, "mom3"), (mom4, "mom4")):
        if on:
            v += ["rho" + sfx, "velx" + sfx, "vely" + sfx, "velz" + sfx, "rhoE" + sfx] + sp("Yk" + sfx + "_")
            v += ["T" + sfx]
    if deltay != -1:
        v += sp("deltaYk_")
    # nplot of writePlotFileStag.cpp:37-99
    nvars = 5 + ns
    nplot = nvars + 3 + 5 + 2 * ns + 3 + 2 + (1 if abs(p.visc_type) == 3 else 0)
    nplot += (nvars + 3 + 5 + 2 * ns + 3 + 3) if means else 0
    nplot += (nvars + 3 + 9 + ns + 3) if varz else 0
    nplot += 26 if covars else 0
    nplot += (nvars + 1) * (int(mom3) + int(mom4))
    nplot += ns if deltay != -1 else 0
    assert len(v) == nplot
    return v


def reference_composition(p, st, stats=None, means=False, varz=False, covars=False, mom3=False, mom4=False,
                          deltay=-1):
    """writePlotFileStag.cpp:111-281 on the valid box: list of (ncomp, nz, ny, nx) arrays
    (MultiFab::Copy of cell components; ShiftFaceToCC copies face (i,j,k) to cell (i,j,k))."""
    ns = p.nspecies
    nprim = 6 + 2 * ns
    N = p.n_cells
    cell = lambda mf, c: mf.valid()[c].cpu().numpy()
    face = lambda mf: mf.valid()[0][:N[2], :N[1], :N[0]].cpu().numpy()
    out = [cell(st.cu, c) for c in range(5 + ns)]
    out += [face(st.cumom[d]) for d in range(3)]
    out += [cell(st.prim, 1 + c) for c in range(5 + 2 * ns)]
    out += [face(st.vel[d]) for d in range(3)]
    out += [cell(st.eta, 0), cell(st.kappa, 0)]
    if abs(p.visc_type) == 3:
        out += [cell(st.zeta, 0)]
    if means:
        out += [cell(stats.cuMeans, c) for c in range(5 + ns)]
        out += [face(stats.cumomMeans[d]) for d in range(3)]
        out += [cell(stats.primMeans, 1 + c) for c in range(5 + 2 * ns)]
        out += [face(stats.velMeans[d]) for d in range(3)]
        out += [cell(stats.primMeans, nprim + c) for c in range(3)]
    if varz:
        out += [cell(stats.cuVars, c) for c in range(5 + ns)]
        out += [face(stats.cumomVars[d]) for d in range(3)]
        out += [cell(stats.primVars, 1 + c) for c in range(4)]
        out += [cell(stats.primVars, 6 + c) for c in range(ns)]
        out += [cell(stats.primVars, nprim + c) for c in range(5)]
        out += [face(stats.velVars[d]) for d in range(3)]
    if covars:
        out += [cell(stats.coVars, c) for c in range(26)]
    if mom3:
        out += [cell(stats.mom3, c) for c in range(6 + ns)]
    if mom4:
        out += [cell(stats.mom4, c) for c in range(6 + ns)]
    if deltay != -1:
        # WriteHorizontalAverageToMF (ComputeAverages.cpp:96-190): per plane r the
        # sequential sum in loop order k, j, i (np.cumsum adds one term at a time),
        # divided by the plane's cell count; then (-average) + Y_k
        for c in range(ns):
            y = cell(st.prim, 6 + c)                      # (z, y, x)
            avg = np.empty(N[deltay])
            for r in range(N[deltay]):
                plane = (y[:, :, r] if deltay == 0 else (y[:, r, :] if deltay == 1 else y[r, :, :])).ravel()
                navg = plane.size
                avg[r] = np.cumsum(plane)[-1] / navg
            shape = [1, 1, 1]
            shape[2 - deltay] = N[deltay]
            out.append((-avg).reshape(shape) + y)
    return np.stack(out)
