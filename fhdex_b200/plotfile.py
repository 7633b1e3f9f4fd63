"""WritePlotFileStag (writePlotFileStag.cpp:7-527) through the C ABI.

``plotfile_names`` gives the reference's variable list for a set of flags,
``pack`` assembles the plotfile MultiFab on the GPU (fhd_plotfile_pack) and
``write_plotfile_stag`` writes the AMReX plotfile directory
``<base><step, 9 digits>/`` (fhd_write_plotfile_stag).  Flags follow the
reference's plot_means / plot_vars / plot_covars / plot_mom3 / plot_mom4 inputs.
"""
from __future__ import annotations

import ctypes as C

from . import capi
from .capi import check
from .fab import CELL, MultiFab

MEANS, VARS, COVARS, MOM3, MOM4 = 1, 2, 4, 8, 16
DELTAY = (32, 64, 128)   # plot_deltaY_dir = 0, 1, 2


def flags_of(plot_means=False, plot_vars=False, plot_covars=False, plot_mom3=False, plot_mom4=False,
             plot_deltaY_dir=-1) -> int:
    return ((MEANS if plot_means else 0) | (VARS if plot_vars else 0) | (COVARS if plot_covars else 0)
            | (MOM3 if plot_mom3 else 0) | (MOM4 if plot_mom4 else 0)
            | (DELTAY[plot_deltaY_dir] if plot_deltaY_dir in (0, 1, 2) else 0))


def plotfile_names(p, flags: int = 0) -> list[str]:
    """The reference's variable names of the plotfile for Params ``p`` and ``flags``."""
    lib = capi.load()
    cp = p.to_c()
    n = lib.fhd_plotfile_ncomp(C.byref(cp), flags)
    if n < 0:
        check(-n, "fhd_plotfile_ncomp")
    buf = C.create_string_buffer(64)
    out = []
    for c in range(n):
        check(lib.fhd_plotfile_varname(C.byref(cp), flags, c, buf, 64), "fhd_plotfile_varname")
        out.append(buf.value.decode())
    return out


def write_plotfile_host(p, dirname: str, data, flags: int, time: float, step: int) -> None:
    """Writes the plotfile directory from a packed host array (ncomp, nz, ny, nx)."""
    import torch
    arr = data.detach().to("cpu", torch.float64).contiguous()
    cp = p.to_c()
    check(capi.load().fhd_plotfile_write_host(C.byref(cp), dirname.encode(),
                                              C.cast(arr.data_ptr(), C.POINTER(C.c_double)), flags, time, step),
          "fhd_plotfile_write_host")


def _args(st, stats, flags):
    nf = capi.FhdFab()
    zeta = st.zeta.fab() if getattr(st, "aux", False) else nf
    sp = C.byref(stats.c_struct()) if (stats is not None and flags) else None
    return (st.cu.fab(), st.mom_fabs(), st.prim.fab(), st.vel_fabs(), st.eta.fab(), st.kappa.fab(), zeta), sp


def pack(ctx, st, stats=None, flags: int = 0, out: MultiFab | None = None) -> MultiFab:
    """The plotfile MultiFab (cell-centred, no ghosts) on the state's device, into
    ``out`` when given.  ``st`` needs its transport coefficients (a StagState with
    aux=True)."""
    ctx._stream()
    if out is None:
        n = len(plotfile_names(ctx.p, flags))
        out = MultiFab(st.cu.n_cells, CELL, n, 0, device=st.cu.arr.device)
    a, sp = _args(st, stats, flags)
    check(ctx.lib.fhd_plotfile_pack(ctx._h, flags, out.fab(), *a, sp), "fhd_plotfile_pack")
    return out


def write_plotfile_stag(ctx, plot_base_name: str, step: int, time: float, st, stats=None, flags: int = 0) -> str:
    """Writes <plot_base_name><step:09d>/ and returns its path."""
    ctx._stream()
    a, sp = _args(st, stats, flags)
    check(ctx.lib.fhd_write_plotfile_stag(ctx._h, plot_base_name.encode(), step, time, flags, *a, sp),
          "fhd_write_plotfile_stag")
    return f"{plot_base_name}{step:09d}"
