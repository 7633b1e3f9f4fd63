"""Static structure factor (the reference's StructFact, src_analysis/StructFact.cpp)
over ``fhd_sf_*``: covariances of the Fourier transforms of cell-centred
variables, accumulated on the device (cuFFT + one fused accumulation kernel).

    sf = StructFact(p.n_cells, ["rho", "T"], var_scaling=[1.0] * 3)
    for step in ...:
        sf.fort_structure(variables)          # MultiFab with the variables as components
    real, imag, mag = sf.finalize(zero_avg=1)  # k = 0 at n_cells // 2

A quasi-2-D run's per-z-slice or a quasi-1-D run's per-x-pencil structure factors
(main_driver.cpp:923-993) are one stacked object: ``StructFact(p.n_cells, names,
scaling, stack="z_slices" | "x_pencils")`` takes the whole box's variables, and
``stack_average()`` gives the reference's averaged (mag, realimag) output.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import capi
from .capi import check
from .fab import CELL, MultiFab


def default_pairs(nvar: int):
    """All nvar (nvar + 1) / 2 pairs (A = j, B = i for i <= j), StructFact.cpp:45-69."""
    a, b = [], []
    for i in range(nvar):
        for j in range(i, nvar):
            a.append(j)
            b.append(i)
    return a, b


STACKS = {None: 0, "z_slices": 1, "x_pencils": 2}


class StructFact:
    def __init__(self, n_cells, var_names, var_scaling, pairs=None, device: int = 0, stack=None):
        self.lib = capi.load()
        self.n_cells = tuple(int(x) for x in n_cells)
        self.stack = stack
        nx, ny, nz = self.n_cells
        self.member = {None: (nx, ny, nz), "z_slices": (nx, ny, 1), "x_pencils": (nx, 1, 1)}[stack]
        self.var_names = list(var_names)
        self.device = device
        nvar = len(self.var_names)
        pa, pb = pairs if pairs is not None else default_pairs(nvar)
        if len(pa) != len(pb) or len(var_scaling) != len(pa):
            raise ValueError("pairs and var_scaling must have one entry per covariance")
        self.pairs = (list(pa), list(pb))
        # StructFact.cpp:165-177: names struct_fact_<B>_<A>
        self.cov_names = [f"struct_fact_{self.var_names[b]}_{self.var_names[a]}" for a, b in zip(pa, pb)]
        n = (C.c_int * 3)(*self.n_cells)
        ca = (C.c_int * len(pa))(*pa)
        cb = (C.c_int * len(pb))(*pb)
        sc = (C.c_double * len(pa))(*var_scaling)
        self._h = C.c_void_p()
        check(self.lib.fhd_sf_create_stack(C.byref(self._h), n, STACKS[stack], nvar, len(pa), ca, cb, sc, device),
              "fhd_sf_create_stack")

    @property
    def ncov(self) -> int:
        return self.lib.fhd_sf_ncov(self._h)

    @property
    def nsamples(self) -> int:
        return self.lib.fhd_sf_nsamples(self._h)

    def _stream(self):
        s = torch.cuda.current_stream(self.device).cuda_stream
        check(self.lib.fhd_sf_set_stream(self._h, C.c_void_p(s)), "fhd_sf_set_stream")

    def fort_structure(self, variables: MultiFab, reset: int = 0):
        """One sample (StructFact::FortStructure); variables holds the nvar fields."""
        self._stream()
        check(self.lib.fhd_sf_fort_structure(self._h, variables.fab(), reset), "fhd_sf_fort_structure")

    def finalize(self, zero_avg: int = 1):
        """(cov_real, cov_imag, cov_mag) MultiFabs, StructFact::CallFinalize."""
        self._stream()
        out = [MultiFab(self.n_cells, CELL, self.ncov, 0, device=f"cuda:{self.device}") for _ in range(3)]
        check(self.lib.fhd_sf_finalize(self._h, out[0].fab(), out[1].fab(), out[2].fab(), zero_avg),
              "fhd_sf_finalize")
        return tuple(out)

    def stack_average(self, zero_avg: int = 1):
        """(mag, realimag) MultiFabs of the member shape: AddToExternal of every
        member in order, then times 1/members (main_driver.cpp:1592-1618, 1683-1711)."""
        self._stream()
        dev = f"cuda:{self.device}"
        mag = MultiFab(self.member, CELL, self.ncov, 0, device=dev)
        ri = MultiFab(self.member, CELL, 2 * self.ncov, 0, device=dev)
        check(self.lib.fhd_sf_stack_average(self._h, mag.fab(), ri.fab(), zero_avg), "fhd_sf_stack_average")
        return mag, ri

    def close(self):
        if self._h:
            self.lib.fhd_sf_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
