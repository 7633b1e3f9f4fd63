"""Single-box MultiFab mirror over a torch tensor in AMReX Array4 layout.

A ``MultiFab`` here is one box of the reference's ``amrex::MultiFab``: valid
region ``0..n_cells[d]-1`` (cell-centred) or ``0..n_cells[d]`` (nodal in d),
``ngrow`` ghost points on every side, ``ncomp`` components.  Storage is a torch
tensor of shape ``(ncomp, nz, ny, nx)`` (C order), which is exactly Array4's
Fortran order with the component slowest, so ``data_ptr()`` can be handed to the
C ABI unchanged.  ``mf[i, j, k, n]`` indexes with the reference's (ghost-aware)
indices.
"""
from __future__ import annotations

import torch

from .capi import FHD_F32, FHD_F64, FhdFab

CELL = (0, 0, 0)
NODAL_X = (1, 0, 0)
NODAL_Y = (0, 1, 0)
NODAL_Z = (0, 0, 1)
NODAL_XY = (1, 1, 0)
NODAL_XZ = (1, 0, 1)
NODAL_YZ = (0, 1, 1)
FACE = (NODAL_X, NODAL_Y, NODAL_Z)
EDGE = (NODAL_XY, NODAL_XZ, NODAL_YZ)


class MultiFab:
    def __init__(self, n_cells, nodal=CELL, ncomp=1, ngrow=0, *, dtype=torch.float64,
                 device="cpu", pin_memory=False, tensor=None):
        self.n_cells = tuple(int(n) for n in n_cells)
        self.nodal = tuple(int(x) for x in nodal)
        self.ncomp = int(ncomp)
        self.ngrow = int(ngrow)
        shape = (self.ncomp,) + tuple(
            self.n_cells[d] + self.nodal[d] + 2 * self.ngrow for d in (2, 1, 0))
        if tensor is not None:
            if tuple(tensor.shape) != shape:
                raise ValueError(f"tensor shape {tuple(tensor.shape)} != {shape}")
            self.arr = tensor
        else:
            self.arr = torch.zeros(shape, dtype=dtype, device=device,
                                   pin_memory=pin_memory and device == "cpu")

    # -- geometry ---------------------------------------------------------------
    @property
    def lo(self):
        return (-self.ngrow,) * 3

    @property
    def hi(self):
        return tuple(self.n_cells[d] - 1 + self.nodal[d] + self.ngrow for d in range(3))

    def valid_shape(self):
        return tuple(self.n_cells[d] + self.nodal[d] for d in range(3))

    def valid(self, comp=None):
        """View of the valid region, shape (ncomp, nz, ny, nx) or (nz, ny, nx)."""
        g = self.ngrow
        nx, ny, nz = self.valid_shape()
        v = self.arr[:, g:g + nz, g:g + ny, g:g + nx]
        return v if comp is None else v[comp]

    def __getitem__(self, idx):
        i, j, k, *n = idx
        g = self.ngrow
        return self.arr[n[0] if n else 0, k + g, j + g, i + g]

    def __setitem__(self, idx, value):
        i, j, k, *n = idx
        g = self.ngrow
        self.arr[n[0] if n else 0, k + g, j + g, i + g] = value

    # -- C ABI --------------------------------------------------------------------
    def fab(self) -> FhdFab:
        f = FhdFab()
        f.data = self.arr.data_ptr()
        lo, hi = self.lo, self.hi
        for d in range(3):
            f.lo[d] = lo[d]
            f.hi[d] = hi[d]
            f.nodal[d] = self.nodal[d]
        f.ncomp = self.ncomp
        if self.arr.dtype == torch.float64:
            f.dtype = FHD_F64
        elif self.arr.dtype == torch.float32:
            f.dtype = FHD_F32
        else:
            raise TypeError(f"unsupported dtype {self.arr.dtype}")
        if not self.arr.is_contiguous():
            raise ValueError("MultiFab storage must be contiguous")
        return f

    # -- helpers --------------------------------------------------------------------
    def like(self, *, device=None, dtype=None, pin_memory=False):
        return MultiFab(self.n_cells, self.nodal, self.ncomp, self.ngrow,
                        dtype=dtype or self.arr.dtype, device=device or self.arr.device,
                        pin_memory=pin_memory)

    def copy(self, *, device=None, pin_memory=False):
        m = self.like(device=device, pin_memory=pin_memory)
        m.arr.copy_(self.arr)
        return m

    def to(self, device):
        return self.copy(device=device)

    def setVal(self, v, comp=None):
        if comp is None:
            self.arr.fill_(v)
        else:
            self.arr[comp].fill_(v)

    def nbytes(self):
        return self.arr.numel() * self.arr.element_size()


def fab_array(mfs, ctype):
    a = ctype()
    for q, m in enumerate(mfs):
        a[q] = m.fab() if m is not None else FhdFab()
    return a
