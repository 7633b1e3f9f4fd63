"""NumPy restatement of the reference's StructFact (TEST INFRASTRUCTURE ONLY:
loaded by tests/ as the checker of fhd_sf_*).

Follows src_analysis/StructFact.cpp: FortStructure (:231-311) with ComputeFFT's
real-to-complex transform over x and its unpacking of the Hermitian half
(:322-519: the conjugate of the mirror point for i > nx/2, then division by
sqrt(N)), the pair accumulation in the reference's operation order, and
CallFinalize/Finalize (:598-641) with ShiftFFT (:643-719).  Arrays are indexed
[k, j, i] (x fastest in memory).
"""
from __future__ import annotations

import numpy as np


def default_pairs(nvar):
    a, b = [], []
    for i in range(nvar):
        for j in range(i, nvar):
            a.append(j)
            b.append(i)
    return a, b


def unpacked_spectrum(field):
    """ComputeFFT for one variable: full-grid (re, im) / sqrt(N)."""
    nz, ny, nx = field.shape
    half = np.fft.rfftn(field)                     # [k, j, 0..nx/2]
    re = np.empty(field.shape)
    im = np.empty(field.shape)
    h = nx // 2
    re[:, :, :h + 1] = half.real
    im[:, :, :h + 1] = half.imag
    for i in range(h + 1, nx):
        iloc = nx - i
        jloc = (ny - np.arange(ny)) % ny
        kloc = (nz - np.arange(nz)) % nz
        mirror = half[np.ix_(kloc, jloc, [iloc])][:, :, 0]
        re[:, :, i] = mirror.real
        im[:, :, i] = -mirror.imag
    sqrtnpts = np.sqrt(float(nx * ny * nz))
    return re / sqrtnpts, im / sqrtnpts


class StructFactOracle:
    def __init__(self, shape_zyx, nvar, var_scaling, pairs=None):
        self.pa, self.pb = pairs if pairs is not None else default_pairs(nvar)
        self.ncov = len(self.pa)
        self.scaling = [1.0 / s for s in var_scaling]
        self.re = np.zeros((self.ncov,) + tuple(shape_zyx))
        self.im = np.zeros((self.ncov,) + tuple(shape_zyx))
        self.nsamples = 0

    def fort_structure(self, variables, reset=0):
        """variables: array [nvar, nz, ny, nx] (valid region)."""
        spec = {v: unpacked_spectrum(variables[v]) for v in sorted(set(self.pa) | set(self.pb))}
        for c, (a, b) in enumerate(zip(self.pa, self.pb)):
            rA, iA = spec[a]
            rB, iB = spec[b]
            tr = 0.0 + rA * rB
            tr = tr + iA * iB
            ti = 0.0 + iA * rB
            ti = ti * -1.0
            ti = ti + rA * iB
            if reset == 1 or self.nsamples == 0:
                self.re[c] = tr
                self.im[c] = ti
            else:
                self.re[c] = self.re[c] + tr
                self.im[c] = self.im[c] + ti
        self.nsamples = 1 if reset == 1 else self.nsamples + 1

    def finalize(self, zero_avg=1):
        nsinv = 1.0 / self.nsamples
        out = []
        for acc in (self.re, self.im):
            x = acc.copy()
            if zero_avg == 1:
                x[:, 0, 0, 0] = 0.0
            nz, ny, nx = x.shape[1:]
            x = np.roll(x, (nz // 2, ny // 2, nx // 2), axis=(1, 2, 3))
            for c in range(self.ncov):
                x[c] = x[c] * nsinv
                x[c] = x[c] * self.scaling[c]
            out.append(x)
        mag = 0.0 + out[0] * out[0]
        mag = mag + out[1] * out[1]
        return out[0], out[1], np.sqrt(mag)


class StructFactStackOracle:
    """The quasi-2-D runs' per-z-slice and the quasi-1-D runs' per-x-pencil
    StructFact vectors (main_driver.cpp:923-993, 1503-1557) and their averaged
    output (AddToExternal of every member, StructFact.cpp:979-1009, then the mult
    by 1/members, main_driver.cpp:1592-1618, 1683-1711)."""

    def __init__(self, shape_zyx, kind, nvar, var_scaling, pairs=None):
        nz, ny, nx = shape_zyx
        self.kind = kind
        if kind == "z_slices":
            # member z = i: ExtractSlice(mf, Flattened, 2, i, ...)
            self.take = [(lambda v, z=z: v[:, z:z + 1, :, :]) for z in range(nz)]
            mshape = (1, ny, nx)
        else:
            # member i: ExtractXPencil(mf, pencil, i / ny, i % ny, ...) (y, z)
            assert ny == nz
            self.take = [(lambda v, i=i: v[:, i % ny:i % ny + 1, i // ny:i // ny + 1, :]) for i in range(ny * nz)]
            mshape = (1, 1, nx)
        self.members = [StructFactOracle(mshape, nvar, var_scaling, pairs) for _ in self.take]

    @property
    def nsamples(self):
        return self.members[0].nsamples

    def fort_structure(self, variables, reset=0):
        for m, take in zip(self.members, self.take):
            m.fort_structure(take(variables), reset=reset)

    def stack_average(self, zero_avg=1):
        sm = sr = si = 0.0
        for m in self.members:
            re, im, mag = m.finalize(zero_avg)
            sm = sm + mag
            sr = sr + re
            si = si + im
        inv = 1.0 / len(self.members)
        return sm * inv, np.concatenate([sr, si]) * inv
