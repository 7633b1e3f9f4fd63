"""WritePlotFileStag's variable list and the on-disk plotfile, without a GPU.

The names and their count are the reference's (writePlotFileStag.cpp:37-99,
313-447, restated in tests/plotfile_reader.py); the Header is read back in the
token order of the reference's own post-processing reader
(TURB_PDFS/main.cpp:66-115) and the FAB data round-trips bit for bit.  The
directory layout beyond the Header's leading fields follows AMReX's published
single-level format; no AMReX reader exists here to check it against.
"""
import numpy as np
import pytest
import torch

from fhdex_b200.params import argon, mixture4
from fhdex_b200.plotfile import COVARS, MEANS, MOM3, MOM4, VARS, plotfile_names, write_plotfile_host
from tests.plotfile_reader import read_cell_data, read_cell_h, read_header, reference_names

CASES = [
    (argon(4), 0),
    (argon(4), MEANS | VARS),
    (mixture4((5, 4, 3)), MEANS | VARS | COVARS | MOM3 | MOM4),
    (mixture4((3, 3, 3), visc_type=3, zeta_ratio=1.0), COVARS | MOM4),
    (argon(4), MEANS | 64),
]


@pytest.mark.parametrize("p,flags", CASES)
def test_names_are_the_references(p, flags):
    dy = {32: 0, 64: 1, 128: 2}.get(flags & 224, -1)
    want = reference_names(p, means=bool(flags & MEANS), varz=bool(flags & VARS), covars=bool(flags & COVARS),
                           mom3=bool(flags & MOM3), mom4=bool(flags & MOM4), deltay=dy)
    assert plotfile_names(p, flags) == want


def test_plotfile_round_trip(tmp_path):
    p = mixture4((6, 5, 4), dx=8e-6)
    flags = MEANS | MOM3
    names = plotfile_names(p, flags)
    g = torch.Generator().manual_seed(3)
    data = torch.randn((len(names), 4, 5, 6), generator=g, dtype=torch.float64) * 1e3
    d = str(tmp_path / "plt000000012")
    write_plotfile_host(p, d, data, flags, 3.25e-9, 12)
    h = read_header(d)
    assert h["version"] == "HyperCLaw-V1.1"
    assert h["names"] == names and h["dim"] == 3 and h["finest_level"] == 0
    assert h["time"] == 3.25e-9 and h["level_time"] == 3.25e-9 and h["step"] == 12 and h["level_step"] == 12
    assert h["prob_lo"] == list(p.prob_lo) and h["prob_hi"] == list(p.prob_hi)
    assert h["domain"] == "((0,0,0)(5,4,3)(0,0,0))"
    assert h["dx"] == list(p.dx) and h["nboxes"] == 1 and h["cell_path"] == "Level_0/Cell"
    got = read_cell_data(d)
    assert np.array_equal(got, data.numpy())
    nc, mins, maxs = read_cell_h(d)
    assert nc == len(names)
    assert mins == [float(x) for x in data.reshape(nc, -1).min(1).values]
    assert maxs == [float(x) for x in data.reshape(nc, -1).max(1).values]


def test_bad_flags_are_rejected():
    from fhdex_b200 import capi
    import ctypes as C
    cp = argon(4).to_c()
    assert capi.load().fhd_plotfile_ncomp(C.byref(cp), 256) == -capi.FHD_ERR_BAD_ARG
    assert capi.load().fhd_plotfile_ncomp(C.byref(cp), 32 | 64) == -capi.FHD_ERR_BAD_ARG  # two deltaY directions


def test_plotfile_directory_parents_are_created(tmp_path):
    p = argon((3, 3, 3), dx=8e-6)
    data = torch.zeros((len(plotfile_names(p, 0)), 3, 3, 3), dtype=torch.float64)
    d = str(tmp_path / "runs" / "case1" / "plt000000000")
    write_plotfile_host(p, d, data, 0, 0.0, 0)
    assert read_header(d)["names"] == plotfile_names(p, 0)
