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


@pytest.mark.parametrize("make,flags", [(lambda: argon((5, 4, 3), dx=8e-6), 0),
                                        (lambda: argon((5, 4, 3), dx=8e-6), MEANS | VARS | COVARS | MOM3 | MOM4),
                                        (lambda: mixture4((4, 3, 5), dx=8e-6, visc_type=3, zeta_ratio=1.0),
                                         MEANS | VARS | COVARS | MOM3 | MOM4),
                                        (lambda: mixture4((4, 5, 3), dx=8e-6), MEANS | 32),
                                        (lambda: mixture4((3, 4, 5), dx=8e-6), VARS | 64),
                                        (lambda: argon((5, 3, 4), dx=8e-6), MOM4 | 128)])
def test_restated_composition_and_names_equal_the_references(oracle, make, flags):
    """The reference's own WritePlotFileStag (oracle/_ref, its plotfile MultiFab
    captured before the AMReX writer) on random states and statistics: the
    restated composition (tests/plotfile_reader.py, which the GPU pack is held
    to) and fhd_plotfile_varname's names equal it bit for bit."""
    from oracle import ref as R
    from fhdex_b200.stats import StatsState
    from tests.helpers import perturbed_state
    from tests.plotfile_reader import reference_composition
    if not R.available():
        pytest.skip("oracle/_ref was not built")
    p = make()
    st = perturbed_state(oracle, p, seed=11, amp=0.05)
    stats = StatsState(p)
    g = torch.Generator().manual_seed(12)
    for m in [st.eta, st.kappa, st.zeta] + list(stats.named().values()):
        m.arr.copy_(torch.rand(m.arr.shape, generator=g, dtype=torch.float64) + 0.5)
    data, names = R.plotfile(st, stats, flags, step=7, time=1e-9)
    dy = {32: 0, 64: 1, 128: 2}.get(flags & 224, -1)
    want = reference_composition(p, st, stats, means=bool(flags & MEANS), varz=bool(flags & VARS),
                                 covars=bool(flags & COVARS), mom3=bool(flags & MOM3), mom4=bool(flags & MOM4),
                                 deltay=dy)
    assert names == plotfile_names(p, flags)
    assert np.array_equal(data.numpy(), want)
