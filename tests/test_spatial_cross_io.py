"""WriteSpatialCross3D (writePlotFileStag.cpp:528-549) without a GPU: the text
file spatialCross<step, 9 digits> written by fhd_write_spatial_cross from host
memory, one line per x cell with the cell centre and the ncross entries in the
reference's stream formatting (the first centre at the default 6 significant
digits, every later number at 16, each followed by a space), and the crossMeans
rows (main_driver.cpp:1284-1288)."""
import os

import torch

from fhdex_b200.params import argon, mixture4
from fhdex_b200.stats import StatsState, ncross, nstats


def test_spatial_cross_file_format(tmp_path):
    p = mixture4((6, 3, 4), dx=8e-6).replace(prob_lo=(1e-5, 0.0, 0.0), prob_hi=(1e-5 + 4.8e-5, 2.4e-5, 3.2e-5))
    s = StatsState(p, cross=True)
    g = torch.Generator().manual_seed(5)
    s.spatialCross.copy_(torch.randn(s.spatialCross.shape, generator=g, dtype=torch.float64))
    s.write_spatial_cross(12, str(tmp_path) + "/")
    text = open(tmp_path / "spatialCross000000012").read()
    h = (p.prob_hi[0] - p.prob_lo[0]) / p.n_cells[0]
    want = ""
    for i in range(p.n_cells[0]):
        x = p.prob_lo[0] + (i + 0.5) * h
        want += (f"{x:g} " if i == 0 else f"{x:.16g} ")
        want += "".join(f"{v:.16g} " for v in s.spatialCross[i].tolist()) + "\n"
    assert text == want
    assert s.spatialCross.shape == (6, ncross(4)) and ncross(4) == 44


def test_cross_means_rows(tmp_path):
    p = argon((4, 3, 3), dx=8e-6)
    s = StatsState(p, cross=True)
    assert s.dataSliceMeans_xcross.numel() == nstats(2) == 26
    s.dataSliceMeans_xcross.copy_(torch.arange(26, dtype=torch.float64) * 1.2345678e-3 + 1.0)
    path = str(tmp_path / "crossMeans")
    s.append_cross_means(path, 100)
    s.append_cross_means(path, 200)
    rows = open(path).read().split("\n")
    assert rows[0].startswith("100 1 1.00123 1.00247 ") and rows[0].endswith(" ")
    assert rows[1].startswith("200 ") and rows[2] == "" and len(rows[0].split()) == 27
    assert os.path.getsize(path) > 0


def test_spatial_cross_file_equals_the_references(tmp_path, monkeypatch):
    """fhd_write_spatial_cross against the reference's own WriteSpatialCross3D
    (oracle/_ref), byte for byte."""
    from oracle import ref as R
    if not R.available():
        import pytest
        pytest.skip("oracle/_ref was not built")
    p = mixture4((7, 3, 4), dx=8e-6).replace(prob_lo=(-2e-5, 0.0, 0.0), prob_hi=(-2e-5 + 5.6e-5, 2.4e-5, 3.2e-5))
    s = StatsState(p, cross=True)
    g = torch.Generator().manual_seed(9)
    s.spatialCross.copy_(torch.randn(s.spatialCross.shape, generator=g, dtype=torch.float64) * 1e-9)
    s.spatialCross[2, 5] = 0.0
    s.spatialCross[3, 7] = 1.0
    mine, theirs = tmp_path / "mine", tmp_path / "ref"
    mine.mkdir()
    theirs.mkdir()
    s.write_spatial_cross(40, str(mine) + "/")
    monkeypatch.chdir(theirs)
    R.write_spatial_cross(p, s.spatialCross, 40)
    name = "spatialCross000000040"
    assert (mine / name).read_bytes() == (theirs / name).read_bytes()
