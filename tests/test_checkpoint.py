"""Checkpoints without a GPU: host MultiFabs written by fhd_write_checkpoint come
back bit for bit through fhd_read_checkpoint, under the reference's file names
(Checkpoint.cpp:172-239), with the restart step = saved step + 1
(Checkpoint.cpp:328-329); mismatched shapes are refused."""
import os

import pytest
import torch

from fhdex_b200.capi import FhdError
from fhdex_b200.checkpoint import read_checkpoint, write_checkpoint
from fhdex_b200.params import mixture4
from fhdex_b200.state import StagState
from fhdex_b200.stats import StatsState


def randomized(p, seed):
    g = torch.Generator().manual_seed(seed)
    st, stats = StagState(p), StatsState(p)
    for m in st.state_mfs() + list(stats.named().values()):
        m.arr.copy_(torch.randn(m.arr.shape, generator=g, dtype=torch.float64))
    return st, stats


def test_checkpoint_round_trip(tmp_path):
    p = mixture4((5, 4, 6), dx=8e-6)
    st, stats = randomized(p, 1)
    base = str(tmp_path / "chk")
    path = write_checkpoint(p, base, 7, 2.5e-10, st, stats, stats_count=7)
    assert path.endswith("chk000000007")
    names = sorted(f[:-2] for f in os.listdir(os.path.join(path, "Level_0")) if f.endswith("_H"))
    want = ["coVars", "cu", "cuMeans", "cuVars", "mom3", "mom4", "prim", "primMeans", "primVars"]
    for stem in ("vel", "velmean", "velvar", "cumom", "cumommean", "cumomvar"):
        want += [stem + c for c in "xyz"]
    assert names == sorted(want)
    assert open(os.path.join(path, "Header")).readline() == "Checkpoint file for FHDeX/compressStag\n"
    st2, stats2 = StagState(p), StatsState(p)
    step, time, count = read_checkpoint(p, base, 7, st2, stats2)
    assert (step, time, count) == (8, 2.5e-10, 7)
    for a, b in zip(st2.state_mfs() + list(stats2.named().values()), st.state_mfs() + list(stats.named().values())):
        assert torch.equal(a.arr, b.arr)


def test_checkpoint_refuses_other_shapes(tmp_path):
    p = mixture4((5, 4, 6), dx=8e-6)
    st, _ = randomized(p, 2)
    base = str(tmp_path / "chk")
    write_checkpoint(p, base, 1, 0.0, st)
    q = mixture4((5, 4, 7), dx=8e-6)
    with pytest.raises(FhdError):
        read_checkpoint(q, base, 1, StagState(q))
    with pytest.raises(FhdError):
        read_checkpoint(p, base, 2, StagState(p))   # no such checkpoint


def test_checkpoint_keeps_spatial_cross_in_the_header(tmp_path):
    """With plot_cross the Header carries spatialCrossVec after the BoxArray, one
    value per line at 16 significant digits (Checkpoint.cpp:112-118), and the
    restart reads those decimal values back (:343-358)."""
    p = mixture4((5, 4, 6), dx=8e-6)
    st, _ = randomized(p, 3)
    stats = StatsState(p, cross=True)
    g = torch.Generator().manual_seed(4)
    stats.spatialCross.copy_(torch.randn(stats.spatialCross.shape, generator=g, dtype=torch.float64) * 1e-7)
    base = str(tmp_path / "chk")
    path = write_checkpoint(p, base, 3, 1e-10, st, stats, stats_count=3)
    lines = open(os.path.join(path, "Header")).read().split("\n")
    end = lines.index(")")
    vals = [v for v in lines[end + 1:] if v]
    want = [f"{v:.16g}" for v in stats.spatialCross.flatten().tolist()]
    assert vals == want
    back = StatsState(p, cross=True)
    step, _, count = read_checkpoint(p, base, 3, StagState(p), back)
    assert (step, count) == (4, 3)
    assert back.spatialCross.flatten().tolist() == [float(v) for v in want]
    # without plot_cross nothing follows the BoxArray
    path = write_checkpoint(p, base, 4, 1e-10, st, StatsState(p), stats_count=3)
    lines = open(os.path.join(path, "Header")).read().split("\n")
    assert not [v for v in lines[lines.index(")") + 1:] if v]


def test_file_failures_are_io_errors(tmp_path):
    """A missing checkpoint or an output directory that cannot be created gives
    FHD_ERR_IO, a checkpoint of other shapes FHD_ERR_BAD_ARG."""
    from fhdex_b200 import capi
    p = mixture4((5, 4, 6), dx=8e-6)
    st, stats = randomized(p, 3)
    base = str(tmp_path / "chk")
    write_checkpoint(p, base, 2, 0.0, st)
    with pytest.raises(FhdError) as e:
        read_checkpoint(p, base, 3, StagState(p))
    assert e.value.code == capi.FHD_ERR_IO
    q = mixture4((5, 4, 7), dx=8e-6)
    with pytest.raises(FhdError) as e:
        read_checkpoint(q, base, 2, StagState(q))
    assert e.value.code == capi.FHD_ERR_BAD_ARG
    blocker = tmp_path / "file"
    blocker.write_text("x")
    with pytest.raises(FhdError) as e:
        write_checkpoint(p, str(blocker / "chk"), 1, 0.0, st)
    assert e.value.code == capi.FHD_ERR_IO
    s = StatsState(p, cross=True)
    with pytest.raises(FhdError) as e:
        s.write_spatial_cross(1, str(blocker) + "/")
    assert e.value.code == capi.FHD_ERR_IO
