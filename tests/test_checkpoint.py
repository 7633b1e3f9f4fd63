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
