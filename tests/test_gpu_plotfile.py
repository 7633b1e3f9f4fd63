"""WritePlotFileStag on the GPU: fhd_plotfile_pack's plotfile MultiFab equals the
reference's composition (writePlotFileStag.cpp:111-281, restated in
tests/plotfile_reader.py) bit for bit: every component is a copy of one source
component, face fields shifted to cells; fhd_write_plotfile_stag writes exactly
that data under the reference's names."""
import numpy as np
import pytest
import torch

from fhdex_b200.context import Context
from fhdex_b200.params import argon, mixture4, stable_dt
from fhdex_b200.plotfile import COVARS, MEANS, MOM3, MOM4, VARS, pack, plotfile_names, write_plotfile_stag
from fhdex_b200.stats import StatsState
from tests.helpers import perturbed_state
from tests.plotfile_reader import read_cell_data, read_header, reference_composition

pytestmark = pytest.mark.gpu

ALL = MEANS | VARS | COVARS | MOM3 | MOM4


def evolved(oracle, p, nsteps=3):
    st = perturbed_state(oracle, p, seed=2).clone(device="cuda")
    ctx = Context(p)
    stats = StatsState(p, "cuda")
    dt = stable_dt(p)
    for s in range(nsteps):
        ctx.rk3_step(st, dt, s, aux=True)
        ctx.stats_stag(st, stats, s + 1, 15)
    torch.cuda.synchronize()
    return ctx, st, stats


@pytest.mark.parametrize("make,flags", [(lambda: argon((6, 5, 4), dx=8e-6), 0),
                                        (lambda: argon((6, 5, 4), dx=8e-6), ALL),
                                        (lambda: mixture4((5, 4, 6), dx=8e-6, visc_type=3, zeta_ratio=1.0), ALL),
                                        (lambda: argon((6, 5, 4), dx=8e-6), ALL | 32),
                                        (lambda: mixture4((7, 5, 6), dx=8e-6), MEANS | 64),
                                        (lambda: mixture4((5, 6, 7), dx=8e-6), 128)])
def test_pack_is_the_references_composition(oracle, make, flags):
    p = make()
    ctx, st, stats = evolved(oracle, p)
    out = pack(ctx, st, stats, flags)
    torch.cuda.synchronize()
    dy = {32: 0, 64: 1, 128: 2}.get(flags & 224, -1)
    want = reference_composition(p, st, stats, means=bool(flags & MEANS), varz=bool(flags & VARS),
                                 covars=bool(flags & COVARS), mom3=bool(flags & MOM3), mom4=bool(flags & MOM4),
                                 deltay=dy)
    got = out.arr.cpu().numpy()
    assert got.shape == want.shape
    assert np.array_equal(got, want)
    assert ctx.status() == 0
    ctx.close()


def test_write_plotfile_stag_writes_the_packed_data(oracle, tmp_path):
    p = mixture4((6, 5, 4), dx=8e-6)
    ctx, st, stats = evolved(oracle, p)
    flags = MEANS | VARS | COVARS
    packed = pack(ctx, st, stats, flags).arr.cpu().numpy()
    path = write_plotfile_stag(ctx, str(tmp_path / "plt"), 3, 1.5e-10, st, stats, flags)
    assert path.endswith("plt000000003")
    h = read_header(path)
    assert h["names"] == plotfile_names(p, flags) and h["step"] == 3 and h["time"] == 1.5e-10
    assert np.array_equal(read_cell_data(path), packed)
    ctx.close()


def test_pack_rejects_pageable_host_memory(oracle):
    """A source in pageable host memory is refused on the host, never read by the kernel."""
    from fhdex_b200.capi import FhdError
    p = argon((4, 4, 4), dx=8e-6)
    ctx, st, _ = evolved(oracle, p, nsteps=1)
    host = st.clone(device="cpu")
    with pytest.raises(FhdError):
        pack(ctx, host, None, 0)
    ctx.close()
