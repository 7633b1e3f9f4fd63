"""MultiFabFillRandomNormal / MultiFabFillRandomUniform (MultiFabFillRandom.cpp:
34-50, 53-66) through the C ABI: moments of the filled values, determinism per
stream id and independence across stream ids and components, OverrideSync
(periodic duplicates of nodal points equal) and FillBoundary (ghosts equal to the
periodic images of valid values)."""
import math

import pytest
import torch

from fhdex_b200.context import Context
from fhdex_b200.fab import MultiFab
from fhdex_b200.params import argon

pytestmark = pytest.mark.gpu

N = 24
CELL, FACEX = (0, 0, 0), (1, 0, 0)


def ctx_and_fab(nodal, ncomp=2, ngrow=2):
    p = argon(N, dx=8e-6, seed=99)
    return Context(p), MultiFab(p.n_cells, nodal, ncomp, ngrow, device="cuda")


def periodic_image(mf):
    """Expected full array: every ghost the periodic image of a valid value, with
    the valid region's low-side nodal point standing for its high-side duplicate."""
    g = mf.ngrow
    full = mf.arr
    out = torch.empty_like(full)
    shape = full.shape[1:]
    idx = []
    for ax, d in ((0, 2), (1, 1), (2, 0)):
        n = N
        i = torch.arange(shape[ax], device=full.device) - g
        idx.append(torch.remainder(i, n) + g)
    out[:] = full[:, idx[0]][:, :, idx[1]][:, :, :, idx[2]]
    return out


@pytest.mark.parametrize("nodal", [CELL, FACEX])
def test_fill_random_normal(nodal):
    ctx, mf = ctx_and_fab(nodal)
    ctx.fill_random_normal(mf, 0, 2, 1.5, 4.0, stream_id=7)
    torch.cuda.synchronize()
    v = mf.valid()
    n = v[0].numel()
    for c in range(2):
        x = v[c].flatten()
        mean, var = x.mean().item(), x.var().item()
        assert abs(mean - 1.5) < 5 * math.sqrt(4.0 / n), (c, mean)
        assert abs(var / 4.0 - 1.0) < 5 * math.sqrt(2.0 / n), (c, var)
    assert torch.corrcoef(torch.stack([v[0].flatten(), v[1].flatten()]))[0, 1].abs().item() < 5 / math.sqrt(n)
    # OverrideSync + FillBoundary: the whole array is the periodic image of the cells 0..N-1
    assert torch.equal(mf.arr, periodic_image(mf))
    # deterministic per stream id, independent across ids
    again = mf.like()
    ctx.fill_random_normal(again, 0, 2, 1.5, 4.0, stream_id=7)
    other = mf.like()
    ctx.fill_random_normal(other, 0, 2, 1.5, 4.0, stream_id=8)
    torch.cuda.synchronize()
    assert torch.equal(again.arr, mf.arr)
    assert not torch.equal(other.valid(), mf.valid())
    ctx.close()


@pytest.mark.parametrize("nodal", [CELL, FACEX])
def test_fill_random_uniform(nodal):
    ctx, mf = ctx_and_fab(nodal)
    ctx.fill_random_uniform(mf, 0, 2, stream_id=3)
    torch.cuda.synchronize()
    v = mf.valid()
    n = v[0].numel()
    assert v.min().item() >= 0.0 and v.max().item() < 1.0
    for c in range(2):
        x = v[c].flatten()
        assert abs(x.mean().item() - 0.5) < 5 * math.sqrt(1.0 / 12.0 / n)
        assert abs(x.var().item() * 12.0 - 1.0) < 0.05
        # 53-bit resolution: no repeated values among the ~1e4 independent draws
        # (the high-side nodal plane duplicates the low side)
        own = v[c][:, :, :N].flatten()
        assert torch.unique(own).numel() == own.numel()
    assert torch.equal(mf.arr, periodic_image(mf))
    again = mf.like()
    ctx.fill_random_uniform(again, 0, 2, stream_id=3)
    other = mf.like()
    ctx.fill_random_uniform(other, 0, 2, stream_id=4)
    torch.cuda.synchronize()
    assert torch.equal(again.arr, mf.arr)
    assert not torch.equal(other.valid(), mf.valid())
    ctx.close()
