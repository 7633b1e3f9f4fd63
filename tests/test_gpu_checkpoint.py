"""Restart from a checkpoint on the GPU: N steps with statistics, a checkpoint, a
fresh context reading it back into new device MultiFabs, and M more steps equal
N + M uninterrupted steps bit for bit (state and running statistics).  The
in-kernel noise is a function of (seed, step), so the restart step carries the
whole generator state."""
import pytest
import torch

from fhdex_b200.checkpoint import read_checkpoint, write_checkpoint
from fhdex_b200.context import Context
from fhdex_b200.params import argon, no2_dimerization, stable_dt
from fhdex_b200.state import StagState
from fhdex_b200.stats import StatsState
from tests.helpers import compare_named, perturbed_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [lambda: argon((10, 8, 6), dx=8e-6), lambda: no2_dimerization((8, 8, 8), dx=8e-6)])
def test_restart_continues_bitwise(oracle, tmp_path, make):
    p = make()
    dt = stable_dt(p)
    init = perturbed_state(oracle, p, seed=3)
    n1, n2 = 3, 3
    # uninterrupted
    ctx = Context(p)
    a = init.clone(device="cuda")
    sa = StatsState(p, "cuda")
    for s in range(n1 + n2):
        ctx.rk3_step(a, dt, s, aux=False)
        ctx.stats_stag(a, sa, s + 1, 15)
    torch.cuda.synchronize()
    ctx.close()
    # interrupted: checkpoint after step n1 - 1, restart in a fresh context
    ctx = Context(p)
    b = init.clone(device="cuda")
    sb = StatsState(p, "cuda")
    for s in range(n1):
        ctx.rk3_step(b, dt, s, aux=False)
        ctx.stats_stag(b, sb, s + 1, 15)
    torch.cuda.synchronize()
    write_checkpoint(p, str(tmp_path / "chk"), n1 - 1, n1 * dt, b, sb, stats_count=n1)
    ctx.close()
    del b, sb
    ctx = Context(p)
    c = StagState(p, "cuda")
    sc = StatsState(p, "cuda")
    step, time, count = read_checkpoint(p, str(tmp_path / "chk"), n1 - 1, c, sc)
    assert (step, count) == (n1, n1) and time == n1 * dt
    for s in range(step, n1 + n2):
        ctx.rk3_step(c, dt, s, aux=False)
        count += 1
        ctx.stats_stag(c, sc, count, 15)
    torch.cuda.synchronize()
    bad, _ = compare_named(c.named(), a.named())
    assert not bad, bad[:8]
    bad, _ = compare_named(sc.named(), sa.named())
    assert not bad, bad[:8]
    assert ctx.status() == 0
    ctx.close()
