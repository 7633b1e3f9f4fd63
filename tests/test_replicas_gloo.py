"""The N > 1 path of the benchmark (replicas, no data-path collective) on CPU:
two gloo ranks take the same collective steps, agree on the slowest rank's time
and on the whole-job rate, and run distinct Philox keys."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from fhdex_b200 import replicas
from fhdex_b200.params import argon


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    env = replicas.rank_env()
    assert (env.world, env.rank) == (world, rank)
    replicas.init(env, "gloo", timeout_s=30)
    replicas.barrier(env)
    ms = 10.0 + 5.0 * rank            # rank 1 is the slow one
    ms_max = replicas.max_over_ranks(ms, env)
    rate = replicas.whole_job_rate(1000 * 4, env, ms_max)
    seed = replicas.replica_params(argon(8, seed=7), rank).seed
    replicas.finish(env)
    out.put((rank, ms_max, rate, seed))


def test_two_gloo_ranks_agree_on_slowest_time_and_rate():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [r[1] for r in res] == [15.0, 15.0]
    assert [r[2] for r in res] == pytest.approx([2 * 4000 / 0.015] * 2)
    assert res[0][3] == 7 and res[1][3] != res[0][3]


def test_single_rank_needs_no_process_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    env = replicas.rank_env()
    assert env.world == 1
    replicas.init(env, "gloo")
    assert replicas.max_over_ranks(3.5, env) == 3.5
    assert replicas.whole_job_rate(100, env, 1000.0) == 100.0
    replicas.finish(env)
