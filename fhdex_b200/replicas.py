"""Replicas across GPUs: one process per GPU, each advancing its own independent
run (the staggered step has no cross-run exchange), with no collective on the
data path.  The only collectives are host-side: a barrier around the timed
region and a MAX-reduction of the per-rank device times, so that the whole-job
rate is (units all ranks processed) / (slowest rank's time).

Every rank takes the same collective steps in the same order; the process group
gets a short timeout so that a rank that never arrives ends the others' wait
with an error instead of a hang.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass

import torch
import torch.distributed as dist

from .params import Params

_GOLDEN = 0x9E3779B97F4A7C15
_MASK64 = (1 << 64) - 1


@dataclass(frozen=True)
class RankEnv:
    world: int
    rank: int
    local: int


def rank_env() -> RankEnv:
    """WORLD_SIZE / RANK / LOCAL_RANK as torchrun sets them (1 / 0 / 0 alone)."""
    return RankEnv(int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                   int(os.environ.get("LOCAL_RANK", "0")))


def init(env: RankEnv, backend: str = "nccl", timeout_s: float = 120.0):
    """Joins the process group when world > 1 (MASTER_ADDR/PORT from the env)."""
    if env.world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, rank=env.rank, world_size=env.world,
                                timeout=datetime.timedelta(seconds=timeout_s))


def finish(env: RankEnv):
    if env.world > 1 and dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()


def replica_params(p: Params, rank: int) -> Params:
    """The run of `rank`: the same gas and box, its own Philox key (the seed
    advanced by rank x the 64-bit golden-ratio constant), so replicas draw
    independent noise.  Rank 0 keeps the seed unchanged."""
    return p.replace(seed=(p.seed + rank * _GOLDEN) & _MASK64)


def barrier(env: RankEnv):
    if env.world > 1:
        dist.barrier()


def max_over_ranks(x: float, env: RankEnv, device=None) -> float:
    """MAX of a per-rank scalar over all ranks (the slowest rank's time)."""
    if env.world == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, env: RankEnv, ms_max: float) -> float:
    """Units processed by all ranks per second of the slowest rank."""
    return units_per_rank * env.world / (ms_max / 1e3)
