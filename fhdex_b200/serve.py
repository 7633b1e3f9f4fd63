"""Ensemble and serving front ends over ``Batch``.

``ensemble``: many independent realisations of one gas (per-member density,
temperature, dt and seed) advanced together.

``Server``: continuous batching of simulation requests.  Requests (box edge,
species count, number of steps, precision) arrive on a Poisson trace; a request
is admitted as soon as its HBM footprint fits the budget, joins the batch of its
(species count, precision) class between two step chunks, and leaves it when its
steps are done.  Each class batch runs on its own CUDA stream, so the classes'
kernels overlap on the device; within a class the members share every launch.
``run_alone`` is the baseline: the same trace served one request at a time with
the plain FP64 step.

A one-species request runs in the reference's parity form of a single gas: two
identical species (the reference cannot run nspecies = 1; its transport routine
aborts on Y = 1).
"""
from __future__ import annotations

import math
import random
import time
from dataclasses import dataclass, field

import torch

from .batch import Batch
from .context import Context
from .params import Params, argon, mixture4, stable_dt
from .state import StagState


@dataclass
class Request:
    rid: int
    arrival: float          # seconds after the start of the trace
    n: int                  # box edge (cells)
    ns: int                 # species count requested (1, 2 or 4)
    steps: int
    precision: int          # 0 FP64, 1 mixed
    seed: int
    # filled by the server
    start: float = math.nan
    finish: float = math.nan
    status: int = 0


def request_params(r: Request, dx=8e-6) -> Params:
    if r.ns in (1, 2):
        return argon(r.n, dx=dx, precision=r.precision, seed=r.seed)
    if r.ns == 4:
        return mixture4(r.n, dx=dx, precision=r.precision, seed=r.seed)
    raise ValueError("nspecies must be 1, 2 or 4")


def poisson_trace(nreq: int, rate: float = 50.0, seed: int = 0, edge=(16, 128), steps=(100, 2000),
                  ns_choices=(1, 2, 4), precisions=(0, 1)) -> list[Request]:
    """Poisson arrivals at `rate`/s; box edge log-uniform in `edge`; species count
    uniform in `ns_choices`; steps uniform in `steps`; precision uniform."""
    rng = random.Random(seed)
    t = 0.0
    out = []
    for q in range(nreq):
        t += rng.expovariate(rate)
        n = int(round(math.exp(rng.uniform(math.log(edge[0]), math.log(edge[1])))))
        out.append(Request(q, t, n, rng.choice(ns_choices), rng.randint(steps[0], steps[1]), rng.choice(precisions),
                           seed=(seed << 20) + q + 1))
    return out


def footprint_bytes(p: Params) -> int:
    """Device bytes of one run: the state MultiFabs plus the batch's stage scratch."""
    n = p.n_cells
    g = [c + 4 for c in n]
    cells_g = g[0] * g[1] * g[2]
    faces_g = sum((g[0] + (d == 0)) * (g[1] + (d == 1)) * (g[2] + (d == 2)) for d in range(3))
    pts = (n[0] + 1) * (n[1] + 1) * (n[2] + 1)
    ns = p.nspecies
    re = 4 if p.precision == 1 else 8
    state = 8 * (cells_g * (p.nvars + p.nprimvars) + 2 * faces_g)
    scratch = (8 * (2 * cells_g * p.nvars + 2 * faces_g + 3 * pts * (2 + ns) + 3 * cells_g + 6 * pts)
               + re * (cells_g * (3 + ns + ns * ns) + 6 * cells_g + 6 * pts))
    return state + scratch


def ensemble(members: int = 512, seed: int = 0, precision: int = 1, sizes=(32, 64), dx=8e-6, device=0):
    """The batched ensemble: `members` realisations of argon, half at each box
    size, T0 ~ U(250, 350) K and rho0 ~ U(1e-3, 3e-3) g/cm^3 drawn from `seed`."""
    rng = random.Random(seed)
    b = Batch(2, precision, device)
    states = []
    cells = 0
    for q in range(members):
        n = sizes[0] if q < members // 2 else sizes[1]
        p = argon(n, dx=dx, precision=precision, seed=(seed << 20) + q + 1,
                  T_init=rng.uniform(250.0, 350.0), rho0=rng.uniform(1e-3, 3e-3))
        st = StagState(p, f"cuda:{device}", aux=False)
        b.add(p, st, stable_dt(p))
        states.append((p, st))
        cells += n ** 3
    return b, states, cells


class Server:
    def __init__(self, device: int = 0, hbm_budget: int | None = None, chunk: int = 20):
        self.device = device
        free, total = torch.cuda.mem_get_info(device)
        self.budget = hbm_budget if hbm_budget is not None else int(0.6 * free)
        self.chunk = chunk
        self.batches: dict = {}

    def _batch(self, ns, precision):
        key = (ns, precision)
        if key not in self.batches:
            self.batches[key] = Batch(ns, precision, self.device)
        return self.batches[key]

    def run(self, trace: list[Request], keep_states: bool = False):
        """Serve `trace` in real time; returns the requests with start/finish filled
        and, when keep_states, {rid: StagState} of the final states."""
        pending = sorted(trace, key=lambda r: r.arrival)
        active = {}      # rid -> (req, batch, mid, remaining, state, bytes)
        used = 0
        finals = {}
        cell_updates = 0
        t0 = time.perf_counter()
        while pending or active:
            now = time.perf_counter() - t0
            # admission: FIFO, as memory frees up
            while pending and pending[0].arrival <= now:
                r = pending[0]
                p = request_params(r)
                fb = footprint_bytes(p)
                if used + fb > self.budget and active:
                    break
                pending.pop(0)
                b = self._batch(p.nspecies, p.precision)
                st = StagState(p, f"cuda:{self.device}", aux=False)
                mid = b.add(p, st, stable_dt(p))
                r.start = time.perf_counter() - t0
                active[r.rid] = [r, b, mid, r.steps, st, fb, p]
                used += fb
            if not active:
                if pending:
                    time.sleep(max(0.0, min(0.005, pending[0].arrival - now)))
                continue
            # one chunk per class batch; classes run concurrently on their streams
            chunks = {}
            for key, b in self.batches.items():
                rem = [v[3] for v in active.values() if v[1] is b]
                if rem:
                    k = min(self.chunk, min(rem))
                    b.step(k, graph=True)
                    chunks[key] = k
            for key, k in chunks.items():
                self.batches[key].synchronize()
            now = time.perf_counter() - t0
            for rid in list(active):
                v = active[rid]
                k = chunks[(v[6].nspecies, v[6].precision)]
                v[3] -= k
                cell_updates += k * v[6].n_cells[0] * v[6].n_cells[1] * v[6].n_cells[2]
                if v[3] <= 0:
                    r, b, mid = v[0], v[1], v[2]
                    r.status = b.status(mid)
                    b.remove(mid)
                    r.finish = now
                    used -= v[5]
                    if keep_states:
                        finals[rid] = v[4]
                    del active[rid]
        elapsed = time.perf_counter() - t0
        return trace, finals, cell_updates, elapsed

    def close(self):
        for b in self.batches.values():
            b.close()
        self.batches = {}


def run_alone(trace: list[Request], device: int = 0, fp64: bool = True):
    """Baseline: the same trace served one request at a time (FIFO) with the plain
    single-run step (FP64 unless fp64=False)."""
    reqs = sorted(trace, key=lambda r: r.arrival)
    t0 = time.perf_counter()
    cell_updates = 0
    ctxs = {}
    for r in reqs:
        now = time.perf_counter() - t0
        if now < r.arrival:
            time.sleep(r.arrival - now)
        p = request_params(r)
        if fp64:
            p = p.replace(precision=0)
        r.start = time.perf_counter() - t0
        ctx = Context(p, device)
        st = StagState(p, f"cuda:{device}", aux=False)
        ctx.init_state(st)
        dt = stable_dt(p)
        for s in range(r.steps):
            ctx.rk3_step(st, dt, s, aux=False)
        torch.cuda.synchronize(device)
        r.status = ctx.status()
        r.finish = time.perf_counter() - t0
        cell_updates += r.steps * p.n_cells[0] * p.n_cells[1] * p.n_cells[2]
        ctx.close()
        del st
    return reqs, cell_updates, time.perf_counter() - t0


def latency_stats(reqs):
    ttc = sorted(r.finish - r.arrival for r in reqs)

    def pct(q):
        if not ttc:
            return math.nan
        i = min(len(ttc) - 1, max(0, int(math.ceil(q * len(ttc))) - 1))
        return ttc[i]

    return {"p50_s": pct(0.50), "p99_s": pct(0.99), "max_s": ttc[-1] if ttc else math.nan, "n": len(ttc)}
