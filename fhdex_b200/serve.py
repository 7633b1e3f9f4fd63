"""Ensemble and serving front ends over ``Batch``.

``ensemble``: many independent realisations of one gas (per-member density,
temperature, dt and seed) advanced together.

``Server``: continuous batching of simulation requests.  Requests (box edge,
species count, number of steps, precision) arrive on a Poisson trace; a request
is admitted as soon as its HBM footprint fits the budget, joins the batch of its
(species count, precision) class between two step chunks, and leaves it when its
steps are done.  Each class batch runs on its own CUDA stream and advances as
soon as its previous chunk has finished, so the classes' kernels overlap on the
device; within a class the members share every launch.  A request whose box
already fills the GPU (``solo_cells``) runs the single-run step on a stream of
its own instead of joining a batch.
``run_alone`` is the baseline: the same trace served one request at a time with
the plain FP64 step.

A one-species request runs the single-gas fast path (nspecies = 1: no species
flux); the reference itself cannot run nspecies = 1 (its transport routine aborts
on Y = 1) and models a single gas as two identical species, which two-species
requests do.
"""
from __future__ import annotations

import math
import random
import time
from dataclasses import dataclass, field

import torch

from .batch import Batch
from .context import Context
from .params import Params, argon, argon_single, mixture4, stable_dt
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
    if r.ns == 1:
        return argon_single(r.n, dx=dx, precision=r.precision, seed=r.seed)
    if r.ns == 2:
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


def warm_kernels(device: int = 0, ns_choices=(1, 2, 4), precisions=(0, 1), n: int = 16):
    """Loads every kernel a served trace can use before anything is timed (CUDA
    loads a kernel's module on its first launch): per (species count, precision)
    one n^3 member through the batched step (graph and direct launches) and one
    single-run step, as the solo lane and the one-at-a-time baseline use."""
    for ns in ns_choices:
        for prec in precisions:
            p = request_params(Request(0, 0.0, n, ns, 1, prec, seed=1))
            dt = stable_dt(p)
            b = Batch(ns, prec, device)
            st = StagState(p, f"cuda:{device}", aux=False)
            b.add(p, st, dt)
            b.step(1, graph=True)
            b.step(1, graph=False)
            b.synchronize()
            b.close()
            ctx = Context(p, device)
            st1 = StagState(p, f"cuda:{device}", aux=False)
            ctx.init_state(st1)
            ctx.rk3_step(st1, dt, 0, aux=False)
            torch.cuda.synchronize(device)
            ctx.close()


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


class _Class:
    """One (species count, precision, size bucket) class: its batch, stream and the
    chunk in flight."""

    def __init__(self, ns, precision, device, priority=-1):
        self.batch = Batch(ns, precision, device)
        # batched requests: higher-priority streams than the solo runs (the smaller
        # the boxes, the higher), so short requests are not held back by long ones
        self.stream = torch.cuda.Stream(device, priority=priority)
        self.batch.set_stream(self.stream)
        self.event = torch.cuda.Event()
        self.inflight = 0          # steps of the chunk in flight (0 = idle)
        self.queue = []            # admitted requests waiting to join: (req, params, state, bytes)
        self.active = {}           # rid -> [req, member id, remaining steps, state, bytes, params]


class _Solo:
    """A request large enough to fill the GPU by itself: the single-run step on a
    stream of its own, advanced in chunks like a class batch."""

    def __init__(self, req, p, st, fb, device):
        self.req, self.p, self.st, self.fb = req, p, st, fb
        self.ctx = Context(p, device)
        self.stream = torch.cuda.Stream(device, priority=0)
        self.event = torch.cuda.Event()
        self.dt = stable_dt(p)
        self.done_steps = 0
        self.inflight = 0

    def launch(self, k):
        with torch.cuda.stream(self.stream):
            self.ctx.rk3_steps(self.st, self.dt, self.done_steps, k)
            self.event.record(self.stream)
        self.inflight = k


class Server:
    """solo_cells: requests with at least this many cells run alone on their own
    stream with the single-run kernels (batching brings nothing to a launch that
    already fills the GPU); smaller ones join the batch of their class (species
    count, precision, size bucket).  small_cells splits the batched requests into
    two size buckets (0: one bucket): a batch advances all its members together, so
    a small box batched with a large one would move at the large one's pace.
    Batched classes run on priority -1 streams (the small bucket on small_priority),
    solo runs on priority 0."""

    def __init__(self, device: int = 0, hbm_budget: int | None = None, chunk: int = 20,
                 solo_cells: int = 96 ** 3, small_cells: int = 40 ** 3, small_priority: int = -3):
        self.device = device
        free, total = torch.cuda.mem_get_info(device)
        self.budget = hbm_budget if hbm_budget is not None else int(0.6 * free)
        self.chunk = chunk
        self.solo_cells = solo_cells
        self.small_cells = small_cells
        self.small_priority = small_priority
        self.classes: dict = {}
        self.solos: list = []

    def _class(self, ns, precision, cells) -> _Class:
        bucket = 0 if cells < self.small_cells else 1
        key = (ns, precision, bucket)
        if key not in self.classes:
            self.classes[key] = _Class(ns, precision, self.device,
                                       priority=self.small_priority if bucket == 0 else -1)
        return self.classes[key]

    def _busy(self):
        return bool(self.solos) or any(c.inflight or c.queue or c.active for c in self.classes.values())

    def run(self, trace: list[Request], keep_states: bool = False):
        """Serve `trace` in real time; returns the requests with start/finish filled,
        {rid: StagState} of the final states (when keep_states), the cell-updates
        done and the elapsed seconds.

        Admission is FIFO by HBM footprint.  Every class batch and every solo run
        advances independently: when its chunk in flight has finished (CUDA event
        query, no blocking), its completed requests leave, the requests admitted
        since join, and the next chunk of min(chunk, fewest remaining steps) steps
        is launched on its stream.  Members join and leave only while their class
        is idle."""
        pending = sorted(trace, key=lambda r: r.arrival)
        used = 0
        finals = {}
        cell_updates = 0
        t0 = time.perf_counter()
        while pending or self._busy():
            now = time.perf_counter() - t0
            # admission: FIFO, as memory frees up
            while pending and pending[0].arrival <= now:
                r = pending[0]
                p = request_params(r)
                fb = footprint_bytes(p)
                if used + fb > self.budget and self._busy():
                    break
                pending.pop(0)
                used += fb
                st = StagState(p, f"cuda:{self.device}", aux=False)
                cells = p.n_cells[0] * p.n_cells[1] * p.n_cells[2]
                if cells >= self.solo_cells:
                    torch.cuda.current_stream(self.device).synchronize()
                    s = _Solo(r, p, st, fb, self.device)
                    s.ctx.init_state(st)
                    torch.cuda.current_stream(self.device).synchronize()
                    r.start = time.perf_counter() - t0
                    self.solos.append(s)
                else:
                    self._class(p.nspecies, p.precision, cells).queue.append((r, p, st, fb))
            progressed = False
            for s in list(self.solos):
                if s.inflight:
                    if not s.event.query():
                        continue
                    n = s.p.n_cells
                    cell_updates += s.inflight * n[0] * n[1] * n[2]
                    s.done_steps += s.inflight
                    s.inflight = 0
                    if s.done_steps >= s.req.steps:
                        s.req.status = s.ctx.status()
                        s.req.finish = time.perf_counter() - t0
                        used -= s.fb
                        if keep_states:
                            finals[s.req.rid] = s.st
                        s.ctx.close()
                        self.solos.remove(s)
                        continue
                s.launch(min(self.chunk, s.req.steps - s.done_steps))
                progressed = True
            for c in self.classes.values():
                if c.inflight:
                    if not c.event.query():
                        continue
                    k, c.inflight = c.inflight, 0
                    t = time.perf_counter() - t0
                    for rid in list(c.active):
                        v = c.active[rid]
                        v[2] -= k
                        n = v[5].n_cells
                        cell_updates += k * n[0] * n[1] * n[2]
                        if v[2] <= 0:
                            r = v[0]
                            r.status = c.batch.status(v[1])
                            c.batch.remove(v[1])
                            r.finish = t
                            used -= v[4]
                            if keep_states:
                                finals[rid] = v[3]
                            del c.active[rid]
                for r, p, st, fb in c.queue:
                    mid = c.batch.add(p, st, stable_dt(p))
                    r.start = time.perf_counter() - t0
                    c.active[r.rid] = [r, mid, r.steps, st, fb, p]
                c.queue = []
                if c.active:
                    k = min(self.chunk, min(v[2] for v in c.active.values()))
                    c.batch.step(k, graph=True)
                    c.event.record(c.stream)
                    c.inflight = k
                    progressed = True
            if not progressed:
                idle = pending and not self._busy()
                nxt = pending[0].arrival - (time.perf_counter() - t0) if idle else 0.0002
                time.sleep(max(0.0, min(0.005, nxt)))
        return trace, finals, cell_updates, time.perf_counter() - t0

    def close(self):
        for c in self.classes.values():
            c.batch.synchronize()
            c.batch.close()
        self.classes = {}


def run_alone(trace: list[Request], device: int = 0, fp64: bool = True):
    """Baseline: the same trace served one request at a time (FIFO) with the plain
    single-run step (FP64 unless fp64=False), its steps replayed from the
    context's CUDA graph (fhd_rk3_steps_stag), the fastest single-run path."""
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
        ctx.rk3_steps(st, dt, 0, r.steps)
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
