#!/usr/bin/env python
"""Benchmark of the compressible staggered FHD RK3 step (cell-updates/s).

Workload (default): 'single-species' argon in the reference's parity form (two
identical species), 256^3 cells, dx = 8e-6 cm (the reference decks' spacing; at
dx = 1e-6 cm a cell holds ~27 molecules and the reference's own mass-fraction
guard trips after the first step), fully periodic, FP64, in-kernel Philox
noise, dt from the acoustic + diffusive stability rule.  One step = one
SSP-RK3 step of the whole box.  value = cells * steps * ranks / max-over-ranks
device time; e2e = the same metric through the host-buffer C-ABI call
(fhd_rk3_step_stag_host: H2D of cu and mom from pinned memory, step, D2H of
cu, mom, prim and vel).

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
                  [--n 256] [--ns 1|2|4] [--precision fp64|mixed] [--tile auto|<idx>]
                  [--mode step|ensemble|serve|stats|sf]

--ns 1 is the single-gas fast path (no CPU baseline: the reference cannot run
one species).  The other modes time the batched ensemble, the continuous-
batching server, the running statistics and the structure factor.

N > 1 runs one independent replica per GPU (weak scaling, no data-path
collective; the runs do not exchange data).  --impl reference times the
reference's own CPU implementation of the step (FHDeX's sources compiled
unmodified into oracle/_ref), one process per host core, on a bounded sample of
the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

try:
    _CORES = len(os.sched_getaffinity(0))
except AttributeError:  # pragma: no cover
    _CORES = os.cpu_count() or 1
os.environ.setdefault("OMP_NUM_THREADS", str(_CORES))

HBM_FALLBACK_GBS = 6650.0
METRIC = "cell-updates/s (RK3 steps x cells)"
UNIT = "cell-updates/s"

# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one RK stage
# (k_cellprep + k_taus + 3 x k_faces + k_update) per cell, keyed
# "nspecies:precision": ncu, 128^3, one full timed step captured, scaled to the
# box by the cell count (every operand exceeds L2 at both sizes).  Absent for
# configurations not captured.
STAGE_TRAFFIC_BYTES_PER_CELL = {"2:fp64": 1592.1, "2:mixed": 1232.5}
# DRAM traffic of one statistics update per cell (all flags), keyed "nspecies":
# ncu, 128^3, the three statistics kernels captured, scaled by the cell count.
STATS_TRAFFIC_BYTES_PER_CELL = {"2": 1639.1}
# FP64 flops of one RK stage per cell (dadd + dmul + 2 x dfma thread instructions
# of k_cellprep, k_taus, 3 x k_faces and k_update; ncu at 128^3, divided by the
# cells), keyed "nspecies:precision".
STAGE_FP64_FLOPS_PER_CELL = {"2:fp64": 3042.4}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def make_params(args):
    from fhdex_b200.params import argon, argon_single, mixture4, no2_dimerization
    prec = 1 if args.precision == "mixed" else 0
    if args.gas == "no2":
        p = no2_dimerization(args.n, dx=args.dx, precision=prec, seed=args.seed)
    elif args.ns == 1:
        p = argon_single(args.n, dx=args.dx, precision=prec, seed=args.seed)
    elif args.ns == 2:
        p = argon(args.n, dx=args.dx, precision=prec, seed=args.seed)
    elif args.ns == 4:
        p = mixture4(args.n, dx=args.dx, precision=prec, seed=args.seed)
    else:
        raise SystemExit("--ns must be 1 (single gas), 2 (argon parity form) or 4 (mixture)")
    p = with_bench_walls(p, getattr(args, "walls", "none"))
    # quasi-1-D / 2-D runs and the other transport models take the reference-ordered pipeline
    mode = getattr(args, "lowdim", "none")
    if mode != "none":
        p = p.replace(do_1D=int(mode == "1d"), do_2D=int(mode == "2d"))
    model = getattr(args, "transport", "gio")
    if model != "gio":
        p = p.replace(transport_type={"vw": 2, "hcb": 3}[model])
    return p


def with_bench_walls(p, kind):
    """The boundary set-ups of the reference's regression runs on the bench box:
    tempgrad (no-slip isothermal x walls at 0.9 / 1.1 T0, slip adiabatic y and z
    walls, all impermeable) and reservoir (reservoirs of the initial composition
    on all six sides, no-slip, at 0.95 / 1.05 T0)."""
    from fhdex_b200.params import with_walls
    if kind == "tempgrad":
        slip = dict(vel=1, therm=1, mass=1)
        return with_walls(p, x=dict(vel=2, therm=2, mass=1, t=(0.9 * p.T_init, 1.1 * p.T_init)), y=slip, z=slip)
    if kind == "reservoir":
        y = tuple(p.rhobar[:p.nspecies])
        res = dict(vel=2, therm=2, mass=3, t=(0.95 * p.T_init, 1.05 * p.T_init), Yk=(y, y))
        return with_walls(p, x=res, y=res, z=res)
    return p


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_oracle_rate(p, target_s=15.0, max_n=None, threads=0):
    """Oracle (CPU restatement of the reference step, OpenMP over `threads` host
    cores, 0 = all) on a bounded sample: a smaller box of the same gas, enough
    steps for about target_s seconds.  Returns (cell-updates/s, sample description)."""
    from oracle import oracle as O
    from fhdex_b200.params import stable_dt
    from fhdex_b200.state import StagState, StepNoise
    O.build()
    O.set_threads(threads)
    n = min(64, p.n_cells[0]) if max_n is None else max_n
    q = p.replace(n_cells=(n, n, n), prob_hi=tuple(p.dx[0] * n for _ in range(3)))
    st = StagState(q)
    O.init_state(st, q)
    dt = stable_dt(p)
    nz = StepNoise(q)
    O.fill_step_noise(nz, q.seed, 0)
    t = time.perf_counter()
    O.rk3_step(st, nz, dt)  # calibration step (not counted)
    one = time.perf_counter() - t
    steps = max(1, int(target_s / max(one, 1e-3)))
    t = time.perf_counter()
    for s in range(steps):
        O.fill_step_noise(nz, q.seed, s + 1)  # the reference fills its A/B noise every step
        rc = O.rk3_step(st, nz, dt)
        assert rc == 0
    el = time.perf_counter() - t
    O.set_threads(0)
    return n ** 3 * steps / el, f"{n}^3 box of the same gas, {steps} RK3 steps incl. per-step noise fill, {el:.1f} s"


def _ref_worker(p, n, warmup, steps, rank, barrier, out_q):
    """One host process advancing its own n^3 box of p's gas with the reference's
    own RK3stepStag (oracle/_ref: FHDeX's sources compiled unmodified); each timed
    step includes the step's A/B noise generation (in the reference, its 24
    MultiFabFillRandomNormal calls)."""
    try:
        from oracle import oracle as O
        from oracle import ref as R
        from fhdex_b200.params import stable_dt
        from fhdex_b200.state import StagState, StepNoise
        O.set_threads(1)
        q = p.replace(n_cells=(n, n, n), prob_hi=tuple(p.dx[0] * n for _ in range(3)), seed=p.seed + rank)
        st = StagState(q)
        R.init_cons_var_stag(st)
        R.conserved_to_primitive(st)
        for m in [st.cu, st.prim] + st.cumom + st.vel:
            O.fill_boundary(m)
        nz = StepNoise(q)
        dt = stable_dt(q)
        for s in range(warmup):
            O.fill_step_noise(nz, q.seed, s)
            R.rk3_step(st, nz, dt, s)
        barrier.wait(timeout=600)
        t = time.perf_counter()
        for s in range(steps):
            O.fill_step_noise(nz, q.seed, warmup + s)
            R.rk3_step(st, nz, dt, warmup + s)
        out_q.put((rank, time.perf_counter() - t, None))
    except Exception as e:  # reported to the parent
        out_q.put((rank, None, repr(e)))


def reference_rate(p, procs, warmup, steps, step_budget_s):
    """cell-updates/s of the reference's own CPU code (oracle/_ref) on `procs`
    host processes at once, each advancing its own box of p's gas (the
    reference's hot path has no OpenMP and scales by one rank per core; the
    processes exchange nothing, so their halo exchange is not counted).  The box
    edge n is chosen so that one step of one process takes about step_budget_s.
    Returns (rate, n, description), or None when oracle/_ref is absent."""
    import multiprocessing as mp
    from oracle import oracle as O
    from oracle import ref as R
    from fhdex_b200.params import stable_dt
    from fhdex_b200.state import StagState, StepNoise
    if not R.available():
        R.build()
    if not R.available():
        return None
    O.build()
    # calibrate: one reference step of a 24^3 box in this process
    n0 = 24
    q = p.replace(n_cells=(n0, n0, n0), prob_hi=tuple(p.dx[0] * n0 for _ in range(3)))
    st = StagState(q)
    R.init_cons_var_stag(st)
    R.conserved_to_primitive(st)
    for m in [st.cu, st.prim] + st.cumom + st.vel:
        O.fill_boundary(m)
    nz = StepNoise(q)
    O.set_threads(1)
    O.fill_step_noise(nz, q.seed, 0)
    t = time.perf_counter()
    R.rk3_step(st, nz, stable_dt(q), 0)
    per_cell = (time.perf_counter() - t) / n0 ** 3
    n = int((step_budget_s / per_cell) ** (1.0 / 3.0))
    n = max(16, min(p.n_cells[0], (n // 4) * 4))
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(procs)
    out_q = ctx.Queue()
    ps = [ctx.Process(target=_ref_worker, args=(p, n, warmup, steps, r, barrier, out_q)) for r in range(procs)]
    for pr in ps:
        pr.start()
    res = [out_q.get(timeout=1800) for _ in range(procs)]
    for pr in ps:
        pr.join(timeout=60)
    errs = [e for _, _, e in res if e]
    if errs:
        raise RuntimeError(f"reference worker failed: {errs[0]}")
    el = max(t for _, t, _ in res)
    rate = procs * n ** 3 * steps / el
    desc = (f"{procs} host processes at once, each one {n}^3 box of the same gas advanced by the reference's own "
            f"RK3stepStag (FHDeX sources compiled unmodified, oracle/_ref), {steps} timed steps each incl. the "
            f"step's A/B noise generation, {el:.1f} s")
    return rate, n, desc


def run_reference(args):
    """--impl reference: the reference's own CPU implementation of the step
    (oracle/_ref) on all host cores, rank 0 only; each step is a bounded sample
    of the workload (one box per core).  Falls back to the oracle restatement
    when oracle/_ref is absent."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    p = make_params(args)
    from fhdex_b200.params import stable_dt
    dt = stable_dt(p)
    budget = 100.0 / max(1, args.steps + args.warmup)
    r = reference_rate(p, _CORES, args.warmup, args.steps, budget) if p.nspecies > 1 else None
    if r is not None:
        val, n, sample = r
        kind = "reference"
        ms = 1e3 * (_CORES * n ** 3) / val
    else:
        val, sample = cpu_oracle_rate(p, target_s=60.0)
        kind = "port"
        ms = None
    out = {
        "metric": METRIC, "value": val, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(args, p, dt, None),
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": _CORES, "kind": kind, "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def config_dict(args, p, dt, tile):
    return {
        "workload": (("2 NO2 <-> N2O4 (chemistry source, CLE)" if p.nreaction > 0 else
                      {1: "argon (single gas)", 2: "argon (2 identical species)"}.get(p.nspecies, "4-species mixture"))
                     + f" {p.n_cells[0]}^3, dx={p.dx[0]:g} cm, {'periodic' if getattr(args, 'walls', 'none') == 'none' else args.walls + ' walls'}, {args.precision}, in-kernel Philox noise"
                     + ("" if getattr(args, "lowdim", "none") == "none" else f", quasi-{args.lowdim[0]}-D run")
                     + ("" if getattr(args, "transport", "gio") == "gio" else
                        {"vw": ", Valk/Waldmann transport", "hcb": ", HCB binary transport"}[args.transport])),
        "n_cells": list(p.n_cells), "nspecies": p.nspecies, "precision": args.precision, "dt_s": dt,
        "noise": "philox-4x32-10 in kernel", "tile": tile,
        "l2": "inputs larger than L2 (state ~%.1f GB)" % (state_gb(p)),
        "parallelism": f"replicas x{args.gpus}",
    }


def state_gb(p):
    n = [c + 4 for c in p.n_cells]
    cells = n[0] * n[1] * n[2]
    return (p.nvars + p.nprimvars + 6) * cells * 8 / 1e9


def autotune(ctx, st, dt, steps=2):
    """Own tile autotuner: time each tile shape of the fused stage kernel on this
    problem and keep the fastest."""
    import torch
    from fhdex_b200.context import Context
    best = None
    table = {}
    for t, name in enumerate(Context.tiles()):
        ctx.set_tile(t)
        ctx.rk3_step(st, dt, 0, aux=False)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for s in range(steps):
            ctx.rk3_step(st, dt, s, aux=False)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        table[name] = round(ms, 3)
        if best is None or ms < best[1]:
            best = (t, ms, name)
    ctx.set_tile(best[0])
    return best[0], best[1], best[2], table


def fma_peaks(device):
    """FP64 / FP32 FMA throughput of this GPU, measured now (fhd_measure_fma_peak),
    with the committed measurement (MEASURED_FMA.json) beside it."""
    from fhdex_b200.peaks import measure_fma_peaks
    try:
        live = measure_fma_peaks(device)
    except Exception as e:  # pragma: no cover - reported, not fatal
        live = {"error": repr(e)}
    committed = None
    try:
        with open(os.path.join(ROOT, "MEASURED_FMA.json")) as f:
            committed = json.load(f)
    except Exception:
        pass
    return live, committed


def step_extras(args, p, dt, local, peak, peak_kind):
    """The forms the benchmark's metric compares, measured in the same call after
    the headline step (untimed for the headline): the 256^3 step in the mixed
    precision, the FP64 step with its by-products (aux), the batched ensemble and
    the continuous-batching server, each against the plain FP64 one-at-a-time
    path of the same call, and the batched mixed form's equilibrium variances."""
    import torch
    from fhdex_b200.context import Context
    from fhdex_b200.state import StagState
    out = {}
    cells = p.n_cells[0] * p.n_cells[1] * p.n_cells[2]
    S = 5 + p.nspecies

    def timed(ctx, st, nsteps, aux=False):
        for s in range(2):
            ctx.rk3_step(st, dt, s, aux=aux)
        torch.cuda.synchronize()
        ctx.profile(True)
        ctx.profile_read()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for s in range(nsteps):
            ctx.rk3_step(st, dt, 2 + s, aux=aux)
        e1.record()
        torch.cuda.synchronize()
        prof = ctx.profile_read()
        ctx.profile(False)
        return e0.elapsed_time(e1) / nsteps, prof

    # the same step with the by-products RK3stepStag writes (coefficients, fluxes)
    ctx = Context(p, local)
    st = StagState(p, f"cuda:{local}", aux=True)
    ctx.init_state(st)
    t, _, tname, _ = autotune(ctx, st, dt)
    ms_aux, _ = timed(ctx, st, 3, aux=True)
    out["aux_true"] = {"ms_per_step": ms_aux, "value": cells / (ms_aux / 1e3), "tile": tname,
                       "writes": "stage-3 eta, zeta, kappa, chi, D, face/edge/centre fluxes (the reference's "
                                 "RK3stepStag outputs besides the state)"}
    ctx.close()
    del st
    torch.cuda.empty_cache()

    # the mixed-precision step on the same box
    pm = p.replace(precision=1)
    ctx = Context(pm, local)
    st = StagState(pm, f"cuda:{local}", aux=False)
    ctx.init_state(st)
    t, _, tname, _ = autotune(ctx, st, dt)
    ms_mx, prof = timed(ctx, st, max(3, min(args.steps, 10)))
    stage_ms = sum(prof[k][0] for k in ("cellprep", "taus", "faces", "update", "fused"))
    nst = max(prof["taus"][1] + prof["fused"][1], 1)
    ach = (2 + 3 + 3) / 3.0 * S * 8 * cells / (stage_ms / 1e3 / nst) / 1e9
    out["mixed"] = {"ms_per_step": ms_mx, "value": cells / (ms_mx / 1e3), "tile": tname,
                    "dtype": "f32 fluxes/coefficients + f64 state", "status": ctx.status(),
                    "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                 "peak_kind": peak_kind, "kernel_ms_per_launch": stage_ms / nst}}
    ctx.close()
    del st
    torch.cuda.empty_cache()

    # batched ensemble (reduced: --members members x --bench-batch-steps steps)
    from fhdex_b200.params import stable_dt
    from fhdex_b200.serve import ensemble, latency_stats, poisson_trace, run_alone, Server, warm_kernels
    nb = args.bench_batch_steps
    batched = {"config": {"members": args.members, "sizes": "half 32^3, half 64^3", "gas": "argon (2 species)",
                          "T0": "U(250, 350) K", "rho0": "U(1e-3, 3e-3) g/cm^3", "steps": nb,
                          "launch": "fp64 / mixed: 23 batched kernels per step, one CUDA graph replay per step; "
                                    "*_persistent: one persistent launch per step (k_batch_persist), graph replay"}}
    members = None
    for prec, key in ((0, "fp64"), (1, "mixed")):
        b, states, bcells = ensemble(args.members, seed=args.seed, precision=prec)
        members = [q for q, _ in states]
        s_ = torch.cuda.Stream(local)
        b.set_stream(s_)
        for form in ("", "_persistent"):
            b.set_persistent(form == "_persistent")
            b.step(3, graph=True)
            b.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(s_):
                e0.record()
            b.step(nb, graph=True)
            with torch.cuda.stream(s_):
                e1.record()
            b.synchronize()
            ms = e0.elapsed_time(e1)
            bad = sum(1 for mid in list(b.members) if b.status(mid) != 0)
            batched[key + form] = {"value": bcells * nb / (ms / 1e3), "ms_per_step": ms / nb,
                                   "members_with_status": bad}
        b.close()
        del states
        torch.cuda.empty_cache()
    # the plain FP64 path, one member at a time (graph replay of its own step)
    tot = 0.0
    acells = 0
    for q in members:
        q = q.replace(precision=0)
        c = Context(q, local)
        st = StagState(q, f"cuda:{local}", aux=False)
        c.init_state(st)
        qdt = stable_dt(q)
        c.rk3_steps(st, qdt, 0, 1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        c.rk3_steps(st, qdt, 1, nb)
        torch.cuda.synchronize()
        tot += time.perf_counter() - t0
        acells += q.n_cells[0] * q.n_cells[1] * q.n_cells[2]
        c.close()
        del st
    batched["alone_fp64"] = {"value": acells * nb / tot, "elapsed_s": tot,
                             "path": "each member alone: fhd_rk3_steps_stag (graph replay), FP64, one after another"}
    from fhdex_b200.equilibrium import batch_variance_ratios
    ratios, m = batch_variance_ratios(members=8, precision=1, dt_scale=0.5, warm=2000, every=10)
    batched["equilibrium_mixed"] = {"members": 8, "n": 32, "dt": "stable_dt/2", "samples_per_field": m,
                                    "variance_over_theory": {k: round(v, 5) for k, v in ratios.items()},
                                    "max_abs_error": round(max(abs(v - 1.0) for v in ratios.values()), 5)}
    out["batched"] = batched

    # continuous-batching server against one request at a time (plain FP64)
    warm_kernels(local)
    steps = (args.serve_min_steps, args.bench_serve_max_steps)
    trace = poisson_trace(args.bench_requests, rate=args.rate, seed=args.seed, steps=steps)
    srv = Server(device=local, chunk=args.chunk)
    reqs, _, cu_b, el_b = srv.run(trace)
    srv.close()
    torch.cuda.empty_cache()
    trace2 = poisson_trace(args.bench_requests, rate=args.rate, seed=args.seed, steps=steps)
    reqs2, cu_a, el_a = run_alone(trace2, device=local)
    out["served"] = {
        "config": {"requests": args.bench_requests, "arrivals": f"Poisson, {args.rate:g} per s",
                   "box_edge": "log-uniform 16-128", "nspecies": "{1, 2, 4}", "steps": f"U{{{steps[0]}..{steps[1]}}}",
                   "precision": "FP64 or mixed per request", "chunk_steps": args.chunk},
        "served": {"value": cu_b / el_b, "elapsed_s": el_b, **latency_stats(reqs),
                   "bad_status": sum(1 for r in reqs if r.status)},
        "alone_fp64": {"value": cu_a / el_a, "elapsed_s": el_a, **latency_stats(reqs2),
                       "bad_status": sum(1 for r in reqs2 if r.status)},
    }
    return out


def run_ours(args):
    import torch
    from fhdex_b200.context import Context
    from fhdex_b200.params import stable_dt
    from fhdex_b200.state import StagState

    from fhdex_b200 import replicas
    env = replicas.rank_env()
    world, rank, local = env.world, env.rank, env.local
    torch.cuda.set_device(local)
    replicas.init(env, "nccl")
    # replicas: every rank advances its own run (own Philox key), no data-path collective
    p = replicas.replica_params(make_params(args), rank)
    dt = stable_dt(p)
    ctx = Context(p, local)
    st = StagState(p, f"cuda:{local}", aux=False)
    ctx.init_state(st)
    tune = None
    if args.tile == "auto":
        t, ms, tname, tune = autotune(ctx, st, dt)
    else:
        ctx.set_tile(int(args.tile))
        tname = Context.tiles()[int(args.tile)]
    for s in range(args.warmup):
        ctx.rk3_step(st, dt, s, aux=False)
    torch.cuda.synchronize()
    ctx.profile(True)
    ctx.profile_read()
    clocks = ClockSampler(local)
    replicas.barrier(env)
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for s in range(args.steps):
        ctx.rk3_step(st, dt, args.warmup + s, aux=False)
    e1.record()
    torch.cuda.synchronize()
    replicas.barrier(env)
    clk = clocks.stop()
    prof = ctx.profile_read()
    ctx.profile(False)
    ms = e0.elapsed_time(e1)
    status = ctx.status()
    ms = replicas.max_over_ranks(ms, env, device=f"cuda:{local}")
    cells = p.n_cells[0] * p.n_cells[1] * p.n_cells[2]
    value = replicas.whole_job_rate(cells * args.steps, env, ms)
    # every bracketed profile scope is one launch, except the face-flux scope (3 launches)
    launches = sum(v[1] for v in prof.values()) + 2 * prof["faces"][1]
    if p.nreaction > 0:  # k_chem runs inside each stage's cellprep scope
        launches += prof["cellprep"][1]

    # roofline of the dominant kernel group: one RK stage = k_cellprep + k_taus +
    # 3 x k_faces + k_update (conversion, transport coefficients, calculateFluxStag
    # and the stage update of the reference).
    # Algorithmic bytes per stage: the conserved state S = 5 + nspecies doubles per
    # cell read once (stage 1) or twice (U^s and U^0, stages 2-3) and written once;
    # averaged over the three stages: (2 + 3 + 3)/3 * S * 8 bytes per cell.
    S = 5 + p.nspecies
    stage_ms = prof["cellprep"][0] + prof["taus"][0] + prof["faces"][0] + prof["update"][0] + prof["fused"][0]
    nstages = max(prof["taus"][1] + prof["fused"][1], 1)
    avg_stage_s = stage_ms / 1e3 / nstages
    alg_bytes = (2 + 3 + 3) / 3.0 * S * 8 * cells
    peak, peak_kind = measured_peak()
    achieved = alg_bytes / avg_stage_s / 1e9
    key = f"{p.nspecies}:{args.precision}"
    traffic = None if prof["fused"][1] else STAGE_TRAFFIC_BYTES_PER_CELL.get(key)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic * cells if traffic else None, "peak_kind": peak_kind,
            "traffic_source": "ncu, 128^3, one timed step, per cell, scaled to this box" if traffic else None,
            "traffic_gbs": traffic * cells / avg_stage_s / 1e9 if traffic else None,
            "kernel": ("RK stage (k_cellprep + k_stage_zm), per stage" if prof["fused"][1] else
                       "RK stage (k_cellprep + k_taus + 3x k_faces + k_update), per stage"),
            "kernel_ms_per_launch": 1e3 * avg_stage_s,
            "algorithmic_bytes_per_launch": alg_bytes,
            "step_breakdown_ms": {k: v[0] / args.steps for k, v in prof.items()}}

    # the same steps replayed from a CUDA graph the context captures once
    # (fhd_rk3_steps_stag): what small, launch-bound boxes gain
    side = torch.cuda.Stream(local)
    with torch.cuda.stream(side):
        ctx.rk3_steps(st, dt, args.warmup + args.steps, 1)   # capture + one untimed replay
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record()
        ctx.rk3_steps(st, dt, args.warmup + args.steps + 1, args.steps)
        g1.record()
    side.synchronize()
    gms = replicas.max_over_ranks(g0.elapsed_time(g1), env, device=f"cuda:{local}")
    graph = {"ms_per_step": gms / args.steps, "value": replicas.whole_job_rate(cells * args.steps, env, gms),
             "path": "fhd_rk3_steps_stag (one captured step replayed per step)"}

    # the chemistry kernel alone (fhd_chemistry_source_cle on the state's prim):
    # reads T, p and X (2 + ns doubles) and the nreaction noises, writes ns doubles
    chem = None
    if p.nreaction > 0:
        from fhdex_b200.fab import CELL, MultiFab
        src = MultiFab(p.n_cells, CELL, p.nvars, 0, device=f"cuda:{local}")
        W = MultiFab(p.n_cells, CELL, p.nreaction, 0, device=f"cuda:{local}")
        ctx.fill_random_normal(W, 0, p.nreaction, 0.0, 1.0, overridesync=False, fillboundary=False, stream_id=5)
        dV = p.dx[0] * p.dx[1] * p.dx[2]
        for _ in range(3):
            ctx.chemistry_source_cle(st.prim, src, W, dt, dV)
        reps = 20
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        cs = torch.cuda.current_stream(local)
        c0.record(cs)
        for _ in range(reps):
            ctx.chemistry_source_cle(st.prim, src, W, dt, dV)
        c1.record(cs)
        torch.cuda.synchronize()
        cms = c0.elapsed_time(c1) / reps
        cbytes = 8.0 * cells * (2 + p.nspecies + p.nreaction + p.nspecies)
        chem = {"kernel": "k_chem (fhd_chemistry_source_cle)", "ms_per_launch": cms,
                "algorithmic_bytes_per_launch": cbytes, "achieved_gbs": cbytes / cms / 1e6,
                "frac": cbytes / cms / 1e6 / peak, "peak": peak, "peak_kind": peak_kind,
                "note": "in the step it runs once per stage inside the cellprep scope (in-kernel noise: no W reads)"}
        del src, W

    # e2e through the host-buffer C-ABI call (H2D + step + D2H, pinned memory)
    ctx.close()
    del st
    torch.cuda.empty_cache()
    e2e = None
    if not args.no_e2e:
        ctx = Context(p, local)
        hs = StagState(p, "cpu", aux=False, pin_memory=True)
        tmp = StagState(p, f"cuda:{local}", aux=False)
        ctx.init_state(tmp)
        torch.cuda.synchronize()
        hs.copy_from(tmp)
        del tmp
        torch.cuda.empty_cache()
        ctx.rk3_step_host(hs, dt, 0)  # warm
        ne = max(2, min(args.steps, 5))
        replicas.barrier(env)
        t = time.perf_counter()
        for s in range(ne):
            h2d, d2h = ctx.rk3_step_host(hs, dt, 1 + s)
        el = replicas.max_over_ranks(time.perf_counter() - t, env, device=f"cuda:{local}")
        e2e = {"value": replicas.whole_job_rate(cells * ne, env, 1e3 * el), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "steps": ne, "path": "fhd_rk3_step_stag_host (pinned host fabs)"}
        ctx.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and p.nspecies > 1:
        r = reference_rate(p, _CORES, 1, 2, 6.0)
        if r is not None:
            v, _, sample = r
            v1, _, sample1 = reference_rate(p, 1, 1, 2, 4.0)
            kind = "reference"
        else:
            v, sample = cpu_oracle_rate(p)
            v1, sample1 = cpu_oracle_rate(p, target_s=8.0, max_n=32, threads=1)
            kind = "port"
        cpu = {"value": v, "unit": UNIT, "cores": _CORES, "kind": kind, "sample": sample,
               "single_core": {"value": v1, "unit": UNIT, "cores": 1, "sample": sample1}}

    extras = None
    fma = None
    if rank == 0 and world == 1:
        fma_live, fma_file = fma_peaks(local)
        fma = {"measured_now": fma_live, "committed": fma_file}
        if not args.no_extras:
            extras = step_extras(args, p, dt, local, peak, peak_kind)
    replicas.finish(env)
    if rank != 0:
        return
    if fma and "fp64_tflops" in fma["measured_now"]:
        # FP64 denominator: FP64 flops per cell per stage counted by ncu (dadd +
        # dmul + 2 dfma, split pipeline, argon, in-kernel noise), over the stage time
        fl = STAGE_FP64_FLOPS_PER_CELL.get(f"{p.nspecies}:{args.precision}")
        if fl:
            tf = fl * cells / avg_stage_s / 1e12
            pk = fma["measured_now"]["fp64_tflops"]
            roof["fp64"] = {"achieved": tf, "peak": pk, "unit": "TFLOP/s", "frac": tf / pk,
                            "flops_per_cell_stage": fl, "peak_kind": "measured (fhd_measure_fma_peak)",
                            "flops_source": "ncu instruction count of one stage at 128^3, per cell"}
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": ("synthetic (uniform NO2/N2O4 at chemical equilibrium + in-kernel Philox noise; no dataset)"
                 if p.nreaction > 0 else "synthetic (uniform argon at rest + in-kernel Philox noise; no dataset)"),
        "config": dict(config_dict(args, p, dt, tname), autotune_ms_per_step=tune),
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "graph_replay": graph, "gpu_launches": launches,
        "chemistry": chem, "aux": False, "fma_peaks": fma,
        "clocks": clk, "status": status,
    }
    if extras:
        out.update(extras)
    print(json.dumps(out), flush=True)


def stats_alg_bytes_per_cell(p):
    """Algorithmic bytes of one statistics update per cell: the state read once
    (cu, prim, the three face momenta) and every statistic read and written once
    (cuMeans, cuVars, primMeans, primVars, coVars, mom3, mom4 and the four
    face-centred statistics in three directions)."""
    nv, npv = p.nvars, p.nprimvars
    reads = nv + npv + 3
    stats = 2 * nv + (npv + 3) + (npv + 5) + 26 + 2 * (nv + 1) + 4 * 3
    return 8 * (reads + 2 * stats)


def run_stats(args):
    """Running statistics (fhd_stats_stag, all flags) after the step, timed alone:
    --steps updates with CUDA events on the launching stream; HBM roofline."""
    import torch
    from fhdex_b200 import capi
    from fhdex_b200.context import Context
    from fhdex_b200.params import stable_dt
    from fhdex_b200.state import StagState
    from fhdex_b200.stats import StatsState
    torch.cuda.set_device(0)
    p = make_params(args)
    ctx = Context(p, 0)
    st = StagState(p, "cuda:0", aux=False)
    ctx.init_state(st)
    dt = stable_dt(p)
    ctx.rk3_step(st, dt, 0, aux=False)
    stats = StatsState(p, "cuda:0", cross=True)
    flags = capi.STATS_MEANS | capi.STATS_VARS | capi.STATS_MOM3 | capi.STATS_MOM4
    for s in range(1, args.warmup + 1):
        ctx.stats_stag(st, stats, s, flags | capi.STATS_CROSS)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for s in range(args.steps):
        ctx.stats_stag(st, stats, args.warmup + 1 + s, flags)
    e1.record()
    # the same updates with the yz-averaged spatial cross-correlations (plot_cross)
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record()
    for s in range(args.steps):
        ctx.stats_stag(st, stats, args.warmup + args.steps + 1 + s, flags | capi.STATS_CROSS)
    e3.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    ms_cross = e2.elapsed_time(e3) / args.steps - ms
    assert ctx.status() == 0
    cells = p.n_cells[0] * p.n_cells[1] * p.n_cells[2]
    alg = stats_alg_bytes_per_cell(p) * cells
    # k_sum_to_line streams cu, cuMeans (nvars each) and nspecies+4 components of prim and primMeans once
    line_bytes = 8 * (2 * p.nvars + 2 * (p.nspecies + 4)) * cells
    peak, peak_kind = measured_peak()
    achieved = alg / (ms / 1e3) / 1e9
    traffic = STATS_TRAFFIC_BYTES_PER_CELL.get(f"{p.nspecies}")
    print(json.dumps({"mode": "stats", "metric": "statistics updates/s (cells x updates)", "unit": "cell-updates/s",
                      "value": cells / (ms / 1e3), "ms_per_update": ms, "steps": args.steps, "warmup": args.warmup,
                      "dtype": "f64", "config": {"workload": f"running statistics, all flags, {p.n_cells[0]}^3, "
                                                             f"{p.nspecies} species"},
                      "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                   "frac": achieved / peak, "peak_kind": peak_kind,
                                   "traffic": traffic * cells if traffic else None,
                                   "algorithmic_bytes_per_launch": alg,
                                   "kernel": "k_stats_means_a + k_stats_means_b + k_stats_vars + 4 ghost fills"},
                      "cross": {"ms_per_update": ms_cross, "kernels": "k_sum_to_line + k_spatial_cross",
                                "algorithmic_bytes": line_bytes,
                                "achieved_GBs": line_bytes / (ms_cross / 1e3) / 1e9,
                                "frac": line_bytes / (ms_cross / 1e3) / 1e9 / peak},
                      "clocks": clk}), flush=True)


def run_plot(args):
    """WritePlotFileStag: the GPU composition of the plotfile MultiFab (all
    statistics flags) timed over --steps launches with CUDA events (HBM roofline:
    every component read once and written once), and one plotfile written to disk
    at 64^3 (wall clock, pack + copy + file writes)."""
    import shutil
    import tempfile
    import torch
    from fhdex_b200.context import Context
    from fhdex_b200.params import stable_dt
    from fhdex_b200.plotfile import COVARS, MEANS, MOM3, MOM4, VARS, pack, plotfile_names, write_plotfile_stag
    from fhdex_b200.state import StagState
    from fhdex_b200.stats import StatsState
    flags = MEANS | VARS | COVARS | MOM3 | MOM4

    def prepared(p):
        ctx = Context(p, 0)
        st = StagState(p, "cuda:0", aux=True)
        ctx.init_state(st)
        ctx.rk3_step(st, stable_dt(p), 0, aux=True)
        stats = StatsState(p, "cuda:0")
        ctx.stats_stag(st, stats, 1, 15)
        return ctx, st, stats

    torch.cuda.set_device(0)
    p = make_params(args)
    ctx, st, stats = prepared(p)
    out = pack(ctx, st, stats, flags)
    for _ in range(args.warmup):
        pack(ctx, st, stats, flags, out=out)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        pack(ctx, st, stats, flags, out=out)
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    assert ctx.status() == 0
    # plot_deltaY_dir: the same pack with Y_k minus its plane average in each direction
    # (one thread per plane and species sums the plane in the reference's order)
    from fhdex_b200.plotfile import DELTAY
    deltay_ms = {}
    for d, fl in enumerate(DELTAY):
        o2 = pack(ctx, st, stats, flags | fl)
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        for _ in range(args.steps):
            pack(ctx, st, stats, flags | fl, out=o2)
        f1.record()
        torch.cuda.synchronize()
        deltay_ms["xyz"[d]] = f0.elapsed_time(f1) / args.steps
        del o2
    assert ctx.status() == 0
    ncomp = out.ncomp
    cells = p.n_cells[0] * p.n_cells[1] * p.n_cells[2]
    alg = 2 * 8 * ncomp * cells
    peak, peak_kind = measured_peak()
    achieved = alg / (ms / 1e3) / 1e9
    ctx.close()
    del st, stats, out
    torch.cuda.empty_cache()
    # one plotfile on disk at 64^3
    q = p.replace(n_cells=(64, 64, 64), prob_hi=tuple(p.dx[0] * 64 for _ in range(3)))
    ctx, st, stats = prepared(q)
    tmp = tempfile.mkdtemp(prefix="fhdplt")
    t = time.perf_counter()
    path = write_plotfile_stag(ctx, os.path.join(tmp, "plt"), 1, 0.0, st, stats, flags)
    wall = time.perf_counter() - t
    nbytes = sum(os.path.getsize(os.path.join(dp, f)) for dp, _, fs in os.walk(path) for f in fs)
    shutil.rmtree(tmp, ignore_errors=True)
    ctx.close()
    print(json.dumps({"mode": "plot", "metric": "plotfile components packed/s (cells x components)",
                      "unit": "cell-components/s", "value": cells * ncomp / (ms / 1e3), "ms_per_pack": ms,
                      "deltaY_ms_per_pack": deltay_ms,
                      "steps": args.steps, "warmup": args.warmup, "dtype": "f64",
                      "config": {"workload": f"WritePlotFileStag composition, all statistics flags, "
                                             f"{p.n_cells[0]}^3, {p.nspecies} species, {ncomp} components"},
                      "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                   "frac": achieved / peak, "peak_kind": peak_kind,
                                   "algorithmic_bytes_per_launch": alg, "kernel": "k_plot_pack"},
                      "write_64": {"seconds": wall, "bytes": nbytes, "names": len(plotfile_names(q, flags)),
                                   "path": "fhd_write_plotfile_stag (pack + D2H + Header/Cell_H/Cell_D files)"},
                      "clocks": clk}), flush=True)


def run_sf(args):
    """Static structure factor (fhd_sf_fort_structure): rho, rhoE, T and jx of the
    stepped state, all 10 pairs, --steps samples timed with CUDA events."""
    import torch
    from fhdex_b200.context import Context
    from fhdex_b200.fab import CELL, MultiFab
    from fhdex_b200.params import stable_dt
    from fhdex_b200.state import StagState
    from fhdex_b200.structfact import StructFact
    torch.cuda.set_device(0)
    p = make_params(args)
    ctx = Context(p, 0)
    st = StagState(p, "cuda:0", aux=False)
    ctx.init_state(st)
    ctx.rk3_step(st, stable_dt(p), 0, aux=False)
    nvar = 4
    var = MultiFab(p.n_cells, CELL, nvar, 0, device="cuda:0")
    var.valid(0).copy_(st.cu.valid(0))
    var.valid(1).copy_(st.cu.valid(4))
    var.valid(2).copy_(st.prim.valid(4))
    var.valid(3).copy_(st.cu.valid(1))
    stack = None if args.sf_stack == "none" else args.sf_stack
    nmem = {None: 1, "z_slices": p.n_cells[2], "x_pencils": p.n_cells[1] * p.n_cells[2]}[stack]
    sf = StructFact(p.n_cells, ["rho", "rhoE", "T", "jx"], [1.0] * (nvar * (nvar + 1) // 2), stack=stack)
    for s in range(args.warmup):
        sf.fort_structure(var)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for s in range(args.steps):
        sf.fort_structure(var)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    avg_ms = None
    if stack is not None:   # the output loop, once (it runs at plot time, not per sample)
        e0.record()
        sf.stack_average()
        e1.record()
        torch.cuda.synchronize()
        avg_ms = e0.elapsed_time(e1)
    cells = p.n_cells[0] * p.n_cells[1] * p.n_cells[2]
    # per point: pack (read + write 8 B), FFT (read 8 B, write the 8 B half spectrum) and
    # the accumulation's spectrum read (8 B) per variable; covariance read + write per pair
    alg = cells * (40 * nvar + 32 * sf.ncov)
    peak, peak_kind = measured_peak()
    achieved = alg / (ms / 1e3) / 1e9
    print(json.dumps({"mode": "sf", "metric": "structure-factor samples x cells / s", "unit": "cell-samples/s",
                      "value": cells / (ms / 1e3), "ms_per_sample": ms, "stack_average_ms": avg_ms,
                      "steps": args.steps, "nvar": nvar,
                      "ncov": sf.ncov, "config": {"workload": f"StructFact of 4 variables, 10 pairs, "
                                                              f"{p.n_cells[0]}^3"
                                                              + ("" if stack is None else
                                                                 f", one per {stack[2:-1]} ({nmem} members)")},
                      "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                   "frac": achieved / peak, "peak_kind": peak_kind,
                                   "algorithmic_bytes_per_launch": alg,
                                   "kernel": "4 x (k_sf_pack + cuFFT D2Z) + k_sf_accumulate"}}), flush=True)
    sf.close()


def equilibrium_check(args, precision):
    """Equilibrium-variance error of the batched form: a batch of --eq-members
    independent 32^3 argon runs, variances over cells, members and 150 snapshots
    divided by the fluctuation theory (fhdex_b200/equilibrium.py), at the
    benchmark's dt (1000 warm-up steps, snapshots 5 steps apart) and at dt/2 (2000,
    10): the time-discretisation error of the temperature variance falls from ~1.3 %
    to ~0.2 % (the same in FP64 and mixed), while cell-updates/s do not depend on
    dt.  Untimed; None when --eq-members is 0."""
    if args.eq_members <= 0:
        return None
    from fhdex_b200.equilibrium import batch_variance_ratios
    out = {"form": "batched " + ("mixed" if precision else "fp64"), "members": args.eq_members, "n": 32}
    for key, sc, warm, every in (("dt", 1.0, 1000, 5), ("dt_half", 0.5, 2000, 10)):
        ratios, m = batch_variance_ratios(members=args.eq_members, precision=precision, dt_scale=sc, warm=warm,
                                          every=every)
        out[key] = {"steps": warm + 150 * every, "samples_per_field": m,
                    "variance_over_theory": {k: round(v, 5) for k, v in ratios.items()},
                    "max_abs_error": round(max(abs(v - 1.0) for v in ratios.values()), 5)}
    return out


def run_ensemble(args):
    """Batched ensemble: --members realisations of argon, half 32^3 and half 64^3,
    T0 ~ U(250,350) K, rho0 ~ U(1e-3,3e-3) g/cm^3, one graph replay per step."""
    import torch
    from fhdex_b200.serve import ensemble
    torch.cuda.set_device(0)
    prec = 1 if args.precision == "mixed" else 0
    b, states, cells = ensemble(args.members, seed=args.seed, precision=prec)
    s = torch.cuda.Stream()
    b.set_stream(s)
    b.step(args.warmup, graph=True)
    b.synchronize()
    # the batch's autotuner picks the face kernels' register cap on these members
    tile, tune_ms = b.autotune()
    persist_ms = {}
    if args.persistent:
        # the persistent kernel's register cap, each timed over 3 graph-replayed steps
        for t in range(len(b.TILE_REGS)):
            b.set_persistent(True, t)
            b.step(1, graph=True)
            b.synchronize()
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(s):
                f0.record()
            b.step(3, graph=True)
            with torch.cuda.stream(s):
                f1.record()
            b.synchronize()
            persist_ms[b.TILE_REGS[t]] = f0.elapsed_time(f1) / 3
        tile = min(range(len(b.TILE_REGS)), key=lambda t: persist_ms[b.TILE_REGS[t]])
        b.set_persistent(True, tile)
    b.step(1, graph=True)            # re-capture the step graph with the chosen shape (untimed)
    b.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(s):
        e0.record()
    b.step(args.steps, graph=True)
    with torch.cuda.stream(s):
        e1.record()
    b.synchronize()
    ms = e0.elapsed_time(e1)
    bad = sum(1 for mid in list(b.members) if b.status(mid) != 0)
    b.close()
    eq = equilibrium_check(args, prec)
    print(json.dumps({"mode": "ensemble", "metric": METRIC, "value": cells * args.steps / (ms / 1e3), "unit": UNIT,
                      "members": args.members, "cells_total": cells, "steps": args.steps, "ms_per_step": ms / args.steps,
                      "precision": args.precision, "members_with_status": bad,
                      "face_tile_regs": b.TILE_REGS[tile], "autotune_face_ms_per_stage": tune_ms,
                      "persistent_ms_per_step_by_regs": persist_ms or None,
                      "launch": ("one persistent launch per step (k_batch_persist), graph replay" if args.persistent
                                 else "23 batched kernels per step, one CUDA graph replay per step"),
                      "equilibrium": eq}), flush=True)


def run_serve(args):
    """Serving: Poisson arrivals (rate --rate), box edge log-uniform 16-128,
    nspecies in {1,2,4}, steps U{100..2000}, precision FP64/mixed; continuous
    batching vs serving one request at a time with the plain FP64 step."""
    import torch
    from fhdex_b200.serve import Server, latency_stats, poisson_trace, run_alone, warm_kernels
    torch.cuda.set_device(0)
    warm_kernels(0)                  # both paths start with every kernel loaded
    steps = (args.serve_min_steps, args.serve_max_steps)
    trace = poisson_trace(args.requests, rate=args.rate, seed=args.seed, steps=steps)
    srv = Server(chunk=args.chunk)
    reqs, _, cu_b, el_b = srv.run(trace)
    srv.close()
    torch.cuda.empty_cache()
    lb = latency_stats(reqs)
    trace2 = poisson_trace(args.requests, rate=args.rate, seed=args.seed, steps=steps)
    reqs2, cu_a, el_a = run_alone(trace2)
    la = latency_stats(reqs2)
    print(json.dumps({"mode": "serve", "metric": METRIC, "unit": UNIT, "requests": args.requests, "rate_per_s": args.rate,
                      "steps_range": list(steps),
                      "served": {"value": cu_b / el_b, "elapsed_s": el_b, **lb,
                                 "bad_status": sum(1 for r in reqs if r.status)},
                      "alone_fp64": {"value": cu_a / el_a, "elapsed_s": el_a, **la,
                                     "bad_status": sum(1 for r in reqs2 if r.status)},
                      "equilibrium": equilibrium_check(args, 1)}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", default="step", choices=["step", "ensemble", "serve", "stats", "sf", "plot"])
    ap.add_argument("--members", type=int, default=512)
    ap.add_argument("--requests", type=int, default=48)
    ap.add_argument("--rate", type=float, default=50.0)
    ap.add_argument("--chunk", type=int, default=20)
    ap.add_argument("--serve-min-steps", type=int, default=100)
    ap.add_argument("--serve-max-steps", type=int, default=2000)
    ap.add_argument("--eq-members", type=int, default=16,
                    help="members of the batched equilibrium check (ensemble/serve modes; 0: skip)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--ns", type=int, default=2)
    ap.add_argument("--walls", default="none", choices=["none", "tempgrad", "reservoir"],
                    help="step mode: physical boundaries of the reference's regression runs (FP64)")
    ap.add_argument("--lowdim", default="none", choices=["none", "1d", "2d"],
                    help="quasi-1-D / 2-D run (do_1D / do_2D) on the same box")
    ap.add_argument("--transport", default="gio", choices=["gio", "vw", "hcb"],
                    help="transport model: Giovangigli (default), Valk/Waldmann, HCB binary")
    ap.add_argument("--gas", default="argon", choices=["argon", "no2"],
                    help="argon: --ns selects the species form; no2: 2 NO2 <-> N2O4 with the chemistry source")
    ap.add_argument("--dx", type=float, default=8e-6)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--tile", default="auto")
    ap.add_argument("--sf-stack", default="none", choices=["none", "z_slices", "x_pencils"],
                    help="--mode sf: the quasi-2-D per-slice or quasi-1-D per-pencil stack")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed / aux / batched / served objects of the step line")
    ap.add_argument("--persistent", action="store_true",
                    help="ensemble mode: one persistent launch per step instead of the per-kind launches")
    ap.add_argument("--bench-batch-steps", type=int, default=20)
    ap.add_argument("--bench-requests", type=int, default=50)
    ap.add_argument("--bench-serve-max-steps", type=int, default=600)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.mode == "ensemble":
        run_ensemble(args)
    elif args.mode == "serve":
        run_serve(args)
    elif args.mode == "stats":
        run_stats(args)
    elif args.mode == "sf":
        run_sf(args)
    elif args.mode == "plot":
        run_plot(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
