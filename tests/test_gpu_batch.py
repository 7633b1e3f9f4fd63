"""Batched ensembles / served runs: every member's result equals the same run
alone, also when members join and leave between steps (continuous batching).
FP64: bit for bit (the batched kernels run the same point functions in the same
order with the member's own Philox key and step counter).  Mixed precision: the
FP32 units are built with FMA contraction, which the compiler may apply
differently in the batched and the single-run kernels, so members agree with the
run alone within a norm-relative error of MIXED_TOL per field: FP32 rounding
(6e-8) amplified over the steps, a tenth of the mixed path's own 1e-4 bound
against the FP64 result."""
import pytest
import torch

from fhdex_b200.batch import Batch
from fhdex_b200.context import Context
from fhdex_b200.params import argon, mixture4, stable_dt
from fhdex_b200.state import StagState

pytestmark = pytest.mark.gpu


def alone(p, dt, steps, first=0):
    st = StagState(p, "cuda", aux=False)
    ctx = Context(p)
    ctx.init_state(st)
    for s in range(first, first + steps):
        ctx.rk3_step(st, dt, s, aux=False)
    torch.cuda.synchronize()
    ctx.close()
    return st


MIXED_TOL = 1e-5


def same(a, b, tol=0.0):
    """names of the fields of a that differ from b (tol = 0: bitwise)."""
    from tests.helpers import max_rel
    bad = []
    for n, m in a.named().items():
        r = b.named()[n]
        if tol == 0.0:
            if not torch.equal(m.arr, r.arr):
                bad.append(n)
        else:
            for c in range(m.ncomp):
                e = max_rel(m.valid(c), r.valid(c))
                if not e <= tol:
                    bad.append((n, c, e))
    return bad


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_members_match_runs_alone(precision):
    ps = [argon(16, dx=8e-6, T_init=260.0, rho0=1.2e-3, seed=11, precision=precision),
          argon((20, 12, 8), dx=8e-6, T_init=330.0, rho0=2.5e-3, seed=12, precision=precision),
          argon(12, dx=8e-6, T_init=300.0, rho0=1.78e-3, seed=13, precision=precision)]
    dts = [stable_dt(p) for p in ps]
    b = Batch(2, precision)
    sts = [StagState(p, "cuda", aux=False) for p in ps]
    ids = [b.add(p, st, dt) for p, st, dt in zip(ps, sts, dts)]
    b.step(3, graph=True)
    b.synchronize()
    for p, st, dt, mid in zip(ps, sts, dts, ids):
        assert b.status(mid) == 0
        ref = alone(p, dt, 3)
        tol = 0.0 if precision == 0 else MIXED_TOL
        assert not same(st, ref, tol), (p.n_cells, same(st, ref, tol))
    b.close()


def test_fp64_batch_after_mixed_runs_matches_alone():
    """FP64 members stay bit-exact after mixed-precision work in the same process.
    (Kernels that do not depend on the precision are instantiated by both the FP64
    and the FMA-contracting mixed units; with external linkage a launch could run
    the mixed unit's copy once that module was loaded.)"""
    pm = argon(12, dx=8e-6, seed=5, precision=1)
    alone(pm, stable_dt(pm), 2)                    # loads the mixed kernels
    bm = Batch(2, 1)
    sm = StagState(pm, "cuda", aux=False)
    bm.add(pm, sm, stable_dt(pm))
    bm.step(2, graph=True)
    bm.synchronize()
    bm.close()
    p = argon(16, dx=8e-6, T_init=260.0, rho0=1.2e-3, seed=11)
    dt = stable_dt(p)
    b = Batch(2, 0)
    st = StagState(p, "cuda", aux=False)
    b.add(p, st, dt)
    b.step(3, graph=True)
    b.synchronize()
    assert not same(st, alone(p, dt, 3))
    b.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_every_face_tile_and_the_autotuner_keep_member_results(precision):
    """Each register cap of the batched face kernels gives the members the result
    they get alone (FP64 bit for bit), and the autotuner, run between steps,
    changes no member's state."""
    ps = [argon(12, dx=8e-6, T_init=280.0, seed=31, precision=precision),
          argon((10, 14, 8), dx=8e-6, rho0=2.2e-3, seed=32, precision=precision)]
    dts = [stable_dt(p) for p in ps]
    refs = [alone(p, dt, 3) for p, dt in zip(ps, dts)]
    tol = 0.0 if precision == 0 else MIXED_TOL
    for tile in [0, 1, 2, "auto"]:
        b = Batch(2, precision)
        sts = [StagState(p, "cuda", aux=False) for p in ps]
        for p, st, dt in zip(ps, sts, dts):
            b.add(p, st, dt)
        if tile == "auto":
            b.step(1, graph=True)
            best, ms = b.autotune(reps=2)
            assert best in (0, 1, 2) and sorted(ms) == list(Batch.TILE_REGS)
            assert all(v > 0 for v in ms.values()), ms
            b.step(2, graph=True)
        else:
            b.set_tile(tile)
            b.step(3, graph=True)
        b.synchronize()
        for st, ref in zip(sts, refs):
            assert not same(st, ref, tol), (tile, same(st, ref, tol))
        b.close()


def test_members_join_and_leave_between_steps():
    pa = argon(16, dx=8e-6, seed=21)
    pb = mixture4(12, dx=8e-6, seed=22)
    pc = argon(10, dx=8e-6, seed=23, T_init=290.0)
    # two classes: ns=2 batch (a, c) and ns=4 batch (b)
    b2 = Batch(2, 0)
    b4 = Batch(4, 0)
    sa, sb, sc = (StagState(p, "cuda", aux=False) for p in (pa, pb, pc))
    da, db, dc = stable_dt(pa), stable_dt(pb), stable_dt(pc)
    ia = b2.add(pa, sa, da)
    b2.step(2)
    ib = b4.add(pb, sb, db)
    ic = b2.add(pc, sc, dc)          # joins while a is running
    b2.step(2)
    b4.step(2)
    b2.remove(ia)                    # a leaves after 4 steps
    b2.step(1, graph=False)
    b2.synchronize()
    b4.synchronize()
    assert not same(sa, alone(pa, da, 4))
    assert not same(sb, alone(pb, db, 2))
    assert not same(sc, alone(pc, dc, 3))
    b2.close()
    b4.close()


def test_server_results_match_runs_alone():
    """Requests served with continuous batching (joining and leaving batches of
    both precisions, species counts and size buckets at different times, and boxes of
    11^3 cells or more on the solo lane) end in exactly the state they reach when run
    alone."""
    from fhdex_b200.serve import Server, poisson_trace, request_params
    trace = poisson_trace(8, rate=400.0, seed=3, edge=(8, 14), steps=(3, 9))
    srv = Server(chunk=2, solo_cells=11 ** 3, small_cells=9 ** 3)
    reqs, finals, cell_updates, elapsed = srv.run(trace, keep_states=True)
    assert all(r.status == 0 for r in reqs)
    sizes = [r.n for r in reqs]
    assert any(n >= 11 for n in sizes) and any(n < 11 for n in sizes), sizes
    assert cell_updates == sum(r.steps * r.n ** 3 for r in reqs)
    for r in reqs:
        p = request_params(r)
        ref = alone(p, stable_dt(p), r.steps)
        tol = 0.0 if p.precision == 0 else MIXED_TOL
        assert not same(finals[r.rid], ref, tol), (r, same(finals[r.rid], ref, tol))
    srv.close()


@pytest.mark.parametrize("precision,ns", [(0, 2), (1, 2), (0, 4)])
def test_persistent_step_equals_the_per_kind_launches(precision, ns):
    """One persistent launch per step (k_batch_persist: chunks of every member's
    phases from one device counter, bounded waits on the member's previous phase)
    gives the per-kind launches' results bit for bit, with and without graph
    replay, on members of different sizes."""
    mk = argon if ns == 2 else mixture4
    ps = [mk(16, dx=8e-6, T_init=260.0, rho0=1.2e-3, seed=21, precision=precision),
          mk((20, 12, 8), dx=8e-6, T_init=330.0, rho0=2.5e-3, seed=22, precision=precision),
          mk((9, 7, 13), dx=8e-6, seed=23, precision=precision)]
    dts = [stable_dt(p) for p in ps]
    out = []
    for persistent in (False, True):
        b = Batch(ns, precision)
        b.set_persistent(persistent)
        sts = [StagState(p, "cuda", aux=False) for p in ps]
        ids = [b.add(p, st, dt) for p, st, dt in zip(ps, sts, dts)]
        b.step(2, graph=False)
        b.step(2, graph=True)
        b.synchronize()
        assert all(b.status(i) == 0 for i in ids)
        out.append(sts)
        b.close()
    for a, r in zip(out[1], out[0]):
        assert not same(a, r), same(a, r)


def test_persistent_wait_runs_out_and_the_batch_stays_usable():
    """The failure path of the persistent step's waits: with the completions of
    phase 3 (the x face fluxes of stage 1) never published, the wait of phase 4
    runs out after the 50 ms limit, the member's status reads FHD_ERR_TIMEOUT and
    the launch ends; afterwards the batch steps normally again."""
    from fhdex_b200 import capi
    ps = [argon(12, dx=8e-6, seed=31), argon(10, dx=8e-6, seed=32)]
    b = Batch(2, 0)
    b.set_persistent(True)
    sts = [StagState(p, "cuda", aux=False) for p in ps]
    ids = [b.add(p, st, stable_dt(p)) for p, st in zip(ps, sts)]
    b.set_wait_limit(0.05, hold_phase=3)
    b.step(1, graph=False)
    b.synchronize()
    codes = [b.status(i) for i in ids]
    assert capi.FHD_ERR_TIMEOUT in codes and all(c in (0, capi.FHD_ERR_TIMEOUT) for c in codes)
    b.set_wait_limit(1.0, hold_phase=-1)
    # a fresh batch of the same members' sizes steps cleanly after the timeout
    b2 = Batch(2, 0)
    b2.set_persistent(True)
    st2 = StagState(ps[0], "cuda", aux=False)
    i2 = b2.add(ps[0], st2, stable_dt(ps[0]))
    b2.step(2, graph=True)
    b2.synchronize()
    assert b2.status(i2) == 0
    ref = alone(ps[0], stable_dt(ps[0]), 2)
    assert not same(st2, ref)
    b.step(1, graph=False)
    b.synchronize()
    b.close()
    b2.close()
