"""Ensembles and served runs: many independent runs stepped together.

``Batch`` wraps ``fhd_batch_*``: members of one species count and precision,
each with its own box size, gas state, dt, seed and step counter, are advanced
by batched kernels (one launch per kernel for all members) replayed from a
captured CUDA graph.  A member's result is the one it would get alone through
``Context.rk3_step`` with in-kernel noise.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import capi
from .capi import check
from .params import Params
from .state import StagState


class Batch:
    def __init__(self, nspecies: int, precision: int = 0, device: int = 0):
        self.lib = capi.load()
        self.device = device
        self.ns = nspecies
        self.precision = precision
        self._h = C.c_void_p()
        check(self.lib.fhd_batch_create(C.byref(self._h), nspecies, precision, device), "fhd_batch_create")
        self.members = {}   # id -> (Params, StagState)

    def close(self):
        if self._h:
            self.lib.fhd_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, p: Params, st: StagState, dt: float, first_step: int = 0, init: bool = True) -> int:
        """Register a run.  init=True sets the uniform rest state of p (rho0,
        T_init, rhobar) in st; otherwise st must hold a converted, ghost-filled state."""
        torch.cuda.current_stream(self.device).synchronize()
        ini = (C.c_double * (2 + p.nspecies))(p.rho0, p.T_init, *p.rhobar[:p.nspecies]) if init else None
        mid = C.c_int(-1)
        cp = p.to_c()
        check(self.lib.fhd_batch_add(self._h, C.byref(cp), st.cu.fab(), st.mom_fabs(), st.prim.fab(), st.vel_fabs(),
                                     dt, first_step, ini, C.byref(mid)), "fhd_batch_add")
        self.members[mid.value] = (p, st)
        return mid.value

    def remove(self, mid: int):
        check(self.lib.fhd_batch_remove(self._h, mid), "fhd_batch_remove")
        self.members.pop(mid, None)

    def step(self, nsteps: int = 1, graph: bool = True):
        check(self.lib.fhd_batch_step(self._h, nsteps, int(graph)), "fhd_batch_step")

    def set_stream(self, stream: "torch.cuda.Stream"):
        """Run on a torch CUDA stream (not the legacy default stream: graphs are
        captured on it)."""
        self._stream = stream
        check(self.lib.fhd_batch_set_stream(self._h, C.c_void_p(stream.cuda_stream)), "fhd_batch_set_stream")

    def set_persistent(self, enable: bool = True, tile: int = -1):
        """One persistent launch per step (k_batch_persist) instead of the per-kind
        launches; bitwise the same results.  tile: the kernel's register cap
        (TILE_REGS; -1 the default)."""
        check(self.lib.fhd_batch_set_persistent(self._h, int(enable), tile), "fhd_batch_set_persistent")

    def set_wait_limit(self, seconds: float, hold_phase: int = -1):
        """Time limit of the persistent step's waits; hold_phase >= 0 never publishes
        that phase's completions (a failure-injection hook for tests)."""
        check(self.lib.fhd_batch_set_wait_limit(self._h, seconds, hold_phase), "fhd_batch_set_wait_limit")

    def synchronize(self):
        check(self.lib.fhd_batch_synchronize(self._h), "fhd_batch_synchronize")

    def status(self, mid: int) -> int:
        return self.lib.fhd_batch_member_status(self._h, mid)

    def __len__(self):
        return self.lib.fhd_batch_size(self._h)

    # register caps of the batched face-flux kernels (registers per thread)
    TILE_REGS = (64, 80, 128)

    def set_tile(self, tile: int):
        """Face-kernel launch shape: an index into TILE_REGS, or -1 for the default."""
        check(self.lib.fhd_batch_set_tile(self._h, tile), "fhd_batch_set_tile")

    def autotune(self, reps: int = 3):
        """Time the batched face-flux kernels of one stage for every register cap on
        the current members and keep the fastest (members' states do not change;
        run after at least one step).  Returns (best tile, {regs: ms})."""
        nt = self.lib.fhd_batch_num_tiles()
        ms = (C.c_double * nt)()
        best = C.c_int(-1)
        check(self.lib.fhd_batch_autotune(self._h, reps, ms, C.byref(best)), "fhd_batch_autotune")
        return best.value, {self.TILE_REGS[t]: round(ms[t], 4) for t in range(nt)}
