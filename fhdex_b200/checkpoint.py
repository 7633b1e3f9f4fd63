"""WriteCheckPoint / ReadCheckPoint (Checkpoint.cpp:28-257, 259-575) through the C
ABI: ``write_checkpoint`` saves the state (and the running statistics) under
``<chk_base><step:09d>/``; ``read_checkpoint`` fills states of the same shapes
and returns (step to run next, time, statsCount), as the reference's restart
does.  Device and host MultiFabs both work."""
from __future__ import annotations

import ctypes as C

from . import capi
from .capi import check


def _args(st, stats):
    sp = C.byref(stats.c_struct()) if stats is not None else None
    return st.cu.fab(), st.mom_fabs(), st.prim.fab(), st.vel_fabs(), sp


def write_checkpoint(p, chk_base: str, step: int, time: float, st, stats=None, stats_count: int = 0) -> str:
    cp = p.to_c()
    check(capi.load().fhd_write_checkpoint(C.byref(cp), chk_base.encode(), step, time, stats_count,
                                           *_args(st, stats)), "fhd_write_checkpoint")
    return f"{chk_base}{step:09d}"


def read_checkpoint(p, chk_base: str, restart: int, st, stats=None):
    cp = p.to_c()
    step, stats_count = C.c_int(), C.c_int()
    time = C.c_double()
    check(capi.load().fhd_read_checkpoint(C.byref(cp), chk_base.encode(), restart, C.byref(step), C.byref(time),
                                          C.byref(stats_count), *_args(st, stats)), "fhd_read_checkpoint")
    return step.value, time.value, stats_count.value
