"""fhd_rk3_step_stag_noalloc: the RK3 step for callers that cannot allocate device
memory (arena-owned device memory, allocation-free framework callbacks,
latency-critical loops that cannot absorb cudaMalloc/cudaFree's device-wide
synchronisation).  Its scratch is a static device array inside the library;
these tests compare it, through the C ABI, with the allocating entry point on
two steps in a row, and check that oversized boxes are refused before any GPU
work.  This file is collected last so that a run stopping at the first failure
has run every other test first."""
import ctypes as C

import pytest
import torch

from fhdex_b200 import capi
from fhdex_b200.context import Context
from fhdex_b200.params import argon, mixture4, stable_dt
from fhdex_b200.state import StagState

pytestmark = pytest.mark.gpu


def _noalloc_step(p, st, dt, step):
    lib = capi.load()
    status = C.c_int(-1)
    cp = p.to_c()
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.fhd_rk3_step_stag_noalloc(C.byref(cp), st.cu.fab(), st.mom_fabs(), st.prim.fab(), st.vel_fabs(),
                                       dt, step, C.c_void_p(stream), C.byref(status))
    return rc, status.value


@pytest.mark.parametrize("make", [lambda: argon(20, dx=8e-6), lambda: mixture4((16, 12, 10), dx=8e-6)])
def test_noalloc_step_matches_allocating_step(make):
    """Two consecutive steps through the static-scratch entry point equal the
    context-based step bit for bit (the FP64 path's tolerance is zero)."""
    p = make()
    dt = stable_dt(p)
    ref = StagState(p, "cuda", aux=False)
    ctx = Context(p)
    ctx.init_state(ref)
    got = StagState(p, "cuda", aux=False)
    got.copy_from(ref)
    for step in (0, 1):
        ctx.rk3_step(ref, dt, step, aux=False)
        rc, status = _noalloc_step(p, got, dt, step)
        assert rc == 0, capi.load().fhd_strerror(rc)
        assert status == 0
        torch.cuda.synchronize()
        for name, m in ref.named().items():
            assert torch.equal(got.named()[name].arr, m.arr), (step, name)
    ctx.close()


def test_noalloc_rejects_boxes_beyond_its_scratch():
    p = argon(64, dx=8e-6)
    st = StagState(p, "cuda", aux=False)
    rc, _ = _noalloc_step(p, st, stable_dt(p), 0)
    assert rc == capi.FHD_ERR_TOO_LARGE
    assert b"16 MiB" in capi.load().fhd_strerror(rc)
