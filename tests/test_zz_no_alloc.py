"""fhd_rk3_step_stag_noalloc: the RK3 step for callers that cannot allocate device
memory (arena-owned device memory, allocation-free framework callbacks,
latency-critical loops that cannot absorb cudaMalloc/cudaFree's device-wide
synchronisation).  Its scratch is a static device array inside the library;
these tests compare it, through the C ABI, with the allocating entry point on
two steps in a row (boxes up to the scratch's limit, with and without
stochastic forcing, 2- and 3-cell ghosts), check that it allocates no device
memory, and that oversized boxes and host memory are refused before any GPU
work.  This file is collected last so that a run stopping at the first failure
has run every other test first."""
import ctypes as C

import pytest
import torch

from fhdex_b200 import capi
from fhdex_b200.context import Context
from fhdex_b200.params import argon, mixture4, stable_dt
from fhdex_b200.state import StagState
from tests.helpers import perturbed_state

pytestmark = pytest.mark.gpu


def _noalloc_step(p, st, dt, step):
    lib = capi.load()
    status = C.c_int(-1)
    cp = p.to_c()
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.fhd_rk3_step_stag_noalloc(C.byref(cp), st.cu.fab(), st.mom_fabs(), st.prim.fab(), st.vel_fabs(),
                                       dt, step, C.c_void_p(stream), C.byref(status))
    return rc, status.value


# (30, 30, 29) with 2 species fills the 16 MiB scratch to within 48 KiB, so the
# last fab carved from it ends next to the array's end.
@pytest.mark.parametrize("make", [lambda: argon(20, dx=8e-6), lambda: mixture4((16, 12, 10), dx=8e-6),
                                  lambda: argon((30, 30, 29), dx=8e-6), lambda: mixture4(26, dx=8e-6),
                                  lambda: mixture4((12, 10, 9), dx=8e-6, stoch_stress_form=0)])
def test_noalloc_step_matches_allocating_step(oracle, make):
    """Two consecutive steps through the static-scratch entry point equal the
    context-based step bit for bit (the FP64 path's tolerance is zero), from a
    perturbed state, with and without stochastic forcing, and for boxes that
    nearly fill the scratch."""
    p = make()
    dt = stable_dt(p)
    ref = perturbed_state(oracle, p, seed=21).clone(device="cuda")
    ctx = Context(p)
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


@pytest.mark.parametrize("n", [64, 30])
def test_noalloc_rejects_boxes_beyond_its_scratch(n):
    p = argon(n, dx=8e-6)
    st = StagState(p, "cuda", aux=False)
    rc, _ = _noalloc_step(p, st, stable_dt(p), 0)
    assert rc == capi.FHD_ERR_TOO_LARGE
    assert b"16 MiB" in capi.load().fhd_strerror(rc)


def test_noalloc_step_allocates_no_device_memory():
    """After a first call (which loads the library's module and with it the static
    scratch), further calls leave the device's free memory and torch's allocator
    untouched: the step's 16 MiB of stage scratch would show as a drop of at least
    one 2 MiB allocation granule."""
    p = argon(24, dx=8e-6)
    st = StagState(p, "cuda", aux=False)
    Context(p).init_state(st)
    dt = stable_dt(p)
    rc, status = _noalloc_step(p, st, dt, 0)
    assert rc == 0 and status == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    torch0 = torch.cuda.memory_allocated()
    for step in (1, 2, 3):
        rc, status = _noalloc_step(p, st, dt, step)
        assert rc == 0 and status == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert torch.cuda.memory_allocated() == torch0
    assert free0 - free1 < (2 << 20), (free0, free1)


def test_noalloc_accepts_wider_ghosts_and_rejects_host_memory(oracle):
    """Fabs with 3 ghost cells (the context entry point accepts any width >= 2)
    step to the same valid values; host memory is refused with FHD_ERR_BAD_ARG."""
    p = argon(10, dx=8e-6)
    dt = stable_dt(p)
    ref = perturbed_state(oracle, p, seed=22).clone(device="cuda")
    wide = StagState(p.replace(ngc=3), "cuda", aux=False)
    for a, b in zip(wide.state_mfs(), ref.state_mfs()):
        a.valid().copy_(b.valid())
    for m in wide.state_mfs():
        Context(p).fill_boundary(m)
    ctx = Context(p)
    for step in (0, 1):
        ctx.rk3_step(ref, dt, step, aux=False)
        rc, status = _noalloc_step(p, wide, dt, step)
        assert rc == 0 and status == 0
    torch.cuda.synchronize()
    for a, b in zip(wide.state_mfs(), ref.state_mfs()):
        assert torch.equal(a.valid(), b.valid())
    host = StagState(p, "cpu", aux=False)
    rc, _ = _noalloc_step(p, host, dt, 0)
    assert rc == capi.FHD_ERR_BAD_ARG
