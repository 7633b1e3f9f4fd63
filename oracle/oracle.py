"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
reference arm as the checker; the product library never calls it.  Works on
host (CPU) MultiFabs from ``fhdex_b200.state``.  The restated functions and the
reference lines they follow are cited in ``fhd_oracle.cpp``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from fhdex_b200.capi import FabArr3, FabArr6, FhdFab, FhdNoise, FhdParams, FhdStats
from fhdex_b200.fab import fab_array

_DIR = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_DIR, "lib", "libfhd_oracle.so")
_lib = None


def build(force=False):
    src = os.path.join(_DIR, "fhd_oracle.cpp")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _DIR])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P = C.POINTER
        fab, pfab, d, i = FhdFab, P(FhdFab), C.c_double, C.c_int
        L.orc_set_params.argtypes = [P(FhdParams)]
        L.orc_get_hc.argtypes = [P(d), P(d)]
        L.orc_fill_boundary.argtypes = [fab]
        L.orc_override_sync.argtypes = [fab]
        L.orc_init_cons_var_stag.argtypes = [fab, pfab, d, d, P(d)]
        L.orc_conserved_to_primitive_stag.argtypes = [fab, pfab, fab, pfab]
        L.orc_transport_coeffs.argtypes = [fab] * 6
        L.orc_flux_stag.argtypes = [fab, pfab, fab, pfab, fab, fab, fab, fab, fab, pfab, pfab, pfab,
                                    pfab, pfab, pfab, d]
        L.orc_rk3_step_stag.argtypes = [fab, pfab, fab, pfab, fab, fab, fab, fab, fab, fab, pfab, pfab,
                                        pfab, P(FhdNoise), d]
        L.orc_fill_random_normal.argtypes = [fab, i, i, d, d, C.c_uint64, C.c_uint64]
        L.orc_chemistry_source_cle.argtypes = [d, d, fab, fab, fab]
        L.orc_philox4x32_10.argtypes = [P(C.c_uint32), P(C.c_uint32), P(C.c_uint32)]
        L.orc_philox4x32_10.restype = None
        L.orc_fill_noise_mt64.argtypes = [P(FhdNoise), C.c_uint64]
        L.orc_stats_stag.argtypes = [fab, fab, pfab, P(FhdStats), C.c_int64, i]
        L.orc_set_threads.argtypes = [i]
        L.orc_set_threads.restype = i
        L.orc_max_acoustic_cfl.argtypes = [fab, pfab, d]
        L.orc_max_acoustic_cfl.restype = d
        _lib = L
    return _lib


def _chk(rc, what):
    if rc != 0:
        raise RuntimeError(f"oracle {what} returned {rc}")


def set_params(p):
    _chk(lib().orc_set_params(C.byref(p.to_c())), "set_params")


def hc():
    a = (C.c_double * 8)()
    b = (C.c_double * 8)()
    lib().orc_get_hc(a, b)
    return list(a), list(b)


def fill_boundary(mf):
    _chk(lib().orc_fill_boundary(mf.fab()), "fill_boundary")


def override_sync(mf):
    _chk(lib().orc_override_sync(mf.fab()), "override_sync")


def init_cons_var_stag(st, p):
    rb = (C.c_double * 8)(*p.rhobar)
    _chk(lib().orc_init_cons_var_stag(st.cu.fab(), st.mom_fabs(), p.rho0, p.T_init, rb), "init")


def conserved_to_primitive(st, cu=None, mom=None):
    set_params(st.p)
    cu = cu or st.cu
    mom = mom or st.cumom
    return lib().orc_conserved_to_primitive_stag(st.prim.fab(), st.vel_fabs(), cu.fab(),
                                                 fab_array(mom, FabArr3))


def transport_coeffs(st):
    set_params(st.p)
    return lib().orc_transport_coeffs(st.prim.fab(), st.eta.fab(), st.zeta.fab(), st.kappa.fab(),
                                      st.chi.fab(), st.D.fab())


def flux_stag(st, sf, se, sc, dt):
    set_params(st.p)
    return lib().orc_flux_stag(st.cu.fab(), st.mom_fabs(), st.prim.fab(), st.vel_fabs(), st.eta.fab(),
                               st.zeta.fab(), st.kappa.fab(), st.chi.fab(), st.D.fab(),
                               st.faceflux_fabs(), st.edgeflux_fabs(), st.cenflux_fabs(),
                               fab_array(sf, FabArr3), fab_array(se, FabArr3), fab_array(sc, FabArr3), dt)


def rk3_step(st, noise, dt):
    """One RK3stepStag with injected A/B noise (``noise`` = StepNoise or None)."""
    set_params(st.p)
    nz = C.byref(noise.c_struct()) if noise is not None else None
    return lib().orc_rk3_step_stag(st.cu.fab(), st.mom_fabs(), st.prim.fab(), st.vel_fabs(),
                                   st.source.fab(), st.eta.fab(), st.zeta.fab(), st.kappa.fab(),
                                   st.chi.fab(), st.D.fab(), st.faceflux_fabs(), st.edgeflux_fabs(),
                                   st.cenflux_fabs(), nz, dt)


def chemistry_source_cle(p, dt, dV, prim, source, ranchem=None):
    """compute_compressible_chemistry_source_CLE (chemistry_functions.cpp:128-193)."""
    set_params(p)
    rf = ranchem.fab() if ranchem is not None else FhdFab()
    return lib().orc_chemistry_source_cle(dt, dV, prim.fab(), source.fab(), rf)


def fill_random_normal(mf, scomp, ncomp, mean, variance, seed, stream_id):
    _chk(lib().orc_fill_random_normal(mf.fab(), scomp, ncomp, mean, variance, seed, stream_id), "fill")


def fill_step_noise(noise, seed, step):
    """The reference's per-step noise fill (timeStepStag.cpp:183-222): faces and edges
    variance 1, centres variance 2, each OverrideSync'ed and FillBoundary'ed."""
    set_params(noise.p)
    ns = noise.p.nspecies
    sid = 0
    for s in range(2):
        for d in range(3):
            fill_random_normal(noise.face[s][d], 0, ns + 1, 0.0, 1.0, seed, (step << 8) | sid); sid += 1
            fill_random_normal(noise.edge[s][d], 0, 1, 0.0, 1.0, seed, (step << 8) | sid); sid += 1
            fill_random_normal(noise.cen[s][d], 0, 1, 0.0, 2.0, seed, (step << 8) | sid); sid += 1
    # ranchem_A / ranchem_B, variance 1 (timeStepStag.cpp:225-229)
    for s in range(2):
        if noise.chem[s] is not None:
            fill_random_normal(noise.chem[s], 0, noise.p.nreaction, 0.0, 1.0, seed, (step << 8) | sid); sid += 1


def stats_stag(st, stats, steps, flags=15):
    """evaluateStatsStag3D's per-cell statistics (statsStag.cpp:10-77) on host
    MultiFabs; returns the FHD_* code."""
    set_params(st.p)
    s = stats.c_struct()
    return lib().orc_stats_stag(st.cu.fab(), st.prim.fab(), st.mom_fabs(), C.byref(s), steps, flags)


def set_threads(n=0):
    """OpenMP threads of the oracle's loops (0: all host cores); returns the count."""
    return lib().orc_set_threads(int(n))


def fill_noise_mt64(noise, seed=1):
    """Injected-noise A/B fields drawn on the host from std::mt19937_64(seed) with
    Box-Muller (faces/edges variance 1, centres variance 2), OverrideSync'ed and
    FillBoundary'ed: the noise of the injected-noise parity runs."""
    set_params(noise.p)
    nz = noise.c_struct()
    _chk(lib().orc_fill_noise_mt64(C.byref(nz), seed), "fill_noise_mt64")


def philox4x32_10(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return list(o)


def max_acoustic_cfl(st, dt):
    return lib().orc_max_acoustic_cfl(st.prim.fab(), st.vel_fabs(), dt)


def init_state(st, p):
    """main_driver init: InitConsVarStag -> conservedToPrimitiveStag -> FillBoundary
    (main_driver.cpp:757-790)."""
    set_params(p)
    init_cons_var_stag(st, p)
    _chk(conserved_to_primitive(st), "convert")
    for m in [st.cu, st.prim] + st.cumom + st.vel:
        fill_boundary(m)
