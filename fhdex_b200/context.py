"""Python binding of the C ABI (ctypes) over single-box MultiFabs.

``Context`` owns one ``fhd_ctx``.  Every call is enqueued on torch's current CUDA
stream, so library work and torch work stay ordered without extra syncs.  The
CUDA library is required: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import capi
from .capi import FabArr3, FabArr6, FhdParams, check
from .fab import fab_array
from .params import Params
from .state import StagState, StepNoise


class Context:
    def __init__(self, p: Params, device: int = 0):
        if not torch.cuda.is_available():
            raise RuntimeError("fhdex_b200 needs a CUDA device (no CPU fallback)")
        self.lib = capi.load()
        self.p = p
        self.device = device
        self._h = C.c_void_p()
        self._cparams = p.to_c()
        check(self.lib.fhd_create(C.byref(self._h), C.byref(self._cparams), device), "fhd_create")

    # -- plumbing -----------------------------------------------------------------
    def _stream(self):
        s = torch.cuda.current_stream(self.device).cuda_stream
        check(self.lib.fhd_set_stream(self._h, C.c_void_p(s)), "fhd_set_stream")

    def close(self):
        if self._h:
            self.lib.fhd_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        check(self.lib.fhd_synchronize(self._h), "fhd_synchronize")

    def status(self) -> int:
        self._stream()
        return self.lib.fhd_status(self._h)

    def effective_params(self) -> FhdParams:
        out = FhdParams()
        check(self.lib.fhd_get_params(self._h, C.byref(out)), "fhd_get_params")
        return out

    def set_tile(self, t: int):
        check(self.lib.fhd_set_tile(self._h, t), "fhd_set_tile")

    @staticmethod
    def tiles():
        lib = capi.load()
        return [lib.fhd_tile_name(t).decode() for t in range(lib.fhd_num_tiles())]

    def profile(self, enable: bool):
        check(self.lib.fhd_profile(self._h, int(enable)), "fhd_profile")

    def profile_read(self):
        """{kind: (ms, launches)} since the last read (CUDA events, launching stream)."""
        ms = (C.c_double * len(capi.PROF_KINDS))()
        n = (C.c_int64 * len(capi.PROF_KINDS))()
        check(self.lib.fhd_profile_read(self._h, ms, n), "fhd_profile_read")
        return {k: (ms[q], n[q]) for q, k in enumerate(capi.PROF_KINDS)}

    def rk3_step_host(self, st: StagState, dt: float, step: int, noise: StepNoise | None = None):
        """RK3stepStag on host MultiFabs (copies in and out).  Returns (h2d, d2h) bytes."""
        nz = noise.c_struct() if noise is not None else None
        self._noise_struct = nz
        hb = C.c_int64()
        db = C.c_int64()
        check(self.lib.fhd_rk3_step_stag_host(self._h, st.cu.fab(), st.mom_fabs(), st.prim.fab(), st.vel_fabs(),
                                              C.byref(nz) if nz is not None else None, dt, step,
                                              C.byref(hb), C.byref(db)), "fhd_rk3_step_stag_host")
        return hb.value, db.value

    # -- reference operators --------------------------------------------------------
    def init_cons_var_stag(self, st: StagState):
        self._stream()
        rb = (C.c_double * 8)(*self.p.rhobar)
        check(self.lib.fhd_init_cons_var_stag(self._h, st.cu.fab(), st.mom_fabs(), self.p.rho0, self.p.T_init, rb),
              "fhd_init_cons_var_stag")

    def conserved_to_primitive(self, st: StagState, cu=None, mom=None):
        self._stream()
        cu = cu or st.cu
        mom = mom or st.cumom
        check(self.lib.fhd_conserved_to_primitive_stag(self._h, st.prim.fab(), st.vel_fabs(), cu.fab(),
                                                       fab_array(mom, FabArr3)), "fhd_conserved_to_primitive_stag")

    def transport_coeffs(self, st: StagState):
        self._stream()
        check(self.lib.fhd_transport_coeffs(self._h, st.prim.fab(), st.eta.fab(), st.zeta.fab(), st.kappa.fab(),
                                            st.chi.fab(), st.D.fab()), "fhd_transport_coeffs")

    def flux_stag(self, st: StagState, sf, se, sc, dt):
        self._stream()
        check(self.lib.fhd_flux_stag(self._h, st.cu.fab(), st.mom_fabs(), st.prim.fab(), st.vel_fabs(),
                                     st.eta.fab(), st.zeta.fab(), st.kappa.fab(), st.chi.fab(), st.D.fab(),
                                     st.faceflux_fabs(), st.edgeflux_fabs(), st.cenflux_fabs(),
                                     fab_array(sf, FabArr3), fab_array(se, FabArr3), fab_array(sc, FabArr3), dt),
              "fhd_flux_stag")

    def fill_boundary(self, mf):
        self._stream()
        check(self.lib.fhd_fill_boundary(self._h, mf.fab()), "fhd_fill_boundary")

    def set_bc(self, st: StagState, cu=None, mom=None):
        """setBCStag on (prim, cu, cumom, vel); nothing on a fully periodic box."""
        self._stream()
        cu = cu or st.cu
        mom = mom or st.cumom
        mf = FabArr3(*[m.fab() for m in mom])
        check(self.lib.fhd_set_bc_stag(self._h, st.prim.fab(), cu.fab(), mf, st.vel_fabs()), "fhd_set_bc_stag")

    def set_reservoir_record(self, buf=None, cap: int = 0):
        """Test hook: record the particle reservoir's draws of the next steps into buf
        (a CUDA float64 tensor of 3 x interface faces x cap values); None stops it."""
        ptr = C.c_void_p(buf.data_ptr()) if buf is not None else None
        check(self.lib.fhd_set_reservoir_record(self._h, ptr, cap if buf is not None else 0),
              "fhd_set_reservoir_record")

    def override_sync(self, mf):
        self._stream()
        check(self.lib.fhd_override_sync(self._h, mf.fab()), "fhd_override_sync")

    def fill_random_normal(self, mf, scomp, ncomp, mean, variance, overridesync=True, fillboundary=True,
                           stream_id=0):
        self._stream()
        check(self.lib.fhd_fill_random_normal(self._h, mf.fab(), scomp, ncomp, mean, variance, int(overridesync),
                                              int(fillboundary), stream_id), "fhd_fill_random_normal")

    def fill_random_uniform(self, mf, scomp, ncomp, overridesync=True, fillboundary=True, stream_id=0):
        """MultiFabFillRandomUniform: uniforms in [0, 1) on the valid region."""
        self._stream()
        check(self.lib.fhd_fill_random_uniform(self._h, mf.fab(), scomp, ncomp, int(overridesync),
                                               int(fillboundary), stream_id), "fhd_fill_random_uniform")

    def chemistry_source_cle(self, prim, source, ranchem, dt: float, dV: float | None = None):
        """compute_compressible_chemistry_source_CLE (chemistry_functions.cpp:128-193):
        species comps 5.. of ``source`` from ``prim`` and the reaction noises
        ``ranchem`` (None for reaction_type 0); dV defaults to the cell volume."""
        self._stream()
        if dV is None:
            dx = self.p.dx
            dV = dx[0] * dx[1] * dx[2]
        rf = ranchem.fab() if ranchem is not None else capi.FhdFab()
        check(self.lib.fhd_chemistry_source_cle(self._h, dt, dV, prim.fab(), source.fab(), rf),
              "fhd_chemistry_source_cle")

    def fill_step_noise(self, noise: StepNoise, step: int):
        self._stream()
        self._noise_struct = noise.c_struct()
        check(self.lib.fhd_fill_step_noise(self._h, C.byref(self._noise_struct), step), "fhd_fill_step_noise")

    def rk3_step(self, st: StagState, dt: float, step: int, noise: StepNoise | None = None, aux: bool = True):
        """RK3stepStag.  aux=True also writes the stage-3 coefficients and fluxes into
        st (the reference's by-products); aux=False skips them (the fast path)."""
        self._stream()
        nz = noise.c_struct() if noise is not None else None
        self._noise_struct = nz
        if aux and st.aux:
            args = (st.eta.fab(), st.zeta.fab(), st.kappa.fab(), st.chi.fab(), st.D.fab(),
                    st.faceflux_fabs(), st.edgeflux_fabs(), st.cenflux_fabs())
        else:
            nf = capi.FhdFab()
            args = (nf, nf, nf, nf, nf, None, None, None)
        src = st.source.fab() if st.aux else capi.FhdFab()
        rc = self.lib.fhd_rk3_step_stag(self._h, st.cu.fab(), st.mom_fabs(), st.prim.fab(), st.vel_fabs(), src,
                                        *args, C.byref(nz) if nz is not None else None, dt, step)
        check(rc, "fhd_rk3_step_stag")

    def rk3_steps(self, st: StagState, dt: float, step0: int, nsteps: int):
        """nsteps RK3stepStag steps with in-kernel noise (steps step0 .. step0+nsteps-1),
        replayed from a CUDA graph the context captures and keeps (fhd_rk3_steps_stag);
        bitwise the same as nsteps rk3_step(..., aux=False) calls.  The legacy default
        stream cannot be captured, so from it the steps run on a side stream ordered
        after and before the caller's stream."""
        cur = torch.cuda.current_stream(self.device)
        if cur.cuda_stream != 0:
            self._stream()
            check(self.lib.fhd_rk3_steps_stag(self._h, st.cu.fab(), st.mom_fabs(), st.prim.fab(), st.vel_fabs(), dt,
                                              step0, nsteps), "fhd_rk3_steps_stag")
            return
        if getattr(self, "_side", None) is None:
            self._side = torch.cuda.Stream(self.device)
        self._side.wait_stream(cur)
        with torch.cuda.stream(self._side):
            self.rk3_steps(st, dt, step0, nsteps)
        cur.wait_stream(self._side)

    def stats_stag(self, st: StagState, stats, steps: int, flags: int = 15):
        """evaluateStatsStag3D's update (fhd_stats_stag) with sample count `steps`
        (1 for the first sample after a reset); flags = capi.STATS_* (STATS_CROSS
        needs a StatsState made with cross=True and uses Params.cross_cell)."""
        self._stream()
        s = stats.c_struct()
        self._stats_struct = s
        check(self.lib.fhd_stats_stag(self._h, st.cu.fab(), st.prim.fab(), st.vel_fabs(), st.mom_fabs(),
                                      C.byref(s), steps, flags), "fhd_stats_stag")

    def init_state(self, st: StagState):
        """main_driver init: InitConsVarStag -> conservedToPrimitiveStag ->
        FillBoundary -> setBCStag (main_driver.cpp:766-780)."""
        self.init_cons_var_stag(st)
        self.conserved_to_primitive(st)
        for m in [st.cu, st.prim] + st.cumom + st.vel:
            self.fill_boundary(m)
        if self.p.walls:
            self.set_bc(st)
