"""ctypes mirror of ``include/fhd_capi.h`` and the loader of ``libfhd_b200.so``.

The C structs here must match the header field for field; ``tests/test_capi_load``
checks the sizes against the compiled library.
"""
from __future__ import annotations

import ctypes as C
import os

MAX_SPECIES = 8
MAX_REACTIONS = 8

FHD_OK = 0
FHD_ERR_BAD_ARG = 1
FHD_ERR_MASSFRAC = 2
FHD_ERR_NONFINITE = 3
FHD_ERR_OOM = 4
FHD_ERR_TIMEOUT = 5
FHD_ERR_CUDA = 6
FHD_ERR_UNSUPPORTED = 7
FHD_ERR_TOO_LARGE = 8
FHD_ERR_SINGULAR = 9
FHD_ERR_IO = 10

FHD_F64 = 0
FHD_F32 = 1

FHD_PREC_FP64 = 0
FHD_PREC_MIXED = 1


class FhdFab(C.Structure):
    _fields_ = [
        ("data", C.c_void_p),
        ("lo", C.c_int * 3),
        ("hi", C.c_int * 3),
        ("ncomp", C.c_int),
        ("nodal", C.c_int * 3),
        ("dtype", C.c_int),
    ]


NULL_FAB = FhdFab()


class FhdParams(C.Structure):
    _fields_ = [
        ("nspecies", C.c_int),
        ("n_cells", C.c_int * 3),
        ("prob_lo", C.c_double * 3),
        ("prob_hi", C.c_double * 3),
        ("molmass", C.c_double * MAX_SPECIES),
        ("diameter", C.c_double * MAX_SPECIES),
        ("dof", C.c_double * MAX_SPECIES),
        ("e0", C.c_double * MAX_SPECIES),
        ("hcv", C.c_double * MAX_SPECIES),
        ("hcp", C.c_double * MAX_SPECIES),
        ("k_B", C.c_double),
        ("Runiv", C.c_double),
        ("grav", C.c_double * 3),
        ("zeta_ratio", C.c_double),
        ("algorithm_type", C.c_int),
        ("visc_type", C.c_int),
        ("advection_type", C.c_int),
        ("transport_type", C.c_int),
        ("stoch_stress_form", C.c_int),
        ("precision", C.c_int),
        ("seed", C.c_uint64),
        ("nreaction", C.c_int),
        ("reaction_type", C.c_int),
        ("stoich_R", (C.c_int * MAX_SPECIES) * MAX_REACTIONS),
        ("stoich_P", (C.c_int * MAX_SPECIES) * MAX_REACTIONS),
        ("rate_const", C.c_double * MAX_REACTIONS),
        ("alpha_param", C.c_double * MAX_REACTIONS),
        ("beta_param", C.c_double * MAX_REACTIONS),
        ("T0_chem", C.c_double),
        ("avogadro", C.c_double),
        ("walls", C.c_int),
        ("bc_vel_lo", C.c_int * 3),
        ("bc_vel_hi", C.c_int * 3),
        ("bc_mass_lo", C.c_int * 3),
        ("bc_mass_hi", C.c_int * 3),
        ("bc_therm_lo", C.c_int * 3),
        ("bc_therm_hi", C.c_int * 3),
        ("t_lo", C.c_double * 3),
        ("t_hi", C.c_double * 3),
        ("bc_Yk_lo", (C.c_double * MAX_SPECIES) * 3),
        ("bc_Yk_hi", (C.c_double * MAX_SPECIES) * 3),
        ("bc_Xk_lo", (C.c_double * MAX_SPECIES) * 3),
        ("bc_Xk_hi", (C.c_double * MAX_SPECIES) * 3),
        ("p_lo", C.c_double * 3),
        ("p_hi", C.c_double * 3),
        ("rho_lo", C.c_double * 3),
        ("rho_hi", C.c_double * 3),
        ("rho0", C.c_double),
        ("T_init", C.c_double),
        ("rhobar", C.c_double * MAX_SPECIES),
        ("cross_cell", C.c_int),
        ("do_1D", C.c_int),
        ("do_2D", C.c_int),
        ("all_correl", C.c_int),
    ]


class FhdNoise(C.Structure):
    _fields_ = [
        ("face", (FhdFab * 3) * 2),
        ("edge", (FhdFab * 3) * 2),
        ("cen", (FhdFab * 3) * 2),
        ("chem", FhdFab * 2),
    ]


PROF_KINDS = ("cellprep", "taus", "faces", "update", "ghosts", "convert", "aux_fluxes", "fused")

FabArr3 = FhdFab * 3
FabArr6 = FhdFab * 6


class FhdStats(C.Structure):
    """fhd_stats: the reference's statistics MultiFabs (one box each)."""
    _fields_ = [("cuMeans", FhdFab), ("cuVars", FhdFab), ("primMeans", FhdFab), ("primVars", FhdFab),
                ("coVars", FhdFab), ("mom3", FhdFab), ("mom4", FhdFab),
                ("velMeans", FhdFab * 3), ("velVars", FhdFab * 3), ("cumomMeans", FhdFab * 3),
                ("cumomVars", FhdFab * 3), ("spatialCross", C.c_void_p), ("dataSliceMeans_xcross", C.c_void_p)]


STATS_MEANS, STATS_VARS, STATS_MOM3, STATS_MOM4, STATS_CROSS = 1, 2, 4, 8, 16

_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG_DIR, "lib", "libfhd_b200.so")

_lib = None


def _declare(lib):
    P = C.POINTER
    fab = FhdFab
    pfab = P(FhdFab)
    i = C.c_int
    d = C.c_double
    vp = C.c_void_p
    sigs = {
        "fhd_create": (i, [P(vp), P(FhdParams), i]),
        "fhd_destroy": (i, [vp]),
        "fhd_strerror": (C.c_char_p, [i]),
        "fhd_set_stream": (i, [vp, vp]),
        "fhd_synchronize": (i, [vp]),
        "fhd_status": (i, [vp]),
        "fhd_get_params": (i, [vp, P(FhdParams)]),
        "fhd_init_cons_var_stag": (i, [vp, fab, pfab, d, d, P(d)]),
        "fhd_conserved_to_primitive_stag": (i, [vp, fab, pfab, fab, pfab]),
        "fhd_transport_coeffs": (i, [vp, fab, fab, fab, fab, fab, fab]),
        "fhd_flux_stag": (i, [vp, fab, pfab, fab, pfab, fab, fab, fab, fab, fab,
                              pfab, pfab, pfab, pfab, pfab, pfab, d]),
        "fhd_fill_boundary": (i, [vp, fab]),
        "fhd_override_sync": (i, [vp, fab]),
        "fhd_set_bc_stag": (i, [vp, fab, fab, pfab, pfab]),
        "fhd_set_reservoir_record": (i, [vp, vp, i]),
        "fhd_fill_random_normal": (i, [vp, fab, i, i, d, d, i, i, C.c_uint64]),
        "fhd_fill_random_uniform": (i, [vp, fab, i, i, i, i, C.c_uint64]),
        "fhd_rk3_steps_stag": (i, [vp, fab, pfab, fab, pfab, d, C.c_int64, i]),
        "fhd_fill_step_noise": (i, [vp, P(FhdNoise), C.c_int64]),
        "fhd_chemistry_source_cle": (i, [vp, d, d, fab, fab, fab]),
        "fhd_plotfile_ncomp": (i, [P(FhdParams), i]),
        "fhd_plotfile_varname": (i, [P(FhdParams), i, i, C.c_char_p, i]),
        "fhd_plotfile_write_host": (i, [P(FhdParams), C.c_char_p, P(d), i, d, i]),
        "fhd_write_checkpoint": (i, [P(FhdParams), C.c_char_p, i, d, i, fab, pfab, fab, pfab, P(FhdStats)]),
        "fhd_read_checkpoint": (i, [P(FhdParams), C.c_char_p, i, P(i), P(d), P(i), fab, pfab, fab, pfab,
                                    P(FhdStats)]),
        "fhd_plotfile_pack": (i, [vp, i, fab, fab, pfab, fab, pfab, fab, fab, fab, P(FhdStats)]),
        "fhd_write_plotfile_stag": (i, [vp, C.c_char_p, i, d, i, fab, pfab, fab, pfab, fab, fab, fab,
                                        P(FhdStats)]),
        "fhd_rk3_step_stag": (i, [vp, fab, pfab, fab, pfab, fab, fab, fab, fab, fab, fab,
                                  pfab, pfab, pfab, P(FhdNoise), d, C.c_int64]),
        "fhd_rk3_step_stag_host": (i, [vp, fab, pfab, fab, pfab, P(FhdNoise), d, C.c_int64,
                                       P(C.c_int64), P(C.c_int64)]),
        "fhd_set_tile": (i, [vp, i]),
        "fhd_num_tiles": (i, []),
        "fhd_tile_name": (C.c_char_p, [i]),
        "fhd_profile": (i, [vp, i]),
        "fhd_profile_read": (i, [vp, P(d), P(C.c_int64)]),
        "fhd_measure_fma_peak": (i, [i, i, P(d)]),
        "fhd_rk3_step_stag_noalloc": (i, [P(FhdParams), fab, pfab, fab, pfab, d, C.c_int64, vp, P(i)]),
        "fhd_stats_stag": (i, [vp, fab, fab, pfab, pfab, P(FhdStats), C.c_int64, i]),
        "fhd_spatial_cross_ncross": (i, [i]),
        "fhd_spatial_cross_nstats": (i, [i]),
        "fhd_write_spatial_cross": (i, [P(FhdParams), C.c_char_p, i, vp]),
        "fhd_sf_create": (i, [P(vp), P(i), i, i, P(i), P(i), P(d), i]),
        "fhd_sf_destroy": (i, [vp]),
        "fhd_sf_set_stream": (i, [vp, vp]),
        "fhd_sf_synchronize": (i, [vp]),
        "fhd_sf_ncov": (i, [vp]),
        "fhd_sf_nsamples": (C.c_int64, [vp]),
        "fhd_sf_fort_structure": (i, [vp, fab, i]),
        "fhd_sf_finalize": (i, [vp, fab, fab, fab, i]),
        "fhd_sf_create_stack": (i, [P(vp), P(i), i, i, i, P(i), P(i), P(d), i]),
        "fhd_sf_stack_average": (i, [vp, fab, fab, i]),
        "fhd_batch_create": (i, [P(vp), i, i, i]),
        "fhd_batch_destroy": (i, [vp]),
        "fhd_batch_set_stream": (i, [vp, vp]),
        "fhd_batch_add": (i, [vp, P(FhdParams), fab, pfab, fab, pfab, d, C.c_int64, P(d), P(i)]),
        "fhd_batch_remove": (i, [vp, i]),
        "fhd_batch_step": (i, [vp, i, i]),
        "fhd_batch_size": (i, [vp]),
        "fhd_batch_set_persistent": (i, [vp, i, i]),
        "fhd_batch_set_wait_limit": (i, [vp, d, i]),
        "fhd_batch_member_status": (i, [vp, i]),
        "fhd_batch_synchronize": (i, [vp]),
        "fhd_batch_num_tiles": (i, []),
        "fhd_batch_set_tile": (i, [vp, i]),
        "fhd_batch_autotune": (i, [vp, i, P(d), P(i)]),
    }
    for name, (res, args) in sigs.items():
        if hasattr(lib, name):
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
    return lib


def load(path: str | None = None):
    """Load the compiled C-ABI library (raises if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"{p} is missing: build the CUDA library first (python -m fhdex_b200.build)")
    lib = _declare(C.CDLL(p))
    if path is None:
        _lib = lib
    return lib


class FhdError(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        self.code = code
        try:
            msg = load().fhd_strerror(code).decode()
        except Exception:  # pragma: no cover - only when the library is absent
            msg = f"code {code}"
        super().__init__(f"{where}: {msg} ({code})" if where else f"{msg} ({code})")


def check(code: int, where: str = "") -> None:
    if code != FHD_OK:
        raise FhdError(code, where)
