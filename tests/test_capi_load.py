"""CPU checks of the drop-in boundary: the sm_100a library loads, exports every
entry point include/fhd_capi.h declares, and its structs match the ctypes mirror.
No compute calls (no GPU here)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from fhdex_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fhd_capi.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(fhd_\w+)\s*\(", txt, flags=re.M)))


def test_library_exists_and_loads():
    assert os.path.exists(capi.LIB_PATH), "build the library first (python -m fhdex_b200.build)"
    capi.load()


def test_every_declared_entry_point_is_exported():
    syms = declared_symbols()
    assert len(syms) >= 15
    lib = C.CDLL(capi.LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_struct_layouts_match_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text(f'#include "{HEADER}"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(fhd_fab), sizeof(fhd_params), '
                   'sizeof(fhd_noise), offsetof(fhd_params, seed), sizeof(fhd_stats), '
                   'offsetof(fhd_stats, cumomVars), offsetof(fhd_params, stoich_P), offsetof(fhd_params, avogadro), '
                   'offsetof(fhd_noise, chem));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.check_call(["gcc", str(src), "-o", str(exe)])
    vals = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    assert vals == [C.sizeof(capi.FhdFab), C.sizeof(capi.FhdParams), C.sizeof(capi.FhdNoise),
                    capi.FhdParams.seed.offset, C.sizeof(capi.FhdStats), capi.FhdStats.cumomVars.offset,
                    capi.FhdParams.stoich_P.offset, capi.FhdParams.avogadro.offset, capi.FhdNoise.chem.offset]


def test_strerror_is_callable_without_gpu():
    lib = capi.load()
    assert lib.fhd_strerror(capi.FHD_ERR_MASSFRAC).startswith(b"mass fraction")


@pytest.mark.parametrize("change,code", [
    (dict(nspecies=5), "FHD_ERR_UNSUPPORTED"),
    (dict(nspecies=0), "FHD_ERR_UNSUPPORTED"),
    (dict(n_cells=(1, 8, 8)), "FHD_ERR_BAD_ARG"),
    (dict(n_cells=(2048, 2048, 1024)), "FHD_ERR_UNSUPPORTED"),   # 2^32 cells
    (dict(algorithm_type=0), "FHD_ERR_UNSUPPORTED"),
    (dict(stoch_stress_form=2), "FHD_ERR_UNSUPPORTED"),
    (dict(advection_type=3), "FHD_ERR_UNSUPPORTED"),
    (dict(precision=7), "FHD_ERR_BAD_ARG"),
    (dict(visc_type=3, zeta_ratio=-1.0), "FHD_ERR_BAD_ARG"),
    (dict(transport_type=4), "FHD_ERR_UNSUPPORTED"),
    (dict(transport_type=0), "FHD_ERR_UNSUPPORTED"),
    (dict(transport_type=2, precision=1), "FHD_ERR_UNSUPPORTED"),
])
def test_create_rejects_out_of_scope_parameters_without_gpu(change, code):
    """fhd_create validates the run before touching a device: out-of-scope options
    and impossible boxes come back as error codes, never as a crash."""
    from fhdex_b200.params import argon
    p = argon(8, dx=8e-6)
    for k, v in change.items():
        setattr(p, k, v)
    if "n_cells" in change:
        p.prob_hi = tuple(p.prob_lo[d] + 8e-6 * p.n_cells[d] for d in range(3))
    cp = p.to_c()
    h = C.c_void_p()
    lib = capi.load()
    assert lib.fhd_create(C.byref(h), C.byref(cp), 0) == getattr(capi, code)
    assert not h.value


@pytest.mark.parametrize("field,value,code", [
    ("nreaction", 9, "FHD_ERR_BAD_ARG"),
    ("nreaction", -1, "FHD_ERR_BAD_ARG"),
    ("reaction_type", 2, "FHD_ERR_UNSUPPORTED"),   # SSA / tau leaping (chemistry_functions.cpp:131-133)
    ("T0_chem", 0.0, "FHD_ERR_BAD_ARG"),           # chemistry_functions.cpp:135
    ("stoich_R", -1, "FHD_ERR_BAD_ARG"),
])
def test_create_rejects_bad_chemistry_without_gpu(field, value, code):
    from fhdex_b200.params import no2_dimerization
    cp = no2_dimerization(8).to_c()
    if field == "stoich_R":
        cp.stoich_R[1][0] = value
    else:
        setattr(cp, field, value)
    h = C.c_void_p()
    lib = capi.load()
    assert lib.fhd_create(C.byref(h), C.byref(cp), 0) == getattr(capi, code)
    assert not h.value


def test_chemistry_operator_validates_without_gpu():
    lib = capi.load()
    nf = capi.FhdFab()
    assert lib.fhd_chemistry_source_cle(None, 1e-12, 1e-15, nf, nf, nf) == capi.FHD_ERR_BAD_ARG


def test_batch_tile_entry_points_validate_without_gpu():
    """The batch's launch-shape choices and the argument checks of its tile calls
    (no batch object needed, so no GPU)."""
    lib = capi.load()
    assert lib.fhd_batch_num_tiles() == 3
    assert lib.fhd_batch_set_tile(None, 0) == capi.FHD_ERR_BAD_ARG
    assert lib.fhd_batch_autotune(None, 3, None, None) == capi.FHD_ERR_BAD_ARG
    assert lib.fhd_batch_set_persistent(None, 1, -1) == capi.FHD_ERR_BAD_ARG
    assert lib.fhd_batch_set_wait_limit(None, 1.0, -1) == capi.FHD_ERR_BAD_ARG
