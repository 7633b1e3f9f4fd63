"""Build ``fhdex_b200/lib/libfhd_b200.so`` for sm_100a with nvcc (in-tree).

The kernels are compiled once per (species count, precision) in parallel:
the exact FP64 units with ``-fmad=false`` (no contraction of a*b+c, so the
reference's operation order is kept), the mixed-precision units with FMA
contraction allowed.  ``python -m fhdex_b200.build`` rebuilds what is stale.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "_build", "obj")
LIB = os.path.join(PKG, "lib", "libfhd_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
BASE = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
               "-Xptxas", "-v", f"-I{CSRC}", f"-I{os.path.join(ROOT, 'include')}"]
SPECIES = (1, 2, 3, 4)

HEADERS = ["fhd_div.h", "fhd_device.cuh", "philox.cuh", "fhd_flux.cuh", "fhd_kernels.cuh", "fhd_launch.cuh", "fhd_fused.cuh", "fhd_host.h", "fhd_chem.cuh", "fhd_vismf.h", "fhd_walls.cuh"]


def _units():
    u = []
    for ns in SPECIES:
        u.append((f"kern_exact_ns{ns}", "fhd_kern_ns.cu", [f"-DFHD_NS={ns}", "-fmad=false"]))
        u.append((f"kern_mixed_ns{ns}", "fhd_kern_ns.cu", [f"-DFHD_NS={ns}", "-DFHD_MIXED=1", "-fmad=true"]))
    u.append(("exact_util", "fhd_exact.cu", ["-fmad=false"]))
    u.append(("capi", "fhd_capi.cu", ["-fmad=false"]))
    u.append(("noalloc", "fhd_noalloc.cu", ["-fmad=false"]))
    u.append(("batch", "fhd_batch.cu", ["-fmad=false"]))
    u.append(("stats", "fhd_stats.cu", ["-fmad=false"]))
    u.append(("sf", "fhd_sf.cu", ["-fmad=false"]))
    u.append(("chem", "fhd_chem.cu", ["-fmad=false"]))
    u.append(("plot", "fhd_plot.cu", ["-fmad=false"]))
    u.append(("chk", "fhd_chk.cu", []))
    u.append(("peak", "fhd_peak.cu", []))
    return u


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(ROOT, "include", "fhd_capi.h"), __file__]
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(name, src, flags, verbose):
    obj = os.path.join(OBJ, name + ".o")
    if not _stale(obj, src):
        return obj, None
    cmd = [NVCC] + BASE + flags + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    with open(os.path.join(OBJ, name + ".ptxas.log"), "w") as f:
        f.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {name}:\n{r.stderr[-4000:]}")
    return obj, name


def build(verbose=False, jobs=None):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    units = _units()
    jobs = jobs or min(len(units), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda u: _compile(*u, verbose), units))
    objs = [o for o, _ in results]
    rebuilt = [n for _, n in results if n]
    if rebuilt or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cudalib = os.path.join(os.path.dirname(os.path.dirname(NVCC)), "lib64")
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-L" + cudalib, "-lcufft", "-Xlinker",
                                                             "-rpath=" + cudalib]
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
