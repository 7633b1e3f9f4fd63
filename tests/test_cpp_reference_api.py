"""The C++ reference-signature layer (include/fhd/reference_api.hpp over
include/fhd/amrex_compat.hpp): a driver that calls InitConsVarStag,
conservedToPrimitiveStag, FillBoundary, calculateTransportCoeffs and
RK3stepStag by the reference's names must give the same MultiFab shapes as the
Python layer (CPU) and the same state, bit for bit, as the Python path through
the C ABI (GPU), also when its MultiFabs live in pinned host memory."""
import os
import shutil
import subprocess

import numpy as np
import pytest
import torch

from fhdex_b200.params import argon, no2_dimerization, stable_dt
from fhdex_b200.state import StagState

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "fhdex_b200", "lib")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if not os.path.exists(os.path.join(LIBDIR, "libfhd_b200.so")):
        pytest.skip("libfhd_b200.so not built")
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no g++")
    exe = str(tmp_path_factory.mktemp("cpp") / "reference_driver")
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-Wno-unused-parameter",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", "reference_driver.cpp"), "-o", exe,
           "-L", LIBDIR, "-lfhd_b200", f"-Wl,-rpath,{LIBDIR}",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_compat_shapes_match_python_layer(driver):
    n = 6
    r = subprocess.run([driver, "shapes", str(n)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    rows = {}
    for line in r.stdout.splitlines():
        name, *v = line.split()
        rows[name] = [int(x) for x in v]
    assert rows.pop("array4") == [1, 1]
    st = StagState(argon(n, dx=8e-6), "cpu")
    names = {"cu": st.cu, "prim": st.prim, "source": st.source, "eta": st.eta, "chi": st.chi, "D": st.D,
             "edgeflux_x0": st.edgeflux[0], "edgeflux_x1": st.edgeflux[1], "edgeflux_y1": st.edgeflux[3]}
    for d in range(3):
        names[f"cumom{d}"] = st.cumom[d]
        names[f"vel{d}"] = st.vel[d]
        names[f"faceflux{d}"] = st.faceflux[d]
        names[f"cenflux{d}"] = st.cenflux[d]
    for name, mf in names.items():
        f = mf.fab()
        want = list(f.lo) + list(f.hi) + [f.ncomp] + list(f.nodal)
        assert rows[name] == want, (name, rows[name], want)


def read_state(path, st):
    """Split the driver's output into arrays shaped like the MultiFabs of `st`."""
    raw = np.fromfile(path, dtype=np.float64)
    off = 0
    out = []
    for m in [st.cu] + st.cumom + [st.prim] + st.vel:
        k = m.arr.numel()
        out.append(torch.from_numpy(raw[off:off + k].copy()).view(m.arr.shape))
        off += k
    assert off == raw.size
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("arena,gas", [("device", "argon"), ("pinned", "argon"), ("device", "no2"), ("pinned", "no2")])
def test_reference_driver_equals_c_abi_path(driver, tmp_path, arena, gas):
    """The reference-named API (RK3stepStag over the compat MultiFabs, parameters in
    the common::/compressible::/chemistry:: globals) equals the C ABI bit for bit;
    no2 runs the chemistry source inside every stage."""
    from fhdex_b200.context import Context
    n, nsteps, seed = 12, 3, 7
    p = no2_dimerization(n, dx=8e-6, seed=seed) if gas == "no2" else argon(n, dx=8e-6, seed=seed)
    dt = stable_dt(p)
    out = str(tmp_path / "state.bin")
    r = subprocess.run([driver, "run", arena, str(n), str(nsteps), str(seed), repr(dt), out, gas],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    ctx = Context(p)
    st = StagState(p, "cuda", aux=False)
    ctx.init_state(st)
    for step in range(nsteps):
        ctx.rk3_step(st, dt, step, aux=False)
    torch.cuda.synchronize()
    assert ctx.status() == 0
    got = read_state(out, st)
    names = ["cu", "cumom0", "cumom1", "cumom2", "prim", "vel0", "vel1", "vel2"]
    mfs = [st.cu] + st.cumom + [st.prim] + st.vel
    bad = [nm for nm, g, m in zip(names, got, mfs) if not torch.equal(g, m.arr.cpu())]
    assert not bad, bad
    # the state moved (the comparison is not between two initial states)
    init = StagState(p, "cuda", aux=False)
    ctx.init_state(init)
    assert not torch.equal(init.cu.arr, st.cu.arr)


@pytest.mark.gpu
def test_reference_driver_reports_massfrac_through_abort_handler(driver):
    r = subprocess.run([driver, "massfrac", "8"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 3, (r.returncode, r.stdout, r.stderr)
    assert "calculateTransportCoeffs" in r.stdout and "mass fraction" in r.stdout.lower(), r.stdout


@pytest.mark.gpu
def test_reference_driver_plotfile_equals_c_abi_plotfile(driver, tmp_path):
    """WritePlotFileStag through the reference-named layer writes the same files,
    byte for byte, as fhd_write_plotfile_stag on the same steps."""
    from fhdex_b200.context import Context
    from fhdex_b200.plotfile import write_plotfile_stag
    n, nsteps, seed = 8, 2, 5
    p = argon(n, dx=8e-6, seed=seed)
    dt = stable_dt(p)
    base = str(tmp_path / "ref_plt")
    r = subprocess.run([driver, "plot", str(n), str(nsteps), str(seed), repr(dt), base],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    ctx = Context(p)
    st = StagState(p, "cuda")
    ctx.init_state(st)
    for step in range(nsteps):
        ctx.rk3_step(st, dt, step, aux=True)
    ours = write_plotfile_stag(ctx, str(tmp_path / "abi_plt"), nsteps, nsteps * dt, st)
    theirs = base + f"{nsteps:09d}"
    for rel in ("Header", "Level_0/Cell_H", "Level_0/Cell_D_00000"):
        a = open(os.path.join(ours, rel), "rb").read()
        b = open(os.path.join(theirs, rel), "rb").read()
        assert a == b, rel


@pytest.mark.gpu
def test_reference_driver_checkpoint_restart_equals_uninterrupted_run(driver, tmp_path):
    """WriteCheckPoint, ReadCheckPoint into new MultiFabs and the remaining steps,
    all through the reference-named layer, end bitwise where n1 + n2 uninterrupted
    C-ABI steps end."""
    from fhdex_b200.context import Context
    n, n1, n2, seed = 10, 2, 3, 11
    p = argon(n, dx=8e-6, seed=seed)
    dt = stable_dt(p)
    out = str(tmp_path / "state.bin")
    r = subprocess.run([driver, "chk", str(n), str(n1), str(n2), str(seed), repr(dt), out],
                       capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert r.returncode == 0, (r.returncode, r.stderr)
    assert os.path.isdir(tmp_path / f"chk{n1 - 1:09d}")
    ctx = Context(p)
    st = StagState(p, "cuda", aux=False)
    ctx.init_state(st)
    for step in range(n1 + n2):
        ctx.rk3_step(st, dt, step, aux=False)
    torch.cuda.synchronize()
    got = read_state(out, st)
    mfs = [st.cu] + st.cumom + [st.prim] + st.vel
    bad = [k for k, (g, m) in enumerate(zip(got, mfs)) if not torch.equal(g, m.arr.cpu())]
    assert not bad, bad


@pytest.mark.gpu
def test_reference_driver_statistics_equal_c_abi_statistics(driver, tmp_path):
    """evaluateStatsStag3D through the reference-named layer (plot_means, plot_vars,
    plot_mom3, plot_mom4, plot_cross) after every step equals fhd_stats_stag bit
    for bit, and its WriteSpatialCross3D file equals fhd_write_spatial_cross's."""
    from fhdex_b200 import capi
    from fhdex_b200.context import Context
    from fhdex_b200.stats import StatsState
    n, nsteps, seed = 8, 3, 13
    p = argon(n, dx=8e-6, seed=seed).replace(cross_cell=n // 2)
    dt = stable_dt(p)
    out = str(tmp_path / "stats.bin")
    run_dir = tmp_path / "run"
    run_dir.mkdir()
    r = subprocess.run([driver, "stats", str(n), str(nsteps), str(seed), repr(dt), out],
                       capture_output=True, text=True, timeout=300, cwd=str(run_dir))
    assert r.returncode == 0, (r.returncode, r.stderr)
    ctx = Context(p)
    st = StagState(p, "cuda")
    ctx.init_state(st)
    stats = StatsState(p, "cuda", cross=True)
    for step in range(nsteps):
        ctx.rk3_step(st, dt, step, aux=True)
        ctx.stats_stag(st, stats, step + 1, 15 | capi.STATS_CROSS)
    torch.cuda.synchronize()
    stats.write_spatial_cross(nsteps, str(tmp_path) + "/")
    fname = f"spatialCross{nsteps:09d}"
    assert open(run_dir / fname).read() == open(tmp_path / fname).read()
    mfs = [stats.cuMeans, stats.cuVars, stats.primMeans, stats.primVars, stats.coVars, stats.mom3, stats.mom4]
    mfs += stats.velMeans + stats.velVars + stats.cumomMeans + stats.cumomVars
    arrs = [m.arr for m in mfs] + [stats.spatialCross, stats.dataSliceMeans_xcross]
    raw = np.fromfile(out, dtype=np.float64)
    off = 0
    bad = []
    for k, a in enumerate(arrs):
        size = a.numel()
        got = torch.from_numpy(raw[off:off + size].copy()).view(a.shape)
        off += size
        if not torch.equal(got, a.cpu()):
            bad.append(k)
    assert off == raw.size
    assert not bad, bad
    assert stats.cuVars.arr.abs().max().item() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("all_correl", [0, 1])
def test_reference_driver_lowdim_statistics_equal_c_abi_statistics(driver, tmp_path, all_correl):
    """A quasi-1-D run through the reference-named layer: evaluateStatsStag1D after
    every step equals fhd_stats_stag bit for bit (per-pencil correlations in
    spatialCrossMF, one x* or the five of all_correl), WriteSpatialCross1D's files
    equal fhd_write_spatial_cross's, and WriteCheckPoint / ReadCheckPoint carry
    spatialCrossMF through a restart (checked inside the driver)."""
    from fhdex_b200 import capi
    from fhdex_b200.context import Context
    from fhdex_b200.stats import StatsState
    nx, ny, nsteps, seed = 16, 4, 3, 17
    p = argon((nx, ny, ny), dx=8e-6, seed=seed).replace(do_1D=1, cross_cell=3, all_correl=all_correl)
    dt = stable_dt(p)
    out = str(tmp_path / "stats1d.bin")
    run_dir = tmp_path / "run"
    run_dir.mkdir()
    r = subprocess.run([driver, "stats1d", str(nx), str(ny), str(nsteps), str(seed), repr(dt), str(all_correl), out],
                       capture_output=True, text=True, timeout=300, cwd=str(run_dir))
    assert r.returncode == 0, (r.returncode, r.stderr)
    ctx = Context(p)
    st = StagState(p, "cuda")
    ctx.init_state(st)
    stats = StatsState(p, "cuda", cross=True)
    for step in range(nsteps):
        ctx.rk3_step(st, dt, step, aux=True)
        ctx.stats_stag(st, stats, step + 1, 15 | capi.STATS_CROSS)
    torch.cuda.synchronize()
    stats.write_spatial_cross(nsteps, str(tmp_path) + "/")
    names = [f"{s}_spatialCross1D_{nsteps:09d}" for s in range(5)] if all_correl else [f"spatialCross1D_{nsteps:09d}"]
    for fname in names:
        assert open(run_dir / fname).read() == open(tmp_path / fname).read(), fname
    arrs = [m.arr for m in (stats.cuMeans, stats.cuVars, stats.primMeans, stats.primVars, stats.coVars,
                            stats.mom3, stats.mom4)] + [stats.spatialCross]
    raw = np.fromfile(out, dtype=np.float64)
    off = 0
    bad = []
    for k, a in enumerate(arrs):
        size = a.numel()
        got = torch.from_numpy(raw[off:off + size].copy()).view(a.shape)
        off += size
        if not torch.equal(got, a.cpu()):
            bad.append(k)
    assert off == raw.size
    assert not bad, bad
    assert stats.spatialCross.abs().max().item() > 0
