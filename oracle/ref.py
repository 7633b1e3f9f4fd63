"""ctypes front end of oracle/_ref/libfhd_ref.so (TEST INFRASTRUCTURE ONLY).

The library is FHDeX's own hot-path sources (timeStepStag.cpp, fluxStag.cpp,
conservedPrimitiveConversionsStag.cpp, transCoeffs.cpp, boundaryStag.cpp,
compressible_functions*.cpp, MultiFabFillRandom.cpp, chemistry_functions.cpp,
common_functions.cpp, reservoirStag.cpp) compiled unmodified against the
host-only AMReX stand-in in ``oracle/amrex_host`` (recipe: ``make -C oracle
ref``), with ``oracle/ref_driver.cpp`` as its C ABI.  The tests run it beside
the restated oracle (``oracle/fhd_oracle.cpp``) on the same inputs to pin the
restatement to the reference's code.  It is built where the reference tree
exists; the built library travels with the repository to machines without it.

Functions take host MultiFabs from ``fhdex_b200.state`` (the geometry the
reference's main_driver gives them) and a ``Params`` whose ``to_inputs()`` deck
the reference's own namespace initialisers read.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import torch

_DIR = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_DIR, "_ref", "libfhd_ref.so")
REF_TREE = os.environ.get("FHD_REFERENCE_TREE", "/root/reference")
_lib = None
_params = None


def build():
    """Compile the reference sources where the reference tree exists."""
    if os.path.isdir(REF_TREE):
        subprocess.check_call(["make", "-s", "-C", _DIR, "ref", f"REF={REF_TREE}", f"-j{os.cpu_count() or 4}"])


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P = C.POINTER
        d, i, vp = C.c_double, C.c_int, C.c_void_p
        pp = P(vp)
        L.fhdref_error.restype = C.c_char_p
        L.fhdref_init.argtypes = [C.c_char_p]
        L.fhdref_globals.argtypes = [P(i), P(i), P(i), P(i), P(d), P(d), P(i)]
        L.fhdref_init_cons_var_stag.argtypes = [vp, pp]
        L.fhdref_conserved_to_primitive.argtypes = [vp, pp, vp, pp]
        L.fhdref_set_bc.argtypes = [vp, vp, pp, pp]
        L.fhdref_transport.argtypes = [vp] * 6
        L.fhdref_flux.argtypes = [vp, pp, vp, pp, vp, vp, vp, vp, vp, pp, pp, pp, pp, pp, pp, d, d, d]
        L.fhdref_rk3_step.argtypes = [vp, pp, vp, pp, vp, vp, vp, vp, vp, vp, pp, pp, pp, vp, pp, pp, d, i]
        L.fhdref_noise_log.argtypes = [P(i), P(i), P(d), i]
        L.fhdref_chemistry_source.argtypes = [d, d, vp, vp, vp]
        L.fhdref_max_acoustic_cfl.argtypes = [vp, pp, d, P(d)]
        L.fhdref_fill_boundary.argtypes = [vp, P(i), i, i, i]
        L.fhdref_wall_composition.argtypes = [i, P(d), P(d)]
        L.fhdref_wall_state.argtypes = [i, P(d)]
        L.fhdref_set_reservoir_draws.argtypes = [vp, i]
        L.fhdref_eval_stats3d.argtypes = [vp, vp, pp, pp, pp, P(i), pp, vp, vp, i, i]
        L.fhdref_write_spatial_cross.argtypes = [vp, i, i]
        L.fhdref_eval_stats_lowdim.argtypes = [vp, vp, pp, pp, pp, P(i), pp, vp, i, i, i]
        L.fhdref_write_spatial_cross_1d.argtypes = [vp, i, i, i]
        L.fhdref_plotfile.argtypes = [vp, pp, vp, pp, vp, vp, vp, pp, P(i), pp, i, d, vp, C.c_long, C.c_char_p, i,
                                      P(i)]
        _lib = L
    return _lib


def _chk(rc, what):
    if rc != 0:
        raise RuntimeError(f"reference {what}: {lib().fhdref_error().decode()}")


def _ptr(t: torch.Tensor):
    assert t.device.type == "cpu" and t.dtype == torch.float64 and t.is_contiguous()
    return C.c_void_p(t.data_ptr())


def _ptrs(tensors):
    arr = (C.c_void_p * len(tensors))()
    for q, t in enumerate(tensors):
        arr[q] = None if t is None else _ptr(t).value
    return arr


def init(p):
    """Read ``p``'s deck through the reference's namespace initialisers."""
    global _params
    if _params is not p:
        _chk(lib().fhdref_init(p.to_inputs().encode()), "init")
        _params = p


def globals_(p):
    """(nspecies, nvars, nprimvars, ngc, hcv[:ns], hcp[:ns], nreaction) as the
    reference derives them (GetHcGas, compressible_functions.cpp:91-100)."""
    init(p)
    ns, nv, npv, ng, nr = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
    hv = (C.c_double * 8)()
    hp = (C.c_double * 8)()
    _chk(lib().fhdref_globals(C.byref(ns), C.byref(nv), C.byref(npv), C.byref(ng), hv, hp, C.byref(nr)), "globals")
    return ns.value, nv.value, npv.value, ng.value, list(hv[:ns.value]), list(hp[:ns.value]), nr.value


def init_cons_var_stag(st):
    init(st.p)
    _chk(lib().fhdref_init_cons_var_stag(_ptr(st.cu.arr), _ptrs([m.arr for m in st.cumom])), "InitConsVarStag")


def conserved_to_primitive(st):
    init(st.p)
    _chk(lib().fhdref_conserved_to_primitive(_ptr(st.prim.arr), _ptrs([m.arr for m in st.vel]), _ptr(st.cu.arr),
                                             _ptrs([m.arr for m in st.cumom])), "conservedToPrimitiveStag")


def set_bc(st):
    init(st.p)
    _chk(lib().fhdref_set_bc(_ptr(st.prim.arr), _ptr(st.cu.arr), _ptrs([m.arr for m in st.cumom]),
                             _ptrs([m.arr for m in st.vel])), "setBCStag")


def transport(st):
    init(st.p)
    _chk(lib().fhdref_transport(_ptr(st.prim.arr), _ptr(st.eta.arr), _ptr(st.zeta.arr), _ptr(st.kappa.arr),
                                _ptr(st.chi.arr), _ptr(st.D.arr)), "calculateTransportCoeffs")


def _ref_edges(e3):
    """The reference's six edge MultiFabs (edgeflux_x = {xy, xz}, _y = {xy, yz},
    _z = {xz, yz}) from the three distinct noise fields xy, xz, yz.  The
    reference's flux reads only x[0], x[1] and y[1]; the other three get the
    negated fields, so that a read of them would show as a mismatch."""
    xy, xz, yz = e3
    return [xy, xz, (-xy).contiguous(), yz, (-xz).contiguous(), (-yz).contiguous()]


def flux(st, sf, se, sc, dt, w1=1.0, w2=0.0):
    """calculateFluxStag with the weighted noise W: sf[3] face fields (nspecies+1
    comps: energy, species), se[3] edge fields (xy, xz, yz), sc[3] centre fields
    (one ghost), host MultiFabs in the layout of fhdex_b200.state.StepNoise.
    The reference's face noise MultiFab has nvars components with the energy at
    component 4; the first four are left zero."""
    init(st.p)
    nv = st.p.nvars
    faces = []
    for d in range(3):
        f = torch.zeros((nv,) + tuple(sf[d].arr.shape[1:]), dtype=torch.float64)
        f[4:] = sf[d].arr
        faces.append(f)
    edges = _ref_edges([m.arr for m in se])
    _chk(lib().fhdref_flux(_ptr(st.cu.arr), _ptrs([m.arr for m in st.cumom]), _ptr(st.prim.arr),
                           _ptrs([m.arr for m in st.vel]), _ptr(st.eta.arr), _ptr(st.zeta.arr), _ptr(st.kappa.arr),
                           _ptr(st.chi.arr), _ptr(st.D.arr), _ptrs([m.arr for m in st.faceflux]),
                           _ptrs([m.arr for m in st.edgeflux]), _ptrs([m.arr for m in st.cenflux]), _ptrs(faces),
                           _ptrs(edges), _ptrs([m.arr for m in sc]), w1, w2, dt), "calculateFluxStag")


def step_normals(noise):
    """The fields of RK3stepStag's MultiFabFillRandomNormal calls, in the
    reference's order (timeStepStag.cpp:172-222), from a StepNoise (face[s][d]:
    energy + species comps; edge[s][e]: xy, xz, yz; cen[s][d]: one ghost): 24 in
    3-D; with do_1D the x faces and the first centre field (4); with do_2D the x
    and y faces, the xy edges of stochedge_x and stochedge_y and the first two
    centre fields (12)."""
    p = noise.p
    dims = 1 if p.do_1D else 2 if p.do_2D else 3
    out = []
    for d in range(dims):
        out += [noise.face[0][d].arr, noise.face[1][d].arr]
    eA = _ref_edges([m.arr for m in noise.edge[0]])
    eB = _ref_edges([m.arr for m in noise.edge[1]])
    if dims == 2:
        for e in (0, 2):  # stochedge_x[0], stochedge_y[0] (both xy)
            out += [eA[e], eB[e]]
    elif dims == 3:
        for i in range(2):
            for e in (i, 2 + i, 4 + i):  # stochedge_x[i], _y[i], _z[i]
                out += [eA[e], eB[e]]
    for d in range(dims):
        out += [noise.cen[0][d].arr, noise.cen[1][d].arr]
    return out


def rk3_step(st, noise, dt, step=0):
    """RK3stepStag with the step's noise injected from ``noise`` (StepNoise).
    Returns the log of the 24 noise fills: (scomp, ncomp, mean, stddev, nodal)."""
    init(st.p)
    normals = step_normals(noise)
    chem = []
    nr = st.p.nreaction
    for m in range(nr):
        for s in range(2):
            chem.append(noise.chem[s].arr[m].contiguous())
    _chk(lib().fhdref_rk3_step(_ptr(st.cu.arr), _ptrs([m.arr for m in st.cumom]), _ptr(st.prim.arr),
                               _ptrs([m.arr for m in st.vel]), _ptr(st.source.arr), _ptr(st.eta.arr),
                               _ptr(st.zeta.arr), _ptr(st.kappa.arr), _ptr(st.chi.arr), _ptr(st.D.arr),
                               _ptrs([m.arr for m in st.faceflux]), _ptrs([m.arr for m in st.edgeflux]),
                               _ptrs([m.arr for m in st.cenflux]),
                               _ptr(noise_ranchem(st)) if nr > 0 else None, _ptrs(normals),
                               _ptrs(chem) if nr > 0 else None, dt, step), "RK3stepStag")
    return noise_log()


def noise_ranchem(st):
    """The caller's ranchem MultiFab (nreaction comps, ngc ghosts), as main_driver.cpp:1006-1007 defines it."""
    if getattr(st, "_ref_ranchem", None) is None:
        from fhdex_b200.fab import CELL, MultiFab
        st._ref_ranchem = MultiFab(st.p.n_cells, CELL, st.p.nreaction, st.p.ngc).arr
    return st._ref_ranchem


def noise_log():
    n = C.c_int()
    ints = (C.c_int * (11 * 64))()
    reals = (C.c_double * (2 * 64))()
    lib().fhdref_noise_log(C.byref(n), ints, reals, 64)
    out = []
    for q in range(n.value):
        o = ints[11 * q: 11 * q + 11]
        out.append(dict(scomp=o[0], ncomp=o[1], lo=tuple(o[2:5]), hi=tuple(o[5:8]), nodal=tuple(o[8:11]),
                        mean=reals[2 * q], stddev=reals[2 * q + 1]))
    return out


def chemistry_source(p, dt, dV, prim, source, ranchem):
    init(p)
    _chk(lib().fhdref_chemistry_source(dt, dV, _ptr(prim.arr), _ptr(source.arr), _ptr(ranchem.arr)),
         "compute_compressible_chemistry_source_CLE")


def fill_boundary(p, mf, override_sync=False):
    """The stand-in's FillBoundary (and OverrideSync) of one host MultiFab with p's
    periodicity: ghost points of wall directions are left alone."""
    init(p)
    nod = (C.c_int * 3)(*mf.nodal)
    _chk(lib().fhdref_fill_boundary(_ptr(mf.arr), nod, mf.ncomp, mf.ngrow, int(override_sync)), "FillBoundary")


def wall_composition(p, side):
    """(Yk, Xk) of wall side 2 d + hi after SetupCWallStag."""
    init(p)
    y = (C.c_double * 8)()
    x = (C.c_double * 8)()
    _chk(lib().fhdref_wall_composition(side, y, x), "SetupCWallStag")
    return list(y[:p.nspecies]), list(x[:p.nspecies])


def set_reservoir_draws(rec, cap):
    """Feed the particle reservoir's draws (a contiguous float64 CPU tensor laid out as
    fhd_set_reservoir_record writes them) to the next rk3_step; None turns it off."""
    lib()
    if rec is None:
        _chk(lib().fhdref_set_reservoir_draws(None, 0), "reservoir draws")
        return
    assert rec.dtype == torch.float64 and rec.is_contiguous() and rec.device.type == "cpu"
    _chk(lib().fhdref_set_reservoir_draws(C.c_void_p(rec.data_ptr()), cap), "reservoir draws")


def wall_state(p, side):
    """(t, p, rho) of wall side 2 d + hi after SetupCWallStag (reservoirs)."""
    init(p)
    out = (C.c_double * 3)()
    _chk(lib().fhdref_wall_state(side, out), "SetupCWallStag")
    return tuple(out)


def state_from_reference(p, seed=0, amp=0.02, vel_amp=0.05):
    """A perturbed physical state made with the reference's own operators, valid
    for walls: InitConsVarStag, random perturbations of the valid density,
    composition, energy and face momenta, then conservedToPrimitiveStag,
    FillBoundary (periodic directions) and setBCStag, main_driver's init sequence
    (main_driver.cpp:757-794)."""
    from fhdex_b200.state import StagState
    st = StagState(p)
    init(p)
    init_cons_var_stag(st)
    g = torch.Generator().manual_seed(seed)
    ns = p.nspecies
    vc = st.cu.valid()
    shp = vc.shape[1:]
    rho = vc[0].clone()
    frac = torch.stack([vc[5 + s] / rho for s in range(ns)])
    frac = frac * (1.0 + amp * (2 * torch.rand((ns,) + shp, generator=g, dtype=torch.float64) - 1))
    frac = frac / frac.sum(0)
    rho_new = rho * (1.0 + amp * (2 * torch.rand(shp, generator=g, dtype=torch.float64) - 1))
    vc[0] = rho_new
    for s in range(ns):
        vc[5 + s] = rho_new * frac[s]
    vc[4] = vc[4] * (1.0 + 0.5 * amp * (2 * torch.rand(shp, generator=g, dtype=torch.float64) - 1))
    c = p.sound_speed()
    for d in range(3):
        mv = st.cumom[d].valid(0)
        mv.copy_(p.rho0 * vel_amp * c * (2 * torch.rand(mv.shape, generator=g, dtype=torch.float64) - 1))
        fill_boundary(p, st.cumom[d], override_sync=True)
    fill_boundary(p, st.cu)
    conserved_to_primitive(st)
    for m in [st.cu, st.prim] + st.vel:
        fill_boundary(p, m)
    set_bc(st)
    return st


def step_noise(p, seed):
    """A/B noise of one step as the reference's fills leave it: standard normals
    (faces, edges) and normals of variance 2 (centres, one ghost) at every point of
    each field's storage, then OverrideSync and FillBoundary with p's periodicity
    (wall directions keep their own values, ghosts included)."""
    import math as _m
    from fhdex_b200.state import StepNoise
    nz = StepNoise(p)
    g = torch.Generator().manual_seed(seed)
    # the x centre noise of a quasi-1-D run has variance 1 (timeStepStag.cpp:208-210)
    cvar = [1.0 if p.do_1D else 2.0, 2.0, 2.0]
    for s_ in range(2):
        for d in range(3):
            for mf, var in ((nz.face[s_][d], 1.0), (nz.edge[s_][d], 1.0), (nz.cen[s_][d], cvar[d])):
                mf.arr.copy_(_m.sqrt(var) * torch.randn(mf.arr.shape, generator=g, dtype=torch.float64))
                fill_boundary(p, mf, override_sync=True)
        if nz.chem[s_] is not None:
            nz.chem[s_].arr.copy_(torch.randn(nz.chem[s_].arr.shape, generator=g, dtype=torch.float64))
    return nz


def max_acoustic_cfl(st, dt):
    init(st.p)
    out = C.c_double()
    _chk(lib().fhdref_max_acoustic_cfl(_ptr(st.prim.arr), _ptrs([m.arr for m in st.vel]), dt, C.byref(out)),
         "GetMaxAcousticCFL")
    return out.value


SQRT2 = math.sqrt(2.0)


def eval_stats(st, stats, steps, flags):
    """evaluateStatsStag3D (statsStag.cpp:10-76) of the reference on host state
    ``st`` and host StatsState ``stats`` (mom3 / mom4 allocated; spatialCross with
    FHD_STATS_CROSS), with the deck's plot_* keys set from ``flags`` (the bits of
    fhd_stats_stag) and cross_cell from the Params."""
    p = st.p
    extra = (f"plot_means = {int(bool(flags & 1))}\nplot_vars = {int(bool(flags & 2))}\n"
             f"plot_covars = {int(bool(flags & 2))}\nplot_mom3 = {int(bool(flags & 4))}\n"
             f"plot_mom4 = {int(bool(flags & 8))}\nplot_cross = {int(bool(flags & 16))}\n")
    global _params
    _chk(lib().fhdref_init((p.to_inputs() + extra).encode()), "init")
    _params = None
    cells = [stats.cuMeans, stats.cuVars, stats.primMeans, stats.primVars, stats.coVars, stats.mom3, stats.mom4]
    ng = (C.c_int * 7)(*[m.ngrow for m in cells])
    faces = stats.velMeans + stats.velVars + stats.cumomMeans + stats.cumomVars
    ncross = 37 + p.nspecies + 3
    if p.do_1D or p.do_2D:
        if stats.spatialCross is not None:
            sc = stats.spatialCross
        else:
            N = p.n_cells
            sc = torch.zeros((5 if p.do_1D and p.all_correl == 1 else 1) * ncross, N[2], N[1], N[0],
                             dtype=torch.float64)
        _chk(lib().fhdref_eval_stats_lowdim(_ptr(st.cu.arr), _ptr(st.prim.arr), _ptrs([m.arr for m in st.vel]),
                                            _ptrs([m.arr for m in st.cumom]), _ptrs([m.arr for m in cells]), ng,
                                            _ptrs([m.arr for m in faces]), _ptr(sc), sc.shape[0], ncross, int(steps)),
             "evaluateStatsStag1D/2D")
        return
    if stats.spatialCross is not None:
        sc, xc = stats.spatialCross, stats.dataSliceMeans_xcross
    else:
        sc = torch.zeros(p.n_cells[0], ncross, dtype=torch.float64)
        xc = torch.zeros(2 * p.nvars + 8 + 2 * p.nspecies, dtype=torch.float64)
    _chk(lib().fhdref_eval_stats3d(_ptr(st.cu.arr), _ptr(st.prim.arr), _ptrs([m.arr for m in st.vel]),
                                   _ptrs([m.arr for m in st.cumom]), _ptrs([m.arr for m in cells]), ng,
                                   _ptrs([m.arr for m in faces]), _ptr(sc), _ptr(xc), sc.shape[1], int(steps)),
         "evaluateStatsStag3D")


def plotfile(st, stats, flags, step=0, time=0.0):
    """WritePlotFileStag (writePlotFileStag.cpp:7-527) of the reference on host
    state ``st`` (with eta, kappa, zeta) and host StatsState ``stats``: returns the
    composed plotfile MultiFab's valid cells as a (ncomp, nz, ny, nx) tensor and
    its component names.  ``flags`` are the FHD_PLOT_* bits (plot_means 1,
    plot_vars 2, plot_covars 4, plot_mom3 8, plot_mom4 16, plot_deltaY_dir x/y/z
    32/64/128)."""
    p = st.p
    dy = {32: 0, 64: 1, 128: 2}.get(flags & 224, -1)
    extra = (f"plot_means = {int(bool(flags & 1))}\nplot_vars = {int(bool(flags & 2))}\n"
             f"plot_covars = {int(bool(flags & 4))}\nplot_mom3 = {int(bool(flags & 8))}\n"
             f"plot_mom4 = {int(bool(flags & 16))}\nplot_deltaY_dir = {dy}\n")
    global _params
    _chk(lib().fhdref_init((p.to_inputs() + extra).encode()), "init")
    _params = None
    cells = [stats.cuMeans, stats.cuVars, stats.primMeans, stats.primVars, stats.coVars, stats.mom3, stats.mom4]
    ng = (C.c_int * 7)(*[m.ngrow for m in cells])
    faces = stats.velMeans + stats.velVars + stats.cumomMeans + stats.cumomVars
    N = p.n_cells
    cap = 512 * N[0] * N[1] * N[2]
    out = torch.zeros(cap, dtype=torch.float64)
    names = C.create_string_buffer(1 << 16)
    nc = C.c_int()
    _chk(lib().fhdref_plotfile(_ptr(st.cu.arr), _ptrs([m.arr for m in st.cumom]), _ptr(st.prim.arr),
                               _ptrs([m.arr for m in st.vel]), _ptr(st.eta.arr), _ptr(st.kappa.arr),
                               _ptr(st.zeta.arr), _ptrs([m.arr for m in cells]), ng, _ptrs([m.arr for m in faces]),
                               int(step), float(time), _ptr(out), cap, names, len(names), C.byref(nc)),
         "WritePlotFileStag")
    ncomp = nc.value
    data = out[:ncomp * N[0] * N[1] * N[2]].view(ncomp, N[2], N[1], N[0])
    return data, names.value.decode().split("\n")[:ncomp]


def write_spatial_cross(p, spatial_cross, step):
    """The reference's WriteSpatialCross3D (writePlotFileStag.cpp:528-549): writes
    spatialCross<step, 9 digits> in the current working directory."""
    init(p)
    sc = spatial_cross.contiguous()
    _chk(lib().fhdref_write_spatial_cross(_ptr(sc), int(step), sc.shape[1]), "WriteSpatialCross3D")


def write_spatial_cross_1d(p, spatial_cross, step):
    """The reference's WriteSpatialCross1D (writePlotFileStag.cpp:551-563) into the
    current working directory."""
    init(p)
    sc = spatial_cross.contiguous()
    _chk(lib().fhdref_write_spatial_cross_1d(_ptr(sc), sc.shape[0], int(step), 37 + p.nspecies + 3),
         "WriteSpatialCross1D")
