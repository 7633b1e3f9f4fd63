// ref_driver.cpp — C ABI over FHDeX's own hot-path functions, compiled
// unmodified from the reference sources against the host-only AMReX stand-in
// (oracle/amrex_host).  Test infrastructure: the tests load oracle/_ref/
// libfhd_ref.so to pin the restated oracle (oracle/fhd_oracle.cpp) to the
// reference's code itself.
//
// Every double* argument is the storage of one MultiFab with the geometry that
// main_driver.cpp:596-640, 995-1050 gives it (Array4 layout, component slowest):
// cu, cumom[3], prim, vel[3], eta, zeta, kappa, chi, D, source, ranchem with
// ngc ghost cells; faceflux[3] and edgeflux[6] without ghosts; cenflux[3] with
// one; the step's noise fields with the ghosts of timeStepStag.cpp:68-140.
// Parameters come from an inputs-deck text read by the reference's own
// InitializeCommonNamespace / InitializeCompressibleNamespace /
// InitializeChemistryNamespace and GetHcGas, in main_driver.cpp:43-88's order.
#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "chemistry_functions.H"
#include "common_functions.H"
#include "compressible_functions.H"
#include "compressible_functions_stag.H"
#include "rng_functions.H"
#include "TurbForcingComp.H"

void InitializeChemistryNamespace();

// The step only names TurbForcingComp in its signature (the forcing itself is
// compiled in with -DTURB, which oracle/Makefile does not set); an empty object
// stands in for the one main_driver would construct.
TurbForcingComp::TurbForcingComp() {}

// Debug.cpp's ASCII dump (used only by the reference's PrintFluxes debugging
// aid) is not part of the step; it is not compiled, and a call reports itself.
void outputMFAscii(const MultiFab&, std::string) { Abort("outputMFAscii is not part of the host build"); }

namespace {

std::string g_err;
Geometry g_geom;
BoxArray g_ba;
DistributionMapping g_dm;
bool g_ready = false;

struct NoiseCall {
    int scomp, ncomp;
    double mean, stddev;
    int lo[3], hi[3], nodal[3];
};
std::vector<NoiseCall> g_noise_log;

void throwing_abort(const char* msg) { throw std::runtime_error(std::string("amrex::Abort: ") + msg); }

template <class F>
int guarded(F&& f) {
    try {
        if (!g_ready) throw std::runtime_error("fhdref_init has not been called");
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

Box valid_box(const IntVect& nodal) { return convert(g_ba[0], nodal); }

void wrap(MultiFab& mf, double* p, const IntVect& nodal, int nc, int ng) {
    if (!p) throw std::runtime_error("null MultiFab storage");
    mf.wrap(p, valid_box(nodal), nc, ng);
}

void wrap3(std::array<MultiFab, 3>& a, double* const* p, int nc, int ng, bool faces) {
    for (int d = 0; d < 3; ++d) wrap(a[d], p[d], faces ? nodal_flag_dir[d] : IntVect(0), nc, ng);
}

// edge fluxes in the reference's order: edgeflux_x = {xy, xz}, edgeflux_y =
// {xy, yz}, edgeflux_z = {xz, yz}
void wrap_edges(std::array<MultiFab, 2>& ex, std::array<MultiFab, 2>& ey, std::array<MultiFab, 2>& ez,
                double* const* p, int ng) {
    wrap(ex[0], p[0], nodal_flag_xy, 1, ng);
    wrap(ex[1], p[1], nodal_flag_xz, 1, ng);
    wrap(ey[0], p[2], nodal_flag_xy, 1, ng);
    wrap(ey[1], p[3], nodal_flag_yz, 1, ng);
    wrap(ez[0], p[4], nodal_flag_xz, 1, ng);
    wrap(ez[1], p[5], nodal_flag_yz, 1, ng);
}

}  // namespace

extern "C" {

const char* fhdref_error() { return g_err.c_str(); }

// Reads the deck, initialises the reference's parameter namespaces and the
// one-box geometry (main_driver.cpp:43-99, 289-301).
int fhdref_init(const char* inputs) {
    amrex::abort_handler() = throwing_abort;
    try {
        ParmParse::load(inputs ? inputs : "");
        InitializeCommonNamespace();
        InitializeCompressibleNamespace();
        if (nvars != AMREX_SPACEDIM + 2 + nspecies) Abort("nvars must be equal to AMREX_SPACEDIM + 2 + nspecies");
        if (nprimvars != AMREX_SPACEDIM + 3 + 2 * nspecies)
            Abort("nprimvars must be equal to AMREX_SPACEDIM + 3 + 2*nspecies");
        InitializeChemistryNamespace();
        GetHcGas();
        Array<int, 3> is_periodic{0, 0, 0};
        for (int i = 0; i < 3; ++i)
            if (bc_vel_lo[i] == -1 || bc_vel_hi[i] == -1) {
                if (bc_vel_lo[i] != bc_vel_hi[i]) Abort("Inconsistent periodicity definition in bc_vel_lo/hi");
                is_periodic[i] = 1;
            }
        SetupBCStag();
        if (algorithm_type == 2) SetupCWallStag();  // main_driver.cpp:147-151
        Box domain(IntVect(0, 0, 0), IntVect(n_cells[0] - 1, n_cells[1] - 1, n_cells[2] - 1));
        RealBox real_box({prob_lo[0], prob_lo[1], prob_lo[2]}, {prob_hi[0], prob_hi[1], prob_hi[2]});
        g_geom.define(domain, real_box, 0, is_periodic);
        g_ba = BoxArray(domain);
        g_ready = true;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        g_ready = false;
        return 1;
    }
}

// FillBoundary / OverrideSync of one MultiFab (the stand-in's, with the run's
// periodicity: wall directions are left alone), for the harness's initial states
// and noise fields.
int fhdref_fill_boundary(double* p, const int* nodal, int nc, int ng, int override_sync) {
    return guarded([&] {
        MultiFab m;
        wrap(m, p, IntVect(nodal[0], nodal[1], nodal[2]), nc, ng);
        if (override_sync) m.OverrideSync(g_geom.periodicity());
        m.FillBoundary(g_geom.periodicity());
    });
}

// Wall compositions after SetupCWallStag (bc_Yk / bc_Xk of side s = 2 d + hi).
int fhdref_wall_composition(int s, double* yk, double* xk) {
    return guarded([&] {
        const int d = s / 2, hi = s % 2;
        const GpuArray<Real, MAX_SPECIES>* Y[6] = {&bc_Yk_x_lo, &bc_Yk_x_hi, &bc_Yk_y_lo, &bc_Yk_y_hi, &bc_Yk_z_lo,
                                                   &bc_Yk_z_hi};
        const GpuArray<Real, MAX_SPECIES>* X[6] = {&bc_Xk_x_lo, &bc_Xk_x_hi, &bc_Xk_y_lo, &bc_Xk_y_hi, &bc_Xk_z_lo,
                                                   &bc_Xk_z_hi};
        for (int n = 0; n < nspecies; ++n) {
            yk[n] = (*Y[2 * d + hi])[n];
            xk[n] = (*X[2 * d + hi])[n];
        }
    });
}

// Draws of the particle reservoir (bc_mass 4) for the next fhdref_rk3_step: rec holds
// 3 x (interface faces of the bc_mass-4 sides, x lo .. z hi) x cap values, entry
// (stage, face, n) the n-th draw at that face in that stage, as fhd_set_reservoir_record
// lays them out; the step's ParallelForRNG launches are then the reservoir's (one per
// such side and stage, in that order), so the step must have no chemistry noise.
static const double* g_res_rec = nullptr;
static int g_res_cap = 0;

int fhdref_set_reservoir_draws(const double* rec, int cap) {
    return guarded([&] {
        g_res_rec = rec;
        g_res_cap = cap;
    });
}

// Reservoir state of side s after SetupCWallStag: t, p, rho.
int fhdref_wall_state(int s, double* tpr) {
    return guarded([&] {
        const int d = s / 2, hi = s % 2;
        tpr[0] = hi ? t_hi[d] : t_lo[d];
        tpr[1] = hi ? p_hi[d] : p_lo[d];
        tpr[2] = hi ? rho_hi[d] : rho_lo[d];
    });
}

// Derived globals after GetHcGas, for the harness's consistency checks.
int fhdref_globals(int* ns, int* nv, int* npv, int* ng, double* hcv_out, double* hcp_out, int* nreac) {
    return guarded([&] {
        *ns = nspecies;
        *nv = nvars;
        *npv = nprimvars;
        *ng = ngc[0];
        for (int i = 0; i < nspecies; ++i) { hcv_out[i] = hcv[i]; hcp_out[i] = hcp[i]; }
        *nreac = nreaction;
    });
}

int fhdref_init_cons_var_stag(double* cu, double* const* mom) {
    return guarded([&] {
        MultiFab c;
        std::array<MultiFab, 3> m;
        wrap(c, cu, IntVect(0), nvars, ngc[0]);
        wrap3(m, mom, 1, ngc[0], true);
        InitConsVarStag(c, m, g_geom);
    });
}

int fhdref_conserved_to_primitive(double* prim, double* const* vel, double* cu, double* const* mom) {
    return guarded([&] {
        MultiFab p, c;
        std::array<MultiFab, 3> v, m;
        wrap(p, prim, IntVect(0), nprimvars, ngc[0]);
        wrap(c, cu, IntVect(0), nvars, ngc[0]);
        wrap3(v, vel, 1, ngc[0], true);
        wrap3(m, mom, 1, ngc[0], true);
        conservedToPrimitiveStag(p, v, c, m);
    });
}

int fhdref_set_bc(double* prim, double* cu, double* const* mom, double* const* vel) {
    return guarded([&] {
        MultiFab p, c;
        std::array<MultiFab, 3> v, m;
        wrap(p, prim, IntVect(0), nprimvars, ngc[0]);
        wrap(c, cu, IntVect(0), nvars, ngc[0]);
        wrap3(v, vel, 1, ngc[0], true);
        wrap3(m, mom, 1, ngc[0], true);
        setBCStag(p, c, m, v, g_geom);
    });
}

int fhdref_transport(double* prim, double* eta, double* zeta, double* kappa, double* chi, double* D) {
    return guarded([&] {
        MultiFab p, e, z, k, c, d;
        const int g = ngc[0];
        wrap(p, prim, IntVect(0), nprimvars, g);
        wrap(e, eta, IntVect(0), 1, g);
        wrap(z, zeta, IntVect(0), 1, g);
        wrap(k, kappa, IntVect(0), 1, g);
        wrap(c, chi, IntVect(0), nspecies, g);
        wrap(d, D, IntVect(0), nspecies * nspecies, g);
        calculateTransportCoeffs(p, e, z, k, c, d);
    });
}

// calculateFluxStag with the already weighted noise fields W: stochface[3]
// (nvars comps, no ghosts), stochedge[6] (reference order, no ghosts),
// stochcen[3] (one ghost).
int fhdref_flux(double* cu, double* const* mom, double* prim, double* const* vel, double* eta, double* zeta,
                double* kappa, double* chi, double* D, double* const* faceflux, double* const* edgeflux,
                double* const* cenflux, double* const* stochface, double* const* stochedge,
                double* const* stochcen, double w1, double w2, double dt) {
    return guarded([&] {
        const int g = ngc[0];
        MultiFab c, p, e, z, k, ch, d;
        std::array<MultiFab, 3> m, v, ff, cf, sf, sc;
        std::array<MultiFab, 2> ex, ey, ez, sx, sy, sz;
        wrap(c, cu, IntVect(0), nvars, g);
        wrap(p, prim, IntVect(0), nprimvars, g);
        wrap(e, eta, IntVect(0), 1, g);
        wrap(z, zeta, IntVect(0), 1, g);
        wrap(k, kappa, IntVect(0), 1, g);
        wrap(ch, chi, IntVect(0), nspecies, g);
        wrap(d, D, IntVect(0), nspecies * nspecies, g);
        wrap3(m, mom, 1, g, true);
        wrap3(v, vel, 1, g, true);
        wrap3(ff, faceflux, nvars + 4, 0, true);
        wrap3(cf, cenflux, 1, 1, false);
        wrap3(sf, stochface, nvars, 0, true);
        wrap3(sc, stochcen, 1, 1, false);
        wrap_edges(ex, ey, ez, edgeflux, 0);
        wrap_edges(sx, sy, sz, stochedge, 0);
        Vector<Real> weights{w1, w2};
        calculateFluxStag(c, m, p, v, e, z, k, ch, d, ff, ex, ey, ez, cf, sf, sx, sy, sz, sc, g_geom, weights, dt);
    });
}

// RK3stepStag.  normals[24]: the values of the step's 24 MultiFabFillRandomNormal
// calls in the reference's order (timeStepStag.cpp:183-222: stochface_A[d],
// stochface_B[d] for d = 0..2; then for i = 0..1 stochedge_x_A[i], _x_B[i],
// _y_A[i], _y_B[i], _z_A[i], _z_B[i]; then stochcen_A[i], stochcen_B[i] for
// i = 0..2), each over its MultiFab's whole storage and the filled components
// only; they are copied verbatim (the values a normal draw of the requested
// mean and deviation produced) and the reference then applies its own
// OverrideSync and FillBoundary.  chem[2*nreaction]: for reaction m, the
// standard normals of MultiFabFillRandom(ranchem_A, m) and (ranchem_B, m) over
// the valid cells.  Each fill's mean, deviation, components and box are logged
// (fhdref_noise_log).
int fhdref_rk3_step(double* cu, double* const* mom, double* prim, double* const* vel, double* source, double* eta,
                    double* zeta, double* kappa, double* chi, double* D, double* const* faceflux,
                    double* const* edgeflux, double* const* cenflux, double* ranchem,
                    const double* const* normals, const double* const* chem, double dt, int step) {
    return guarded([&] {
        // RK3stepStag's normal fills: 24 in 3-D, 4 with do_1D, 12 with do_2D (timeStepStag.cpp:172-222)
        const int nfills = do_1D ? 4 : do_2D ? 12 : 24;
        const int g = ngc[0];
        MultiFab c, p, s, e, z, k, ch, d, rc;
        std::array<MultiFab, 3> m, v, ff, cf;
        std::array<MultiFab, 2> ex, ey, ez;
        wrap(c, cu, IntVect(0), nvars, g);
        wrap(p, prim, IntVect(0), nprimvars, g);
        wrap(s, source, IntVect(0), nprimvars, g);
        wrap(e, eta, IntVect(0), 1, g);
        wrap(z, zeta, IntVect(0), 1, g);
        wrap(k, kappa, IntVect(0), 1, g);
        wrap(ch, chi, IntVect(0), nspecies, g);
        wrap(d, D, IntVect(0), nspecies * nspecies, g);
        wrap3(m, mom, 1, g, true);
        wrap3(v, vel, 1, g, true);
        wrap3(ff, faceflux, nvars + 4, 0, true);
        wrap3(cf, cenflux, 1, 1, false);
        wrap_edges(ex, ey, ez, edgeflux, 0);
        if (nreaction > 0) wrap(rc, ranchem, IntVect(0), nreaction, g);
        g_noise_log.clear();
        int call = 0;
        auto& src = amrex::noise_source();
        src.launches = 0;
        src.fill_normal = [&](MultiFab& mf, int scomp, int ncomp, Real mean, Real stddev) {
            if (call >= nfills || !normals || !normals[call]) throw std::runtime_error("missing injected noise field");
            const Box b = mf.fab.box();
            NoiseCall rec{scomp, ncomp, mean, stddev, {}, {}, {}};
            for (int q = 0; q < 3; ++q) { rec.lo[q] = b.lo[q]; rec.hi[q] = b.hi[q]; rec.nodal[q] = b.typ.t[q]; }
            g_noise_log.push_back(rec);
            const double* z0 = normals[call++];
            const Long np = b.numPts();
            auto a = mf.fab.array();
            for (int n = 0; n < ncomp; ++n) {
                Long q = 0;
                for (int kk = b.lo[2]; kk <= b.hi[2]; ++kk)
                    for (int jj = b.lo[1]; jj <= b.hi[1]; ++jj)
                        for (int ii = b.lo[0]; ii <= b.hi[0]; ++ii, ++q) a(ii, jj, kk, scomp + n) = z0[n * np + q];
            }
        };
        src.point_normal = [&](long launch, int i, int j, int kk) -> Real {
            if (!chem || launch >= 2 * nreaction || !chem[launch]) throw std::runtime_error("missing reaction noise");
            const IntVect lo = g_ba[0].lo, hi = g_ba[0].hi;
            const Long nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1;
            return chem[launch][(i - lo[0]) + (j - lo[1]) * nx + (kk - lo[2]) * nx * ny];
        };
        if (g_res_rec) {
            int sides[6], ns4 = 0;
            long pref[7] = {0};
            const int* lo = bc_mass_lo.data();
            const int* hi = bc_mass_hi.data();
            for (int side = 0; side < 6; ++side) {
                const int dd = side / 2;
                if ((side % 2 ? hi[dd] : lo[dd]) != 4) continue;
                const int e1 = dd == 0 ? 1 : 0, e2 = dd == 2 ? 1 : 2;
                sides[ns4] = side;
                pref[ns4 + 1] = pref[ns4] + (long)n_cells[e1] * n_cells[e2];
                ++ns4;
            }
            src.stream = [&, sides, ns4, pref](long launch, int i, int j, int kk, long n, int) -> Real {
                if (ns4 == 0 || launch >= 3L * ns4) throw std::runtime_error("unexpected reservoir launch");
                const int stage = (int)(launch / ns4), li = (int)(launch % ns4), dd = sides[li] / 2;
                const int e1 = dd == 0 ? 1 : 0, e2 = dd == 2 ? 1 : 2;
                const int x[3] = {i, j, kk};
                const long q = pref[li] + x[e1] + (long)n_cells[e1] * x[e2];
                if (n >= g_res_cap) throw std::runtime_error("reservoir draws beyond the recorded capacity");
                return g_res_rec[((long)stage * pref[ns4] + q) * g_res_cap + n];
            };
        }
        TurbForcingComp turb;
        RK3stepStag(c, m, p, v, s, e, z, k, ch, d, ff, ex, ey, ez, cf, rc, g_geom, dt, step, turb);
        src.fill_normal = nullptr;
        src.point_normal = nullptr;
        src.stream = nullptr;
        if (call != nfills) throw std::runtime_error("RK3stepStag made an unexpected number of noise fills");
    });
}

// The noise fills of the last step: per call scomp, ncomp, mean, stddev, the
// storage box (lo, hi) and its index type.
int fhdref_noise_log(int* count, int* ints /* 11 per call */, double* reals /* 2 per call */, int cap) {
    *count = (int)g_noise_log.size();
    for (int q = 0; q < *count && q < cap; ++q) {
        const NoiseCall& r = g_noise_log[q];
        int* o = ints + 11 * q;
        o[0] = r.scomp;
        o[1] = r.ncomp;
        for (int d = 0; d < 3; ++d) { o[2 + d] = r.lo[d]; o[5 + d] = r.hi[d]; o[8 + d] = r.nodal[d]; }
        reals[2 * q] = r.mean;
        reals[2 * q + 1] = r.stddev;
    }
    return 0;
}

// compute_compressible_chemistry_source_CLE (chemistry_functions.cpp:128-193)
int fhdref_chemistry_source(double dt, double dV, double* prim, double* source, double* ranchem) {
    return guarded([&] {
        const int g = ngc[0];
        MultiFab p, s, rc;
        wrap(p, prim, IntVect(0), nprimvars, g);
        wrap(s, source, IntVect(0), nprimvars, g);
        wrap(rc, ranchem, IntVect(0), nreaction, g);
        compute_compressible_chemistry_source_CLE(dt, dV, p, s, rc);
    });
}

// evaluateStatsStag3D (statsStag.cpp:10-76) with the deck's plot_means / plot_vars /
// plot_covars / plot_mom3 / plot_mom4 / plot_cross / cross_cell and no surface
// coverage.  cells[7] = cuMeans, cuVars, primMeans, primVars, coVars, mom3, mom4
// (nvars, nvars, nprimvars+3, nprimvars+5, 26, nvars+1, nvars+1 components) with
// ghost widths ng[7]; faces[12] = velMeans, velVars, cumomMeans, cumomVars (three
// each, no ghosts); spatial_cross (n_cells[0]*ncross) and xcross
// (2*nvars+8+2*nspecies) are the reference's spatialCross3D and
// dataSliceMeans_xcross vectors, updated in place.
int fhdref_eval_stats3d(double* cu, double* prim, double* const* vel, double* const* mom, double* const* cells,
                        const int* ng, double* const* faces, double* spatial_cross, double* xcross, int ncross,
                        int steps) {
    return guarded([&] {
        const int g = ngc[0];
        MultiFab c, p, cm, cv, pm, pv, cov, m3, m4, th, thm, thv, thc;
        std::array<MultiFab, 3> v, m, vm, vv, mm, mv;
        wrap(c, cu, IntVect(0), nvars, g);
        wrap(p, prim, IntVect(0), nprimvars, g);
        wrap3(v, vel, 1, g, true);
        wrap3(m, mom, 1, g, true);
        wrap(cm, cells[0], IntVect(0), nvars, ng[0]);
        wrap(cv, cells[1], IntVect(0), nvars, ng[1]);
        wrap(pm, cells[2], IntVect(0), nprimvars + 3, ng[2]);
        wrap(pv, cells[3], IntVect(0), nprimvars + 5, ng[3]);
        wrap(cov, cells[4], IntVect(0), 26, ng[4]);
        wrap(m3, cells[5], IntVect(0), nvars + 1, ng[5]);
        wrap(m4, cells[6], IntVect(0), nvars + 1, ng[6]);
        wrap3(vm, faces, 1, 0, true);
        wrap3(vv, faces + 3, 1, 0, true);
        wrap3(mm, faces + 6, 1, 0, true);
        wrap3(mv, faces + 9, 1, 0, true);
        const int nstats = 2 * nvars + 8 + 2 * nspecies;
        Vector<Real> sc(spatial_cross, spatial_cross + (size_t)n_cells[0] * ncross);
        Vector<Real> xc(xcross, xcross + nstats);
        const Box domain(IntVect(0, 0, 0), IntVect(n_cells[0] - 1, n_cells[1] - 1, n_cells[2] - 1));
        evaluateStatsStag3D(c, cm, cv, p, pm, pv, v, vm, vv, m, mm, mv, cov, m3, m4, th, thm, thv, thc, xc, sc,
                            ncross, domain, steps, g_geom);
        std::copy(sc.begin(), sc.end(), spatial_cross);
        std::copy(xc.begin(), xc.end(), xcross);
    });
}

// WritePlotFileStag (writePlotFileStag.cpp:7-527) with the deck's plot_means /
// plot_vars / plot_covars / plot_mom3 / plot_mom4 / plot_deltaY_dir, no surface
// coverage: the plotfile MultiFab it composes (valid cells, component slowest)
// into out (capacity cap doubles) and its component names, each ended by '\n',
// into names (capacity ncap bytes); *ncomp receives the component count.  The
// state, eta, kappa and zeta have ngc ghosts; cells / ng / faces as
// fhdref_eval_stats3d.
int fhdref_plotfile(double* cu, double* const* mom, double* prim, double* const* vel, double* eta, double* kappa,
                    double* zeta, double* const* cells, const int* ng, double* const* faces, int step, double time,
                    double* out, long cap, char* names, int ncap, int* ncomp) {
    return guarded([&] {
        const int g = ngc[0];
        MultiFab c, p, e, k, z, cm, cv, pm, pv, cov, m3, m4, sc, scm, scv, scc;
        std::array<MultiFab, 3> v, m, vm, vv, mm, mv;
        wrap(c, cu, IntVect(0), nvars, g);
        wrap(p, prim, IntVect(0), nprimvars, g);
        wrap(e, eta, IntVect(0), 1, g);
        wrap(k, kappa, IntVect(0), 1, g);
        wrap(z, zeta, IntVect(0), 1, g);
        wrap3(v, vel, 1, g, true);
        wrap3(m, mom, 1, g, true);
        wrap(cm, cells[0], IntVect(0), nvars, ng[0]);
        wrap(cv, cells[1], IntVect(0), nvars, ng[1]);
        wrap(pm, cells[2], IntVect(0), nprimvars + 3, ng[2]);
        wrap(pv, cells[3], IntVect(0), nprimvars + 5, ng[3]);
        wrap(cov, cells[4], IntVect(0), 26, ng[4]);
        wrap(m3, cells[5], IntVect(0), nvars + 1, ng[5]);
        wrap(m4, cells[6], IntVect(0), nvars + 1, ng[6]);
        wrap3(vm, faces, 1, 0, true);
        wrap3(vv, faces + 3, 1, 0, true);
        wrap3(mm, faces + 6, 1, 0, true);
        wrap3(mv, faces + 9, 1, 0, true);
        WritePlotFileStag(step, time, g_geom, c, cm, cv, m, mm, mv, p, pm, pv, v, vm, vv, cov, m3, m4, sc, scm, scv,
                          scc, e, k, z);
        const PlotfileCapture& pc = plotfile_capture();
        if ((long)pc.data.size() > cap) throw std::runtime_error("fhdref_plotfile: output buffer too small");
        std::copy(pc.data.begin(), pc.data.end(), out);
        std::string joined;
        for (const std::string& n : pc.names) joined += n + "\n";
        if ((int)joined.size() + 1 > ncap) throw std::runtime_error("fhdref_plotfile: names buffer too small");
        std::copy(joined.begin(), joined.end(), names);
        names[joined.size()] = 0;
        *ncomp = (int)pc.names.size();
    });
}

// evaluateStatsStag1D / evaluateStatsStag2D (statsStag.cpp:78-197) of a quasi-1-D /
// 2-D run (the deck's do_1D / do_2D, all_correl), arguments as fhdref_eval_stats3d;
// spatial_cross is the storage of spatialCrossMF (cell-centred, no ghosts,
// ncomp_cross components).
int fhdref_eval_stats_lowdim(double* cu, double* prim, double* const* vel, double* const* mom, double* const* cells,
                             const int* ng, double* const* faces, double* spatial_cross, int ncomp_cross, int ncross,
                             int steps) {
    return guarded([&] {
        const int g = ngc[0];
        MultiFab c, p, cm, cv, pm, pv, cov, m3, m4, th, thm, thv, thc, sc;
        std::array<MultiFab, 3> v, m, vm, vv, mm, mv;
        wrap(c, cu, IntVect(0), nvars, g);
        wrap(p, prim, IntVect(0), nprimvars, g);
        wrap3(v, vel, 1, g, true);
        wrap3(m, mom, 1, g, true);
        wrap(cm, cells[0], IntVect(0), nvars, ng[0]);
        wrap(cv, cells[1], IntVect(0), nvars, ng[1]);
        wrap(pm, cells[2], IntVect(0), nprimvars + 3, ng[2]);
        wrap(pv, cells[3], IntVect(0), nprimvars + 5, ng[3]);
        wrap(cov, cells[4], IntVect(0), 26, ng[4]);
        wrap(m3, cells[5], IntVect(0), nvars + 1, ng[5]);
        wrap(m4, cells[6], IntVect(0), nvars + 1, ng[6]);
        wrap3(vm, faces, 1, 0, true);
        wrap3(vv, faces + 3, 1, 0, true);
        wrap3(mm, faces + 6, 1, 0, true);
        wrap3(mv, faces + 9, 1, 0, true);
        wrap(sc, spatial_cross, IntVect(0), ncomp_cross, 0);
        if (do_1D)
            evaluateStatsStag1D(c, cm, cv, p, pm, pv, v, vm, vv, m, mm, mv, cov, m3, m4, th, thm, thv, thc, sc, ncross,
                                steps, g_geom);
        else
            evaluateStatsStag2D(c, cm, cv, p, pm, pv, v, vm, vv, m, mm, mv, cov, m3, m4, th, thm, thv, thc, sc, ncross,
                                steps, g_geom);
    });
}

// WriteSpatialCross1D (writePlotFileStag.cpp:551-563) into the working directory
// from the storage of spatialCrossMF.
int fhdref_write_spatial_cross_1d(double* spatial_cross, int ncomp_cross, int step, int ncross) {
    return guarded([&] {
        MultiFab sc;
        wrap(sc, spatial_cross, IntVect(0), ncomp_cross, 0);
        WriteSpatialCross1D(sc, step, g_geom, ncross);
    });
}

// WriteSpatialCross3D (writePlotFileStag.cpp:528-549): spatialCross<step, 9
// digits> in the working directory from n_cells[0]*ncross values.
int fhdref_write_spatial_cross(const double* spatial_cross, int step, int ncross) {
    return guarded([&] {
        const Vector<Real> sc(spatial_cross, spatial_cross + (size_t)n_cells[0] * ncross);
        WriteSpatialCross3D(sc, step, g_geom, ncross);
    });
}

int fhdref_max_acoustic_cfl(double* prim, double* const* vel, double dt, double* out) {
    return guarded([&] {
        MultiFab p;
        std::array<MultiFab, 3> v;
        wrap(p, prim, IntVect(0), nprimvars, ngc[0]);
        wrap3(v, vel, 1, ngc[0], true);
        *out = GetMaxAcousticCFL(p, v, dt, g_geom);
    });
}

}  // extern "C"
