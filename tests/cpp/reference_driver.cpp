// Test driver for fhd/reference_api.hpp: the main_driver sequence of the
// reference (main_driver.cpp: MultiFab set-up, InitConsVarStag,
// conservedToPrimitiveStag, FillBoundary, calculateTransportCoeffs, then
// RK3stepStag in the time loop) written against the reference's function
// names, on an argon box (two identical species, the reference's parity form).
//
//   reference_driver shapes <n>
//       print the Array4 bounds of every MultiFab kind (host arena, no GPU)
//   reference_driver run <device|pinned> <n> <nsteps> <seed> <dt> <out.bin> [argon|no2]
//       run nsteps RK3 steps (steps 0..nsteps-1) and write cu, cumom[0..2],
//       prim, vel[0..2] (whole buffers, ghosts included) to out.bin; no2: the
//       2 NO2 <-> N2O4 gas with the chemistry source (chemistry:: globals)
//   reference_driver plot <n> <nsteps> <seed> <dt> <plot_base_name>
//       run nsteps RK3 steps on device MultiFabs and WritePlotFileStag (step
//       nsteps, time nsteps*dt, no statistics)
//   reference_driver chk <n> <n1> <n2> <seed> <dt> <out.bin>
//       n1 steps, WriteCheckPoint (chk<n1-1> in the working directory, with
//       zeroed statistics MultiFabs), ReadCheckPoint into new MultiFabs, steps
//       n1..n1+n2-1 on them; writes the final state as `run` does
//   reference_driver stats <n> <nsteps> <seed> <dt> <out.bin>
//       nsteps RK3 steps, evaluateStatsStag3D after each (plot_means, plot_vars,
//       plot_mom3, plot_mom4, plot_cross at cross_cell n/2); writes cuMeans,
//       cuVars, primMeans, primVars, coVars, mom3, mom4, velMeans, velVars,
//       cumomMeans, cumomVars, spatialCrossVec and dataSliceMeans_xcross, and
//       WriteSpatialCross3D's spatialCross<nsteps> in the working directory
//   reference_driver stats1d <nx> <ny> <nsteps> <seed> <dt> <all_correl> <out.bin>
//       a quasi-1-D run (do_1D) on an nx x ny x ny box: nsteps RK3 steps,
//       evaluateStatsStag1D after each (every statistic, plot_cross at cross_cell 3),
//       WriteSpatialCross1D at step nsteps in the working directory, then
//       WriteCheckPoint / ReadCheckPoint of chk<nsteps> (spatialCrossMF must come
//       back bit for bit, else exit 6); writes cuMeans, cuVars, primMeans,
//       primVars, coVars, mom3, mom4 and spatialCrossMF
//   reference_driver massfrac <n>
//       start from a state with a zero mass fraction: calculateTransportCoeffs
//       must report it through the abort handler (exit code 3)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "fhd/reference_api.hpp"

using namespace fhd::amrex_compat;

struct Caught : std::runtime_error {
    using std::runtime_error::runtime_error;
};
[[noreturn]] static void throwing_handler(const char* msg) { throw Caught(msg); }

static void set_argon(int n, int seed, int ny = -1) {
    const double dx = 8e-6;
    common::nspecies = 2;
    for (int d = 0; d < 3; ++d) {
        common::n_cells[d] = d == 0 || ny < 0 ? n : ny;
        common::prob_lo[d] = 0.0;
        common::prob_hi[d] = common::n_cells[d] * dx;
    }
    for (int s = 0; s < 2; ++s) {
        common::molmass[s] = 39.95;
        common::diameter[s] = 3.66e-8;
        common::dof[s] = 3.0;
        common::rhobar[s] = 0.5;
        common::T_init[s] = 273.0;
    }
    common::rho0 = 1.78e-3;
    common::algorithm_type = 2;
    common::visc_type = 2;
    common::advection_type = 2;
    common::stoch_stress_form = 1;
    common::seed = seed;
}

// 2 NO2 <-> N2O4 with chemical Langevin noise (the reference's NO2 dimerization
// deck's gas and reactions)
static void set_no2(int n, int seed) {
    set_argon(n, seed);
    const double mm[2] = {46.0055, 92.0110}, di[2] = {3.765e-08, 4.621e-08}, dof[2] = {7.279586, 18.049072},
                 rb[2] = {0.723969, 0.276031};
    for (int s = 0; s < 2; ++s) {
        common::molmass[s] = mm[s];
        common::diameter[s] = di[s];
        common::dof[s] = dof[s];
        common::rhobar[s] = rb[s];
        common::T_init[s] = 350.0;
    }
    common::rho0 = 1.858338e-03;
    common::k_B = 1.38065e-16;
    common::Runiv = 8.31446e7;
    chemistry::nreaction = 2;
    chemistry::reaction_type = 1;
    chemistry::stoich_coeffs_R(0, 0) = 2;  // 2 NO2 -> N2O4
    chemistry::stoich_coeffs_P(0, 1) = 1;
    chemistry::stoich_coeffs_R(1, 1) = 1;  // N2O4 -> 2 NO2
    chemistry::stoich_coeffs_P(1, 0) = 2;
    chemistry::rate_const[0] = 4.065753e+11;
    chemistry::rate_const[1] = 6.236899e+07;
    chemistry::alpha_param[0] = -5.337990e+10;
    chemistry::alpha_param[1] = 5.370000e+11;
    chemistry::beta_param[0] = 0.644950;
    chemistry::beta_param[1] = -1.100000;
    chemistry::T0_chem = 350.0;
}

struct State {
    int ns, nvars, nprimvars, ngc = 2;
    Geometry geom;
    MultiFab cu, prim, source, eta, zeta, kappa, chi, D, ranchem;
    std::array<MultiFab, 3> cumom, vel, faceflux, cenflux;
    std::array<MultiFab, 2> edgeflux_x, edgeflux_y, edgeflux_z;

    // on the box common::n_cells
    State(Arena a, bool byproducts) {
        ns = common::nspecies;
        nvars = 5 + ns;
        nprimvars = 6 + 2 * ns;
        const Box dom(IntVect(0, 0, 0), IntVect(common::n_cells[0] - 1, common::n_cells[1] - 1, common::n_cells[2] - 1));
        RealBox rb;
        for (int d = 0; d < 3; ++d) {
            rb.lo[d] = common::prob_lo[d];
            rb.hi[d] = common::prob_hi[d];
        }
        geom = Geometry(dom, rb);
        cu.define(dom, nvars, ngc, a);
        prim.define(dom, nprimvars, ngc, a);
        for (int d = 0; d < 3; ++d) {
            cumom[d].define(convert(dom, face_nodal(d)), 1, ngc, a);
            vel[d].define(convert(dom, face_nodal(d)), 1, ngc, a);
        }
        if (!byproducts) return;
        source.define(dom, nprimvars, ngc, a);
        eta.define(dom, 1, ngc, a);
        zeta.define(dom, 1, ngc, a);
        kappa.define(dom, 1, ngc, a);
        chi.define(dom, ns, ngc, a);
        D.define(dom, ns * ns, ngc, a);
        for (int d = 0; d < 3; ++d) {
            faceflux[d].define(convert(dom, face_nodal(d)), nvars + 4, 0, a);
            cenflux[d].define(dom, 1, 1, a);
        }
        edgeflux_x[0].define(convert(dom, edge_nodal(0, 1)), 1, 0, a);
        edgeflux_x[1].define(convert(dom, edge_nodal(0, 2)), 1, 0, a);
        edgeflux_y[0].define(convert(dom, edge_nodal(0, 1)), 1, 0, a);
        edgeflux_y[1].define(convert(dom, edge_nodal(1, 2)), 1, 0, a);
        edgeflux_z[0].define(convert(dom, edge_nodal(0, 2)), 1, 0, a);
        edgeflux_z[1].define(convert(dom, edge_nodal(1, 2)), 1, 0, a);
    }

    // main_driver's initialisation on device MultiFabs.
    void init() {
        InitConsVarStag(cu, cumom, geom);
        conservedToPrimitiveStag(prim, vel, cu, cumom);
        cu.FillBoundary(geom.periodicity());
        prim.FillBoundary(geom.periodicity());
        for (int d = 0; d < 3; ++d) {
            cumom[d].FillBoundary(geom.periodicity());
            vel[d].FillBoundary(geom.periodicity());
        }
        calculateTransportCoeffs(prim, eta, zeta, kappa, chi, D);
    }
};

static void print_shape(const char* name, const MultiFab& m) {
    const fhd_fab f = m.fab();
    std::printf("%s %d %d %d %d %d %d %d %d %d %d\n", name, f.lo[0], f.lo[1], f.lo[2], f.hi[0], f.hi[1], f.hi[2],
                f.ncomp, f.nodal[0], f.nodal[1], f.nodal[2]);
}

static int cmd_shapes(int n) {
    set_argon(n, 1);
    State s(Arena::Host, true);
    print_shape("cu", s.cu);
    print_shape("prim", s.prim);
    for (int d = 0; d < 3; ++d) print_shape(("cumom" + std::to_string(d)).c_str(), s.cumom[d]);
    for (int d = 0; d < 3; ++d) print_shape(("vel" + std::to_string(d)).c_str(), s.vel[d]);
    print_shape("source", s.source);
    print_shape("eta", s.eta);
    print_shape("chi", s.chi);
    print_shape("D", s.D);
    for (int d = 0; d < 3; ++d) print_shape(("faceflux" + std::to_string(d)).c_str(), s.faceflux[d]);
    print_shape("edgeflux_x0", s.edgeflux_x[0]);
    print_shape("edgeflux_x1", s.edgeflux_x[1]);
    print_shape("edgeflux_y1", s.edgeflux_y[1]);
    for (int d = 0; d < 3; ++d) print_shape(("cenflux" + std::to_string(d)).c_str(), s.cenflux[d]);
    // Array4 indexing agrees with the C-ABI layout (first and last element)
    Array4<Real> a = s.cu.array();
    a(-2, -2, -2, 0) = 1.0;
    a(n + 1, n + 1, n + 1, s.nvars - 1) = 2.0;
    const Real* p = s.cu.dataPtr();
    std::printf("array4 %d %d\n", p[0] == 1.0 ? 1 : 0, p[s.cu.size() - 1] == 2.0 ? 1 : 0);
    return 0;
}

static void write_all(FILE* f, const MultiFab& m) {
    std::vector<Real> h;
    m.copyToHost(h);
    if (std::fwrite(h.data(), sizeof(Real), h.size(), f) != h.size()) throw std::runtime_error("short write");
}

static void step_all(State& s, double dt, int nsteps) {
    TurbForcingComp turbforce;
    for (int step = 0; step < nsteps; ++step)
        RK3stepStag(s.cu, s.cumom, s.prim, s.vel, s.source, s.eta, s.zeta, s.kappa, s.chi, s.D, s.faceflux,
                    s.edgeflux_x, s.edgeflux_y, s.edgeflux_z, s.cenflux, s.ranchem, s.geom, dt, step, turbforce);
}

static int cmd_run(const std::string& arena, int n, int nsteps, int seed, double dt, const char* out,
                   const std::string& gas) {
    if (gas == "no2")
        set_no2(n, seed);
    else
        set_argon(n, seed);
    // initialise on the device, as the reference's GPU build does
    State dev(Arena::Device, true);
    dev.init();
    if (arena == "device") {
        step_all(dev, dt, nsteps);
    } else {
        // a CPU build's MultiFabs: state in pinned host memory, no by-products
        State host(Arena::Pinned, false);
        MultiFab::Copy(host.cu, dev.cu);
        MultiFab::Copy(host.prim, dev.prim);
        for (int d = 0; d < 3; ++d) {
            MultiFab::Copy(host.cumom[d], dev.cumom[d]);
            MultiFab::Copy(host.vel[d], dev.vel[d]);
        }
        step_all(host, dt, nsteps);
        MultiFab::Copy(dev.cu, host.cu);
        MultiFab::Copy(dev.prim, host.prim);
        for (int d = 0; d < 3; ++d) {
            MultiFab::Copy(dev.cumom[d], host.cumom[d]);
            MultiFab::Copy(dev.vel[d], host.vel[d]);
        }
    }
    FILE* f = std::fopen(out, "wb");
    if (!f) return 2;
    write_all(f, dev.cu);
    for (int d = 0; d < 3; ++d) write_all(f, dev.cumom[d]);
    write_all(f, dev.prim);
    for (int d = 0; d < 3; ++d) write_all(f, dev.vel[d]);
    std::fclose(f);
    fhd::ref::finalize();
    return 0;
}

static int cmd_plot(int n, int nsteps, int seed, double dt, const char* base) {
    set_argon(n, seed);
    State s(Arena::Device, true);
    s.init();
    step_all(s, dt, nsteps);
    MultiFab none;
    std::array<MultiFab, 3> none3;
    common::plot_base_name = base;
    WritePlotFileStag(nsteps, nsteps * dt, s.geom, s.cu, none, none, s.cumom, none3, none3, s.prim, none, none, s.vel,
                      none3, none3, none, none, none, none, none, none, none, s.eta, s.kappa, s.zeta);
    fhd::ref::finalize();
    return 0;
}

static int cmd_chk(int n, int n1, int n2, int seed, double dt, const char* out) {
    set_argon(n, seed);
    State s(Arena::Device, true);
    s.init();
    step_all(s, dt, n1);
    const Box dom(IntVect(0, 0, 0), IntVect(n - 1, n - 1, n - 1));
    const int nv = s.nvars, np = s.nprimvars;
    MultiFab cuMeans(dom, nv, 2), cuVars(dom, nv, 2), primMeans(dom, np + 3, 2), primVars(dom, np + 5, 2),
        coVars(dom, 26, 0), none;
    std::array<MultiFab, 3> cmm, cmv, vm, vv, none3;
    for (int d = 0; d < 3; ++d) {
        cmm[d].define(convert(dom, face_nodal(d)), 1, 0);
        cmv[d].define(convert(dom, face_nodal(d)), 1, 0);
        vm[d].define(convert(dom, face_nodal(d)), 1, 0);
        vv[d].define(convert(dom, face_nodal(d)), 1, 0);
    }
    Vector<Real> cross;
    TurbForcingComp turb;
    WriteCheckPoint(n1 - 1, n1 * dt, 0, s.geom, s.cu, cuMeans, cuVars, s.prim, primMeans, primVars, s.cumom, cmm, cmv,
                    s.vel, vm, vv, coVars, none, none, none, none, none, none, none, cross, 0, turb);
    // restart into fresh MultiFabs
    State r(Arena::Device, false);
    MultiFab rcm, rcv, rpm, rpv, rco, rm3, rm4, sc0, sc1, sc2, sc3, scross;
    std::array<MultiFab, 3> rcmm, rcmv, rvm, rvv;
    BoxArray ba;
    DistributionMapping dm;
    int step = -1, count = -1;
    Real time = -1.0;
    common::restart = n1 - 1;
    ReadCheckPoint(step, time, count, r.geom, dom, r.cu, rcm, rcv, r.prim, rpm, rpv, r.cumom, rcmm, rcmv, r.vel, rvm,
                   rvv, rco, rm3, rm4, sc0, sc1, sc2, sc3, scross, cross, 0, turb, ba, dm);
    if (step != n1 || count != 0 || time != n1 * dt) return 5;
    TurbForcingComp turbforce;
    for (int st = step; st < n1 + n2; ++st)
        RK3stepStag(r.cu, r.cumom, r.prim, r.vel, r.source, r.eta, r.zeta, r.kappa, r.chi, r.D, r.faceflux,
                    r.edgeflux_x, r.edgeflux_y, r.edgeflux_z, r.cenflux, r.ranchem, r.geom, dt, st, turbforce);
    FILE* f = std::fopen(out, "wb");
    if (!f) return 2;
    write_all(f, r.cu);
    for (int d = 0; d < 3; ++d) write_all(f, r.cumom[d]);
    write_all(f, r.prim);
    for (int d = 0; d < 3; ++d) write_all(f, r.vel[d]);
    std::fclose(f);
    fhd::ref::finalize();
    return 0;
}

static int cmd_stats(int n, int nsteps, int seed, double dt, const char* out) {
    set_argon(n, seed);
    common::plot_means = common::plot_vars = common::plot_mom3 = common::plot_mom4 = 1;
    common::plot_cross = 1;
    common::cross_cell = n / 2;
    State s(Arena::Device, true);
    s.init();
    const Box dom(IntVect(0, 0, 0), IntVect(n - 1, n - 1, n - 1));
    const int nv = s.nvars, np = s.nprimvars;
    MultiFab cuMeans(dom, nv, 2), cuVars(dom, nv, 2), primMeans(dom, np + 3, 2), primVars(dom, np + 5, 2),
        coVars(dom, 26, 0), mom3(dom, nv + 1, 0), mom4(dom, nv + 1, 0), theta;
    std::array<MultiFab, 3> vm, vv, cmm, cmv;
    for (int d = 0; d < 3; ++d) {
        vm[d].define(convert(dom, face_nodal(d)), 1, 0);
        vv[d].define(convert(dom, face_nodal(d)), 1, 0);
        cmm[d].define(convert(dom, face_nodal(d)), 1, 0);
        cmv[d].define(convert(dom, face_nodal(d)), 1, 0);
    }
    // main_driver.cpp:279-285
    const int ncross = 37 + common::nspecies + 3;
    Vector<Real> slice(2 * nv + 8 + 2 * common::nspecies, 0.0), cross((size_t)n * ncross, 0.0);
    TurbForcingComp turb;
    for (int step = 0; step < nsteps; ++step) {
        RK3stepStag(s.cu, s.cumom, s.prim, s.vel, s.source, s.eta, s.zeta, s.kappa, s.chi, s.D, s.faceflux,
                    s.edgeflux_x, s.edgeflux_y, s.edgeflux_z, s.cenflux, s.ranchem, s.geom, dt, step, turb);
        evaluateStatsStag3D(s.cu, cuMeans, cuVars, s.prim, primMeans, primVars, s.vel, vm, vv, s.cumom, cmm, cmv,
                            coVars, mom3, mom4, theta, theta, theta, theta, slice, cross, ncross, dom, step + 1,
                            s.geom);
    }
    WriteSpatialCross3D(cross, nsteps, s.geom, ncross);
    FILE* f = std::fopen(out, "wb");
    if (!f) return 2;
    for (const MultiFab* m : {&cuMeans, &cuVars, &primMeans, &primVars, &coVars, &mom3, &mom4}) write_all(f, *m);
    for (int d = 0; d < 3; ++d) write_all(f, vm[d]);
    for (int d = 0; d < 3; ++d) write_all(f, vv[d]);
    for (int d = 0; d < 3; ++d) write_all(f, cmm[d]);
    for (int d = 0; d < 3; ++d) write_all(f, cmv[d]);
    std::fwrite(cross.data(), sizeof(Real), cross.size(), f);
    std::fwrite(slice.data(), sizeof(Real), slice.size(), f);
    std::fclose(f);
    fhd::ref::finalize();
    return 0;
}

static bool same(const MultiFab& a, const MultiFab& b) {
    std::vector<Real> ha, hb;
    a.copyToHost(ha);
    b.copyToHost(hb);
    return ha.size() == hb.size() && std::memcmp(ha.data(), hb.data(), ha.size() * sizeof(Real)) == 0;
}

static int cmd_stats1d(int nx, int ny, int nsteps, int seed, double dt, int all_correl, const char* out) {
    set_argon(nx, seed, ny);
    compressible::do_1D = 1;
    compressible::all_correl = all_correl;
    common::plot_means = common::plot_vars = common::plot_mom3 = common::plot_mom4 = 1;
    common::plot_cross = 1;
    common::cross_cell = 3;
    State s(Arena::Device, true);
    s.init();
    const Box dom(IntVect(0, 0, 0), IntVect(nx - 1, ny - 1, ny - 1));
    const int nv = s.nvars, np = s.nprimvars;
    MultiFab cuMeans(dom, nv, 2), cuVars(dom, nv, 2), primMeans(dom, np + 3, 2), primVars(dom, np + 5, 2),
        coVars(dom, 26, 0), mom3(dom, nv + 1, 0), mom4(dom, nv + 1, 0), theta;
    std::array<MultiFab, 3> vm, vv, cmm, cmv;
    for (int d = 0; d < 3; ++d) {
        vm[d].define(convert(dom, face_nodal(d)), 1, 0);
        vv[d].define(convert(dom, face_nodal(d)), 1, 0);
        cmm[d].define(convert(dom, face_nodal(d)), 1, 0);
        cmv[d].define(convert(dom, face_nodal(d)), 1, 0);
    }
    // main_driver.cpp:283, 717-723
    const int ncross = 37 + common::nspecies + 3;
    MultiFab crossMF(dom, (all_correl ? 5 : 1) * ncross, 0);
    crossMF.setVal(0.0);
    TurbForcingComp turb;
    for (int step = 0; step < nsteps; ++step) {
        RK3stepStag(s.cu, s.cumom, s.prim, s.vel, s.source, s.eta, s.zeta, s.kappa, s.chi, s.D, s.faceflux,
                    s.edgeflux_x, s.edgeflux_y, s.edgeflux_z, s.cenflux, s.ranchem, s.geom, dt, step, turb);
        evaluateStatsStag1D(s.cu, cuMeans, cuVars, s.prim, primMeans, primVars, s.vel, vm, vv, s.cumom, cmm, cmv,
                            coVars, mom3, mom4, theta, theta, theta, theta, crossMF, ncross, step + 1, s.geom);
    }
    WriteSpatialCross1D(crossMF, nsteps, s.geom, ncross);
    Vector<Real> crossVec;
    MultiFab none;
    WriteCheckPoint(nsteps, nsteps * dt, nsteps, s.geom, s.cu, cuMeans, cuVars, s.prim, primMeans, primVars, s.cumom,
                    cmm, cmv, s.vel, vm, vv, coVars, mom3, mom4, none, none, none, none, crossMF, crossVec, ncross,
                    turb);
    State r(Arena::Device, false);
    MultiFab rcm, rcv, rpm, rpv, rco, rm3, rm4, sc0, rcross;
    std::array<MultiFab, 3> rcmm, rcmv, rvm, rvv;
    BoxArray ba;
    DistributionMapping dm;
    int rstep = -1, count = -1;
    Real time = -1.0;
    common::restart = nsteps;
    ReadCheckPoint(rstep, time, count, r.geom, dom, r.cu, rcm, rcv, r.prim, rpm, rpv, r.cumom, rcmm, rcmv, r.vel, rvm,
                   rvv, rco, rm3, rm4, sc0, sc0, sc0, sc0, rcross, crossVec, ncross, turb, ba, dm);
    if (rstep != nsteps + 1 || count != nsteps || !same(rcross, crossMF) || !same(rcm, cuMeans) || !same(rm4, mom4))
        return 6;
    FILE* f = std::fopen(out, "wb");
    if (!f) return 2;
    for (const MultiFab* m : {&cuMeans, &cuVars, &primMeans, &primVars, &coVars, &mom3, &mom4, &crossMF})
        write_all(f, *m);
    std::fclose(f);
    fhd::ref::finalize();
    return 0;
}

static int cmd_massfrac(int n) {
    set_argon(n, 1);
    common::rhobar[0] = 1.0;  // species 2 absent: Y_2 = 0
    common::rhobar[1] = 0.0;
    fhd::ref::abort_handler = throwing_handler;
    State s(Arena::Device, true);
    try {
        s.init();
    } catch (const Caught& e) {
        std::printf("caught: %s\n", e.what());
        fhd::ref::finalize();
        return 3;
    }
    fhd::ref::finalize();
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s shapes <n> | run <device|pinned> <n> <nsteps> <seed> <dt> <out> | massfrac <n>\n",
                     argv[0]);
        return 1;
    }
    const std::string cmd = argv[1];
    try {
        if (cmd == "shapes") return cmd_shapes(std::atoi(argv[2]));
        if (cmd == "run" && (argc == 8 || argc == 9))
            return cmd_run(argv[2], std::atoi(argv[3]), std::atoi(argv[4]), std::atoi(argv[5]),
                           std::strtod(argv[6], nullptr), argv[7], argc == 9 ? argv[8] : "argon");
        if (cmd == "massfrac") return cmd_massfrac(std::atoi(argv[2]));
        if (cmd == "stats" && argc == 7)
            return cmd_stats(std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4]), std::strtod(argv[5], nullptr),
                             argv[6]);
        if (cmd == "stats1d" && argc == 9)
            return cmd_stats1d(std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4]), std::atoi(argv[5]),
                               std::strtod(argv[6], nullptr), std::atoi(argv[7]), argv[8]);
        if (cmd == "chk" && argc == 8)
            return cmd_chk(std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4]), std::atoi(argv[5]),
                           std::strtod(argv[6], nullptr), argv[7]);
        if (cmd == "plot" && argc == 7)
            return cmd_plot(std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4]), std::strtod(argv[5], nullptr),
                            argv[6]);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 4;
    }
    std::fprintf(stderr, "bad arguments\n");
    return 1;
}
