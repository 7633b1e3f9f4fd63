// reference_api.hpp — FHDeX's compressible staggered-grid interface with the
// reference's own function names and argument lists, over the single-box types
// of fhd/amrex_compat.hpp, forwarding to the C ABI of fhd_capi.h.
//
// A driver written against the reference (main_driver.cpp) keeps its calls:
//
//   RK3stepStag(cu, cumom, prim, vel, source, eta, zeta, kappa, chi, D,
//               faceflux, edgeflux_x, edgeflux_y, edgeflux_z, cenflux,
//               ranchem, geom, dt, step, turbforce);
//
// Reference declarations mirrored here (paths within the FHDeX tree):
//   conservedToPrimitiveStag   src_compressible_stag/compressible_functions_stag.H:69-70
//   InitConsVarStag            src_compressible_stag/compressible_functions_stag.H:72-74
//   RK3stepStag                src_compressible_stag/compressible_functions_stag.H:113-125
//   calculateFluxStag          src_compressible_stag/compressible_functions_stag.H:127-143
//   calculateTransportCoeffs   src_compressible/compressible_functions.H:37-39
//   MultiFabFillRandom,
//   MultiFabFillRandomNormal,
//   MultiFabFillRandomUniform  src_rng/rng_functions.H:13-22
//   compute_compressible_chemistry_source_CLE
//                              src_chemistry/chemistry_functions.H:20-21
//   WritePlotFileStag          src_compressible_stag/compressible_functions_stag.H:15-39
//   WriteCheckPoint,
//   ReadCheckPoint             src_compressible_stag/compressible_functions_stag.H:188-243
//   evaluateStatsStag3D        src_compressible_stag/compressible_functions_stag.H:257-273
//   evaluateStatsStag2D,
//   evaluateStatsStag1D        src_compressible_stag/compressible_functions_stag.H:275-305
//   WriteSpatialCross3D,
//   WriteSpatialCross1D        src_compressible_stag/compressible_functions_stag.H:41-43
//
// As in the reference, physics parameters are process globals in namespaces
// `common`, `compressible` and `chemistry` (src_common/common_namespace.H,
// src_compressible/compressible_namespace.H, src_chemistry/chemistry_namespace.H)
// with the reference's names and defaults (common_functions.cpp:332-550,
// compressible_functions.cpp:15-88, chemistry_functions.cpp:45-124).
// The first call builds one fhd_ctx from them on `fhd::ref::device`; after
// changing a global call fhd::ref::reinitialize().
//
// Errors: the reference calls amrex::Abort (process exit) on a bad mass
// fraction (transCoeffs.cpp:45-46) and on bad input.  Here every failure goes
// to fhd::ref::abort_handler, which by default prints the message and calls
// std::abort(); a caller may install a handler that throws instead.  Device
// physics faults are latched by the kernels; RK3stepStag and
// calculateTransportCoeffs read the status word after their work (one stream
// synchronisation) and report a latched fault the same way.
//
// MultiFabs must live in the device arena, except that RK3stepStag also accepts
// host/pinned cu, cumom, prim and vel (a CPU build's MultiFabs): it then
// copies them through the context's device buffers and leaves the by-product
// MultiFabs (coefficients and fluxes) untouched.
#ifndef FHD_REFERENCE_API_HPP
#define FHD_REFERENCE_API_HPP

#include <cstdio>
#include <cstdlib>
#include <string>

#include "amrex_compat.hpp"

#ifndef MAX_SPECIES
#define MAX_SPECIES FHD_MAX_SPECIES
#endif

// ---- global parameters (reference names, reference defaults) -----------------
namespace common {
using fhd::amrex_compat::GpuArray;
using fhd::amrex_compat::Real;
inline GpuArray<Real, 3> prob_lo{{0.0, 0.0, 0.0}};
inline GpuArray<Real, 3> prob_hi{{1.0, 1.0, 1.0}};
inline GpuArray<int, 3> n_cells{{0, 0, 0}};
inline GpuArray<Real, 3> grav{{0.0, 0.0, 0.0}};
inline int nspecies = 2;
inline GpuArray<Real, MAX_SPECIES> molmass{{1, 1, 1, 1, 1, 1, 1, 1}};
inline GpuArray<Real, MAX_SPECIES> rhobar{{1, 1, 1, 1, 1, 1, 1, 1}};
inline Real rho0 = 1.0;
inline GpuArray<Real, MAX_SPECIES> diameter{{1, 1, 1, 1, 1, 1, 1, 1}};
inline GpuArray<Real, MAX_SPECIES> dof{{0, 0, 0, 0, 0, 0, 0, 0}};          // no default: set it
inline GpuArray<Real, MAX_SPECIES> e0{{0, 0, 0, 0, 0, 0, 0, 0}};
inline GpuArray<Real, MAX_SPECIES> hcv{{-1, -1, -1, -1, -1, -1, -1, -1}};  // < 0: GetHcGas derives it
inline GpuArray<Real, MAX_SPECIES> hcp{{-1, -1, -1, -1, -1, -1, -1, -1}};
inline Real k_B = 1.38064852e-16;
inline Real Runiv = 8.314462175e7;
inline GpuArray<Real, MAX_SPECIES> T_init{{1, 1, 1, 1, 1, 1, 1, 1}};
inline int algorithm_type = 0;  // the staggered decks set 2, the only value the step accepts
inline int advection_type = 0;
inline int seed = 0;
inline int visc_type = 1;
inline int stoch_stress_form = 1;
}  // namespace common

namespace compressible {
using fhd::amrex_compat::Real;
inline int transport_type = 1;
inline Real zeta_ratio = -1.0;
// quasi-1-D / quasi-2-D runs (compressible_functions.cpp:58-66); all_correl: 1-D
// correlations at five x* instead of one
inline int do_1D = 0;
inline int do_2D = 0;
inline int all_correl = 0;
}  // namespace compressible

namespace common {
// <= 0: Runiv / k_B, as InitializeCommonNamespace derives it (common_functions.cpp:775)
inline fhd::amrex_compat::Real avogadro = 0.0;
// checkpoint to restart from, < 0: none (common_functions.cpp; ReadCheckPoint reads chk<restart>)
inline int restart = -1;
// plotfile inputs (common_functions.cpp:390, 614-618)
inline std::string plot_base_name = "plt";
inline int plot_means = 0;
inline int plot_vars = 0;
inline int plot_covars = 0;
inline int plot_mom3 = 0;
inline int plot_mom4 = 0;
inline int plot_deltaY_dir = -1;  // common_functions.cpp:620
// yz-averaged spatial cross-correlations at x = cross_cell (common_functions.cpp:345, 619)
inline int plot_cross = 0;
inline int cross_cell = 0;
// a restart zeroes the statistics instead of reading them (Checkpoint.cpp:346, 500)
inline int reset_stats = 0;
// Physical boundaries (common_namespace.H:150-185, read at common_functions.cpp:800-900).
// A direction whose bc_vel_lo and bc_vel_hi are both -1 is periodic (the default
// here; the staggered decks set every bc_vel); otherwise both sides are walls:
// bc_vel 1 slip / 2 no-slip, bc_therm 1 adiabatic / 2 isothermal at t_lo / t_hi,
// bc_mass 1 impermeable / 2 at the wall composition bc_Yk_* or bc_Xk_* (the one
// that sums to 1) / 3 a reservoir at t, p, rho and that composition / 4 the same
// reservoir with the interface fluxes of the particles crossing it.
inline GpuArray<int, 3> bc_vel_lo{{-1, -1, -1}}, bc_vel_hi{{-1, -1, -1}};
inline GpuArray<int, 3> bc_mass_lo{{-1, -1, -1}}, bc_mass_hi{{-1, -1, -1}};
inline GpuArray<int, 3> bc_therm_lo{{-1, -1, -1}}, bc_therm_hi{{-1, -1, -1}};
inline GpuArray<Real, 3> t_lo{{0., 0., 0.}}, t_hi{{0., 0., 0.}};
// reservoirs (bc_mass 3): pressure (<= 0: the initial state's), density (<= 0: from p, t, Y)
inline GpuArray<Real, 3> p_lo{{0., 0., 0.}}, p_hi{{0., 0., 0.}};
inline GpuArray<Real, 3> rho_lo{{-1., -1., -1.}}, rho_hi{{-1., -1., -1.}};
inline GpuArray<Real, MAX_SPECIES> bc_Yk_x_lo{{-1, -1, -1, -1, -1, -1, -1, -1}}, bc_Yk_x_hi{{-1, -1, -1, -1, -1, -1, -1, -1}};
inline GpuArray<Real, MAX_SPECIES> bc_Yk_y_lo{{-1, -1, -1, -1, -1, -1, -1, -1}}, bc_Yk_y_hi{{-1, -1, -1, -1, -1, -1, -1, -1}};
inline GpuArray<Real, MAX_SPECIES> bc_Yk_z_lo{{-1, -1, -1, -1, -1, -1, -1, -1}}, bc_Yk_z_hi{{-1, -1, -1, -1, -1, -1, -1, -1}};
inline GpuArray<Real, MAX_SPECIES> bc_Xk_x_lo{{-1, -1, -1, -1, -1, -1, -1, -1}}, bc_Xk_x_hi{{-1, -1, -1, -1, -1, -1, -1, -1}};
inline GpuArray<Real, MAX_SPECIES> bc_Xk_y_lo{{-1, -1, -1, -1, -1, -1, -1, -1}}, bc_Xk_y_hi{{-1, -1, -1, -1, -1, -1, -1, -1}};
inline GpuArray<Real, MAX_SPECIES> bc_Xk_z_lo{{-1, -1, -1, -1, -1, -1, -1, -1}}, bc_Xk_z_hi{{-1, -1, -1, -1, -1, -1, -1, -1}};
}  // namespace common

namespace chemistry {
using fhd::amrex_compat::GpuArray;
using fhd::amrex_compat::Real;
// Array2D<int, 0, MAX_REACTION, 0, MAX_SPECIES> of the reference, indexed (reaction, species)
struct StoichTable {
    int v[FHD_MAX_REACTIONS][FHD_MAX_SPECIES] = {};
    int& operator()(int m, int n) { return v[m][n]; }
    int operator()(int m, int n) const { return v[m][n]; }
};
inline int nreaction = 0;
inline int reaction_type = 0;  // 0 deterministic, 1 CLE (the only two the compressible source takes)
inline StoichTable stoich_coeffs_R, stoich_coeffs_P;
inline GpuArray<Real, FHD_MAX_REACTIONS> rate_const{};
inline GpuArray<Real, FHD_MAX_REACTIONS> alpha_param{};
inline GpuArray<Real, FHD_MAX_REACTIONS> beta_param{};
inline Real T0_chem = 0.0;
}  // namespace chemistry

namespace fhd {
namespace ref {

using amrex_compat::Arena;
using amrex_compat::Geometry;
using amrex_compat::MultiFab;
using amrex_compat::Real;
using amrex_compat::Vector;

// Precision of the step (FHD_PREC_FP64 or FHD_PREC_MIXED); not a reference
// parameter.
inline int precision = FHD_PREC_FP64;
// CUDA device of the process-wide context.
inline int device = 0;
// Stream the context enqueues on (cudaStream_t; nullptr = legacy default).
inline void* stream = nullptr;

[[noreturn]] inline void default_abort(const char* msg) {
    std::fprintf(stderr, "fhd::ref abort: %s\n", msg);
    std::fflush(stderr);
    std::abort();
}
// Called on every failure; must not return normally (throw or exit).
inline void (*abort_handler)(const char*) = default_abort;

[[noreturn]] inline void fail(const std::string& where, int rc) {
    const std::string m = where + ": " + fhd_strerror(rc);
    abort_handler(m.c_str());
    std::abort();  // a handler that returns still ends the call
}

inline fhd_params params_from_globals() {
    fhd_params p;
    std::memset(&p, 0, sizeof(p));
    p.nspecies = common::nspecies;
    for (int d = 0; d < 3; ++d) {
        p.n_cells[d] = common::n_cells[d];
        p.prob_lo[d] = common::prob_lo[d];
        p.prob_hi[d] = common::prob_hi[d];
        p.grav[d] = common::grav[d];
    }
    for (int s = 0; s < FHD_MAX_SPECIES; ++s) {
        p.molmass[s] = common::molmass[s];
        p.diameter[s] = common::diameter[s];
        p.dof[s] = common::dof[s];
        p.e0[s] = common::e0[s];
        p.hcv[s] = common::hcv[s];
        p.hcp[s] = common::hcp[s];
    }
    p.k_B = common::k_B;
    p.Runiv = common::Runiv;
    p.zeta_ratio = compressible::zeta_ratio;
    p.algorithm_type = common::algorithm_type;
    p.visc_type = common::visc_type;
    p.advection_type = common::advection_type;
    p.transport_type = compressible::transport_type;
    p.stoch_stress_form = common::stoch_stress_form;
    p.precision = precision;
    p.seed = uint64_t(int64_t(common::seed));
    p.nreaction = chemistry::nreaction;
    p.reaction_type = chemistry::reaction_type;
    for (int m = 0; m < FHD_MAX_REACTIONS; ++m) {
        for (int n = 0; n < FHD_MAX_SPECIES; ++n) {
            p.stoich_R[m][n] = chemistry::stoich_coeffs_R(m, n);
            p.stoich_P[m][n] = chemistry::stoich_coeffs_P(m, n);
        }
        p.rate_const[m] = chemistry::rate_const[m];
        p.alpha_param[m] = chemistry::alpha_param[m];
        p.beta_param[m] = chemistry::beta_param[m];
    }
    p.T0_chem = chemistry::T0_chem;
    p.avogadro = common::avogadro;
    const amrex_compat::GpuArray<Real, MAX_SPECIES>* yk[2][3] = {{&common::bc_Yk_x_lo, &common::bc_Yk_y_lo, &common::bc_Yk_z_lo},
                                                   {&common::bc_Yk_x_hi, &common::bc_Yk_y_hi, &common::bc_Yk_z_hi}};
    const amrex_compat::GpuArray<Real, MAX_SPECIES>* xk[2][3] = {{&common::bc_Xk_x_lo, &common::bc_Xk_y_lo, &common::bc_Xk_z_lo},
                                                   {&common::bc_Xk_x_hi, &common::bc_Xk_y_hi, &common::bc_Xk_z_hi}};
    for (int d = 0; d < 3; ++d) {
        if (common::bc_vel_lo[d] != -1 || common::bc_vel_hi[d] != -1) p.walls = 1;
        p.bc_vel_lo[d] = common::bc_vel_lo[d];
        p.bc_vel_hi[d] = common::bc_vel_hi[d];
        p.bc_mass_lo[d] = common::bc_mass_lo[d];
        p.bc_mass_hi[d] = common::bc_mass_hi[d];
        p.bc_therm_lo[d] = common::bc_therm_lo[d];
        p.bc_therm_hi[d] = common::bc_therm_hi[d];
        p.t_lo[d] = common::t_lo[d];
        p.t_hi[d] = common::t_hi[d];
        p.p_lo[d] = common::p_lo[d];
        p.p_hi[d] = common::p_hi[d];
        p.rho_lo[d] = common::rho_lo[d];
        p.rho_hi[d] = common::rho_hi[d];
        for (int s = 0; s < FHD_MAX_SPECIES; ++s) {
            p.bc_Yk_lo[d][s] = (*yk[0][d])[s];
            p.bc_Yk_hi[d][s] = (*yk[1][d])[s];
            p.bc_Xk_lo[d][s] = (*xk[0][d])[s];
            p.bc_Xk_hi[d][s] = (*xk[1][d])[s];
        }
    }
    p.rho0 = common::rho0;
    p.T_init = common::T_init[0];
    for (int s = 0; s < FHD_MAX_SPECIES; ++s) p.rhobar[s] = common::rhobar[s];
    p.cross_cell = common::cross_cell;
    p.do_1D = compressible::do_1D;
    p.do_2D = compressible::do_2D;
    p.all_correl = compressible::all_correl;
    return p;
}

struct Runtime {
    fhd_ctx* ctx = nullptr;
    uint64_t fill_calls = 0;  // stream ids of successive MultiFabFillRandom* calls
    // device mirror of the host vectors spatialCross3D and dataSliceMeans_xcross
    double* cross = nullptr;
    size_t cross_doubles = 0;
    ~Runtime() {
        if (ctx) fhd_destroy(ctx);
        if (cross) cudaFree(cross);
    }
};
inline Runtime& runtime() {
    static Runtime r;
    return r;
}

inline void finalize() {
    Runtime& r = runtime();
    if (r.ctx) fhd_destroy(r.ctx);
    r.ctx = nullptr;
    if (r.cross) cudaFree(r.cross);
    r.cross = nullptr;
    r.cross_doubles = 0;
}

// The process-wide context, created from the globals on first use.
inline fhd_ctx* context() {
    Runtime& r = runtime();
    if (!r.ctx) {
        const fhd_params p = params_from_globals();
        int rc = fhd_create(&r.ctx, &p, device);
        if (rc != FHD_OK) {
            r.ctx = nullptr;
            fail("fhd_create", rc);
        }
        rc = fhd_set_stream(r.ctx, stream);
        if (rc != FHD_OK) fail("fhd_set_stream", rc);
    }
    return r.ctx;
}

inline void reinitialize() {
    finalize();
    context();
}

inline void check(int rc, const char* where) {
    if (rc != FHD_OK) fail(where, rc);
}

inline void require_device(const MultiFab& mf, const char* where) {
    if (!mf.ok() || mf.arena() != Arena::Device)
        fail(std::string(where) + ": MultiFab must be allocated in the device arena", FHD_ERR_BAD_ARG);
}

template <size_t N>
inline void fabs_of(const std::array<MultiFab, N>& a, fhd_fab* out) {
    for (size_t d = 0; d < N; ++d) out[d] = a[d].fab();
}

// Whether every MultiFab of `a` was allocated (by-product arrays are optional).
template <size_t N>
inline bool all_ok(const std::array<MultiFab, N>& a) {
    for (const auto& m : a)
        if (!m.ok()) return false;
    return true;
}

}  // namespace ref
}  // namespace fhd

// Turbulence forcing object of the reference's RK3stepStag signature; only used
// under -DTURB there and unused here.
struct TurbForcingComp {};

inline void fhd::amrex_compat::MultiFab::FillBoundary(const Periodicity&) {
    fhd::ref::require_device(*this, "FillBoundary");
    fhd::ref::check(fhd_fill_boundary(fhd::ref::context(), fab()), "FillBoundary");
}
inline void fhd::amrex_compat::MultiFab::OverrideSync(const Periodicity&) {
    fhd::ref::require_device(*this, "OverrideSync");
    fhd::ref::check(fhd_override_sync(fhd::ref::context(), fab()), "OverrideSync");
}

// ---- the reference's functions --------------------------------------------------

// InitConsVarStag, prob_type 1 (uniform state at rest)
// (compressible_functions_stag.cpp:36-56): rho0, T_init[0] and rhobar from the
// globals.
inline void InitConsVarStag(fhd::amrex_compat::MultiFab& cons,
                            std::array<fhd::amrex_compat::MultiFab, 3>& momStag,
                            const fhd::amrex_compat::Geometry& /*geom*/) {
    using namespace fhd::ref;
    require_device(cons, "InitConsVarStag");
    for (auto& m : momStag) require_device(m, "InitConsVarStag");
    fhd_fab mom[3];
    fabs_of(momStag, mom);
    check(fhd_init_cons_var_stag(context(), cons.fab(), mom, common::rho0, common::T_init[0],
                                 common::rhobar.data()),
          "InitConsVarStag");
}

// setBCStag (boundaryStag.cpp:268-298): the wall conditions on every ghost of a
// wall direction and the wall faces; nothing on a fully periodic box.
inline void setBCStag(fhd::amrex_compat::MultiFab& prim_in, fhd::amrex_compat::MultiFab& cons_in,
                      std::array<fhd::amrex_compat::MultiFab, 3>& cumom_in,
                      std::array<fhd::amrex_compat::MultiFab, 3>& vel_in,
                      const fhd::amrex_compat::Geometry& /*geom*/) {
    using namespace fhd::ref;
    require_device(prim_in, "setBCStag");
    require_device(cons_in, "setBCStag");
    fhd_fab mom[3], vel[3];
    for (int d = 0; d < 3; ++d) {
        require_device(cumom_in[d], "setBCStag");
        require_device(vel_in[d], "setBCStag");
    }
    fabs_of(cumom_in, mom);
    fabs_of(vel_in, vel);
    check(fhd_set_bc_stag(context(), prim_in.fab(), cons_in.fab(), mom, vel), "setBCStag");
}

// conservedToPrimitiveStag (conservedPrimitiveConversionsStag.cpp:5-144).
inline void conservedToPrimitiveStag(fhd::amrex_compat::MultiFab& prim_in,
                                     std::array<fhd::amrex_compat::MultiFab, 3>& velStag_in,
                                     fhd::amrex_compat::MultiFab& cons_in,
                                     const std::array<fhd::amrex_compat::MultiFab, 3>& momStag_in) {
    using namespace fhd::ref;
    require_device(prim_in, "conservedToPrimitiveStag");
    require_device(cons_in, "conservedToPrimitiveStag");
    fhd_fab vel[3], mom[3];
    fabs_of(velStag_in, vel);
    fabs_of(momStag_in, mom);
    check(fhd_conserved_to_primitive_stag(context(), prim_in.fab(), vel, cons_in.fab(), mom),
          "conservedToPrimitiveStag");
}

// compute_compressible_chemistry_source_CLE (chemistry_functions.cpp:128-193):
// species components 5.. of `source` from `prim` and the reaction noises
// `ranchem` (read for reaction_type 1 only).
inline void compute_compressible_chemistry_source_CLE(fhd::amrex_compat::Real dt, fhd::amrex_compat::Real dV,
                                                      fhd::amrex_compat::MultiFab& prim,
                                                      fhd::amrex_compat::MultiFab& source,
                                                      fhd::amrex_compat::MultiFab& ranchem) {
    using namespace fhd::ref;
    require_device(prim, "compute_compressible_chemistry_source_CLE");
    require_device(source, "compute_compressible_chemistry_source_CLE");
    fhd_fab rf;
    std::memset(&rf, 0, sizeof(rf));
    if (chemistry::reaction_type == 1) {
        require_device(ranchem, "compute_compressible_chemistry_source_CLE");
        rf = ranchem.fab();
    }
    check(fhd_chemistry_source_cle(context(), dt, dV, prim.fab(), source.fab(), rf),
          "compute_compressible_chemistry_source_CLE");
}

// calculateTransportCoeffs (transCoeffs.cpp:7-90).  A bad mass fraction is
// reported through abort_handler, where the reference aborts.
inline void calculateTransportCoeffs(const fhd::amrex_compat::MultiFab& prim_in,
                                     fhd::amrex_compat::MultiFab& eta_in,
                                     fhd::amrex_compat::MultiFab& zeta_in,
                                     fhd::amrex_compat::MultiFab& kappa_in,
                                     fhd::amrex_compat::MultiFab& chi_in,
                                     fhd::amrex_compat::MultiFab& Dij_in) {
    using namespace fhd::ref;
    require_device(prim_in, "calculateTransportCoeffs");
    check(fhd_transport_coeffs(context(), prim_in.fab(), eta_in.fab(), zeta_in.fab(), kappa_in.fab(),
                               chi_in.fab(), Dij_in.fab()),
          "calculateTransportCoeffs");
    check(fhd_status(context()), "calculateTransportCoeffs");
}

// calculateFluxStag (fluxStag.cpp:5-1868).  stochface/stochedge/stochcen are
// the combined noise W = W_A + w_s W_B of the stage, as RK3stepStag passes
// them; the reference reads only stochedge_x[0] (xy), stochedge_x[1] (xz) and
// stochedge_y[1] (yz) (fluxStag.cpp:130-132), and so does this call.
// stoch_weights is accepted for the signature and unused, as in the reference.
inline void calculateFluxStag(
    const fhd::amrex_compat::MultiFab& cons_in, const std::array<fhd::amrex_compat::MultiFab, 3>& momStag_in,
    const fhd::amrex_compat::MultiFab& prim_in, const std::array<fhd::amrex_compat::MultiFab, 3>& velStag_in,
    const fhd::amrex_compat::MultiFab& eta_in, const fhd::amrex_compat::MultiFab& zeta_in,
    const fhd::amrex_compat::MultiFab& kappa_in, const fhd::amrex_compat::MultiFab& chi_in,
    const fhd::amrex_compat::MultiFab& D_in, std::array<fhd::amrex_compat::MultiFab, 3>& faceflux_in,
    std::array<fhd::amrex_compat::MultiFab, 2>& edgeflux_x_in, std::array<fhd::amrex_compat::MultiFab, 2>& edgeflux_y_in,
    std::array<fhd::amrex_compat::MultiFab, 2>& edgeflux_z_in, std::array<fhd::amrex_compat::MultiFab, 3>& cenflux_in,
    std::array<fhd::amrex_compat::MultiFab, 3>& stochface_in, std::array<fhd::amrex_compat::MultiFab, 2>& stochedge_x_in,
    std::array<fhd::amrex_compat::MultiFab, 2>& stochedge_y_in,
    std::array<fhd::amrex_compat::MultiFab, 2>& /*stochedge_z_in*/,
    std::array<fhd::amrex_compat::MultiFab, 3>& stochcen_in, const fhd::amrex_compat::Geometry& /*geom*/,
    const fhd::amrex_compat::Vector<fhd::amrex_compat::Real>& /*stoch_weights*/, const fhd::amrex_compat::Real dt) {
    using namespace fhd::ref;
    fhd_fab mom[3], vel[3], ff[3], ef[6], cf[3], sf[3], se[3], sc[3];
    fabs_of(momStag_in, mom);
    fabs_of(velStag_in, vel);
    fabs_of(faceflux_in, ff);
    ef[0] = edgeflux_x_in[0].fab();
    ef[1] = edgeflux_x_in[1].fab();
    ef[2] = edgeflux_y_in[0].fab();
    ef[3] = edgeflux_y_in[1].fab();
    ef[4] = edgeflux_z_in[0].fab();
    ef[5] = edgeflux_z_in[1].fab();
    fabs_of(cenflux_in, cf);
    fabs_of(stochface_in, sf);
    se[0] = stochedge_x_in[0].fab();
    se[1] = stochedge_x_in[1].fab();
    se[2] = stochedge_y_in[1].fab();
    fabs_of(stochcen_in, sc);
    check(fhd_flux_stag(context(), cons_in.fab(), mom, prim_in.fab(), vel, eta_in.fab(), zeta_in.fab(),
                        kappa_in.fab(), chi_in.fab(), D_in.fab(), ff, ef, cf, sf, se, sc, dt),
          "calculateFluxStag");
}

// RK3stepStag (timeStepStag.cpp:13-1245).  The white noise of step `step` is
// Philox-4x32-10 keyed by common::seed, generated inside the step's kernels.
// Coefficient and flux MultiFabs receive the stage-3 values when allocated;
// leave them undefined (default-constructed) to skip them.  `source` is the
// reference's chemistry source (zero unless chemistry is on; may be
// undefined).  `ranchem` and `turbforce` are unused, as in the reference's
// non-chemistry, non-TURB build.
inline void RK3stepStag(fhd::amrex_compat::MultiFab& cu, std::array<fhd::amrex_compat::MultiFab, 3>& cumom,
                        fhd::amrex_compat::MultiFab& prim, std::array<fhd::amrex_compat::MultiFab, 3>& facevel,
                        fhd::amrex_compat::MultiFab& source, fhd::amrex_compat::MultiFab& eta,
                        fhd::amrex_compat::MultiFab& zeta, fhd::amrex_compat::MultiFab& kappa,
                        fhd::amrex_compat::MultiFab& chi, fhd::amrex_compat::MultiFab& D,
                        std::array<fhd::amrex_compat::MultiFab, 3>& faceflux,
                        std::array<fhd::amrex_compat::MultiFab, 2>& edgeflux_x,
                        std::array<fhd::amrex_compat::MultiFab, 2>& edgeflux_y,
                        std::array<fhd::amrex_compat::MultiFab, 2>& edgeflux_z,
                        std::array<fhd::amrex_compat::MultiFab, 3>& cenflux,
                        fhd::amrex_compat::MultiFab& /*ranchem*/, const fhd::amrex_compat::Geometry& /*geom*/,
                        const fhd::amrex_compat::Real dt, const int step, TurbForcingComp& /*turbforce*/) {
    using namespace fhd::ref;
    fhd_ctx* ctx = context();
    fhd_fab mom[3], vel[3];
    fabs_of(cumom, mom);
    fabs_of(facevel, vel);
    if (cu.arena() != Arena::Device) {
        // host MultiFabs: copies through the context's device buffers
        int64_t h2d = 0, d2h = 0;
        check(fhd_rk3_step_stag_host(ctx, cu.fab(), mom, prim.fab(), vel, nullptr, dt, step, &h2d, &d2h),
              "RK3stepStag");
    } else {
        require_device(prim, "RK3stepStag");
        fhd_fab ff[3], ef[6], cf[3];
        const bool want_ff = all_ok(faceflux);
        const bool want_ef = all_ok(edgeflux_x) && all_ok(edgeflux_y) && all_ok(edgeflux_z);
        const bool want_cf = all_ok(cenflux);
        if (want_ff) fabs_of(faceflux, ff);
        if (want_ef) {
            ef[0] = edgeflux_x[0].fab();
            ef[1] = edgeflux_x[1].fab();
            ef[2] = edgeflux_y[0].fab();
            ef[3] = edgeflux_y[1].fab();
            ef[4] = edgeflux_z[0].fab();
            ef[5] = edgeflux_z[1].fab();
        }
        if (want_cf) fabs_of(cenflux, cf);
        check(fhd_rk3_step_stag(ctx, cu.fab(), mom, prim.fab(), vel, source.fab(), eta.fab(), zeta.fab(),
                                kappa.fab(), chi.fab(), D.fab(), want_ff ? ff : nullptr, want_ef ? ef : nullptr,
                                want_cf ? cf : nullptr, nullptr, dt, step),
              "RK3stepStag");
    }
    check(fhd_status(ctx), "RK3stepStag");
}

// MultiFabFillRandomNormal (MultiFabFillRandom.cpp:34-50): N(mean, variance) in
// components scomp..scomp+ncomp-1 of the valid region, then OverrideSync and
// FillBoundary when asked.  Successive calls draw independent Philox streams,
// as successive calls on the reference's global generator draw new numbers.
inline void MultiFabFillRandomNormal(fhd::amrex_compat::MultiFab& mf, const int& scomp, const int& ncomp,
                                     const fhd::amrex_compat::Real& mean, const fhd::amrex_compat::Real& variance,
                                     const fhd::amrex_compat::Geometry& /*geom*/, bool overridesync = true,
                                     bool fillboundary = true) {
    using namespace fhd::ref;
    require_device(mf, "MultiFabFillRandomNormal");
    const uint64_t id = ++runtime().fill_calls;
    check(fhd_fill_random_normal(context(), mf.fab(), scomp, ncomp, mean, variance, overridesync ? 1 : 0,
                                 fillboundary ? 1 : 0, id),
          "MultiFabFillRandomNormal");
}

// MultiFabFillRandomUniform (MultiFabFillRandom.cpp:53-66): uniforms in [0, 1) in
// components scomp..scomp+ncomp-1 of the valid region, then OverrideSync and
// FillBoundary when asked; independent streams per call as above.
inline void MultiFabFillRandomUniform(fhd::amrex_compat::MultiFab& mf, const int& scomp, const int& ncomp,
                                      const fhd::amrex_compat::Geometry& /*geom*/, bool overridesync = true,
                                      bool fillboundary = true) {
    using namespace fhd::ref;
    require_device(mf, "MultiFabFillRandomUniform");
    const uint64_t id = ++runtime().fill_calls;
    check(fhd_fill_random_uniform(context(), mf.fab(), scomp, ncomp, overridesync ? 1 : 0, fillboundary ? 1 : 0, id),
          "MultiFabFillRandomUniform");
}

// WritePlotFileStag (writePlotFileStag.cpp:7-527): the plotfile
// <plot_base_name><step, 9 digits>/ with the common::plot_means / plot_vars /
// plot_covars / plot_mom3 / plot_mom4 / plot_deltaY_dir selections.  The surface-coverage
// MultiFabs are accepted and ignored (no surface chemistry on this path).
inline void WritePlotFileStag(int step, const fhd::amrex_compat::Real time, const fhd::amrex_compat::Geometry& /*geom*/,
                              const fhd::amrex_compat::MultiFab& cu, const fhd::amrex_compat::MultiFab& cuMeans,
                              const fhd::amrex_compat::MultiFab& cuVars,
                              const std::array<fhd::amrex_compat::MultiFab, 3>& cumom,
                              const std::array<fhd::amrex_compat::MultiFab, 3>& cumomMeans,
                              const std::array<fhd::amrex_compat::MultiFab, 3>& cumomVars,
                              const fhd::amrex_compat::MultiFab& prim, const fhd::amrex_compat::MultiFab& primMeans,
                              const fhd::amrex_compat::MultiFab& primVars,
                              const std::array<fhd::amrex_compat::MultiFab, 3>& vel,
                              const std::array<fhd::amrex_compat::MultiFab, 3>& velMeans,
                              const std::array<fhd::amrex_compat::MultiFab, 3>& velVars,
                              const fhd::amrex_compat::MultiFab& coVars, const fhd::amrex_compat::MultiFab& mom3,
                              const fhd::amrex_compat::MultiFab& mom4, const fhd::amrex_compat::MultiFab& /*surfcov*/,
                              const fhd::amrex_compat::MultiFab& /*surfcovMeans*/,
                              const fhd::amrex_compat::MultiFab& /*surfcovVars*/,
                              const fhd::amrex_compat::MultiFab& /*surfcovcoVars*/,
                              const fhd::amrex_compat::MultiFab& eta, const fhd::amrex_compat::MultiFab& kappa,
                              const fhd::amrex_compat::MultiFab& zeta) {
    using namespace fhd::ref;
    const int flags = (common::plot_means == 1 ? FHD_PLOT_MEANS : 0) | (common::plot_vars == 1 ? FHD_PLOT_VARS : 0) |
                      (common::plot_covars == 1 ? FHD_PLOT_COVARS : 0) | (common::plot_mom3 ? FHD_PLOT_MOM3 : 0) |
                      (common::plot_mom4 ? FHD_PLOT_MOM4 : 0) |
                      (common::plot_deltaY_dir >= 0 && common::plot_deltaY_dir < 3 ? (FHD_PLOT_DELTAY_X << common::plot_deltaY_dir) : 0);
    fhd_stats st;
    std::memset(&st, 0, sizeof(st));
    st.cuMeans = cuMeans.fab();
    st.cuVars = cuVars.fab();
    st.primMeans = primMeans.fab();
    st.primVars = primVars.fab();
    st.coVars = coVars.fab();
    st.mom3 = mom3.fab();
    st.mom4 = mom4.fab();
    for (int d = 0; d < 3; ++d) {
        st.velMeans[d] = velMeans[d].fab();
        st.velVars[d] = velVars[d].fab();
        st.cumomMeans[d] = cumomMeans[d].fab();
        st.cumomVars[d] = cumomVars[d].fab();
    }
    fhd_fab mom[3], vl[3];
    fabs_of(cumom, mom);
    fabs_of(vel, vl);
    check(fhd_write_plotfile_stag(context(), common::plot_base_name.c_str(), step, time, flags, cu.fab(), mom,
                                  prim.fab(), vl, eta.fab(), kappa.fab(), zeta.fab(), &st),
          "WritePlotFileStag");
}

// evaluateStatsStag3D (statsStag.cpp:10-77): the running means (plot_means) and
// the variances, covariances and third / fourth moments (plot_vars or
// plot_covars; plot_mom3 / plot_mom4) with sample count `steps`, each followed by
// the reference's FillBoundary, then with plot_cross the yz-averaged spatial
// cross-correlations at x = cross_cell into the host vectors spatialCross3D
// (n_cells[0] * ncross) and dataSliceMeans_xcross (2*nvars + 8 + 2*nspecies),
// through a device mirror (copied in and out on the context's stream; the call
// then waits for the stream).  Without surface coverage (theta*): those
// arguments are accepted and left untouched.
inline void evaluateStatsStag3D(fhd::amrex_compat::MultiFab& cons, fhd::amrex_compat::MultiFab& consMean,
                                fhd::amrex_compat::MultiFab& consVar, fhd::amrex_compat::MultiFab& prim_in,
                                fhd::amrex_compat::MultiFab& primMean, fhd::amrex_compat::MultiFab& primVar,
                                const std::array<fhd::amrex_compat::MultiFab, 3>& vel,
                                std::array<fhd::amrex_compat::MultiFab, 3>& velMean,
                                std::array<fhd::amrex_compat::MultiFab, 3>& velVar,
                                const std::array<fhd::amrex_compat::MultiFab, 3>& cumom,
                                std::array<fhd::amrex_compat::MultiFab, 3>& cumomMean,
                                std::array<fhd::amrex_compat::MultiFab, 3>& cumomVar,
                                fhd::amrex_compat::MultiFab& coVar, fhd::amrex_compat::MultiFab& mom3,
                                fhd::amrex_compat::MultiFab& mom4, fhd::amrex_compat::MultiFab& /*theta*/,
                                fhd::amrex_compat::MultiFab& /*thetaMean*/, fhd::amrex_compat::MultiFab& /*thetaVar*/,
                                fhd::amrex_compat::MultiFab& /*thetacoVar*/,
                                fhd::amrex_compat::Vector<fhd::amrex_compat::Real>& dataSliceMeans_xcross,
                                fhd::amrex_compat::Vector<fhd::amrex_compat::Real>& spatialCross3D,
                                const int ncross, const fhd::amrex_compat::Box& /*domain*/, const int steps,
                                const fhd::amrex_compat::Geometry& /*geom*/) {
    using namespace fhd::ref;
    const int flags = (common::plot_means ? FHD_STATS_MEANS : 0) |
                      ((common::plot_vars || common::plot_covars) ? FHD_STATS_VARS : 0) |
                      (common::plot_mom3 ? FHD_STATS_MOM3 : 0) | (common::plot_mom4 ? FHD_STATS_MOM4 : 0) |
                      (common::plot_cross ? FHD_STATS_CROSS : 0);
    if (!flags) return;
    const size_t nsc = (size_t)common::n_cells[0] * ncross, nxc = dataSliceMeans_xcross.size();
    if (common::plot_cross) {
        if (ncross != fhd_spatial_cross_ncross(common::nspecies) || spatialCross3D.size() < nsc ||
            (int)nxc < fhd_spatial_cross_nstats(common::nspecies))
            fail("evaluateStatsStag3D", FHD_ERR_BAD_ARG);
        Runtime& r = runtime();
        if (r.cross_doubles < nsc + nxc) {
            if (r.cross) cudaFree(r.cross);
            r.cross = nullptr;
            r.cross_doubles = 0;
            if (cudaMalloc(reinterpret_cast<void**>(&r.cross), (nsc + nxc) * sizeof(double)) != cudaSuccess) {
                cudaGetLastError();
                fail("evaluateStatsStag3D", FHD_ERR_OOM);
            }
            r.cross_doubles = nsc + nxc;
        }
        const cudaStream_t cs = static_cast<cudaStream_t>(stream);
        if (cudaMemcpyAsync(r.cross, spatialCross3D.data(), nsc * sizeof(double), cudaMemcpyHostToDevice, cs) !=
            cudaSuccess)
            fail("evaluateStatsStag3D", FHD_ERR_CUDA);
    }
    fhd_stats st;
    std::memset(&st, 0, sizeof(st));
    st.cuMeans = consMean.fab();
    st.cuVars = consVar.fab();
    st.primMeans = primMean.fab();
    st.primVars = primVar.fab();
    st.coVars = coVar.fab();
    st.mom3 = mom3.fab();
    st.mom4 = mom4.fab();
    for (int d = 0; d < 3; ++d) {
        st.velMeans[d] = velMean[d].fab();
        st.velVars[d] = velVar[d].fab();
        st.cumomMeans[d] = cumomMean[d].fab();
        st.cumomVars[d] = cumomVar[d].fab();
    }
    if (common::plot_cross) {
        st.spatialCross = runtime().cross;
        st.dataSliceMeans_xcross = runtime().cross + nsc;
    }
    fhd_fab vl[3], mom[3];
    fabs_of(vel, vl);
    fabs_of(cumom, mom);
    check(fhd_stats_stag(context(), cons.fab(), prim_in.fab(), vl, mom, &st, steps, flags), "evaluateStatsStag3D");
    if (common::plot_cross) {
        const cudaStream_t cs = static_cast<cudaStream_t>(stream);
        if (cudaMemcpyAsync(spatialCross3D.data(), st.spatialCross, nsc * sizeof(double), cudaMemcpyDeviceToHost,
                            cs) != cudaSuccess ||
            cudaMemcpyAsync(dataSliceMeans_xcross.data(), st.dataSliceMeans_xcross, nxc * sizeof(double),
                            cudaMemcpyDeviceToHost, cs) != cudaSuccess ||
            cudaStreamSynchronize(cs) != cudaSuccess)
            fail("evaluateStatsStag3D", FHD_ERR_CUDA);
    }
}

// WriteSpatialCross3D (writePlotFileStag.cpp:528-549): spatialCross<step, 9 digits>
// in the working directory.
inline void WriteSpatialCross3D(const fhd::amrex_compat::Vector<fhd::amrex_compat::Real>& spatialCross, int step,
                                const fhd::amrex_compat::Geometry& /*geom*/, const int ncross) {
    using namespace fhd::ref;
    const fhd_params p = params_from_globals();
    if (ncross != fhd_spatial_cross_ncross(p.nspecies) || spatialCross.size() < (size_t)p.n_cells[0] * ncross)
        fail("WriteSpatialCross3D", FHD_ERR_BAD_ARG);
    check(fhd_write_spatial_cross(&p, "", step, spatialCross.data()), "WriteSpatialCross3D");
}

// evaluateStatsStag1D / evaluateStatsStag2D (statsStag.cpp:78-197), for quasi-1-D /
// 2-D runs (compressible::do_1D / do_2D): the per-cell statistics as evaluateStatsStag3D,
// and in 1-D with plot_cross the per-pencil spatial correlations into spatialCross1D (a
// cell-centred MultiFab without ghosts in the device arena, ncross components, or
// 5*ncross with compressible::all_correl, as main_driver.cpp:717-727 defines it).
inline void evaluateStatsStagLowDim(fhd::amrex_compat::MultiFab& cons, fhd::amrex_compat::MultiFab& consMean,
                                    fhd::amrex_compat::MultiFab& consVar, fhd::amrex_compat::MultiFab& prim_in,
                                    fhd::amrex_compat::MultiFab& primMean, fhd::amrex_compat::MultiFab& primVar,
                                    const std::array<fhd::amrex_compat::MultiFab, 3>& vel,
                                    std::array<fhd::amrex_compat::MultiFab, 3>& velMean,
                                    std::array<fhd::amrex_compat::MultiFab, 3>& velVar,
                                    const std::array<fhd::amrex_compat::MultiFab, 3>& cumom,
                                    std::array<fhd::amrex_compat::MultiFab, 3>& cumomMean,
                                    std::array<fhd::amrex_compat::MultiFab, 3>& cumomVar,
                                    fhd::amrex_compat::MultiFab& coVar, fhd::amrex_compat::MultiFab& mom3,
                                    fhd::amrex_compat::MultiFab& mom4, fhd::amrex_compat::MultiFab& spatialCross,
                                    const int ncross, const int steps, const char* where) {
    using namespace fhd::ref;
    const bool cross = common::plot_cross && compressible::do_1D;
    const int flags = (common::plot_means ? FHD_STATS_MEANS : 0) |
                      ((common::plot_vars || common::plot_covars) ? FHD_STATS_VARS : 0) |
                      (common::plot_mom3 ? FHD_STATS_MOM3 : 0) | (common::plot_mom4 ? FHD_STATS_MOM4 : 0) |
                      (cross ? FHD_STATS_CROSS : 0);
    if (!flags) return;
    fhd_stats st;
    std::memset(&st, 0, sizeof(st));
    st.cuMeans = consMean.fab();
    st.cuVars = consVar.fab();
    st.primMeans = primMean.fab();
    st.primVars = primVar.fab();
    st.coVars = coVar.fab();
    st.mom3 = mom3.fab();
    st.mom4 = mom4.fab();
    for (int d = 0; d < 3; ++d) {
        st.velMeans[d] = velMean[d].fab();
        st.velVars[d] = velVar[d].fab();
        st.cumomMeans[d] = cumomMean[d].fab();
        st.cumomVars[d] = cumomVar[d].fab();
    }
    if (cross) {
        const int want = (compressible::all_correl == 1 ? 5 : 1) * ncross;
        if (ncross != fhd_spatial_cross_ncross(common::nspecies) || spatialCross.nComp() != want ||
            spatialCross.nGrow() != 0)
            fail(where, FHD_ERR_BAD_ARG);
        require_device(spatialCross, where);
        st.spatialCross = spatialCross.dataPtr();
    }
    fhd_fab vl[3], mom[3];
    fabs_of(vel, vl);
    fabs_of(cumom, mom);
    check(fhd_stats_stag(context(), cons.fab(), prim_in.fab(), vl, mom, &st, steps, flags), where);
}

#define FHD_REF_STATS_LOWDIM_ARGS                                                                                \
    fhd::amrex_compat::MultiFab &cons, fhd::amrex_compat::MultiFab &consMean, fhd::amrex_compat::MultiFab &consVar, \
        fhd::amrex_compat::MultiFab &prim_in, fhd::amrex_compat::MultiFab &primMean,                              \
        fhd::amrex_compat::MultiFab &primVar, const std::array<fhd::amrex_compat::MultiFab, 3> &vel,              \
        std::array<fhd::amrex_compat::MultiFab, 3> &velMean, std::array<fhd::amrex_compat::MultiFab, 3> &velVar,  \
        const std::array<fhd::amrex_compat::MultiFab, 3> &cumom,                                                  \
        std::array<fhd::amrex_compat::MultiFab, 3> &cumomMean, std::array<fhd::amrex_compat::MultiFab, 3> &cumomVar, \
        fhd::amrex_compat::MultiFab &coVar, fhd::amrex_compat::MultiFab &mom3, fhd::amrex_compat::MultiFab &mom4,  \
        fhd::amrex_compat::MultiFab & /*theta*/, fhd::amrex_compat::MultiFab & /*thetaMean*/,                     \
        fhd::amrex_compat::MultiFab & /*thetaVar*/, fhd::amrex_compat::MultiFab & /*thetacoVar*/,                  \
        fhd::amrex_compat::MultiFab &spatialCross, const int ncross, const int steps,                             \
        const fhd::amrex_compat::Geometry & /*geom*/

inline void evaluateStatsStag1D(FHD_REF_STATS_LOWDIM_ARGS) {
    evaluateStatsStagLowDim(cons, consMean, consVar, prim_in, primMean, primVar, vel, velMean, velVar, cumom,
                            cumomMean, cumomVar, coVar, mom3, mom4, spatialCross, ncross, steps, "evaluateStatsStag1D");
}
inline void evaluateStatsStag2D(FHD_REF_STATS_LOWDIM_ARGS) {
    evaluateStatsStagLowDim(cons, consMean, consVar, prim_in, primMean, primVar, vel, velMean, velVar, cumom,
                            cumomMean, cumomVar, coVar, mom3, mom4, spatialCross, ncross, steps, "evaluateStatsStag2D");
}
#undef FHD_REF_STATS_LOWDIM_ARGS

// WriteSpatialCross1D (writePlotFileStag.cpp:551-563): spatialCross1D_<step, 9 digits>
// (five <s>_spatialCross1D_<step> files with compressible::all_correl) in the working
// directory, from the device MultiFab evaluateStatsStag1D updates.
inline void WriteSpatialCross1D(const fhd::amrex_compat::MultiFab& spatialCross, int step,
                                const fhd::amrex_compat::Geometry& /*geom*/, const int ncross) {
    using namespace fhd::ref;
    const fhd_params p = params_from_globals();
    const int want = (p.all_correl == 1 ? 5 : 1) * ncross;
    if (!p.do_1D || ncross != fhd_spatial_cross_ncross(p.nspecies) || spatialCross.nComp() != want ||
        spatialCross.nGrow() != 0)
        fail("WriteSpatialCross1D", FHD_ERR_BAD_ARG);
    check(fhd_write_spatial_cross(&p, "", step, spatialCross.dataPtr()), "WriteSpatialCross1D");
}

// WriteCheckPoint (Checkpoint.cpp:28-257): chk<step, 9 digits>/ in the working
// directory with the state, every defined statistics MultiFab and, with
// plot_cross, spatialCrossVec in the Header; a quasi-1-D / 2-D run also writes
// spatialCrossMF (Level_0/spatialCrossMF, whether or not plot_cross is set, as
// Checkpoint.cpp:251-256 does).  The surface-coverage and turbulence-forcing records
// are not written (neither exists on this path); the noise needs no generator state.
inline void WriteCheckPoint(int step, const fhd::amrex_compat::Real time, int statsCount,
                            const fhd::amrex_compat::Geometry& /*geom*/, const fhd::amrex_compat::MultiFab& cu,
                            const fhd::amrex_compat::MultiFab& cuMeans, const fhd::amrex_compat::MultiFab& cuVars,
                            const fhd::amrex_compat::MultiFab& prim, const fhd::amrex_compat::MultiFab& primMeans,
                            const fhd::amrex_compat::MultiFab& primVars,
                            const std::array<fhd::amrex_compat::MultiFab, 3>& cumom,
                            const std::array<fhd::amrex_compat::MultiFab, 3>& cumomMeans,
                            const std::array<fhd::amrex_compat::MultiFab, 3>& cumomVars,
                            const std::array<fhd::amrex_compat::MultiFab, 3>& vel,
                            const std::array<fhd::amrex_compat::MultiFab, 3>& velMeans,
                            const std::array<fhd::amrex_compat::MultiFab, 3>& velVars,
                            const fhd::amrex_compat::MultiFab& coVars, const fhd::amrex_compat::MultiFab& mom3,
                            const fhd::amrex_compat::MultiFab& mom4, const fhd::amrex_compat::MultiFab& /*surfcov*/,
                            const fhd::amrex_compat::MultiFab& /*surfcovMeans*/,
                            const fhd::amrex_compat::MultiFab& /*surfcovVars*/,
                            const fhd::amrex_compat::MultiFab& /*surfcovcoVars*/,
                            const fhd::amrex_compat::MultiFab& spatialCrossMF,
                            const fhd::amrex_compat::Vector<fhd::amrex_compat::Real>& spatialCrossVec,
                            int ncross, TurbForcingComp& /*turbforce*/) {
    using namespace fhd::ref;
    fhd_stats st;
    std::memset(&st, 0, sizeof(st));
    st.cuMeans = cuMeans.fab();
    st.cuVars = cuVars.fab();
    st.primMeans = primMeans.fab();
    st.primVars = primVars.fab();
    st.coVars = coVars.fab();
    st.mom3 = mom3.fab();
    st.mom4 = mom4.fab();
    for (int d = 0; d < 3; ++d) {
        st.velMeans[d] = velMeans[d].fab();
        st.velVars[d] = velVars[d].fab();
        st.cumomMeans[d] = cumomMeans[d].fab();
        st.cumomVars[d] = cumomVars[d].fab();
    }
    fhd_fab mom[3], vl[3];
    fabs_of(cumom, mom);
    fabs_of(vel, vl);
    const fhd_params p = params_from_globals();
    if (p.do_1D || p.do_2D) {
        if (ncross != fhd_spatial_cross_ncross(p.nspecies) ||
            spatialCrossMF.nComp() != (p.do_1D && p.all_correl == 1 ? 5 : 1) * ncross || spatialCrossMF.nGrow() != 0)
            fail("WriteCheckPoint", FHD_ERR_BAD_ARG);
        st.spatialCross = spatialCrossMF.dataPtr();
    } else if (common::plot_cross) {
        if (ncross != fhd_spatial_cross_ncross(p.nspecies) || spatialCrossVec.size() < (size_t)p.n_cells[0] * ncross)
            fail("WriteCheckPoint", FHD_ERR_BAD_ARG);
        st.spatialCross = const_cast<double*>(spatialCrossVec.data());
    }
    check(fhd_write_checkpoint(&p, "chk", step, time, statsCount, cu.fab(), mom, prim.fab(), vl, &st),
          "WriteCheckPoint");
}

// ReadCheckPoint (Checkpoint.cpp:259-575): defines every MultiFab with the
// reference's shapes on `domain` (device memory, 2 ghost cells for the state and
// the cell-centred means/variances, none for the others; mom3 / mom4 only with
// plot_mom3 / plot_mom4), reads chk<common::restart, 9 digits>/ into them and sets
// step to the saved step + 1, time and statsCount.  With plot_cross the Header's
// spatialCrossVec is read into spatialCrossVec (n_cells[0] * ncross entries); a
// quasi-1-D / 2-D run defines spatialCrossMF (ncross components, 5 * ncross with
// do_1D and all_correl; no ghosts) and reads it (Checkpoint.cpp:529-533).  With
// reset_stats the statistics, spatialCrossVec and spatialCrossMF are zeroed instead
// of read (Checkpoint.cpp:343-358, 498-519).
inline void ReadCheckPoint(int& step, fhd::amrex_compat::Real& time, int& statsCount,
                           fhd::amrex_compat::Geometry& /*geom*/, const fhd::amrex_compat::Box& domain,
                           fhd::amrex_compat::MultiFab& cu, fhd::amrex_compat::MultiFab& cuMeans,
                           fhd::amrex_compat::MultiFab& cuVars, fhd::amrex_compat::MultiFab& prim,
                           fhd::amrex_compat::MultiFab& primMeans, fhd::amrex_compat::MultiFab& primVars,
                           std::array<fhd::amrex_compat::MultiFab, 3>& cumom,
                           std::array<fhd::amrex_compat::MultiFab, 3>& cumomMeans,
                           std::array<fhd::amrex_compat::MultiFab, 3>& cumomVars,
                           std::array<fhd::amrex_compat::MultiFab, 3>& vel,
                           std::array<fhd::amrex_compat::MultiFab, 3>& velMeans,
                           std::array<fhd::amrex_compat::MultiFab, 3>& velVars,
                           fhd::amrex_compat::MultiFab& coVars, fhd::amrex_compat::MultiFab& mom3,
                           fhd::amrex_compat::MultiFab& mom4, fhd::amrex_compat::MultiFab& /*surfcov*/,
                           fhd::amrex_compat::MultiFab& /*surfcovMeans*/, fhd::amrex_compat::MultiFab& /*surfcovVars*/,
                           fhd::amrex_compat::MultiFab& /*surfcovcoVars*/,
                           fhd::amrex_compat::MultiFab& spatialCrossMF,
                           fhd::amrex_compat::Vector<fhd::amrex_compat::Real>& spatialCrossVec, int ncross,
                           TurbForcingComp& /*turbforce*/, fhd::amrex_compat::BoxArray& ba,
                           fhd::amrex_compat::DistributionMapping& /*dmap*/) {
    using namespace fhd::ref;
    using fhd::amrex_compat::convert;
    using fhd::amrex_compat::face_nodal;
    const int ns = common::nspecies, nvars = 5 + ns, nprim = 6 + 2 * ns, ngc = 2;
    ba.define(domain);
    cu.define(domain, nvars, ngc);
    cuMeans.define(domain, nvars, ngc);
    cuVars.define(domain, nvars, ngc);
    prim.define(domain, nprim, ngc);
    primMeans.define(domain, nprim + 3, ngc);
    primVars.define(domain, nprim + 5, ngc);
    for (int d = 0; d < 3; ++d) {
        const fhd::amrex_compat::Box fb = convert(domain, face_nodal(d));
        vel[d].define(fb, 1, ngc);
        cumom[d].define(fb, 1, ngc);
        velMeans[d].define(fb, 1, 0);
        cumomMeans[d].define(fb, 1, 0);
        velVars[d].define(fb, 1, 0);
        cumomVars[d].define(fb, 1, 0);
    }
    coVars.define(domain, 26, 0);
    if (common::plot_mom3) mom3.define(domain, nvars + 1, 0);
    if (common::plot_mom4) mom4.define(domain, nvars + 1, 0);
    fhd_stats st;
    std::memset(&st, 0, sizeof(st));
    st.cuMeans = cuMeans.fab();
    st.cuVars = cuVars.fab();
    st.primMeans = primMeans.fab();
    st.primVars = primVars.fab();
    st.coVars = coVars.fab();
    st.mom3 = mom3.fab();
    st.mom4 = mom4.fab();
    for (int d = 0; d < 3; ++d) {
        st.velMeans[d] = velMeans[d].fab();
        st.velVars[d] = velVars[d].fab();
        st.cumomMeans[d] = cumomMeans[d].fab();
        st.cumomVars[d] = cumomVars[d].fab();
    }
    fhd_fab mom[3], vl[3];
    fabs_of(cumom, mom);
    fabs_of(vel, vl);
    const fhd_params p = params_from_globals();
    const bool reset = common::reset_stats == 1;
    if (p.do_1D || p.do_2D) {
        if (ncross != fhd_spatial_cross_ncross(ns)) fail("ReadCheckPoint", FHD_ERR_BAD_ARG);
        spatialCrossMF.define(domain, (p.do_1D && p.all_correl == 1 ? 5 : 1) * ncross, 0);
        spatialCrossMF.setVal(0.0);
        if (!reset) st.spatialCross = spatialCrossMF.dataPtr();
    } else if (common::plot_cross) {
        if (ncross != fhd_spatial_cross_ncross(ns)) fail("ReadCheckPoint", FHD_ERR_BAD_ARG);
        spatialCrossVec.resize((size_t)common::n_cells[0] * ncross);
        if (!reset) st.spatialCross = spatialCrossVec.data();
    }
    double t = 0.0;
    check(fhd_read_checkpoint(&p, "chk", common::restart, &step, &t, &statsCount, cu.fab(), mom, prim.fab(), vl,
                              reset ? nullptr : &st),
          "ReadCheckPoint");
    time = t;
    if (reset) {
        for (fhd::amrex_compat::MultiFab* m : {&cuMeans, &cuVars, &primMeans, &primVars, &coVars})
            m->setVal(0.0);
        for (int d = 0; d < 3; ++d) {
            velMeans[d].setVal(0.0);
            velVars[d].setVal(0.0);
            cumomMeans[d].setVal(0.0);
            cumomVars[d].setVal(0.0);
        }
        if (common::plot_mom3) mom3.setVal(0.0);
        if (common::plot_mom4) mom4.setVal(0.0);
        if (common::plot_cross && !p.do_1D && !p.do_2D) spatialCrossVec.assign(spatialCrossVec.size(), 0.0);
    }
}

// MultiFabFillRandom (MultiFabFillRandom.cpp:5-31): N(0, variance) in one
// component, then OverrideSync and FillBoundary (which leaves every ghost,
// `ng` or not, the periodic image of a valid value on a periodic box).
inline void MultiFabFillRandom(fhd::amrex_compat::MultiFab& mf, const int& comp,
                               const fhd::amrex_compat::Real& variance, const fhd::amrex_compat::Geometry& geom,
                               const int& /*ng*/ = 0) {
    MultiFabFillRandomNormal(mf, comp, 1, 0.0, variance, geom, true, true);
}

#endif
