// fhd_host.h — host-side launch descriptors shared by the C ABI and the kernel
// translation units (fhd_exact.cu: FP64 in the reference's operation order,
// built with -fmad=false; fhd_mixed.cu: FP32 fluxes/coefficients).
#pragma once
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/fhd_capi.h"
#include "fhd_device.cuh"

namespace fhd {

enum NoiseMode { NM_OFF = 0, NM_W = 1, NM_AB = 2, NM_PHILOX = 3 };

struct NoiseFabs {
    fhd_fab fa[3], fb[3];   // faces (W or A/B)
    fhd_fab ea[3], eb[3];   // xy, xz, yz edges
    fhd_fab ca[3], cb[3];   // centres
};

// a box with a physical wall in some direction (both sides of a periodic
// direction have bc_vel -1)
inline bool has_walls(const fhd_params& p) {
    if (!p.walls) return false;
    for (int d = 0; d < 3; ++d)
        if (p.bc_vel_lo[d] != -1 || p.bc_vel_hi[d] != -1) return true;
    return false;
}

// runs that take the reference-ordered pipeline: walls, or a quasi-1-D / 2-D run
inline bool reference_order(const fhd_params& p) { return has_walls(p) || p.do_1D || p.do_2D; }

// Kernel parameters of a run (after GetHcGas): cell widths, the transport model's
// cell-independent constants in the reference's own operation order
// (compressible_functions.H:1180-1222), the Philox key and the reciprocals of the
// constant divisors.
inline DevParams dev_params(const fhd_params& p, double dt, uint64_t step) {
    DevParams P;
    std::memset(&P, 0, sizeof(P));
    P.ns = p.nspecies;
    P.nvars = 5 + p.nspecies;
    P.nprim = 6 + 2 * p.nspecies;
    for (int d = 0; d < 3; ++d) {
        P.n[d] = p.n_cells[d];
        P.dx[d] = (p.prob_hi[d] - p.prob_lo[d]) / p.n_cells[d];
        P.grav[d] = p.grav[d];
    }
    P.dt = dt;
    P.volinv = 1. / (P.dx[0] * P.dx[1] * P.dx[2]);
    P.dtinv = 1. / dt;
    P.k_B = p.k_B;
    P.Runiv = p.Runiv;
    P.zeta_ratio = p.zeta_ratio;
    P.visc_type = p.visc_type;
    P.advection_type = p.advection_type;
    P.stoch = p.stoch_stress_form;
    const double AKL = 1.0, BKL = 1.0, CKL = 1.0;
    for (int i = 0; i < MAXS; ++i) {
        P.molmass[i] = p.molmass[i];
        P.hcv[i] = p.hcv[i];
        P.hcp[i] = p.hcp[i];
        P.e0[i] = p.e0[i];
        P.mm[i] = p.molmass[i] * (p.k_B / p.Runiv);
        P.mmkB[i] = P.mm[i] * p.k_B;
    }
    for (int i = 0; i < MAXS; ++i)
        for (int j = 0; j < MAXS; ++j) {
            P.diam[i][j] = 0.5 * (p.diameter[i] + p.diameter[j]);
            P.mu[i][j] = P.mm[i] * P.mm[j] / (P.mm[i] + P.mm[j]);
            P.msum[i][j] = P.mm[i] + P.mm[j];
            P.vfac[i][j] = 1.0 + 0.6 * P.mm[j] / P.mm[i] * AKL;
            P.kfac[i][j] = 7.5 * P.mm[i] / P.mm[j] + 6.25 * P.mm[j] / P.mm[i] - 3.0 * P.mm[j] / P.mm[i] * BKL + 4.0 * AKL;
        }
    for (int i = 0; i < MAXS; ++i) P.eta1pre[i] = 5.0 / (16.0 * P.diam[i][i] * P.diam[i][i]);
    P.koff = 55.0 / 4.0 - 3.0 * BKL - 4.0 * AKL;
    P.voff = 0.6 * AKL - 1.0;
    P.cfac = 6.0 * CKL - 5.0;
    P.sqrt2 = sqrt(2.0);
    P.sqrt3 = sqrt(3.0);
    P.dim = p.do_1D ? 1 : (p.do_2D ? 2 : 3);
    P.fac2d = (3.0 + sqrt(3.0)) / 2.0;
    P.csd0 = p.do_1D ? 1.0 : sqrt(2.0);
    P.transport_type = p.transport_type;
    P.vwt = nullptr;
    P.walls = p.walls ? 1 : 0;
    for (int d = 0; d < 3; ++d) {
        P.periodic[d] = !P.walls || (p.bc_vel_lo[d] == -1 && p.bc_vel_hi[d] == -1);
        const int* lo[3] = {p.bc_vel_lo, p.bc_mass_lo, p.bc_therm_lo};
        const int* hi[3] = {p.bc_vel_hi, p.bc_mass_hi, p.bc_therm_hi};
        int* dst[3] = {P.bc_vel, P.bc_mass, P.bc_therm};
        for (int q = 0; q < 3; ++q) {
            dst[q][2 * d] = P.periodic[d] ? -1 : lo[q][d];
            dst[q][2 * d + 1] = P.periodic[d] ? -1 : hi[q][d];
        }
        P.hdx[d] = 0.5 * P.dx[d];
    }
    P.key0 = (uint32_t)p.seed;
    P.key1 = (uint32_t)(p.seed >> 32);
    P.step = step;
    P.step_ptr = nullptr;
    // reciprocals of the constant divisors for div_rcp (fhd_div.h)
    bool in_window = true;
    auto rcp = [&](double b) {
        in_window = in_window && div_divisor_ok(b);
        return 1.0 / b;
    };
    for (int d = 0; d < 3; ++d) P.rdx[d] = rcp(P.dx[d]);
    for (int i = 0; i < P.ns; ++i) {
        P.rmolmass[i] = rcp(P.molmass[i]);
        P.rmm[i] = rcp(P.mm[i]);
        for (int j = 0; j < P.ns; ++j) {
            P.rmu[i][j] = rcp(P.mu[i][j]);
            P.rmsum[i][j] = rcp(P.msum[i][j]);
        }
    }
    P.rRdt = rcp(P.Runiv * P.dt);
    P.rpi = rcp(3.1415926535897932);
    for (int d = 0; d < 3; ++d) P.rhdx[d] = rcp(P.hdx[d]);
    P.r3 = rcp(3.0);
    P.div_lo = kDivAlo;
    P.div_span = in_window ? kDivAspan : 0u;
    return P;
}

// Everything one stage (or one flux-operator call) reads and writes.
struct StageCall {
    DevParams P;
    int mode;               // NoiseMode
    double w;               // stage weight of B
    int stage;              // 1..3 (0: flux operator only)
    fhd_fab cons_s, mom_s[3];   // stage input U^s
    fhd_fab cons0, mom0[3];     // U^0
    fhd_fab cons_o, mom_o[3];   // U^{s+1}
    fhd_fab pr;             // T at comp pT, p, Y, X follow
    int pT;
    fhd_fab vel[3];
    fhd_fab eta, zeta, kappa, chi, D;   // coefficient fabs (f64, or f32 when mixed)
    fhd_fab src;            // data == NULL: no source
    NoiseFabs nz;
    fhd_fab ff[3], ef[6], cf[3];        // flux outputs of the operator path
    fhd_fab ct, et, sff[3];             // stage scratch: cell/edge stresses, face fluxes
    fhd_fab smc, sme;                   // stage scratch: total centre / edge momentum fluxes
    int* status;
    cudaStream_t stream;
    int tile;               // tile-shape index of k_stage (autotuned)
};

// exact (FP64) translation unit
int exact_cellprep(const StageCall& c);
int exact_stage_part(const StageCall& c, int part);  // 0 stresses, 1 face fluxes, 2 update, 3 fused (all three)
int exact_aux_fluxes(const StageCall& c);
int exact_transport(const DevParams& P, fhd_fab prim, fhd_fab eta, fhd_fab zeta, fhd_fab kappa, fhd_fab chi,
                    fhd_fab D, int* status, cudaStream_t s);
int exact_convert(const DevParams& P, fhd_fab prim, const fhd_fab vel[3], fhd_fab cons, const fhd_fab mom[3],
                  int* status, cudaStream_t s);
// boxes with physical walls (FP64): the stage parts (0 stresses, 1 face fluxes, 2
// update), BCMassTempPress + BCRhoRhoE on prim / cons, BCMomNormal + BCMomTrans on
// the face momenta and velocities
int exact_walls_part(const StageCall& c, int part);
int exact_bc_prim(const DevParams& P, const WallParams& W, fhd_fab prim, fhd_fab cons, const fhd_fab mom[3],
                  cudaStream_t s);
int bc_mom(const DevParams& P, const fhd_fab mom[3], const fhd_fab vel[3], cudaStream_t s);
// the particle reservoir's buffers: faceflux_res[d] (nvars comps) and cumom_res[d] in
// the reference's layout (faces of direction d, no ghost cells), particle masses
struct ResBuffers {
    void* base;
    size_t bytes;
    double* f[3];
    double* m[3];
    int sy[3], sz[3], sn[3];
    double mass[MAXS];
};
int exact_reservoir(const DevParams& P, const ResBuffers& r, const fhd_fab& cons, const fhd_fab& prim,
                    const fhd_fab vel[3], double dt, int stage, double* rec, int rec_cap, int* status,
                    cudaStream_t s);
// ff: three face-flux fabs with the conserved comps 0 / 4 / 5.. at fc_rho / fc_rhoE / fc_Y;
// ef: six edge-flux fabs, or one fab of six comps from ef_comp_base (-1: six fabs)
int exact_res_reset(const DevParams& P, const ResBuffers& r, const fhd_fab* ff, int fc_rho, int fc_rhoE, int fc_Y,
                    const fhd_fab* ef, int ef_comp_base, cudaStream_t s);
int exact_res_mom(const DevParams& P, const ResBuffers& r, const fhd_fab mom[3], cudaStream_t s);
// the reference's boundary passes one by one (boxes with reservoirs): setBCStag
// (rre) or the passes before the conversion
int exact_bc_seq(const DevParams& P, const WallParams& W, fhd_fab prim, fhd_fab cons, const fhd_fab mom[3],
                 const fhd_fab vel[3], bool rre, cudaStream_t s);
// mixed translation unit (coefficient fabs are f32)
int mixed_cellprep(const StageCall& c);
int mixed_stage_part(const StageCall& c, int part);

// utilities (exact TU)
struct GhostReq {
    fhd_fab f;
    int c0, nc;
};
// periodic: the periodic directions (nullptr: all); mode 0 FillBoundary, 1 noise
// fields with wall ghosts of their own (k_ghosts)
int fill_ghosts(const GhostReq* reqs, int n, const int ncell[3], cudaStream_t s, const int* periodic = nullptr,
                int mode = 0);
// chemistry source (fhd_chem.cu): writes species comps 5.. of `source` at the valid
// cells from `prim`; na/nb: the A/B (mode CN_AB) or W (CN_W) noise fabs
struct ChemParams;
// plotfiles (fhd_plot.cu)
int plot_pack(const fhd_params& prm, int flags, fhd_fab out, const fhd_fab& cu, const fhd_fab* cumom,
              const fhd_fab& prim, const fhd_fab* vel, const fhd_fab& eta, const fhd_fab& kappa, const fhd_fab& zeta,
              const fhd_stats* st, cudaStream_t s);
int plot_names(const fhd_params& prm, int flags, std::vector<std::string>& names);
int plot_write(const fhd_params& prm, const char* dir, const double* host, const std::vector<std::string>& names,
               double time, int step);
int chem_launch(const DevParams& P, const ChemParams& C, const fhd_fab& prim, const fhd_fab& source,
                const fhd_fab* na, const fhd_fab* nb, int mode, double w, cudaStream_t s);
// running statistics (fhd_stats.cu, exact TU)
// stars: the x* of FHD_STATS_CROSS (one in 3-D; one or five in a quasi-1-D run);
// lines: device scratch of stats_line_doubles(ns, n_cells[0]) doubles (3-D FHD_STATS_CROSS only)
int exact_stats(const DevParams& P, const fhd_fab& cu, const fhd_fab& prim, const fhd_fab vel[3], const fhd_fab mom[3],
                const fhd_stats& st, int64_t steps, int flags, const int* stars, int nstars, double* lines,
                cudaStream_t s);
int64_t stats_line_doubles(int ns, int nx);
int override_sync(const fhd_fab& f, const int ncell[3], cudaStream_t s, const int* periodic = nullptr);
// wall_ghosts: also fill the first ghost layer of the wall directions (centre noise)
int noise_fill(const DevParams& P, const fhd_fab& f, int c0, int nc, double mean, double sd, uint32_t fid0, int use_b,
               cudaStream_t s, int wall_ghosts = 0);
int init_uniform(const fhd_fab& cu, int ns, double rho0, double rhoE, const double* rhoY, cudaStream_t s);

// batched launches (kinds: 0 cellprep, 1 stresses, 2-4 faces, 5 update, 6 conversion)
size_t batch_args_size(int ns, bool mixed, int kind, int mode);
void batch_pack(int ns, bool mixed, int kind, int mode, const StageCall& c, void* dst);
// tile: register cap of the face kinds (batch_face_tiles() choices; -1 the default)
int batch_launch(int ns, bool mixed, int kind, int mode, int tile, const void* dargs, const int* dbpref, int nmem,
                 int nblocks, cudaStream_t s);
int batch_face_tiles();
// the persistent batched step (k_batch_persist): one launch per RK3 step
// tile: register cap as the batch face tiles (-1 the default for the species count)
int batch_persist(int ns, bool mixed, int mode, int tile, const PersistArgs& a, cudaStream_t s);
int batch_face_min_blocks(int tile);
struct GhostFabDesc;  // opaque to the host code
int ghost_desc_size();
int64_t ghost_pack(const fhd_fab& f, int c0, int nc, const int ncell[3], void* dst);  // returns work items
int ghost_launch_b(const void* dfabs, const int* dbpref, int nfab, int nblocks, cudaStream_t s);
int steps_inc(uint64_t* steps, int n, cudaStream_t s);
int steps_set(uint64_t* step, uint64_t v, cudaStream_t s);

int num_tiles();
const char* tile_name(int t);
bool tile_fused(int t);  // the tile selects the fused stage kernel (stage part 3)

}  // namespace fhd
