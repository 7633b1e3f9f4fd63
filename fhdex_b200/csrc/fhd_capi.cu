// fhd_capi.cu — the C ABI declared in include/fhd_capi.h: context, argument
// validation, the fused RK3 step and the drop-in operators.  Host code only; the
// kernels live in fhd_kern_ns.cu / fhd_exact.cu.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "fhd_host.h"
#include "fhd_chem.cuh"
#include "fhd_transport_alt.cuh"
#include "philox.cuh"

using namespace fhd;

struct fhd_ctx {
    fhd_params prm;
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    int* d_status = nullptr;
    // stage scratch: cup, cup2 (cells, nvars comps, 2 ghosts) and their face momenta
    double* scratch = nullptr;
    size_t scratch_bytes = 0;
    fhd_fab cup{}, cup2{}, cupm[3]{}, cup2m[3]{};
    // coefficient scratch (f64 for the exact path when the caller passes none; f32 mixed)
    void* coef = nullptr;
    size_t coef_bytes = 0;
    int coef_dtype = -1;
    fhd_fab ceta{}, czeta{}, ckappa{}, cchi{}, cD{};
    fhd_fab ct{}, et{};          // stage stresses (coefficient precision)
    fhd_fab sff[3]{};            // stage conservative face fluxes (f64)
    fhd_fab smc{}, sme{};        // stage total centre / edge momentum fluxes (f64)
    fhd_fab csrc{};              // zeroed source of a step given none (chemistry on)
    int tile = 0;
    // physical boundaries: the periodic directions and the walls' values
    int per[3] = {1, 1, 1};
    bool walls = false;
    bool refpipe = false;        // walls or a quasi-1-D / 2-D run: the reference-ordered pipeline
    bool reservoir = false;      // a side with bc_mass 3 or 4: the boundary passes run one by one
    bool res4 = false;           // a particle reservoir side (bc_mass 4)
    ResBuffers res{};
    double* res_rec = nullptr;   // test hook: the particle reservoir's draws
    int res_cap = 0;
    WallParams wall{};
    // the Valk/Waldmann model's pair constants (transport_type 2), device memory
    VWTable* vwt = nullptr;
    // x-line scratch of the spatial cross-correlations (fhd_stats_stag, FHD_STATS_CROSS)
    double* lines = nullptr;
    size_t lines_bytes = 0;
    // device mirrors for the host-buffer step
    double* hbuf = nullptr;
    size_t hbuf_bytes = 0;
    // graph replay of whole steps (fhd_rk3_steps_stag): the captured step, the device
    // word its noise reads the step number from, and what the capture was made for
    cudaGraph_t sgraph = nullptr;
    cudaGraphExec_t sgexec = nullptr;
    uint64_t* d_step = nullptr;
    std::vector<uint64_t> skey;
    // CUDA-event timing per kernel kind
    bool prof = false;
    struct Ev { cudaEvent_t a, b; int kind; };
    std::vector<Ev> evs;
    size_t nev = 0;
};

namespace {

const int NGC = 2;

int64_t fab_points(const fhd_fab& f) {
    int64_t n = 1;
    for (int d = 0; d < 3; ++d) n *= (int64_t)(f.hi[d] - f.lo[d] + 1);
    return n;
}

fhd_fab make_fab(void* data, const int n[3], const int nodal[3], int ng, int nc, int dtype) {
    fhd_fab f;
    f.data = data;
    for (int d = 0; d < 3; ++d) {
        f.lo[d] = -ng;
        f.hi[d] = n[d] - 1 + nodal[d] + ng;
        f.nodal[d] = nodal[d];
    }
    f.ncomp = nc;
    f.dtype = dtype;
    return f;
}

const int CELLN[3] = {0, 0, 0};
const int FACEN[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
const int EDGEN[3][3] = {{1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
const int EFLUXN[6][3] = {{1, 1, 0}, {1, 0, 1}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1}, {0, 1, 1}};

// A fab must be a one-box MultiFab of the context's domain with the given
// centring, a uniform ghost width >= min_ng and >= min_nc components.
bool fab_ok(const fhd_ctx* c, const fhd_fab& f, const int nodal[3], int min_ng, int min_nc, int dtype,
            int exact_ng = -1) {
    if (!f.data || f.dtype != dtype || f.ncomp < min_nc) return false;
    if (fab_points(f) * f.ncomp >= ((int64_t)1 << 31)) return false;  // kernels index with 32 bits
    const int g = -f.lo[0];
    if (g < min_ng || (exact_ng >= 0 && g != exact_ng)) return false;
    for (int d = 0; d < 3; ++d) {
        if (f.lo[d] != -g || f.nodal[d] != nodal[d]) return false;
        if (f.hi[d] != c->prm.n_cells[d] - 1 + nodal[d] + g) return false;
    }
    return true;
}

DevParams make_dev(const fhd_ctx* c, double dt, uint64_t step) {
    DevParams P = dev_params(c->prm, dt, step);
    P.vwt = c->vwt;
    return P;
}

// IdealMixtureTransportVW's cell-independent parts (compressible_functions.H:1047-1121)
// and the powers ViscLin and LambdaLin take of the molecular masses, by the reference's
// own expressions (the host's pow, as the reference's CPU build has it)
void vw_table(const fhd_params& p, VWTable& t) {
    std::memset(&t, 0, sizeof(t));
    const double pi = 3.1415926535897932, k_B = p.k_B;
    const int ns = p.nspecies;
    double m[MAXS];
    for (int n = 0; n < ns; ++n) m[n] = p.molmass[n] * (k_B / p.Runiv);
    const double Fijstar = -27. / 5.;
    for (int i = 0; i < ns; ++i) {
        t.pm2[i] = std::pow(m[i], 2.);
        for (int j = 0; j < ns; ++j) {
            const int q = i * MAXS + j;
            const double diamat = 0.5 * (p.diameter[i] + p.diameter[j]);
            const double mu = m[i] * m[j] / (m[i] + m[j]);
            const double Fij = (6.0 * m[i] * m[i] + 13.0 / 5.0 * m[j] * m[j] + 16.0 / 5.0 * m[i] * m[j]) /
                               (std::pow(m[i] + m[j], 2.));
            const double sigma11bar = std::sqrt(k_B / (2.0 * pi * mu)) * pi * std::pow(diamat, 2.);
            t.alphabar[q] = 8.0 / (3.0 * k_B) * mu * mu * (-.5 * sigma11bar);
            t.DbinC[q] = 3.0 / 16.0 * std::sqrt(2.0 * pi * std::pow(k_B, 3.) * (m[i] + m[j]) / m[i] / m[j]) /
                         (pi * std::pow(diamat, 2.));
            t.omegaC[q] = std::sqrt(pi * k_B / (2.0 * mu)) * std::pow(diamat, 2.);
            t.a1C[q] = 5.0 / (k_B)*m[i] * m[j] / (m[i] + m[j]) * Fij * sigma11bar;
            t.a2C[q] = 5.0 / (k_B)*m[i] * m[j] * m[i] * m[j] / (std::pow(m[i] + m[j], 3.)) * Fijstar * sigma11bar;
            t.ps2[q] = std::pow(m[i] + m[j], 2.);
            t.ps3[q] = std::pow(m[i] + m[j], 3.);
        }
    }
}

// With walls the state has the reference's ghost width exactly (the conditions
// fill every ghost layer, as the stage buffers have NGC of them)
bool walls_ghosts_ok(const fhd_fab& cu, const fhd_fab* mom, const fhd_fab& prim, const fhd_fab* vel) {
    if (-cu.lo[0] != NGC || -prim.lo[0] != NGC) return false;
    for (int d = 0; d < 3; ++d)
        if (-mom[d].lo[0] != NGC || -vel[d].lo[0] != NGC) return false;
    return true;
}

int ensure_scratch(fhd_ctx* c) {
    const int* n = c->prm.n_cells;
    const int nvars = 5 + c->prm.nspecies;
    fhd_fab tmpl = make_fab(nullptr, n, CELLN, NGC, nvars, FHD_F64);
    const int64_t cellpts = fab_points(tmpl);
    int64_t fpts[3];
    for (int d = 0; d < 3; ++d) fpts[d] = fab_points(make_fab(nullptr, n, FACEN[d], NGC, 1, FHD_F64));
    const int ns = c->prm.nspecies;
    const int allnod[3] = {1, 1, 1};
    const int64_t npts = fab_points(make_fab(nullptr, n, allnod, 0, 1, FHD_F64));  // [0, n]^3
    const int64_t c1pts = fab_points(make_fab(nullptr, n, CELLN, 1, 1, FHD_F64));  // cells grown by 1
    const int64_t vpts = (int64_t)n[0] * n[1] * n[2];
    const int64_t srcpts = c->prm.nreaction > 0 ? vpts * nvars : 0;  // chemistry's source when the caller has none
    const size_t need = (size_t)(2 * cellpts * nvars + 2 * (fpts[0] + fpts[1] + fpts[2]) + 3 * npts * (2 + ns) +
                                 3 * c1pts + 6 * npts + srcpts) * sizeof(double);
    if (c->scratch && c->scratch_bytes >= need) return FHD_OK;
    if (c->scratch) cudaFree(c->scratch);
    c->scratch = nullptr;
    if (cudaMalloc(&c->scratch, need) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_OOM; }
    // zero once so that components never written (1..3 of cup/cup2) are defined
    if (cudaMemsetAsync(c->scratch, 0, need, c->stream) != cudaSuccess) return FHD_ERR_CUDA;
    c->scratch_bytes = need;
    double* p = c->scratch;
    c->cup = make_fab(p, n, CELLN, NGC, nvars, FHD_F64); p += cellpts * nvars;
    c->cup2 = make_fab(p, n, CELLN, NGC, nvars, FHD_F64); p += cellpts * nvars;
    for (int d = 0; d < 3; ++d) { c->cupm[d] = make_fab(p, n, FACEN[d], NGC, 1, FHD_F64); p += fpts[d]; }
    for (int d = 0; d < 3; ++d) { c->cup2m[d] = make_fab(p, n, FACEN[d], NGC, 1, FHD_F64); p += fpts[d]; }
    // face fluxes on [0, n]^3 (lo = 0, hi = n: every face box fits)
    for (int d = 0; d < 3; ++d) {
        c->sff[d] = make_fab(p, n, allnod, 0, 2 + ns, FHD_F64);
        p += npts * (2 + ns);
    }
    c->smc = make_fab(p, n, CELLN, 1, 3, FHD_F64); p += c1pts * 3;
    c->sme = make_fab(p, n, allnod, 0, 6, FHD_F64); p += npts * 6;
    c->csrc = srcpts ? make_fab(p, n, CELLN, 0, nvars, FHD_F64) : fhd_fab{};
    return FHD_OK;
}

// the particle reservoir's faceflux_res / cumom_res (reference layout: the faces of
// each direction, no ghosts; nvars comps / one comp)
int ensure_res(fhd_ctx* c) {
    if (!c->res4 || c->res.base) return FHD_OK;
    const int* n = c->prm.n_cells;
    const int nvars = 5 + c->prm.nspecies;
    size_t tot = 0;
    int64_t pts[3];
    for (int d = 0; d < 3; ++d) {
        c->res.sy[d] = n[0] + (d == 0);
        c->res.sz[d] = c->res.sy[d] * (n[1] + (d == 1));
        c->res.sn[d] = c->res.sz[d] * (n[2] + (d == 2));
        pts[d] = c->res.sn[d];
        tot += (size_t)pts[d] * (nvars + 1);
    }
    void* b = nullptr;
    if (cudaMalloc(&b, tot * sizeof(double)) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_OOM; }
    c->res.base = b;
    c->res.bytes = tot * sizeof(double);
    double* q = static_cast<double*>(b);
    for (int d = 0; d < 3; ++d) { c->res.f[d] = q; q += pts[d] * nvars; }
    for (int d = 0; d < 3; ++d) { c->res.m[d] = q; q += pts[d]; }
    // particle masses molmass / avogadro (reservoirStag.cpp:24-27)
    const double navo = c->prm.avogadro > 0 ? c->prm.avogadro : c->prm.Runiv / c->prm.k_B;
    for (int i = 0; i < MAXS; ++i) c->res.mass[i] = i < c->prm.nspecies ? c->prm.molmass[i] / navo : 0.0;
    return FHD_OK;
}

int ensure_coef(fhd_ctx* c, int dtype) {
    const int* n = c->prm.n_cells;
    const int ns = c->prm.nspecies;
    const int ncomp = 3 + ns + ns * ns;
    const int64_t pts = fab_points(make_fab(nullptr, n, CELLN, NGC, 1, dtype));
    const int allnod[3] = {1, 1, 1};
    const int64_t ctpts = fab_points(make_fab(nullptr, n, CELLN, 1, 1, dtype));
    const int64_t etpts = fab_points(make_fab(nullptr, n, allnod, 0, 1, dtype));
    const size_t es = dtype == FHD_F64 ? 8 : 4;
    const size_t need = ((size_t)pts * ncomp + 6 * (size_t)(ctpts + etpts)) * es;
    if (c->coef && c->coef_bytes >= need && c->coef_dtype == dtype) return FHD_OK;
    if (c->coef) cudaFree(c->coef);
    c->coef = nullptr;
    if (cudaMalloc(&c->coef, need) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_OOM; }
    c->coef_bytes = need;
    c->coef_dtype = dtype;
    char* p = static_cast<char*>(c->coef);
    c->ceta = make_fab(p, n, CELLN, NGC, 1, dtype); p += pts * es;
    c->czeta = make_fab(p, n, CELLN, NGC, 1, dtype); p += pts * es;
    c->ckappa = make_fab(p, n, CELLN, NGC, 1, dtype); p += pts * es;
    c->cchi = make_fab(p, n, CELLN, NGC, ns, dtype); p += pts * ns * es;
    c->cD = make_fab(p, n, CELLN, NGC, ns * ns, dtype); p += pts * ns * ns * es;
    c->ct = make_fab(p, n, CELLN, 1, 6, dtype); p += ctpts * 6 * es;
    c->et = make_fab(p, n, allnod, 0, 6, dtype);
    return FHD_OK;
}

// brackets one launch with events when profiling is on
struct ProfScope {
    fhd_ctx* c;
    fhd_ctx::Ev* ev = nullptr;
    ProfScope(fhd_ctx* c_, int kind) : c(c_) {
        if (!c->prof) return;
        if (c->nev == c->evs.size()) {
            fhd_ctx::Ev e;
            cudaEventCreate(&e.a);
            cudaEventCreate(&e.b);
            c->evs.push_back(e);
        }
        ev = &c->evs[c->nev++];
        ev->kind = kind;
        cudaEventRecord(ev->a, c->stream);
    }
    ~ProfScope() {
        if (ev) cudaEventRecord(ev->b, c->stream);
    }
};

int sync_rc(cudaError_t e) {
    if (e == cudaSuccess) return FHD_OK;
    cudaGetLastError();
    return FHD_ERR_CUDA;
}

// the reaction noises of an injected step: required when the step's chemistry
// draws them (nreaction > 0 and reaction_type 1)
bool chem_noise_needed(const fhd_ctx* c) { return c->prm.nreaction > 0 && c->prm.reaction_type == 1; }
bool chem_noise_ok(const fhd_ctx* c, const fhd_noise* nz) {
    for (int s = 0; s < 2; ++s)
        if (!fab_ok(c, nz->chem[s], CELLN, 0, c->prm.nreaction, FHD_F64)) return false;
    return true;
}

bool noise_ok(const fhd_ctx* c, const fhd_noise* nz) {
    const int ns = c->prm.nspecies;
    for (int s = 0; s < 2; ++s)
        for (int d = 0; d < 3; ++d) {
            if (!fab_ok(c, nz->face[s][d], FACEN[d], 0, ns + 1, FHD_F64)) return false;
            if (!fab_ok(c, nz->edge[s][d], EDGEN[d], 0, 1, FHD_F64)) return false;
            if (!fab_ok(c, nz->cen[s][d], CELLN, 1, 1, FHD_F64)) return false;
        }
    return true;
}

void set_noise(StageCall& sc, const fhd_noise* nz, bool W) {
    for (int d = 0; d < 3; ++d) {
        sc.nz.fa[d] = nz->face[0][d];
        sc.nz.fb[d] = W ? nz->face[0][d] : nz->face[1][d];
        sc.nz.ea[d] = nz->edge[0][d];
        sc.nz.eb[d] = W ? nz->edge[0][d] : nz->edge[1][d];
        sc.nz.ca[d] = nz->cen[0][d];
        sc.nz.cb[d] = W ? nz->cen[0][d] : nz->cen[1][d];
    }
}

}  // namespace

extern "C" {

const char* fhd_strerror(int code) {
    switch (code) {
        case FHD_OK: return "ok";
        case FHD_ERR_BAD_ARG: return "bad argument (shape, dtype or parameter)";
        case FHD_ERR_MASSFRAC: return "mass fraction outside (0,1) (reference: amrex::Abort in calculateTransportCoeffs)";
        case FHD_ERR_NONFINITE: return "non-finite temperature or pressure";
        case FHD_ERR_OOM: return "device allocation failed";
        case FHD_ERR_TIMEOUT: return "bounded device wait timed out";
        case FHD_ERR_CUDA: return "CUDA runtime error";
        case FHD_ERR_UNSUPPORTED: return "option outside the implemented scope";
        case FHD_ERR_TOO_LARGE: return "box too large for the 16 MiB static scratch of fhd_rk3_step_stag_noalloc";
        case FHD_ERR_SINGULAR: return "singular Valk/Waldmann transport system (reference: amrex::Abort in Decomp)";
        case FHD_ERR_IO: return "file I/O failed (directory, open, write, read or close)";
        default: return "unknown error";
    }
}

// Wall settings (boundaryStag.cpp SetupBCStag / SetupCWallStag): a direction is
// periodic when both sides have bc_vel -1; otherwise both are walls with slip or
// no-slip velocity, adiabatic or isothermal temperature and impermeable or
// concentration mass conditions.  The concentration walls' Y and X follow from
// whichever of the two sums to 1 (GetMassfrac / GetMolfrac,
// compressible_functions.H:139-167).  Reservoirs (bc_mass >= 3) are not handled.
int setup_walls(const fhd_params& p, int per[3], WallParams& W) {
    std::memset(&W, 0, sizeof(W));
    const int ns = p.nspecies;
    for (int d = 0; d < 3; ++d) {
        per[d] = 1;
        if (!p.walls) continue;
        const bool plo = p.bc_vel_lo[d] == -1, phi = p.bc_vel_hi[d] == -1;
        if (plo && phi) continue;
        if (plo != phi) return FHD_ERR_BAD_ARG;
        per[d] = 0;
        if (p.n_cells[d] < NGC) return FHD_ERR_BAD_ARG;
        for (int h = 0; h < 2; ++h) {
            const int s = 2 * d + h;
            const int v = h ? p.bc_vel_hi[d] : p.bc_vel_lo[d];
            const int m = h ? p.bc_mass_hi[d] : p.bc_mass_lo[d];
            const int t = h ? p.bc_therm_hi[d] : p.bc_therm_lo[d];
            if (m >= 5) return FHD_ERR_UNSUPPORTED;
            if ((v != 1 && v != 2) || (m < 1 || m > 4) || (t != 1 && t != 2)) return FHD_ERR_BAD_ARG;
            W.t[s] = h ? p.t_hi[d] : p.t_lo[d];
            W.p[s] = h ? p.p_hi[d] : p.p_lo[d];
            W.rho[s] = h ? p.rho_hi[d] : p.rho_lo[d];
            if (t == 2 && m < 3 && !(W.t[s] > 0)) return FHD_ERR_BAD_ARG;
            const double* Yk = h ? p.bc_Yk_hi[d] : p.bc_Yk_lo[d];
            const double* Xk = h ? p.bc_Xk_hi[d] : p.bc_Xk_lo[d];
            for (int n = 0; n < ns; ++n) {
                W.Yk[s][n] = Yk[n];
                W.Xk[s][n] = Xk[n];
            }
            if (m == 1) continue;
            double sumx = 0., sumy = 0.;
            for (int n = 0; n < ns; ++n) {
                sumx = sumx + Xk[n];
                sumy = sumy + Yk[n];
            }
            if (std::fabs(sumx - 1) < 1.e-10) {
                double molmix = 0.;
                for (int n = 0; n < ns; ++n) molmix += W.Xk[s][n] * p.molmass[n];
                for (int n = 0; n < ns; ++n) W.Yk[s][n] = W.Xk[s][n] * p.molmass[n] / molmix;
            } else if (std::fabs(sumy - 1) < 1.e-10) {
                double molmix = 0.;
                for (int n = 0; n < ns; ++n) molmix += W.Yk[s][n] / p.molmass[n];
                molmix = 1. / molmix;
                for (int n = 0; n < ns; ++n) W.Xk[s][n] = W.Yk[s][n] * molmix / p.molmass[n];
            } else {
                return FHD_ERR_BAD_ARG;
            }
            if (m < 3) continue;
            // reservoir state (boundaryStag.cpp:39-60): the pressure defaults to the
            // initial state's (GetPressureGas of rhobar, rho0, T_init); then the
            // density from p, t and Y (GetDensity), or, when a density is given and
            // no temperature, the temperature from p and rho
            if (W.p[s] <= 0.0) {
                double molmix = 0.;
                for (int n = 0; n < ns; ++n) molmix += p.rhobar[n] / p.molmass[n];
                molmix = 1. / molmix;
                W.p[s] = p.rho0 * (p.Runiv / molmix) * p.T_init;
            }
            if (W.rho[s] <= 0.0) {
                if (!(W.t[s] > 0)) return FHD_ERR_BAD_ARG;
                double molmix = 0.;
                for (int n = 0; n < ns; ++n) molmix += W.Yk[s][n] / p.molmass[n];
                molmix = 1. / molmix;
                W.rho[s] = W.p[s] / (p.Runiv / molmix) / W.t[s];
            } else if (W.t[s] <= 0.0) {
                double molmix = 0.;
                for (int n = 0; n < ns; ++n) molmix += W.Yk[s][n] / p.molmass[n];
                molmix = 1. / molmix;
                W.t[s] = W.p[s] * (molmix / p.Runiv) / W.rho[s];
            }
            if (!(W.p[s] > 0) || !(W.rho[s] > 0) || !(W.t[s] > 0)) return FHD_ERR_BAD_ARG;
        }
    }
    return FHD_OK;
}

int fhd_create(fhd_ctx** out, const fhd_params* params, int device) {
    if (!out || !params) return FHD_ERR_BAD_ARG;
    *out = nullptr;
    const fhd_params& p = *params;
    if (p.nspecies < 1 || p.nspecies > 4) return FHD_ERR_UNSUPPORTED;
    // one cell is a direction of a quasi-2-D (z) or quasi-1-D (y, z) run, as the reference's
    // driver requires those runs for such boxes (main_driver.cpp:125-140); it stays periodic
    for (int d = 0; d < 3; ++d) {
        const bool thin_ok = (d == 2 && p.do_2D == 1) || (d >= 1 && p.do_1D == 1);
        if (p.n_cells[d] < 1 || (p.n_cells[d] < 2 && !thin_ok) || !(p.prob_hi[d] > p.prob_lo[d]))
            return FHD_ERR_BAD_ARG;
        if (p.n_cells[d] == 1 && p.walls && (p.bc_vel_lo[d] != -1 || p.bc_vel_hi[d] != -1)) return FHD_ERR_BAD_ARG;
    }
    if ((int64_t)p.n_cells[0] * p.n_cells[1] * p.n_cells[2] >= ((int64_t)1 << 32)) return FHD_ERR_UNSUPPORTED;
    // algorithm_type 2 is the multispecies path every staggered deck runs; transport models
    // 1 Giovangigli, 2 Valk/Waldmann, 3 HCB (binary mixtures only)
    if (p.algorithm_type != 2 || p.transport_type < 1 || p.transport_type > 3) return FHD_ERR_UNSUPPORTED;
    if (p.transport_type == 3 && p.nspecies != 2) return FHD_ERR_BAD_ARG;
    if (p.transport_type != 1 && p.precision != FHD_PREC_FP64) return FHD_ERR_UNSUPPORTED;
    if (p.stoch_stress_form != 0 && p.stoch_stress_form != 1) return FHD_ERR_UNSUPPORTED;
    if (p.advection_type < -1 || p.advection_type > 2) return FHD_ERR_UNSUPPORTED;
    if (p.precision != FHD_PREC_FP64 && p.precision != FHD_PREC_MIXED) return FHD_ERR_BAD_ARG;
    if ((p.visc_type == 3 || p.visc_type == -3) && p.zeta_ratio < 0) return FHD_ERR_BAD_ARG;
    // chemistry (chemistry_functions.cpp:50-52, 131-135)
    if (p.nreaction < 0 || p.nreaction > FHD_MAX_REACTIONS) return FHD_ERR_BAD_ARG;
    if (p.nreaction > 0) {
        if (p.reaction_type != 0 && p.reaction_type != 1) return FHD_ERR_UNSUPPORTED;
        if (!(p.T0_chem > 0)) return FHD_ERR_BAD_ARG;
        for (int m = 0; m < p.nreaction; ++m)
            for (int n = 0; n < p.nspecies; ++n)
                if (p.stoich_R[m][n] < 0 || p.stoich_R[m][n] > 16 || p.stoich_P[m][n] < 0 || p.stoich_P[m][n] > 16)
                    return FHD_ERR_BAD_ARG;
    }
    int per[3];
    WallParams wall;
    if (const int rc = setup_walls(p, per, wall)) return rc;
    const bool walls = !(per[0] && per[1] && per[2]);
    if (walls && p.precision != FHD_PREC_FP64) return FHD_ERR_UNSUPPORTED;
    // quasi-1-D / 2-D runs: one mode at most, no bulk viscosity (main_driver.cpp:104-118);
    // FP64 and no particle reservoir here
    if (p.do_1D < 0 || p.do_1D > 1 || p.do_2D < 0 || p.do_2D > 1 || (p.do_1D && p.do_2D)) return FHD_ERR_BAD_ARG;
    const bool lowdim = p.do_1D || p.do_2D;
    if (lowdim && (p.visc_type == 3 || p.visc_type == -3)) return FHD_ERR_BAD_ARG;
    if (lowdim && p.precision != FHD_PREC_FP64) return FHD_ERR_UNSUPPORTED;
    if (lowdim && walls)
        for (int d = 0; d < 3; ++d)
            if (!per[d] && (p.bc_mass_lo[d] == 4 || p.bc_mass_hi[d] == 4)) return FHD_ERR_UNSUPPORTED;
    fhd_ctx* c = new (std::nothrow) fhd_ctx;
    if (!c) return FHD_ERR_OOM;
    c->prm = p;
    c->prm.walls = walls ? 1 : 0;
    // the effective wall compositions and reservoir states (after SetupCWallStag)
    for (int d = 0; d < 3 && walls; ++d) {
        if (per[d]) continue;
        c->prm.t_lo[d] = wall.t[2 * d];
        c->prm.t_hi[d] = wall.t[2 * d + 1];
        c->prm.p_lo[d] = wall.p[2 * d];
        c->prm.p_hi[d] = wall.p[2 * d + 1];
        c->prm.rho_lo[d] = wall.rho[2 * d];
        c->prm.rho_hi[d] = wall.rho[2 * d + 1];
    }
    for (int d = 0; d < 3 && walls; ++d)
        for (int n = 0; n < p.nspecies && !per[d]; ++n) {
            c->prm.bc_Yk_lo[d][n] = wall.Yk[2 * d][n];
            c->prm.bc_Xk_lo[d][n] = wall.Xk[2 * d][n];
            c->prm.bc_Yk_hi[d][n] = wall.Yk[2 * d + 1][n];
            c->prm.bc_Xk_hi[d][n] = wall.Xk[2 * d + 1][n];
        }
    for (int d = 0; d < 3; ++d) c->per[d] = per[d];
    c->walls = walls;
    c->refpipe = walls || lowdim || p.transport_type != 1;
    c->wall = wall;
    for (int d = 0; d < 3; ++d) {
        if (!per[d] && (p.bc_mass_lo[d] >= 3 || p.bc_mass_hi[d] >= 3)) c->reservoir = true;
        if (!per[d] && (p.bc_mass_lo[d] == 4 || p.bc_mass_hi[d] == 4)) c->res4 = true;
    }
    // GetHcGas, compressible_functions.cpp:91-100
    for (int i = 0; i < p.nspecies; ++i) {
        if (c->prm.hcv[i] < 0.) c->prm.hcv[i] = 0.5 * p.dof[i] * p.Runiv / p.molmass[i];
        if (c->prm.hcp[i] < 0.) c->prm.hcp[i] = 0.5 * (2. + p.dof[i]) * p.Runiv / p.molmass[i];
    }
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); delete c; return FHD_ERR_CUDA; }
    if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) { delete c; return FHD_ERR_CUDA; }
    c->stream = c->own;
    if (cudaMalloc(&c->d_status, sizeof(int)) != cudaSuccess) {
        cudaStreamDestroy(c->own);
        delete c;
        return FHD_ERR_OOM;
    }
    cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream);
    if (p.transport_type == 2) {
        VWTable t;
        vw_table(c->prm, t);
        if (cudaMalloc(&c->vwt, sizeof(VWTable)) != cudaSuccess ||
            cudaMemcpy(c->vwt, &t, sizeof(VWTable), cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaGetLastError();
            fhd_destroy(c);
            return FHD_ERR_OOM;
        }
    }
    *out = c;
    return FHD_OK;
}

int fhd_destroy(fhd_ctx* c) {
    if (!c) return FHD_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    if (c->scratch) cudaFree(c->scratch);
    if (c->coef) cudaFree(c->coef);
    if (c->lines) cudaFree(c->lines);
    if (c->vwt) cudaFree(c->vwt);
    if (c->res.base) cudaFree(c->res.base);
    if (c->hbuf) cudaFree(c->hbuf);
    for (auto& e : c->evs) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
    if (c->d_status) cudaFree(c->d_status);
    if (c->sgexec) cudaGraphExecDestroy(c->sgexec);
    if (c->sgraph) cudaGraphDestroy(c->sgraph);
    if (c->d_step) cudaFree(c->d_step);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
    return FHD_OK;
}

int fhd_set_stream(fhd_ctx* c, void* stream) {
    if (!c) return FHD_ERR_BAD_ARG;
    // NULL selects the legacy default stream (cudaStream_t 0), as in the CUDA API
    c->stream = static_cast<cudaStream_t>(stream);
    return FHD_OK;
}

int fhd_synchronize(fhd_ctx* c) {
    if (!c) return FHD_ERR_BAD_ARG;
    return sync_rc(cudaStreamSynchronize(c->stream));
}

int fhd_status(fhd_ctx* c) {
    if (!c) return FHD_ERR_BAD_ARG;
    int h = 0;
    if (cudaMemcpyAsync(&h, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
        return FHD_ERR_CUDA;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_CUDA; }
    cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream);
    return h;
}

int fhd_get_params(const fhd_ctx* c, fhd_params* out) {
    if (!c || !out) return FHD_ERR_BAD_ARG;
    *out = c->prm;
    return FHD_OK;
}

int fhd_set_tile(fhd_ctx* c, int tile) {
    if (!c || tile < 0 || tile >= num_tiles()) return FHD_ERR_BAD_ARG;
    c->tile = tile;
    return FHD_OK;
}

int fhd_num_tiles(void) { return num_tiles(); }
const char* fhd_tile_name(int t) { return tile_name(t); }

int fhd_init_cons_var_stag(fhd_ctx* c, fhd_fab cu, const fhd_fab mom[3], double rho0, double T_init,
                           const double* rhobar) {
    if (!c || !mom || !rhobar) return FHD_ERR_BAD_ARG;
    const int ns = c->prm.nspecies;
    if (!fab_ok(c, cu, CELLN, 0, 5 + ns, FHD_F64)) return FHD_ERR_BAD_ARG;
    for (int d = 0; d < 3; ++d)
        if (!fab_ok(c, mom[d], FACEN[d], 0, 1, FHD_F64)) return FHD_ERR_BAD_ARG;
    // GetEnergy (compressible_functions.H:1497-1510) at T_init with massvec = rhobar
    double cvmix = 0., e0mix = 0.;
    for (int i = 0; i < ns; ++i) {
        cvmix += rhobar[i] * c->prm.hcv[i];
        e0mix += rhobar[i] * c->prm.e0[i];
    }
    const double intEnergy = e0mix + T_init * cvmix;
    double rhoY[FHD_MAX_SPECIES];
    for (int i = 0; i < ns; ++i) rhoY[i] = rho0 * rhobar[i];
    cudaSetDevice(c->device);
    int rc = init_uniform(cu, ns, rho0, rho0 * intEnergy, rhoY, c->stream);
    if (rc) return rc;
    for (int d = 0; d < 3; ++d)
        if (cudaMemsetAsync(mom[d].data, 0, fab_points(mom[d]) * sizeof(double) * mom[d].ncomp, c->stream) !=
            cudaSuccess)
            return FHD_ERR_CUDA;
    return FHD_OK;
}

int fhd_conserved_to_primitive_stag(fhd_ctx* c, fhd_fab prim, const fhd_fab vel[3], fhd_fab cu, const fhd_fab mom[3]) {
    if (!c || !vel || !mom) return FHD_ERR_BAD_ARG;
    const int ns = c->prm.nspecies;
    if (!fab_ok(c, cu, CELLN, 1, 5 + ns, FHD_F64) || !fab_ok(c, prim, CELLN, 0, 6 + 2 * ns, FHD_F64))
        return FHD_ERR_BAD_ARG;
    for (int d = 0; d < 3; ++d)
        if (!fab_ok(c, vel[d], FACEN[d], 0, 1, FHD_F64) || !fab_ok(c, mom[d], FACEN[d], 0, 1, FHD_F64))
            return FHD_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    return exact_convert(make_dev(c, 1.0, 0), prim, vel, cu, mom, c->d_status, c->stream);
}

int fhd_transport_coeffs(fhd_ctx* c, fhd_fab prim, fhd_fab eta, fhd_fab zeta, fhd_fab kappa, fhd_fab chi, fhd_fab D) {
    if (!c) return FHD_ERR_BAD_ARG;
    const int ns = c->prm.nspecies;
    if (!fab_ok(c, prim, CELLN, 0, 6 + 2 * ns, FHD_F64)) return FHD_ERR_BAD_ARG;
    const int g = -prim.lo[0];
    if (!fab_ok(c, eta, CELLN, g, 1, FHD_F64) || !fab_ok(c, zeta, CELLN, g, 1, FHD_F64) ||
        !fab_ok(c, kappa, CELLN, g, 1, FHD_F64) || !fab_ok(c, chi, CELLN, g, ns, FHD_F64) ||
        !fab_ok(c, D, CELLN, g, ns * ns, FHD_F64))
        return FHD_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    return exact_transport(make_dev(c, 1.0, 0), prim, eta, zeta, kappa, chi, D, c->d_status, c->stream);
}

int fhd_flux_stag(fhd_ctx* c, fhd_fab cu, const fhd_fab mom[3], fhd_fab prim, const fhd_fab vel[3], fhd_fab eta,
                  fhd_fab zeta, fhd_fab kappa, fhd_fab chi, fhd_fab D, const fhd_fab faceflux[3],
                  const fhd_fab edgeflux[6], const fhd_fab cenflux[3], const fhd_fab stochface[3],
                  const fhd_fab stochedge[3], const fhd_fab stochcen[3], double dt) {
    if (!c || !mom || !vel || !faceflux || !edgeflux || !cenflux) return FHD_ERR_BAD_ARG;
    const int ns = c->prm.nspecies, nvars = 5 + ns;
    if (!fab_ok(c, cu, CELLN, 1, nvars, FHD_F64) || !fab_ok(c, prim, CELLN, 1, 6 + 2 * ns, FHD_F64))
        return FHD_ERR_BAD_ARG;
    if (!fab_ok(c, eta, CELLN, 1, 1, FHD_F64) || !fab_ok(c, zeta, CELLN, 1, 1, FHD_F64) ||
        !fab_ok(c, kappa, CELLN, 1, 1, FHD_F64) || !fab_ok(c, chi, CELLN, 1, ns, FHD_F64) ||
        !fab_ok(c, D, CELLN, 1, ns * ns, FHD_F64))
        return FHD_ERR_BAD_ARG;
    for (int d = 0; d < 3; ++d) {
        if (!fab_ok(c, vel[d], FACEN[d], 1, 1, FHD_F64) || !fab_ok(c, mom[d], FACEN[d], 1, 1, FHD_F64))
            return FHD_ERR_BAD_ARG;
        if (!fab_ok(c, faceflux[d], FACEN[d], 0, nvars + 4, FHD_F64, 0)) return FHD_ERR_BAD_ARG;
        if (!fab_ok(c, cenflux[d], CELLN, 1, 1, FHD_F64, 1)) return FHD_ERR_BAD_ARG;
    }
    for (int e = 0; e < 6; ++e)
        if (!fab_ok(c, edgeflux[e], EFLUXN[e], 0, 1, FHD_F64, 0)) return FHD_ERR_BAD_ARG;
    const bool stoch = c->prm.stoch_stress_form == 1;
    if (stoch) {
        if (!stochface || !stochedge || !stochcen) return FHD_ERR_BAD_ARG;
        for (int d = 0; d < 3; ++d)
            if (!fab_ok(c, stochface[d], FACEN[d], 0, ns + 1, FHD_F64) ||
                !fab_ok(c, stochedge[d], EDGEN[d], 0, 1, FHD_F64) || !fab_ok(c, stochcen[d], CELLN, 1, 1, FHD_F64))
                return FHD_ERR_BAD_ARG;
    }
    cudaSetDevice(c->device);
    StageCall sc;
    std::memset(&sc, 0, sizeof(sc));
    sc.P = make_dev(c, dt, 0);
    sc.mode = stoch ? NM_W : NM_OFF;
    sc.w = 0.0;
    sc.stage = 0;
    sc.cons_s = cu;
    for (int d = 0; d < 3; ++d) { sc.mom_s[d] = mom[d]; sc.vel[d] = vel[d]; sc.ff[d] = faceflux[d]; sc.cf[d] = cenflux[d]; }
    for (int e = 0; e < 6; ++e) sc.ef[e] = edgeflux[e];
    sc.pr = prim;
    sc.pT = 4;
    sc.eta = eta; sc.zeta = zeta; sc.kappa = kappa; sc.chi = chi; sc.D = D;
    if (stoch) {
        for (int d = 0; d < 3; ++d) {
            sc.nz.fa[d] = sc.nz.fb[d] = stochface[d];
            sc.nz.ea[d] = sc.nz.eb[d] = stochedge[d];
            sc.nz.ca[d] = sc.nz.cb[d] = stochcen[d];
        }
    }
    sc.status = c->d_status;
    sc.stream = c->stream;
    return exact_aux_fluxes(sc);
}

int fhd_fill_boundary(fhd_ctx* c, fhd_fab f) {
    if (!c || !f.data || f.dtype != FHD_F64) return FHD_ERR_BAD_ARG;
    int nodal[3] = {f.nodal[0], f.nodal[1], f.nodal[2]};
    if (!fab_ok(c, f, nodal, 0, 1, FHD_F64)) return FHD_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    GhostReq r{f, 0, f.ncomp};
    return fill_ghosts(&r, 1, c->prm.n_cells, c->stream, c->per, 0);
}

int fhd_set_bc_stag(fhd_ctx* c, fhd_fab prim, fhd_fab cu, const fhd_fab cumom[3], const fhd_fab vel[3]) {
    if (!c || !cumom || !vel) return FHD_ERR_BAD_ARG;
    const int ns = c->prm.nspecies;
    if (!fab_ok(c, prim, CELLN, 0, 6 + 2 * ns, FHD_F64)) return FHD_ERR_BAD_ARG;
    const int g = -prim.lo[0];
    if (!fab_ok(c, cu, CELLN, g, 5 + ns, FHD_F64, g)) return FHD_ERR_BAD_ARG;
    const int gm = -cumom[0].lo[0];
    // BCRhoRhoE reads the face momenta around every ghost cell of prim
    if (gm < g) return FHD_ERR_BAD_ARG;
    for (int d = 0; d < 3; ++d)
        if (!fab_ok(c, cumom[d], FACEN[d], gm, 1, FHD_F64, gm) || !fab_ok(c, vel[d], FACEN[d], gm, 1, FHD_F64, gm))
            return FHD_ERR_BAD_ARG;
    if (!c->walls) return FHD_OK;
    for (int d = 0; d < 3; ++d)
        if (!c->per[d] && (c->prm.n_cells[d] < g || c->prm.n_cells[d] < gm)) return FHD_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    const DevParams P = make_dev(c, 1.0, 0);
    if (c->reservoir) return exact_bc_seq(P, c->wall, prim, cu, cumom, vel, true, c->stream);
    int rc = bc_mom(P, cumom, vel, c->stream);
    if (!rc) rc = exact_bc_prim(P, c->wall, prim, cu, cumom, c->stream);
    return rc;
}

int fhd_set_reservoir_record(fhd_ctx* c, void* buf, int cap) {
    if (!c || cap < 0 || (buf && cap == 0)) return FHD_ERR_BAD_ARG;
    c->res_rec = static_cast<double*>(buf);
    c->res_cap = buf ? cap : 0;
    // the captured step graph embeds the hook
    if (c->sgexec) cudaGraphExecDestroy(c->sgexec);
    if (c->sgraph) cudaGraphDestroy(c->sgraph);
    c->sgexec = nullptr;
    c->sgraph = nullptr;
    c->skey.clear();
    return FHD_OK;
}

int fhd_override_sync(fhd_ctx* c, fhd_fab f) {
    if (!c || !f.data) return FHD_ERR_BAD_ARG;
    int nodal[3] = {f.nodal[0], f.nodal[1], f.nodal[2]};
    if (!fab_ok(c, f, nodal, 0, 1, FHD_F64)) return FHD_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    return override_sync(f, c->prm.n_cells, c->stream, c->per);
}

int fhd_fill_random_normal(fhd_ctx* c, fhd_fab mf, int scomp, int ncomp, double mean, double variance,
                           int overridesync, int fillboundary, uint64_t stream_id) {
    if (!c || !mf.data || scomp < 0 || ncomp < 1 || scomp + ncomp > mf.ncomp || variance < 0) return FHD_ERR_BAD_ARG;
    int nodal[3] = {mf.nodal[0], mf.nodal[1], mf.nodal[2]};
    if (!fab_ok(c, mf, nodal, 0, 1, FHD_F64)) return FHD_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    DevParams P = make_dev(c, 1.0, stream_id);
    // field ids above the step-noise range keep these streams apart from the step's noise
    int rc = noise_fill(P, mf, scomp, ncomp, mean, std::sqrt(variance), 0x1000u + (uint32_t)scomp, 0, c->stream);
    if (rc) return rc;
    if (overridesync) rc = override_sync(mf, c->prm.n_cells, c->stream, c->per);
    if (rc) return rc;
    if (fillboundary && -mf.lo[0] > 0) {
        GhostReq r{mf, scomp, ncomp};
        rc = fill_ghosts(&r, 1, c->prm.n_cells, c->stream, c->per, 0);
    }
    return rc;
}

int fhd_fill_random_uniform(fhd_ctx* c, fhd_fab mf, int scomp, int ncomp, int overridesync, int fillboundary,
                            uint64_t stream_id) {
    if (!c || !mf.data || scomp < 0 || ncomp < 1 || scomp + ncomp > mf.ncomp) return FHD_ERR_BAD_ARG;
    int nodal[3] = {mf.nodal[0], mf.nodal[1], mf.nodal[2]};
    if (!fab_ok(c, mf, nodal, 0, 1, FHD_F64)) return FHD_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    DevParams P = make_dev(c, 1.0, stream_id);
    // counter word 1 is the field id itself here (0x2000 + comp): apart from the
    // normal fills' field pairs and from the step noise
    int rc = noise_fill(P, mf, scomp, ncomp, 0.0, 1.0, 0x2000u + (uint32_t)scomp, 2, c->stream);
    if (rc) return rc;
    if (overridesync) rc = override_sync(mf, c->prm.n_cells, c->stream, c->per);
    if (rc) return rc;
    if (fillboundary && -mf.lo[0] > 0) {
        GhostReq r{mf, scomp, ncomp};
        rc = fill_ghosts(&r, 1, c->prm.n_cells, c->stream, c->per, 0);
    }
    return rc;
}

static bool device_accessible(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged || a.type == cudaMemoryTypeHost;
}

static bool plot_inputs_accessible(int flags, const fhd_fab& cu, const fhd_fab* cumom, const fhd_fab& prim,
                                   const fhd_fab* vel, const fhd_fab& eta, const fhd_fab& kappa, const fhd_fab& zeta,
                                   const fhd_stats* st, int visc3) {
    std::vector<const void*> ptrs = {cu.data, prim.data, eta.data, kappa.data};
    if (visc3) ptrs.push_back(zeta.data);
    for (int d = 0; d < 3; ++d) { ptrs.push_back(cumom[d].data); ptrs.push_back(vel[d].data); }
    if (flags & FHD_PLOT_MEANS) {
        ptrs.push_back(st->cuMeans.data);
        ptrs.push_back(st->primMeans.data);
        for (int d = 0; d < 3; ++d) { ptrs.push_back(st->cumomMeans[d].data); ptrs.push_back(st->velMeans[d].data); }
    }
    if (flags & FHD_PLOT_VARS) {
        ptrs.push_back(st->cuVars.data);
        ptrs.push_back(st->primVars.data);
        for (int d = 0; d < 3; ++d) { ptrs.push_back(st->cumomVars[d].data); ptrs.push_back(st->velVars[d].data); }
    }
    if (flags & FHD_PLOT_COVARS) ptrs.push_back(st->coVars.data);
    if (flags & FHD_PLOT_MOM3) ptrs.push_back(st->mom3.data);
    if (flags & FHD_PLOT_MOM4) ptrs.push_back(st->mom4.data);
    for (const void* p : ptrs)
        if (!p || !device_accessible(p)) return false;
    return true;
}

// FHD_PLOT_* bits, at most one of the three deltaY directions
static bool plot_flags_ok(int flags) {
    if (flags < 0 || flags > 255) return false;
    const int dy = (flags >> 5) & 7;
    return dy == 0 || dy == 1 || dy == 2 || dy == 4;
}

static bool plot_params_ok(const fhd_params* p) {
    if (!p || p->nspecies < 1 || p->nspecies > 4) return false;
    for (int d = 0; d < 3; ++d)
        if (p->n_cells[d] < 1) return false;
    return true;
}

int fhd_plotfile_ncomp(const fhd_params* p, int flags) {
    if (!plot_params_ok(p) || !plot_flags_ok(flags)) return -FHD_ERR_BAD_ARG;
    std::vector<std::string> names;
    const int rc = plot_names(*p, flags, names);
    return rc ? -rc : (int)names.size();
}

int fhd_plotfile_varname(const fhd_params* p, int flags, int comp, char* buf, int buflen) {
    if (!plot_params_ok(p) || !buf || buflen < 1 || !plot_flags_ok(flags)) return FHD_ERR_BAD_ARG;
    std::vector<std::string> names;
    const int rc = plot_names(*p, flags, names);
    if (rc) return rc;
    if (comp < 0 || comp >= (int)names.size() || (int)names[comp].size() >= buflen) return FHD_ERR_BAD_ARG;
    std::memcpy(buf, names[comp].c_str(), names[comp].size() + 1);
    return FHD_OK;
}

int fhd_plotfile_write_host(const fhd_params* p, const char* dir, const double* data, int flags, double time,
                            int step) {
    if (!plot_params_ok(p) || !dir || !data || !plot_flags_ok(flags)) return FHD_ERR_BAD_ARG;
    std::vector<std::string> names;
    const int rc = plot_names(*p, flags, names);
    if (rc) return rc;
    return plot_write(*p, dir, data, names, time, step);
}

int fhd_plotfile_pack(fhd_ctx* c, int flags, fhd_fab out, fhd_fab cu, const fhd_fab cumom[3], fhd_fab prim,
                      const fhd_fab vel[3], fhd_fab eta, fhd_fab kappa, fhd_fab zeta, const fhd_stats* stats) {
    if (!c || !cumom || !vel || !plot_flags_ok(flags) || ((flags & 31) && !stats)) return FHD_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    const int visc3 = c->prm.visc_type == 3 || c->prm.visc_type == -3;
    if (!out.data || !device_accessible(out.data) ||
        !plot_inputs_accessible(flags, cu, cumom, prim, vel, eta, kappa, zeta, stats, visc3))
        return FHD_ERR_BAD_ARG;
    return plot_pack(c->prm, flags, out, cu, cumom, prim, vel, eta, kappa, zeta, stats, c->stream);
}

int fhd_write_plotfile_stag(fhd_ctx* c, const char* plot_base_name, int step, double time, int flags, fhd_fab cu,
                            const fhd_fab cumom[3], fhd_fab prim, const fhd_fab vel[3], fhd_fab eta, fhd_fab kappa,
                            fhd_fab zeta, const fhd_stats* stats) {
    if (!c || !plot_base_name || step < 0) return FHD_ERR_BAD_ARG;
    const int nc = fhd_plotfile_ncomp(&c->prm, flags);
    if (nc <= 0) return nc < 0 ? -nc : FHD_ERR_BAD_ARG;
    std::vector<std::string> names;
    int rc = plot_names(c->prm, flags, names);
    if (rc) return rc;
    cudaSetDevice(c->device);
    const int* n = c->prm.n_cells;
    const size_t cells = (size_t)n[0] * n[1] * n[2];
    double* dbuf = nullptr;
    if (cudaMalloc(&dbuf, cells * nc * sizeof(double)) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_OOM; }
    const fhd_fab out = make_fab(dbuf, n, CELLN, 0, nc, FHD_F64);
    rc = fhd_plotfile_pack(c, flags, out, cu, cumom, prim, vel, eta, kappa, zeta, stats);
    std::vector<double> host;
    if (!rc) {
        host.resize(cells * nc);
        if (cudaMemcpyAsync(host.data(), dbuf, cells * nc * sizeof(double), cudaMemcpyDeviceToHost, c->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(c->stream) != cudaSuccess)
            rc = FHD_ERR_CUDA;
    }
    cudaFree(dbuf);
    if (rc) return rc;
    // amrex::Concatenate(plot_base_name, step, 9)
    char num[32];
    std::snprintf(num, sizeof(num), "%09d", step);
    const std::string dir = std::string(plot_base_name) + num;
    return plot_write(c->prm, dir.c_str(), host.data(), names, time, step);
}

int fhd_chemistry_source_cle(fhd_ctx* c, double dt, double dV, fhd_fab prim, fhd_fab source, fhd_fab ranchem) {
    if (!c || c->prm.nreaction < 1 || !(dt > 0) || !(dV > 0)) return FHD_ERR_BAD_ARG;
    const int ns = c->prm.nspecies, nprim = 6 + 2 * ns;
    if (!fab_ok(c, prim, CELLN, 0, nprim, FHD_F64) || !fab_ok(c, source, CELLN, 0, 5 + ns, FHD_F64)) return FHD_ERR_BAD_ARG;
    const bool cle = c->prm.reaction_type == 1;
    if (cle && !fab_ok(c, ranchem, CELLN, 0, c->prm.nreaction, FHD_F64)) return FHD_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    const DevParams P = make_dev(c, dt, 0);
    const ChemParams cp = chem_params(c->prm, dt, dV);
    return chem_launch(P, cp, prim, source, cle ? &ranchem : nullptr, nullptr, cle ? CN_W : CN_OFF, 0.0, c->stream);
}

int fhd_fill_step_noise(fhd_ctx* c, const fhd_noise* nz, int64_t step) {
    if (!c || !nz) return FHD_ERR_BAD_ARG;
    // the stress fields (when face[0][0] is given) and the reaction fields (when
    // chem[0] is given and the context has reactions); at least one of the two
    const bool stress = nz->face[0][0].data != nullptr;
    const bool chem = nz->chem[0].data != nullptr;
    if (!stress && !chem) return FHD_ERR_BAD_ARG;
    if (stress && !noise_ok(c, nz)) return FHD_ERR_BAD_ARG;
    if (chem && (c->prm.nreaction < 1 || !chem_noise_ok(c, nz))) return FHD_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    const int ns = c->prm.nspecies;
    DevParams P = make_dev(c, 1.0, (uint64_t)step);
    if (chem)
        for (int s = 0; s < 2; ++s) {
            const int rc = noise_fill(P, nz->chem[s], 0, c->prm.nreaction, 0.0, 1.0, fid_chem(0), s, c->stream);
            if (rc) return rc;
        }
    if (!stress) return FHD_OK;
    GhostReq g[6];
    int ng = 0;
    for (int s = 0; s < 2; ++s)
        for (int d = 0; d < 3; ++d) {
            const fhd_fab& f = nz->face[s][d];
            int rc = noise_fill(P, f, f.ncomp - (ns + 1), ns + 1, 0.0, 1.0, fid_face(d, 0), s, c->stream);
            if (!rc) rc = noise_fill(P, nz->edge[s][d], 0, 1, 0.0, 1.0, fid_edge(d), s, c->stream);
            // the centre noise is read on the cells grown by 1: in a wall direction
            // its ghost layer holds values of its own
            if (!rc) rc = noise_fill(P, nz->cen[s][d], 0, 1, 0.0, d == 0 ? P.csd0 : std::sqrt(2.0), fid_cen(d), s,
                                     c->stream, 1);
            if (rc) return rc;
            g[ng++] = GhostReq{nz->cen[s][d], 0, 1};
        }
    return fill_ghosts(g, ng, c->prm.n_cells, c->stream, c->per, 1);
}

// One RK3 step of a box with physical walls (timeStepStag.cpp with setBCStag):
// per stage the coefficients on the whole grown box from the stage's prim, the
// wall variants of the stresses and fluxes, the update, then BCMomNormal /
// BCMomTrans on the new face momenta, FillBoundary of the periodic directions,
// conservedToPrimitiveStag on the valid region, FillBoundary again and setBCStag
// (the conditions of boundaryStag.cpp on every ghost of the wall directions).
// The state's prim and vel carry each stage's primitive fields, as in the
// reference.  (The reference also runs BCMassTempPress on the previous stage's
// prim before the conversion; setBCStag rewrites every value that pass writes
// from the new prim, so it is left out.)
static int walls_step_launches(fhd_ctx* c, fhd_fab cu, const fhd_fab mom[3], fhd_fab prim, const fhd_fab vel[3],
                               fhd_fab source, fhd_fab eta, fhd_fab zeta, fhd_fab kappa, fhd_fab chi, fhd_fab D,
                               const fhd_fab* faceflux, const fhd_fab* edgeflux, const fhd_fab* cenflux,
                               const fhd_noise* injected, double dt, int64_t step, bool aux_coef, bool aux_flux,
                               const uint64_t* step_ptr) {
    const int ns = c->prm.nspecies, nvars = 5 + ns, nprim = 6 + 2 * ns;
    const bool stoch = c->prm.stoch_stress_form == 1;
    int rc = FHD_OK;
    const double w[3] = {(2.0 * std::sqrt(2.0) + 1.0 * std::sqrt(3.0)) / 5.0,
                         (-4.0 * std::sqrt(2.0) + 3.0 * std::sqrt(3.0)) / 5.0,
                         (1.0 * std::sqrt(2.0) - 2.0 * std::sqrt(3.0)) / 10.0};
    StageCall sc;
    std::memset(&sc, 0, sizeof(sc));
    sc.P = make_dev(c, dt, (uint64_t)step);
    sc.P.step_ptr = step_ptr;
    sc.mode = !stoch ? NM_OFF : (injected ? NM_AB : NM_PHILOX);
    if (injected && stoch) set_noise(sc, injected, false);
    sc.pr = prim;
    sc.pT = 4;
    for (int d = 0; d < 3; ++d) { sc.vel[d] = vel[d]; sc.mom0[d] = mom[d]; }
    sc.cons0 = cu;
    sc.src = source;
    const bool chem = c->prm.nreaction > 0;
    ChemParams cp;
    int cmode = CN_OFF;
    if (chem) {
        if (!sc.src.data) sc.src = c->csrc;
        cp = chem_params(c->prm, dt, sc.P.dx[0] * sc.P.dx[1] * sc.P.dx[2]);
        if (c->prm.reaction_type == 1) cmode = injected ? CN_AB : CN_PHILOX;
    }
    sc.status = c->d_status;
    sc.stream = c->stream;
    sc.ct = c->ct;
    sc.et = c->et;
    sc.smc = c->smc;
    sc.sme = c->sme;
    for (int d = 0; d < 3; ++d) sc.sff[d] = c->sff[d];
    const fhd_fab* ins[3] = {&cu, &c->cup, &c->cup2};
    const fhd_fab* insm[3] = {mom, c->cupm, c->cup2m};
    const fhd_fab* outs[3] = {&c->cup, &c->cup2, &cu};
    const fhd_fab* outsm[3] = {c->cupm, c->cup2m, mom};
    if (c->reservoir) {
        // the stage buffers start each step at zero, ghosts included, as RK3stepStag's
        // cup / cup2 do (timeStepStag.cpp:30-62): with reservoirs the boundary passes
        // read ghost corners before they rewrite them
        const size_t stage_bytes = (size_t)((char*)c->sff[0].data - (char*)c->scratch);
        if (cudaMemsetAsync(c->scratch, 0, stage_bytes, c->stream) != cudaSuccess) return FHD_ERR_CUDA;
    }
    for (int s = 0; s < 3; ++s) {
        sc.stage = s + 1;
        sc.w = w[s];
        sc.cons_s = *ins[s];
        sc.cons_o = *outs[s];
        for (int d = 0; d < 3; ++d) { sc.mom_s[d] = insm[s][d]; sc.mom_o[d] = outsm[s][d]; }
        // calculateTransportCoeffs on the grown box (the caller's fabs at stage 3)
        if (s == 2 && aux_coef) { sc.eta = eta; sc.zeta = zeta; sc.kappa = kappa; sc.chi = chi; sc.D = D; }
        else { sc.eta = c->ceta; sc.zeta = c->czeta; sc.kappa = c->ckappa; sc.chi = c->cchi; sc.D = c->cD; }
        {
            ProfScope ps(c, 0);
            rc = exact_transport(sc.P, prim, sc.eta, sc.zeta, sc.kappa, sc.chi, sc.D, c->d_status, c->stream);
            if (!rc && chem)
                rc = chem_launch(sc.P, cp, prim, sc.src, cmode == CN_AB ? &injected->chem[0] : nullptr,
                                 cmode == CN_AB ? &injected->chem[1] : nullptr, cmode, w[s], c->stream);
            // the particle reservoir's fluxes from the stage's input (ComputeFluxMomReservoir
            // with dt, dt / 4, 2 dt / 3: timeStepStag.cpp:341-350, 667-676, 1000-1009)
            if (!rc && c->res4) {
                const double dts = s == 0 ? dt : (s == 1 ? 0.25 * dt : (2.0 / 3.0) * dt);
                rc = exact_reservoir(sc.P, c->res, *ins[s], prim, vel, dts, s, c->res_rec, c->res_cap, c->d_status,
                                     c->stream);
            }
        }
        if (rc) return rc;
        if (s == 2 && aux_flux) {
            for (int d = 0; d < 3; ++d) { sc.ff[d] = faceflux[d]; sc.cf[d] = cenflux[d]; }
            for (int e = 0; e < 6; ++e) sc.ef[e] = edgeflux[e];
            ProfScope ps(c, 6);
            rc = exact_aux_fluxes(sc);
            if (!rc && c->res4) rc = exact_res_reset(sc.P, c->res, faceflux, 0, 4, 5, edgeflux, -1, c->stream);
            if (rc) return rc;
        }
        for (int part = 0; part < 3 && !rc; ++part) {
            ProfScope ps(c, 1 + part);
            // ResetReservoirFluxes between the fluxes and the update
            if (part == 2 && c->res4) rc = exact_res_reset(sc.P, c->res, c->sff, 0, 1, 2, &c->sme, 0, c->stream);
            if (!rc) rc = exact_walls_part(sc, part);
        }
        if (rc) return rc;
        {
            ProfScope ps(c, 4);
            // wall faces of the new momenta (the conversion reads them), then the
            // periodic ghosts that the conversion and the conditions read; with
            // reservoirs every pass RK3stepStag makes here (the reservoir density
            // enters the interface velocity)
            if (c->reservoir) rc = exact_bc_seq(sc.P, c->wall, prim, *outs[s], outsm[s], vel, false, c->stream);
            else rc = bc_mom(sc.P, outsm[s], vel, c->stream);
            // ResetReservoirMom (timeStepStag.cpp:538-540, 871-873, 1212-1214)
            if (!rc && c->res4) rc = exact_res_mom(sc.P, c->res, outsm[s], c->stream);
            GhostReq g[4] = {{*outs[s], 0, nvars}, {outsm[s][0], 0, 1}, {outsm[s][1], 0, 1}, {outsm[s][2], 0, 1}};
            if (!rc) rc = fill_ghosts(g, 4, c->prm.n_cells, c->stream, c->per, 0);
        }
        if (rc) return rc;
        {
            ProfScope ps(c, 5);
            rc = exact_convert(sc.P, prim, vel, *outs[s], outsm[s], c->d_status, c->stream);
        }
        if (rc) return rc;
        {
            ProfScope ps(c, 4);
            GhostReq g[5] = {{*outs[s], 0, nvars}, {prim, 0, nprim}, {vel[0], 0, 1}, {vel[1], 0, 1}, {vel[2], 0, 1}};
            rc = fill_ghosts(g, 5, c->prm.n_cells, c->stream, c->per, 0);
            if (c->reservoir) {
                if (!rc) rc = exact_bc_seq(sc.P, c->wall, prim, *outs[s], outsm[s], vel, true, c->stream);
            } else {
                if (!rc) rc = bc_mom(sc.P, outsm[s], vel, c->stream);
                if (!rc) rc = exact_bc_prim(sc.P, c->wall, prim, *outs[s], outsm[s], c->stream);
            }
        }
        if (rc) return rc;
    }
    return FHD_OK;
}

// The launches of one RK3 step (after validation and scratch set-up); step_ptr,
// when set, is the device word the Philox noise reads its step from (graph replay).
static int step_launches(fhd_ctx* c, fhd_fab cu, const fhd_fab mom[3], fhd_fab prim, const fhd_fab vel[3], fhd_fab source,
                  fhd_fab eta, fhd_fab zeta, fhd_fab kappa, fhd_fab chi, fhd_fab D, const fhd_fab* faceflux,
                  const fhd_fab* edgeflux, const fhd_fab* cenflux, const fhd_noise* injected, double dt, int64_t step,
                  bool aux_coef, bool aux_flux, const uint64_t* step_ptr) {
    if (c->refpipe)
        return walls_step_launches(c, cu, mom, prim, vel, source, eta, zeta, kappa, chi, D, faceflux, edgeflux,
                                   cenflux, injected, dt, step, aux_coef, aux_flux, step_ptr);
    const int ns = c->prm.nspecies, nprim = 6 + 2 * ns;
    const bool mixed = c->prm.precision == FHD_PREC_MIXED;
    const bool stoch = c->prm.stoch_stress_form == 1;
    int rc = FHD_OK;
    const double w[3] = {(2.0 * std::sqrt(2.0) + 1.0 * std::sqrt(3.0)) / 5.0,
                         (-4.0 * std::sqrt(2.0) + 3.0 * std::sqrt(3.0)) / 5.0,
                         (1.0 * std::sqrt(2.0) - 2.0 * std::sqrt(3.0)) / 10.0};
    StageCall sc;
    std::memset(&sc, 0, sizeof(sc));
    sc.P = make_dev(c, dt, (uint64_t)step);
    sc.P.step_ptr = step_ptr;
    sc.mode = !stoch ? NM_OFF : (injected ? NM_AB : NM_PHILOX);
    if (injected && stoch) set_noise(sc, injected, false);
    sc.pr = prim;
    sc.pT = 4;
    for (int d = 0; d < 3; ++d) { sc.vel[d] = vel[d]; sc.mom0[d] = mom[d]; }
    sc.cons0 = cu;
    if (aux_coef && !mixed) { sc.eta = eta; sc.zeta = zeta; sc.kappa = kappa; sc.chi = chi; sc.D = D; }
    else { sc.eta = c->ceta; sc.zeta = c->czeta; sc.kappa = c->ckappa; sc.chi = c->cchi; sc.D = c->cD; }
    sc.src = source;
    // chemistry source (timeStepStag.cpp:354-361): written into the caller's source,
    // or into the context's zeroed one, after each stage's conversion
    const bool chem = c->prm.nreaction > 0;
    ChemParams cp;
    int cmode = CN_OFF;
    if (chem) {
        if (!sc.src.data) sc.src = c->csrc;
        cp = chem_params(c->prm, dt, sc.P.dx[0] * sc.P.dx[1] * sc.P.dx[2]);
        if (c->prm.reaction_type == 1) cmode = injected ? CN_AB : CN_PHILOX;
    }
    sc.status = c->d_status;
    sc.stream = c->stream;
    sc.tile = c->tile;
    sc.ct = c->ct;
    sc.et = c->et;
    sc.smc = c->smc;
    sc.sme = c->sme;
    for (int d = 0; d < 3; ++d) sc.sff[d] = c->sff[d];
    const fhd_fab* ins[3] = {&cu, &c->cup, &c->cup2};
    const fhd_fab* insm[3] = {mom, c->cupm, c->cup2m};
    const fhd_fab* outs[3] = {&c->cup, &c->cup2, &cu};
    const fhd_fab* outsm[3] = {c->cupm, c->cup2m, mom};
    for (int s = 0; s < 3; ++s) {
        sc.stage = s + 1;
        sc.w = w[s];
        sc.cons_s = *ins[s];
        sc.cons_o = *outs[s];
        for (int d = 0; d < 3; ++d) { sc.mom_s[d] = insm[s][d]; sc.mom_o[d] = outsm[s][d]; }
        {
            ProfScope ps(c, 0);
            rc = mixed ? mixed_cellprep(sc) : exact_cellprep(sc);
            if (!rc && chem)
                rc = chem_launch(sc.P, cp, prim, sc.src, cmode == CN_AB ? &injected->chem[0] : nullptr,
                                 cmode == CN_AB ? &injected->chem[1] : nullptr, cmode, w[s], c->stream);
        }
        if (rc) return rc;
        if (s == 2 && aux_flux) {
            for (int d = 0; d < 3; ++d) { sc.ff[d] = faceflux[d]; sc.cf[d] = cenflux[d]; }
            for (int e = 0; e < 6; ++e) sc.ef[e] = edgeflux[e];
            ProfScope ps(c, 6);
            rc = exact_aux_fluxes(sc);
            if (rc) return rc;
        }
        if (tile_fused(c->tile)) {
            ProfScope ps(c, 7);
            rc = mixed ? mixed_stage_part(sc, 3) : exact_stage_part(sc, 3);
        } else {
            for (int part = 0; part < 3 && !rc; ++part) {
                ProfScope ps(c, 1 + part);
                rc = mixed ? mixed_stage_part(sc, part) : exact_stage_part(sc, part);
            }
        }
        if (rc) return rc;
        GhostReq g[5] = {{*outs[s], 0, 1}, {*outs[s], 4, 1 + ns}, {outsm[s][0], 0, 1}, {outsm[s][1], 0, 1},
                         {outsm[s][2], 0, 1}};
        {
            ProfScope ps(c, 4);
            rc = fill_ghosts(g, 5, c->prm.n_cells, c->stream);
        }
        if (rc) return rc;
    }
    // final conservedToPrimitiveStag + FillBoundary (timeStepStag.cpp:1216-1230)
    {
        ProfScope ps(c, 5);
        rc = exact_convert(sc.P, prim, vel, cu, mom, c->d_status, c->stream);
    }
    if (rc) return rc;
    GhostReq g[10];
    int ng = 0;
    g[ng++] = GhostReq{cu, 1, 3};
    g[ng++] = GhostReq{prim, 0, nprim};
    for (int d = 0; d < 3; ++d) g[ng++] = GhostReq{vel[d], 0, 1};
    if (aux_coef) {
        g[ng++] = GhostReq{eta, 0, 1};
        g[ng++] = GhostReq{zeta, 0, 1};
        g[ng++] = GhostReq{kappa, 0, 1};
        g[ng++] = GhostReq{chi, 0, ns};
        g[ng++] = GhostReq{D, 0, ns * ns};
    }
    ProfScope ps(c, 4);
    return fill_ghosts(g, ng, c->prm.n_cells, c->stream);
}


int fhd_rk3_step_stag(fhd_ctx* c, fhd_fab cu, const fhd_fab mom[3], fhd_fab prim, const fhd_fab vel[3], fhd_fab source,
                      fhd_fab eta, fhd_fab zeta, fhd_fab kappa, fhd_fab chi, fhd_fab D, const fhd_fab* faceflux,
                      const fhd_fab* edgeflux, const fhd_fab* cenflux, const fhd_noise* injected, double dt,
                      int64_t step) {
    if (!c || !mom || !vel || !(dt > 0)) return FHD_ERR_BAD_ARG;
    const int ns = c->prm.nspecies, nvars = 5 + ns, nprim = 6 + 2 * ns;
    const bool mixed = c->prm.precision == FHD_PREC_MIXED;
    if (!fab_ok(c, cu, CELLN, NGC, nvars, FHD_F64) || !fab_ok(c, prim, CELLN, NGC, nprim, FHD_F64)) return FHD_ERR_BAD_ARG;
    for (int d = 0; d < 3; ++d)
        if (!fab_ok(c, mom[d], FACEN[d], NGC, 1, FHD_F64) || !fab_ok(c, vel[d], FACEN[d], NGC, 1, FHD_F64))
            return FHD_ERR_BAD_ARG;
    if (source.data && !fab_ok(c, source, CELLN, 0, nvars, FHD_F64)) return FHD_ERR_BAD_ARG;
    if (c->refpipe && !walls_ghosts_ok(cu, mom, prim, vel)) return FHD_ERR_BAD_ARG;
    const bool aux_coef = eta.data != nullptr;
    if (aux_coef) {
        if (mixed) return FHD_ERR_UNSUPPORTED;
        if (!fab_ok(c, eta, CELLN, 1, 1, FHD_F64) || !fab_ok(c, zeta, CELLN, 1, 1, FHD_F64) ||
            !fab_ok(c, kappa, CELLN, 1, 1, FHD_F64) || !fab_ok(c, chi, CELLN, 1, ns, FHD_F64) ||
            !fab_ok(c, D, CELLN, 1, ns * ns, FHD_F64))
            return FHD_ERR_BAD_ARG;
    }
    const bool aux_flux = faceflux && edgeflux && cenflux && faceflux[0].data;
    if (aux_flux) {
        if (mixed || !aux_coef) return FHD_ERR_UNSUPPORTED;
        for (int d = 0; d < 3; ++d)
            if (!fab_ok(c, faceflux[d], FACEN[d], 0, nvars + 4, FHD_F64, 0) || !fab_ok(c, cenflux[d], CELLN, 1, 1, FHD_F64, 1))
                return FHD_ERR_BAD_ARG;
        for (int e = 0; e < 6; ++e)
            if (!fab_ok(c, edgeflux[e], EFLUXN[e], 0, 1, FHD_F64, 0)) return FHD_ERR_BAD_ARG;
    }
    const bool stoch = c->prm.stoch_stress_form == 1;
    if (stoch && injected && !noise_ok(c, injected)) return FHD_ERR_BAD_ARG;
    if (injected && chem_noise_needed(c) && !chem_noise_ok(c, injected)) return FHD_ERR_BAD_ARG;
    if (source.data && c->prm.nreaction > 0 && !fab_ok(c, source, CELLN, 0, nvars, FHD_F64)) return FHD_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    int rc = ensure_scratch(c);
    if (rc) return rc;
    rc = ensure_coef(c, mixed ? FHD_F32 : FHD_F64);
    if (rc) return rc;
    rc = ensure_res(c);
    if (rc) return rc;
    return step_launches(c, cu, mom, prim, vel, source, eta, zeta, kappa, chi, D, faceflux, edgeflux, cenflux, injected,
                         dt, step, aux_coef, aux_flux, nullptr);
}

int fhd_rk3_steps_stag(fhd_ctx* c, fhd_fab cu, const fhd_fab mom[3], fhd_fab prim, const fhd_fab vel[3], double dt,
                       int64_t step0, int nsteps) {
    if (!c || !mom || !vel || !(dt > 0) || nsteps < 0) return FHD_ERR_BAD_ARG;
    const int ns = c->prm.nspecies, nvars = 5 + ns, nprim = 6 + 2 * ns;
    const bool mixed = c->prm.precision == FHD_PREC_MIXED;
    if (!fab_ok(c, cu, CELLN, NGC, nvars, FHD_F64) || !fab_ok(c, prim, CELLN, NGC, nprim, FHD_F64)) return FHD_ERR_BAD_ARG;
    for (int d = 0; d < 3; ++d)
        if (!fab_ok(c, mom[d], FACEN[d], NGC, 1, FHD_F64) || !fab_ok(c, vel[d], FACEN[d], NGC, 1, FHD_F64))
            return FHD_ERR_BAD_ARG;
    if (c->refpipe && !walls_ghosts_ok(cu, mom, prim, vel)) return FHD_ERR_BAD_ARG;
    if (nsteps == 0) return FHD_OK;
    cudaSetDevice(c->device);
    int rc = ensure_scratch(c);
    if (rc) return rc;
    rc = ensure_coef(c, mixed ? FHD_F32 : FHD_F64);
    if (rc) return rc;
    rc = ensure_res(c);
    if (rc) return rc;
    if (!c->d_step && cudaMalloc(&c->d_step, sizeof(uint64_t)) != cudaSuccess) {
        cudaGetLastError();
        c->d_step = nullptr;
        return FHD_ERR_OOM;
    }
    const fhd_fab none{};
    // what the captured launches embed: every pointer, layout, dt and the tile
    std::vector<uint64_t> key;
    auto add_fab = [&](const fhd_fab& f) {
        key.push_back((uint64_t)(uintptr_t)f.data);
        for (int d = 0; d < 3; ++d) key.push_back(((uint64_t)(uint32_t)f.lo[d] << 32) | (uint32_t)f.hi[d]);
    };
    add_fab(cu);
    add_fab(prim);
    for (int d = 0; d < 3; ++d) { add_fab(mom[d]); add_fab(vel[d]); }
    uint64_t dtb;
    std::memcpy(&dtb, &dt, sizeof(dtb));
    key.push_back(dtb);
    key.push_back((uint64_t)c->tile);
    key.push_back((uint64_t)(uintptr_t)c->scratch);
    key.push_back((uint64_t)(uintptr_t)c->coef);
    bool captured = c->sgexec && key == c->skey;
    if (!captured) {
        if (c->sgexec) cudaGraphExecDestroy(c->sgexec);
        if (c->sgraph) cudaGraphDestroy(c->sgraph);
        c->sgexec = nullptr;
        c->sgraph = nullptr;
        c->skey.clear();
        if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const bool prof = c->prof;
            c->prof = false;  // no timing events inside the graph
            rc = step_launches(c, cu, mom, prim, vel, none, none, none, none, none, none, nullptr, nullptr, nullptr,
                               nullptr, dt, step0, false, false, c->d_step);
            if (!rc) rc = steps_inc(c->d_step, 1, c->stream);
            c->prof = prof;
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
            if (!rc && e == cudaSuccess && cudaGraphInstantiate(&c->sgexec, g, 0) == cudaSuccess) {
                c->sgraph = g;
                c->skey = key;
                captured = true;
            } else {
                if (g) cudaGraphDestroy(g);
                c->sgexec = nullptr;
                cudaGetLastError();
                if (rc) return rc;
            }
        } else {
            cudaGetLastError();  // e.g. the legacy default stream: launch step by step below
        }
    }
    if (!captured) {
        for (int s = 0; s < nsteps && !rc; ++s)
            rc = step_launches(c, cu, mom, prim, vel, none, none, none, none, none, none, nullptr, nullptr, nullptr,
                               nullptr, dt, step0 + s, false, false, nullptr);
        return rc;
    }
    rc = steps_set(c->d_step, (uint64_t)step0, c->stream);
    for (int s = 0; s < nsteps && !rc; ++s)
        if (cudaGraphLaunch(c->sgexec, c->stream) != cudaSuccess) { cudaGetLastError(); rc = FHD_ERR_CUDA; }
    return rc;
}

int fhd_stats_stag(fhd_ctx* c, fhd_fab cu, fhd_fab prim, const fhd_fab vel[3], const fhd_fab mom[3],
                   const fhd_stats* st, int64_t steps, int flags) {
    if (!c || !mom || !st || steps < 1) return FHD_ERR_BAD_ARG;
    const bool means = flags & FHD_STATS_MEANS, vars = flags & FHD_STATS_VARS;
    if (vars && !means) return FHD_ERR_BAD_ARG;  // statsStag.cpp:38-39
    const int ns = c->prm.nspecies, nvars = 5 + ns, nprim = 6 + 2 * ns;
    if (!fab_ok(c, cu, CELLN, NGC, nvars, FHD_F64) || !fab_ok(c, prim, CELLN, 0, nprim, FHD_F64)) return FHD_ERR_BAD_ARG;
    for (int d = 0; d < 3; ++d) {
        if (!fab_ok(c, mom[d], FACEN[d], 0, 1, FHD_F64)) return FHD_ERR_BAD_ARG;
        if (!fab_ok(c, st->velMeans[d], FACEN[d], 0, 1, FHD_F64) || !fab_ok(c, st->cumomMeans[d], FACEN[d], 0, 1, FHD_F64))
            return FHD_ERR_BAD_ARG;
        if (vars && (!fab_ok(c, st->velVars[d], FACEN[d], 0, 1, FHD_F64) ||
                     !fab_ok(c, st->cumomVars[d], FACEN[d], 0, 1, FHD_F64)))
            return FHD_ERR_BAD_ARG;
    }
    if (!fab_ok(c, st->cuMeans, CELLN, NGC, nvars, FHD_F64) || !fab_ok(c, st->primMeans, CELLN, 0, nprim + 3, FHD_F64))
        return FHD_ERR_BAD_ARG;
    if (vars) {
        if (!fab_ok(c, st->cuVars, CELLN, 0, nvars, FHD_F64) || !fab_ok(c, st->primVars, CELLN, 0, nprim + 5, FHD_F64) ||
            !fab_ok(c, st->coVars, CELLN, 0, 26, FHD_F64))
            return FHD_ERR_BAD_ARG;
        if ((flags & FHD_STATS_MOM3) && !fab_ok(c, st->mom3, CELLN, 0, nvars + 1, FHD_F64)) return FHD_ERR_BAD_ARG;
        if ((flags & FHD_STATS_MOM4) && !fab_ok(c, st->mom4, CELLN, 0, nvars + 1, FHD_F64)) return FHD_ERR_BAD_ARG;
    }
    const bool cross = (flags & FHD_STATS_CROSS) && !c->prm.do_2D;
    const bool cross1d = cross && c->prm.do_1D;
    // the x* (statsStag.cpp:168-193): cross_cell, or the five equidistant ones with all_correl in 1-D
    int stars[5] = {c->prm.cross_cell, 0, 0, 0, 0};
    int nstars = 1;
    if (cross1d && c->prm.all_correl == 1) {
        const int n0 = c->prm.n_cells[0];
        stars[0] = 0;
        stars[1] = (int)std::floor(1.0 * n0 / 4.0);
        stars[2] = (int)std::floor(2.0 * n0 / 4.0);
        stars[3] = (int)std::floor(3.0 * n0 / 4.0);
        stars[4] = n0 - 1;
        nstars = 5;
    }
    if (cross) {
        // main_driver.cpp:249-251
        if (c->prm.cross_cell < 0 || c->prm.cross_cell > c->prm.n_cells[0] - 1) return FHD_ERR_BAD_ARG;
        if (!st->spatialCross || (!cross1d && !st->dataSliceMeans_xcross)) return FHD_ERR_BAD_ARG;
        if (cross1d) {
            // the 1-D correlations read vel x and the face momentum / velocity means
            for (int d = 0; d < 3; ++d)
                if (!vel || !fab_ok(c, vel[d], FACEN[d], 0, 1, FHD_F64)) return FHD_ERR_BAD_ARG;
        }
    }
    cudaSetDevice(c->device);
    if (cross && !cross1d) {
        const size_t need = (size_t)stats_line_doubles(ns, c->prm.n_cells[0]) * sizeof(double);
        if (c->lines_bytes < need) {
            if (c->lines) {
                if (cudaStreamSynchronize(c->stream) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_CUDA; }
                cudaFree(c->lines);
                c->lines = nullptr;
                c->lines_bytes = 0;
            }
            if (cudaMalloc(&c->lines, need) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_OOM; }
            c->lines_bytes = need;
        }
    }
    const DevParams P = make_dev(c, 1.0, 0);
    return exact_stats(P, cu, prim, vel, mom, *st, steps, cross ? flags : (flags & ~FHD_STATS_CROSS), stars, nstars,
                       c->lines, c->stream);
}

int fhd_spatial_cross_ncross(int nspecies) {
    return nspecies < 1 || nspecies > FHD_MAX_SPECIES ? FHD_ERR_BAD_ARG : 37 + nspecies + 3;
}
int fhd_spatial_cross_nstats(int nspecies) {
    return nspecies < 1 || nspecies > FHD_MAX_SPECIES ? FHD_ERR_BAD_ARG : 2 * (5 + nspecies) + 8 + 2 * nspecies;
}

int fhd_profile(fhd_ctx* c, int enable) {
    if (!c) return FHD_ERR_BAD_ARG;
    c->prof = enable != 0;
    return FHD_OK;
}

int fhd_profile_read(fhd_ctx* c, double* ms, int64_t* launches) {
    if (!c || !ms || !launches) return FHD_ERR_BAD_ARG;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_CUDA; }
    for (int k = 0; k < FHD_PROF_KINDS; ++k) { ms[k] = 0.0; launches[k] = 0; }
    for (size_t q = 0; q < c->nev; ++q) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, c->evs[q].a, c->evs[q].b) != cudaSuccess) { cudaGetLastError(); continue; }
        ms[c->evs[q].kind] += t;
        launches[c->evs[q].kind] += 1;
    }
    c->nev = 0;
    return FHD_OK;
}

int fhd_rk3_step_stag_host(fhd_ctx* c, fhd_fab cu, const fhd_fab mom[3], fhd_fab prim, const fhd_fab vel[3],
                           const fhd_noise* injected, double dt, int64_t step, int64_t* h2d_bytes,
                           int64_t* d2h_bytes) {
    if (!c || !mom || !vel) return FHD_ERR_BAD_ARG;
    const int ns = c->prm.nspecies;
    if (!fab_ok(c, cu, CELLN, NGC, 5 + ns, FHD_F64) || !fab_ok(c, prim, CELLN, NGC, 6 + 2 * ns, FHD_F64))
        return FHD_ERR_BAD_ARG;
    for (int d = 0; d < 3; ++d)
        if (!fab_ok(c, mom[d], FACEN[d], NGC, 1, FHD_F64) || !fab_ok(c, vel[d], FACEN[d], NGC, 1, FHD_F64))
            return FHD_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    // device mirrors with the caller's exact geometry
    const fhd_fab* hf[8] = {&cu, &mom[0], &mom[1], &mom[2], &prim, &vel[0], &vel[1], &vel[2]};
    size_t bytes[8], total = 0;
    for (int q = 0; q < 8; ++q) { bytes[q] = (size_t)fab_points(*hf[q]) * hf[q]->ncomp * sizeof(double); total += bytes[q]; }
    // injected reaction noises are not mirrored here (in-kernel reaction noise is)
    if (injected && chem_noise_needed(c)) return FHD_ERR_UNSUPPORTED;
    fhd_noise dn;
    std::memset(&dn, 0, sizeof(dn));
    size_t nzb = 0;
    const bool inj = injected && c->prm.stoch_stress_form == 1;
    if (inj) {
        if (!noise_ok(c, injected)) return FHD_ERR_BAD_ARG;
        for (int s = 0; s < 2; ++s)
            for (int d = 0; d < 3; ++d)
                nzb += (fab_points(injected->face[s][d]) * injected->face[s][d].ncomp + fab_points(injected->edge[s][d]) +
                        fab_points(injected->cen[s][d])) * sizeof(double);
    }
    if (!c->hbuf || c->hbuf_bytes < total + nzb) {
        if (c->hbuf) cudaFree(c->hbuf);
        c->hbuf = nullptr;
        if (cudaMalloc(&c->hbuf, total + nzb) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_OOM; }
        c->hbuf_bytes = total + nzb;
    }
    fhd_fab df[8];
    char* p = reinterpret_cast<char*>(c->hbuf);
    int64_t h2d = 0, d2h = 0;
    for (int q = 0; q < 8; ++q) {
        df[q] = *hf[q];
        df[q].data = p;
        // only cu and mom go up: the step derives prim and vel from them before
        // reading either, so the input prim/vel contents are dead
        if (q < 4) {
            if (cudaMemcpyAsync(p, hf[q]->data, bytes[q], cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
                return FHD_ERR_CUDA;
            h2d += (int64_t)bytes[q];
        }
        p += bytes[q];
    }
    if (inj) {
        auto mirror = [&](const fhd_fab& h, fhd_fab& d) -> int {
            const size_t b = (size_t)fab_points(h) * h.ncomp * sizeof(double);
            d = h;
            d.data = p;
            if (cudaMemcpyAsync(p, h.data, b, cudaMemcpyHostToDevice, c->stream) != cudaSuccess) return FHD_ERR_CUDA;
            h2d += (int64_t)b;
            p += b;
            return FHD_OK;
        };
        for (int s = 0; s < 2; ++s)
            for (int d = 0; d < 3; ++d)
                if (mirror(injected->face[s][d], dn.face[s][d]) || mirror(injected->edge[s][d], dn.edge[s][d]) ||
                    mirror(injected->cen[s][d], dn.cen[s][d]))
                    return FHD_ERR_CUDA;
    }
    fhd_fab dmom[3] = {df[1], df[2], df[3]}, dvel[3] = {df[5], df[6], df[7]};
    fhd_fab nf;
    std::memset(&nf, 0, sizeof(nf));
    int rc = fhd_rk3_step_stag(c, df[0], dmom, df[4], dvel, nf, nf, nf, nf, nf, nf, nullptr, nullptr, nullptr,
                               inj ? &dn : nullptr, dt, step);
    if (rc) return rc;
    for (int q = 0; q < 8; ++q) {
        if (cudaMemcpyAsync(hf[q]->data, df[q].data, bytes[q], cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
            return FHD_ERR_CUDA;
        d2h += (int64_t)bytes[q];
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_CUDA; }
    if (h2d_bytes) *h2d_bytes = h2d;
    if (d2h_bytes) *d2h_bytes = d2h;
    return FHD_OK;
}

}  // extern "C"
