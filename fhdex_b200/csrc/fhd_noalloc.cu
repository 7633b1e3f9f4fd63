// fhd_noalloc.cu — RK3 step for callers that cannot allocate device memory.
//
// Who needs it: code that runs under a memory arena that owns all of the GPU's
// memory (an AMReX or application pool where a stray cudaMalloc fails or
// fragments the pool), framework callbacks that forbid allocation on their hot
// path, and latency-critical loops that cannot afford the device-wide
// synchronisation that cudaMalloc/cudaFree imply.  This entry point performs no
// cudaMalloc, cudaFree or other allocating call: its stage scratch is the
// file-scope array below, sized for small boxes.
//
// The array lives on every GPU that loads the library until the process exits.
// In host code its name is only a host-side stand-in, so the device address is
// obtained once per device with cudaGetSymbolAddress (on the first call made on
// that device, with that device current) and passed to the kernels.  All calls
// share the array and it keeps the last call's contents: the status word is
// cleared at the start of every call, and every other scratch element is
// written before it is read within a call.  Calls whose GPU work overlaps (other
// streams, other host threads) race on the array and must be serialised by the
// caller.
#include <cmath>
#include <cstring>
#include <mutex>

#include "fhd_host.h"

using namespace fhd;

namespace {

// 16 MiB: room for a 26^3 box with 4 species or a 29^3 box with 2 species
// (30x30x29 with 2 species leaves 48 KiB unused).
constexpr size_t kNoallocBytes = (size_t)16 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_dev_ptr[kMaxDevices] = {};

// Device address of the static scratch on the current device (looked up on the
// first call on each device).
int scratch_address(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_CUDA; }
    if (dev < 0 || dev >= kMaxDevices) return FHD_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_dev_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return FHD_ERR_CUDA;
        }
        g_dev_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_dev_ptr[dev];
    return FHD_OK;
}

int64_t points(const fhd_fab& f) {
    int64_t n = 1;
    for (int d = 0; d < 3; ++d) n *= (int64_t)(f.hi[d] - f.lo[d] + 1);
    return n;
}

fhd_fab box(const int n[3], const int nodal[3], int ng, int nc, int dtype) {
    fhd_fab f;
    f.data = nullptr;
    for (int d = 0; d < 3; ++d) {
        f.lo[d] = -ng;
        f.hi[d] = n[d] - 1 + nodal[d] + ng;
        f.nodal[d] = nodal[d];
    }
    f.ncomp = nc;
    f.dtype = dtype;
    return f;
}

// A caller's fab: FP64, at least min_nc components, the same ghost width g >= min_ng
// on every side (the kernels take each fab's own lo, as fhd_rk3_step_stag does).
bool same_geometry(const fhd_fab& f, const int n[3], const int nodal[3], int min_ng, int min_nc) {
    if (!f.data || f.dtype != FHD_F64 || f.ncomp < min_nc) return false;
    const int g = -f.lo[0];
    if (g < min_ng) return false;
    for (int d = 0; d < 3; ++d)
        if (f.lo[d] != -g || f.hi[d] != n[d] - 1 + nodal[d] + g || f.nodal[d] != nodal[d]) return false;
    return points(f) * f.ncomp < ((int64_t)1 << 31);
}

// Every caller fab must be device memory of the current device: the kernels
// run there and would otherwise mix two devices' memory.
bool on_current_device(const fhd_fab& f, int dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, f.data) != cudaSuccess) { cudaGetLastError(); return false; }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}

// carves fabs out of the static scratch, 256-byte aligned
struct Carver {
    unsigned char* base;
    size_t used = 0;
    bool carve(fhd_fab& f, size_t elem) {
        used = (used + 255) & ~(size_t)255;
        const size_t bytes = (size_t)points(f) * f.ncomp * elem;
        if (used + bytes > kNoallocBytes) return false;
        f.data = base ? base + used : nullptr;
        used += bytes;
        return true;
    }
};

}  // namespace

extern "C" int fhd_rk3_step_stag_noalloc(const fhd_params* params, fhd_fab cu, const fhd_fab mom[3], fhd_fab prim,
                                         const fhd_fab vel[3], double dt, int64_t step, void* stream,
                                         int* status) {
    if (!params || !mom || !vel || !(dt > 0)) return FHD_ERR_BAD_ARG;
    fhd_params p = *params;
    const int ns = p.nspecies;
    if (ns < 1 || ns > 4 || p.algorithm_type != 2 || p.transport_type != 1 || p.precision != FHD_PREC_FP64 ||
        (p.stoch_stress_form != 0 && p.stoch_stress_form != 1) || p.advection_type < -1 || p.advection_type > 2 ||
        ((p.visc_type == 3 || p.visc_type == -3) && p.zeta_ratio < 0) || p.nreaction != 0 || reference_order(p))
        return FHD_ERR_UNSUPPORTED;
    for (int d = 0; d < 3; ++d)
        if (p.n_cells[d] < 2 || !(p.prob_hi[d] > p.prob_lo[d])) return FHD_ERR_BAD_ARG;
    const int* n = p.n_cells;
    const int cell[3] = {0, 0, 0}, all[3] = {1, 1, 1};
    const int face[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    if (!same_geometry(cu, n, cell, 2, 5 + ns) || !same_geometry(prim, n, cell, 2, 6 + 2 * ns)) return FHD_ERR_BAD_ARG;
    for (int d = 0; d < 3; ++d)
        if (!same_geometry(mom[d], n, face[d], 2, 1) || !same_geometry(vel[d], n, face[d], 2, 1))
            return FHD_ERR_BAD_ARG;
    {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_CUDA; }
        const fhd_fab* own[8] = {&cu, &prim, &mom[0], &mom[1], &mom[2], &vel[0], &vel[1], &vel[2]};
        for (const fhd_fab* f : own)
            if (!on_current_device(*f, dev)) return FHD_ERR_BAD_ARG;
    }

    // scratch layout (sizes only first: reject what does not fit before touching the GPU)
    fhd_fab st = box(n, cell, 0, 1, FHD_F64);   // status word
    st.hi[0] = st.hi[1] = st.hi[2] = 0;
    fhd_fab cup = box(n, cell, 2, 5 + ns, FHD_F64), cup2 = cup;
    fhd_fab cupm[3], cup2m[3];
    for (int d = 0; d < 3; ++d) cupm[d] = cup2m[d] = box(n, face[d], 2, 1, FHD_F64);
    fhd_fab eta = box(n, cell, 2, 1, FHD_F64), zeta = eta, kappa = eta;
    fhd_fab chi = box(n, cell, 2, ns, FHD_F64), D = box(n, cell, 2, ns * ns, FHD_F64);
    fhd_fab ct = box(n, cell, 1, 6, FHD_F64), et = box(n, all, 0, 6, FHD_F64);
    fhd_fab sff[3];
    for (int d = 0; d < 3; ++d) sff[d] = box(n, all, 0, 2 + ns, FHD_F64);
    fhd_fab smc = box(n, cell, 1, 3, FHD_F64), sme = box(n, all, 0, 6, FHD_F64);
    fhd_fab* parts[] = {&st, &cup, &cup2, &cupm[0], &cupm[1], &cupm[2], &cup2m[0], &cup2m[1], &cup2m[2], &eta,
                        &zeta, &kappa, &chi, &D, &ct, &et, &sff[0], &sff[1], &sff[2], &smc, &sme};
    {
        Carver dry{nullptr};
        for (fhd_fab* f : parts)
            if (!dry.carve(*f, sizeof(double))) return FHD_ERR_TOO_LARGE;
    }
    unsigned char* base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    Carver cv{base};
    for (fhd_fab* f : parts) cv.carve(*f, sizeof(double));
    int* dstatus = static_cast<int*>(st.data);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(dstatus, 0, sizeof(int), s) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_CUDA; }

    // device parameters: GetHcGas and the host-side constants of the transport model
    for (int i = 0; i < ns; ++i) {
        if (p.hcv[i] < 0.) p.hcv[i] = 0.5 * p.dof[i] * p.Runiv / p.molmass[i];
        if (p.hcp[i] < 0.) p.hcp[i] = 0.5 * (2. + p.dof[i]) * p.Runiv / p.molmass[i];
    }
    StageCall sc;
    std::memset(&sc, 0, sizeof(sc));
    sc.P = dev_params(p, dt, (uint64_t)step);
    sc.mode = p.stoch_stress_form == 1 ? NM_PHILOX : NM_OFF;
    sc.pr = prim;
    sc.pT = 4;
    sc.cons0 = cu;
    for (int d = 0; d < 3; ++d) {
        sc.vel[d] = vel[d];
        sc.mom0[d] = mom[d];
        sc.sff[d] = sff[d];
    }
    sc.eta = eta; sc.zeta = zeta; sc.kappa = kappa; sc.chi = chi; sc.D = D;
    sc.ct = ct;
    sc.et = et;
    sc.smc = smc;
    sc.sme = sme;
    sc.status = dstatus;
    sc.stream = s;
    sc.tile = 0;
    const double w[3] = {(2.0 * std::sqrt(2.0) + 1.0 * std::sqrt(3.0)) / 5.0,
                         (-4.0 * std::sqrt(2.0) + 3.0 * std::sqrt(3.0)) / 5.0,
                         (1.0 * std::sqrt(2.0) - 2.0 * std::sqrt(3.0)) / 10.0};
    const fhd_fab* ins[3] = {&cu, &cup, &cup2};
    const fhd_fab* insm[3] = {mom, cupm, cup2m};
    const fhd_fab* outs[3] = {&cup, &cup2, &cu};
    const fhd_fab* outsm[3] = {cupm, cup2m, mom};
    for (int k = 0; k < 3 && !rc; ++k) {
        sc.stage = k + 1;
        sc.w = w[k];
        sc.cons_s = *ins[k];
        sc.cons_o = *outs[k];
        for (int d = 0; d < 3; ++d) { sc.mom_s[d] = insm[k][d]; sc.mom_o[d] = outsm[k][d]; }
        rc = exact_cellprep(sc);
        for (int part = 0; part < 3 && !rc; ++part) rc = exact_stage_part(sc, part);
        GhostReq g[5] = {{*outs[k], 0, 1}, {*outs[k], 4, 1 + ns}, {outsm[k][0], 0, 1}, {outsm[k][1], 0, 1},
                         {outsm[k][2], 0, 1}};
        if (!rc) rc = fill_ghosts(g, 5, n, s);
    }
    if (!rc) rc = exact_convert(sc.P, prim, vel, cu, mom, dstatus, s);
    if (!rc) {
        GhostReq g[5] = {{cu, 1, 3}, {prim, 0, 6 + 2 * ns}, {vel[0], 0, 1}, {vel[1], 0, 1}, {vel[2], 0, 1}};
        rc = fill_ghosts(g, 5, n, s);
    }
    if (rc) return rc;
    if (status) {
        if (cudaMemcpyAsync(status, dstatus, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            cudaGetLastError();
            return FHD_ERR_CUDA;
        }
    }
    return FHD_OK;
}

