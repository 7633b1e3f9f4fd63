// fhd_sf.cu — static structure factor of cell-centred fields: the reference's
// StructFact (src_analysis/StructFact.cpp) for one periodic box.
//
// FortStructure (StructFact.cpp:231-311): for every variable that appears in a
// pair, a real-to-complex FFT over the box (cuFFT, D2Z; the reference uses
// amrex::FFT::R2C), the Hermitian half spectrum unpacked to the full grid and
// divided by sqrt(N) (ComputeFFT, :322-519), then for each pair (a, b)
//   cov_real += Re_a Re_b + Im_a Im_b,   cov_imag += -(Im_a Re_b) + Re_a Im_b.
// Here the unpacking is not materialised: one fused kernel reads both half
// spectra at the point or at its mirror (conjugated), applies the 1/sqrt(N) and
// accumulates every pair in place — one pass over the spectra and the
// accumulators per sample.
// CallFinalize / Finalize (:598-641) and ShiftFFT (:643-719): optional zeroing of
// k = 0, shift by N/2 in every direction, scaling by 1/nsamples and by
// 1/var_scaling, magnitude sqrt(re^2 + im^2).
//
// Stacks (the quasi-2-D runs' per-slice and the quasi-1-D runs' per-pencil
// StructFact vectors, main_driver.cpp:923-993): the members are independent
// structure factors of one shape; the dense copy of a variable holds them one
// after another, one batched cuFFT transforms them all, and the accumulators
// hold them one after another.  fhd_sf_stack_average fuses the reference's
// output loop (AddToExternal of every member, then the mult by 1/members).
//
// FP64 throughout; the accumulation and finalize arithmetic follow the
// reference's operation order (built with -fmad=false).  FFT values differ
// from another FFT library's at rounding level.
#include <cufft.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "fhd_launch.cuh"

using namespace fhd;

struct fhd_sf {
    int device = 0;
    int n[3] = {0, 0, 0};            // the box the variables fab covers
    int kind = FHD_SF_BOX;
    int m[3] = {0, 0, 0};            // one member's shape (the box itself unless a stack)
    int nmem = 1;                    // members
    int nvar = 0, ncov = 0;
    std::vector<int> pa, pb, varu;   // pairs (A, B) and the unique variables among them
    std::vector<double> scaling;     // 1 / var_scaling (StructFact.cpp:93-96)
    int64_t nsamples = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    double* cov = nullptr;           // [2][ncov][nmem][Nm]: real then imaginary accumulators
    double2* spec = nullptr;         // [nvaru][nmem][mz][my][mx/2+1] half spectra
    double* real = nullptr;          // [nmem][mz][my][mx] dense copy of one variable (FFT input)
    int* dpairs = nullptr;           // [2][ncov] pair -> unique-variable slot
    double* dscale = nullptr;        // [ncov]
    cufftHandle plan = 0;
    bool have_plan = false;
};

namespace {

struct SfArgs {
    int nx, ny, nz, nxh1, ncov;      // one member's shape
    int64_t N, half;                 // points and half-spectrum entries of all members
    int64_t Nm, halfm;               // ... of one member
    double sqrtnpts;
    const double2* spec;
    const int* pairs;                // pa slots then pb slots
    double* cov;
    int reset;
};

// (re, im) of unique variable `v` at full-grid point (i, j, k): the stored half
// spectrum for i <= nx/2, else the conjugate at the mirror point
// (ComputeFFT's unpacking rule, StructFact.cpp:394-421), then divided by sqrt(N).
__device__ __forceinline__ void spec_at(const SfArgs& a, int v, int64_t b, int i, int j, int k, double& re,
                                        double& im) {
    const double2* S = a.spec + (int64_t)v * a.half + b * a.halfm;
    if (i <= a.nx / 2) {
        const double2 s = S[i + (int64_t)a.nxh1 * (j + (int64_t)a.ny * k)];
        re = s.x;
        im = s.y;
    } else {
        const int iloc = a.nx - i;
        const int jloc = (j == 0) ? 0 : a.ny - j;
        const int kloc = (k == 0) ? 0 : a.nz - k;
        const double2 s = S[iloc + (int64_t)a.nxh1 * (jloc + (int64_t)a.ny * kloc)];
        re = s.x;
        im = -s.y;
    }
    re /= a.sqrtnpts;
    im /= a.sqrtnpts;
}

__global__ void __launch_bounds__(256) k_sf_accumulate(SfArgs a) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < a.N; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = q / a.Nm, l = q - b * a.Nm;   // member, point within it
        const int i = int(l % a.nx), j = int((l / a.nx) % a.ny), k = int(l / ((int64_t)a.nx * a.ny));
        for (int c = 0; c < a.ncov; ++c) {
            double rA, iA, rB, iB;
            spec_at(a, a.pairs[c], b, i, j, k, rA, iA);
            spec_at(a, a.pairs[a.ncov + c], b, i, j, k, rB, iB);
            // cov_temp = 0 + Re_a Re_b; += Im_a Im_b   (StructFact.cpp:265-268)
            double tr = 0.0 + rA * rB;
            tr = tr + iA * iB;
            // cov_temp = 0 + Im_a Re_b; *= -1; += Re_a Im_b   (:276-280)
            double ti = 0.0 + iA * rB;
            ti = ti * -1.0;
            ti = ti + rA * iB;
            double* re = a.cov + (int64_t)c * a.N + q;
            double* imv = a.cov + ((int64_t)a.ncov + c) * a.N + q;
            if (a.reset) {
                *re = tr;
                *imv = ti;
            } else {
                *re = *re + tr;
                *imv = *imv + ti;
            }
        }
    }
}

struct SfFinArgs {
    int nx, ny, nz, ncov, zero_avg;
    int64_t N;
    double nsinv;
    const double* cov;
    const double* scale;
    Arr4<double> ore, oim, omag;
};

// Finalize (StructFact.cpp:598-620) with ShiftFFT (:643-719): destination point
// ((i + nx/2) % nx, ...) of source point (i, j, k).
__global__ void __launch_bounds__(256) k_sf_finalize(SfFinArgs a) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < a.N; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = int(q % a.nx), j = int((q / a.nx) % a.ny), k = int(q / ((int64_t)a.nx * a.ny));
        const int ip = (i + a.nx / 2) % a.nx, jp = (j + a.ny / 2) % a.ny, kp = (k + a.nz / 2) % a.nz;
        const bool zero = a.zero_avg == 1 && i == 0 && j == 0 && k == 0;
        for (int c = 0; c < a.ncov; ++c) {
            double re = zero ? 0.0 : a.cov[(int64_t)c * a.N + q];
            double im = zero ? 0.0 : a.cov[((int64_t)a.ncov + c) * a.N + q];
            re = re * a.nsinv;
            re = re * a.scale[c];
            im = im * a.nsinv;
            im = im * a.scale[c];
            double mag = 0.0 + re * re;
            mag = mag + im * im;
            a.ore(ip, jp, kp, c) = re;
            a.oim(ip, jp, kp, c) = im;
            a.omag(ip, jp, kp, c) = sqrt(mag);
        }
    }
}

struct SfAvgArgs {
    int nx, ny, nz, ncov, zero_avg;
    int64_t N, Nm, nmem;
    double nsinv, meminv;
    const double* cov;
    const double* scale;
    Arr4<double> omag, ori;
};

// The reference's stack output loop (main_driver.cpp:1592-1618, 1683-1711): for
// every member in order, AddToExternal (StructFact.cpp:979-1009: Finalize of a
// copy, then x_mag += mag, x_realimag += (re, im), from zero), then both outputs
// times 1/members.  One thread per (pair, member point): it owns that pair's
// shifted destination and walks the members in order (a pencil stack has only
// n_cells[0] points, so the pairs multiply the independent chains).
__global__ void __launch_bounds__(256) k_sf_stack_avg(SfAvgArgs a) {
    const int64_t tot = a.Nm * a.ncov;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
        const int c = int(t / a.Nm);
        const int64_t l = t - (int64_t)c * a.Nm;
        const int i = int(l % a.nx), j = int((l / a.nx) % a.ny), k = int(l / ((int64_t)a.nx * a.ny));
        const int ip = (i + a.nx / 2) % a.nx, jp = (j + a.ny / 2) % a.ny, kp = (k + a.nz / 2) % a.nz;
        const bool zero = a.zero_avg == 1 && i == 0 && j == 0 && k == 0;
        {
            double sm = 0.0, sr = 0.0, si = 0.0;
            for (int64_t b = 0; b < a.nmem; ++b) {
                const int64_t q = b * a.Nm + l;
                double re = zero ? 0.0 : a.cov[(int64_t)c * a.N + q];
                double im = zero ? 0.0 : a.cov[((int64_t)a.ncov + c) * a.N + q];
                re = re * a.nsinv;
                re = re * a.scale[c];
                im = im * a.nsinv;
                im = im * a.scale[c];
                double mag = 0.0 + re * re;
                mag = mag + im * im;
                sm = sm + sqrt(mag);
                sr = sr + re;
                si = si + im;
            }
            a.omag(ip, jp, kp, c) = sm * a.meminv;
            a.ori(ip, jp, kp, c) = sr * a.meminv;
            a.ori(ip, jp, kp, a.ncov + c) = si * a.meminv;
        }
    }
}

}  // namespace

namespace {

int shape_fab_ok(const int n[3], const fhd_fab& f, int min_nc) {
    if (!f.data || f.dtype != FHD_F64 || f.ncomp < min_nc) return 0;
    const int g = -f.lo[0];
    if (g < 0) return 0;
    for (int d = 0; d < 3; ++d)
        if (f.nodal[d] != 0 || f.lo[d] != -g || f.hi[d] != n[d] - 1 + g) return 0;
    return 1;
}
int sf_fab_ok(const fhd_sf* s, const fhd_fab& f, int min_nc) { return shape_fab_ok(s->n, f, min_nc); }

int cufft_rc(cufftResult r) { return r == CUFFT_SUCCESS ? FHD_OK : FHD_ERR_CUDA; }

// Dense D2Z plan over the box (slowest dimension first: cuFFT is row-major),
// writing the packed half spectrum nz x ny x (nx/2+1).  Its input is a dense,
// aligned copy of one variable: cuFFT rejects an input pointer into a
// ghost-inclusive fab whose valid region starts off a 16-byte boundary.
// A stack: one plan of nmem transforms (2-D over a slice, 1-D over a pencil),
// members contiguous in the dense copy and in the half spectra.
int sf_plan(fhd_sf* s) {
    if (s->have_plan) return FHD_OK;
    int rc;
    if (s->kind == FHD_SF_BOX) {
        rc = cufft_rc(cufftPlan3d(&s->plan, s->n[2], s->n[1], s->n[0], CUFFT_D2Z));
    } else if (s->kind == FHD_SF_Z_SLICES) {
        int dims[2] = {s->m[1], s->m[0]}, oemb[2] = {s->m[1], s->m[0] / 2 + 1};
        rc = cufft_rc(cufftPlanMany(&s->plan, 2, dims, dims, 1, s->m[0] * s->m[1], oemb, 1,
                                    s->m[1] * (s->m[0] / 2 + 1), CUFFT_D2Z, s->nmem));
    } else {
        int dims[1] = {s->m[0]}, oemb[1] = {s->m[0] / 2 + 1};
        rc = cufft_rc(cufftPlanMany(&s->plan, 1, dims, dims, 1, s->m[0], oemb, 1, s->m[0] / 2 + 1, CUFFT_D2Z,
                                    s->nmem));
    }
    if (rc) return rc;
    rc = cufft_rc(cufftSetStream(s->plan, s->stream));
    if (rc) {
        cufftDestroy(s->plan);
        return rc;
    }
    s->have_plan = true;
    return FHD_OK;
}

// dense copy of one component; x pencils in the reference's member order
// (member p at y = p / ny, z = p % ny, ExtractXPencil's arguments in
// main_driver.cpp:1551), everything else in the box's own order
__global__ void __launch_bounds__(256) k_sf_pack(Arr4<const double> v, int comp, int nx, int ny, int64_t N,
                                                 int pencils, double* __restrict__ out) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x) {
        if (pencils) {
            const int64_t p = q / nx;
            out[q] = v(int(q - p * nx), int(p / ny), int(p % ny), comp);
        } else {
            const int i = int(q % nx), j = int((q / nx) % ny), k = int(q / ((int64_t)nx * ny));
            out[q] = v(i, j, k, comp);
        }
    }
}

}  // namespace

extern "C" {

int fhd_sf_create(fhd_sf** out, const int n_cells[3], int nvar, int ncov, const int* pairA, const int* pairB,
                  const double* var_scaling, int device) {
    return fhd_sf_create_stack(out, n_cells, FHD_SF_BOX, nvar, ncov, pairA, pairB, var_scaling, device);
}

int fhd_sf_create_stack(fhd_sf** out, const int n_cells[3], int kind, int nvar, int ncov, const int* pairA,
                        const int* pairB, const double* var_scaling, int device) {
    if (!out || !n_cells || nvar < 1 || !var_scaling) return FHD_ERR_BAD_ARG;
    if (kind != FHD_SF_BOX && kind != FHD_SF_Z_SLICES && kind != FHD_SF_X_PENCILS) return FHD_ERR_BAD_ARG;
    for (int d = 0; d < 3; ++d)
        if (n_cells[d] < (kind == FHD_SF_BOX || d == 0 ? 2 : 1)) return FHD_ERR_BAD_ARG;
    if (kind == FHD_SF_Z_SLICES && n_cells[1] < 2) return FHD_ERR_BAD_ARG;
    if (kind == FHD_SF_X_PENCILS && n_cells[1] != n_cells[2]) return FHD_ERR_UNSUPPORTED;
    fhd_sf* s = new (std::nothrow) fhd_sf;
    if (!s) return FHD_ERR_OOM;
    s->device = device;
    s->kind = kind;
    for (int d = 0; d < 3; ++d) s->n[d] = s->m[d] = n_cells[d];
    if (kind == FHD_SF_Z_SLICES) {
        s->m[2] = 1;
        s->nmem = n_cells[2];
    } else if (kind == FHD_SF_X_PENCILS) {
        s->m[1] = s->m[2] = 1;
        s->nmem = n_cells[1] * n_cells[2];
    }
    s->nvar = nvar;
    if (!pairA || !pairB) {
        // all NVAR (NVAR + 1) / 2 pairs: A = j, B = i for i <= j (StructFact.cpp:45-69)
        for (int i = 0; i < nvar; ++i)
            for (int j = i; j < nvar; ++j) {
                s->pa.push_back(j);
                s->pb.push_back(i);
            }
    } else {
        for (int c = 0; c < ncov; ++c) {
            if (pairA[c] < 0 || pairA[c] >= nvar || pairB[c] < 0 || pairB[c] >= nvar) {
                delete s;
                return FHD_ERR_BAD_ARG;  // StructFact.cpp:186-190
            }
            s->pa.push_back(pairA[c]);
            s->pb.push_back(pairB[c]);
        }
    }
    s->ncov = (int)s->pa.size();
    if (s->ncov < 1) {
        delete s;
        return FHD_ERR_BAD_ARG;
    }
    for (int c = 0; c < s->ncov; ++c) s->scaling.push_back(1.0 / var_scaling[c]);
    // unique variables, ascending (StructFact.cpp:100-152)
    std::vector<int> used(nvar, 0);
    for (int c = 0; c < s->ncov; ++c) used[s->pa[c]] = used[s->pb[c]] = 1;
    std::vector<int> slot(nvar, -1);
    for (int v = 0; v < nvar; ++v)
        if (used[v]) {
            slot[v] = (int)s->varu.size();
            s->varu.push_back(v);
        }
    std::vector<int> hp(2 * s->ncov);
    for (int c = 0; c < s->ncov; ++c) {
        hp[c] = slot[s->pa[c]];
        hp[s->ncov + c] = slot[s->pb[c]];
    }
    const int64_t N = (int64_t)s->n[0] * s->n[1] * s->n[2];
    const int64_t half = (int64_t)(s->m[0] / 2 + 1) * s->m[1] * s->m[2] * s->nmem;
    int rc = FHD_OK;
    if (cudaSetDevice(device) != cudaSuccess) rc = FHD_ERR_CUDA;
    if (!rc && cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) rc = FHD_ERR_CUDA;
    if (!rc) s->own_stream = true;
    if (!rc && (cudaMalloc(&s->cov, sizeof(double) * 2 * s->ncov * N) != cudaSuccess ||
                cudaMalloc(&s->spec, sizeof(double2) * s->varu.size() * half) != cudaSuccess ||
                cudaMalloc(&s->real, sizeof(double) * N) != cudaSuccess ||
                cudaMalloc(&s->dpairs, sizeof(int) * hp.size()) != cudaSuccess ||
                cudaMalloc(&s->dscale, sizeof(double) * s->ncov) != cudaSuccess))
        rc = FHD_ERR_OOM;
    if (!rc && (cudaMemcpy(s->dpairs, hp.data(), sizeof(int) * hp.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(s->dscale, s->scaling.data(), sizeof(double) * s->ncov, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemset(s->cov, 0, sizeof(double) * 2 * s->ncov * N) != cudaSuccess))
        rc = FHD_ERR_CUDA;
    if (rc) {
        cudaGetLastError();
        fhd_sf_destroy(s);
        return rc;
    }
    *out = s;
    return FHD_OK;
}

int fhd_sf_destroy(fhd_sf* s) {
    if (!s) return FHD_ERR_BAD_ARG;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->have_plan) cufftDestroy(s->plan);
    cudaFree(s->cov);
    cudaFree(s->spec);
    cudaFree(s->real);
    cudaFree(s->dpairs);
    cudaFree(s->dscale);
    if (s->own_stream) cudaStreamDestroy(s->stream);
    delete s;
    return FHD_OK;
}

int fhd_sf_set_stream(fhd_sf* s, void* stream) {
    if (!s) return FHD_ERR_BAD_ARG;
    if (s->own_stream) {
        cudaStreamSynchronize(s->stream);
        cudaStreamDestroy(s->stream);
        s->own_stream = false;
    }
    s->stream = static_cast<cudaStream_t>(stream);
    if (s->have_plan) return cufft_rc(cufftSetStream(s->plan, s->stream));
    return FHD_OK;
}

int fhd_sf_ncov(const fhd_sf* s) { return s ? s->ncov : -1; }
int64_t fhd_sf_nsamples(const fhd_sf* s) { return s ? s->nsamples : -1; }

int fhd_sf_fort_structure(fhd_sf* s, fhd_fab variables, int reset) {
    if (!s || !sf_fab_ok(s, variables, s->nvar)) return FHD_ERR_BAD_ARG;
    cudaSetDevice(s->device);
    int rc = sf_plan(s);
    if (rc) return rc;
    const Arr4<const double> v = view<const double>(variables);
    const int64_t N = (int64_t)s->n[0] * s->n[1] * s->n[2];
    const int64_t halfm = (int64_t)(s->m[0] / 2 + 1) * s->m[1] * s->m[2], half = halfm * s->nmem;
    for (size_t u = 0; u < s->varu.size(); ++u) {
        k_sf_pack<<<grid_for(N, 256), 256, 0, s->stream>>>(v, s->varu[u], s->n[0], s->n[1], N,
                                                          s->kind == FHD_SF_X_PENCILS ? 1 : 0, s->real);
        rc = cuda_rc(cudaGetLastError());
        if (rc) return rc;
        rc = cufft_rc(cufftExecD2Z(s->plan, s->real, reinterpret_cast<cufftDoubleComplex*>(s->spec + u * half)));
        if (rc) return rc;
    }
    SfArgs a;
    a.nx = s->m[0];
    a.ny = s->m[1];
    a.nz = s->m[2];
    a.nxh1 = s->m[0] / 2 + 1;
    a.ncov = s->ncov;
    a.N = N;
    a.half = half;
    a.Nm = (int64_t)s->m[0] * s->m[1] * s->m[2];
    a.halfm = halfm;
    a.sqrtnpts = std::sqrt((double)a.Nm);  // StructFact.cpp:348-350, over one member's box
    a.spec = s->spec;
    a.pairs = s->dpairs;
    a.cov = s->cov;
    a.reset = (reset == 1 || s->nsamples == 0) ? 1 : 0;
    k_sf_accumulate<<<grid_for(a.N, 256), 256, 0, s->stream>>>(a);
    rc = cuda_rc(cudaGetLastError());
    if (rc) return rc;
    s->nsamples = (reset == 1) ? 1 : s->nsamples + 1;  // :307-311
    return FHD_OK;
}

int fhd_sf_finalize(fhd_sf* s, fhd_fab cov_real, fhd_fab cov_imag, fhd_fab cov_mag, int zero_avg) {
    if (!s || s->nsamples < 1 || s->kind != FHD_SF_BOX) return FHD_ERR_BAD_ARG;
    if (!sf_fab_ok(s, cov_real, s->ncov) || !sf_fab_ok(s, cov_imag, s->ncov) || !sf_fab_ok(s, cov_mag, s->ncov))
        return FHD_ERR_BAD_ARG;
    cudaSetDevice(s->device);
    SfFinArgs a;
    a.nx = s->n[0];
    a.ny = s->n[1];
    a.nz = s->n[2];
    a.ncov = s->ncov;
    a.zero_avg = zero_avg;
    a.N = (int64_t)s->n[0] * s->n[1] * s->n[2];
    a.nsinv = 1.0 / (double)s->nsamples;  // StructFact.cpp:603
    a.cov = s->cov;
    a.scale = s->dscale;
    a.ore = view<double>(cov_real);
    a.oim = view<double>(cov_imag);
    a.omag = view<double>(cov_mag);
    k_sf_finalize<<<grid_for(a.N, 256), 256, 0, s->stream>>>(a);
    return cuda_rc(cudaGetLastError());
}

int fhd_sf_stack_average(fhd_sf* s, fhd_fab mag, fhd_fab realimag, int zero_avg) {
    if (!s || s->nsamples < 1 || s->kind == FHD_SF_BOX) return FHD_ERR_BAD_ARG;
    if (!shape_fab_ok(s->m, mag, s->ncov) || !shape_fab_ok(s->m, realimag, 2 * s->ncov)) return FHD_ERR_BAD_ARG;
    cudaSetDevice(s->device);
    SfAvgArgs a;
    a.nx = s->m[0];
    a.ny = s->m[1];
    a.nz = s->m[2];
    a.ncov = s->ncov;
    a.zero_avg = zero_avg;
    a.Nm = (int64_t)s->m[0] * s->m[1] * s->m[2];
    a.nmem = s->nmem;
    a.N = a.Nm * a.nmem;
    a.nsinv = 1.0 / (double)s->nsamples;  // StructFact.cpp:603
    a.meminv = 1.0 / (double)s->nmem;     // ncellsinv (main_driver.cpp:1610, 1702)
    a.cov = s->cov;
    a.scale = s->dscale;
    a.omag = view<double>(mag);
    a.ori = view<double>(realimag);
    k_sf_stack_avg<<<grid_for(a.Nm * a.ncov, 256), 256, 0, s->stream>>>(a);
    return cuda_rc(cudaGetLastError());
}

int fhd_sf_synchronize(fhd_sf* s) {
    if (!s) return FHD_ERR_BAD_ARG;
    return cuda_rc(cudaStreamSynchronize(s->stream));
}

}  // extern "C"
