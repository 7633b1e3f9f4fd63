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
    int n[3] = {0, 0, 0};
    int nvar = 0, ncov = 0;
    std::vector<int> pa, pb, varu;   // pairs (A, B) and the unique variables among them
    std::vector<double> scaling;     // 1 / var_scaling (StructFact.cpp:93-96)
    int64_t nsamples = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    double* cov = nullptr;           // [2][ncov][N]: real then imaginary accumulators
    double2* spec = nullptr;         // [nvaru][nz][ny][nx/2+1] half spectra
    double* real = nullptr;          // [nz][ny][nx] dense copy of one variable (FFT input)
    int* dpairs = nullptr;           // [2][ncov] pair -> unique-variable slot
    double* dscale = nullptr;        // [ncov]
    cufftHandle plan = 0;
    bool have_plan = false;
};

namespace {

struct SfArgs {
    int nx, ny, nz, nxh1, ncov;
    int64_t N, half;
    double sqrtnpts;
    const double2* spec;
    const int* pairs;                // pa slots then pb slots
    double* cov;
    int reset;
};

// (re, im) of unique variable `v` at full-grid point (i, j, k): the stored half
// spectrum for i <= nx/2, else the conjugate at the mirror point
// (ComputeFFT's unpacking rule, StructFact.cpp:394-421), then divided by sqrt(N).
__device__ __forceinline__ void spec_at(const SfArgs& a, int v, int i, int j, int k, double& re, double& im) {
    const double2* S = a.spec + (int64_t)v * a.half;
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
        const int i = int(q % a.nx), j = int((q / a.nx) % a.ny), k = int(q / ((int64_t)a.nx * a.ny));
        for (int c = 0; c < a.ncov; ++c) {
            double rA, iA, rB, iB;
            spec_at(a, a.pairs[c], i, j, k, rA, iA);
            spec_at(a, a.pairs[a.ncov + c], i, j, k, rB, iB);
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

}  // namespace

namespace {

int sf_fab_ok(const fhd_sf* s, const fhd_fab& f, int min_nc) {
    if (!f.data || f.dtype != FHD_F64 || f.ncomp < min_nc) return 0;
    const int g = -f.lo[0];
    if (g < 0) return 0;
    for (int d = 0; d < 3; ++d)
        if (f.nodal[d] != 0 || f.lo[d] != -g || f.hi[d] != s->n[d] - 1 + g) return 0;
    return 1;
}

int cufft_rc(cufftResult r) { return r == CUFFT_SUCCESS ? FHD_OK : FHD_ERR_CUDA; }

// Dense D2Z plan over the box (slowest dimension first: cuFFT is row-major),
// writing the packed half spectrum nz x ny x (nx/2+1).  Its input is a dense,
// aligned copy of one variable: cuFFT rejects an input pointer into a
// ghost-inclusive fab whose valid region starts off a 16-byte boundary.
int sf_plan(fhd_sf* s) {
    if (s->have_plan) return FHD_OK;
    int rc = cufft_rc(cufftPlan3d(&s->plan, s->n[2], s->n[1], s->n[0], CUFFT_D2Z));
    if (rc) return rc;
    rc = cufft_rc(cufftSetStream(s->plan, s->stream));
    if (rc) {
        cufftDestroy(s->plan);
        return rc;
    }
    s->have_plan = true;
    return FHD_OK;
}

__global__ void __launch_bounds__(256) k_sf_pack(Arr4<const double> v, int comp, int nx, int ny, int64_t N,
                                                 double* __restrict__ out) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = int(q % nx), j = int((q / nx) % ny), k = int(q / ((int64_t)nx * ny));
        out[q] = v(i, j, k, comp);
    }
}

}  // namespace

extern "C" {

int fhd_sf_create(fhd_sf** out, const int n_cells[3], int nvar, int ncov, const int* pairA, const int* pairB,
                  const double* var_scaling, int device) {
    if (!out || !n_cells || nvar < 1 || !var_scaling) return FHD_ERR_BAD_ARG;
    for (int d = 0; d < 3; ++d)
        if (n_cells[d] < 2) return FHD_ERR_BAD_ARG;
    fhd_sf* s = new (std::nothrow) fhd_sf;
    if (!s) return FHD_ERR_OOM;
    s->device = device;
    for (int d = 0; d < 3; ++d) s->n[d] = n_cells[d];
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
    const int64_t half = (int64_t)(s->n[0] / 2 + 1) * s->n[1] * s->n[2];
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
    const int64_t half = (int64_t)(s->n[0] / 2 + 1) * s->n[1] * s->n[2];
    for (size_t u = 0; u < s->varu.size(); ++u) {
        k_sf_pack<<<grid_for(N, 256), 256, 0, s->stream>>>(v, s->varu[u], s->n[0], s->n[1], N, s->real);
        rc = cuda_rc(cudaGetLastError());
        if (rc) return rc;
        rc = cufft_rc(cufftExecD2Z(s->plan, s->real, reinterpret_cast<cufftDoubleComplex*>(s->spec + u * half)));
        if (rc) return rc;
    }
    SfArgs a;
    a.nx = s->n[0];
    a.ny = s->n[1];
    a.nz = s->n[2];
    a.nxh1 = s->n[0] / 2 + 1;
    a.ncov = s->ncov;
    a.N = (int64_t)s->n[0] * s->n[1] * s->n[2];
    a.half = half;
    a.sqrtnpts = std::sqrt((double)a.N);  // StructFact.cpp:350-352
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
    if (!s || s->nsamples < 1) return FHD_ERR_BAD_ARG;
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

int fhd_sf_synchronize(fhd_sf* s) {
    if (!s) return FHD_ERR_BAD_ARG;
    return cuda_rc(cudaStreamSynchronize(s->stream));
}

}  // extern "C"
