// fhd_peak.cu — FMA throughput microbenchmark (FP64 and FP32), the compute
// denominator of the step's roofline next to the measured HBM copy bandwidth.
//
// Each thread runs 8 independent fma chains (enough to cover the FMA pipe's
// latency at full occupancy); the grid is a whole number of waves (resident
// blocks per SM x SM count).  The kernel is timed with CUDA events on its own
// stream after a warm-up launch; clocks and power settings are left alone.
// No reference counterpart.
#include <cuda_runtime.h>

#include "fhd_capi.h"

namespace {

template <class T>
__global__ void __launch_bounds__(256) k_fma_chains(T* sink, int iters, T a, T b) {
    T x0 = T(threadIdx.x) * T(1e-7), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
    T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    const T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (sink && s == T(-1.2345e-30)) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;  // never true; keeps the chains live
}

template <class T>
int measure(int device, double* tflops) {
    if (!tflops) return FHD_ERR_BAD_ARG;
    if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_CUDA; }
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fma_chains<T>, 256, 0) != cudaSuccess) {
        cudaGetLastError();
        return FHD_ERR_CUDA;
    }
    const int blocks = sms * (per_sm > 0 ? per_sm : 1);
    const int iters = 4096;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = FHD_OK;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        rc = FHD_ERR_CUDA;
    } else {
        const T a = T(0.999999), b = T(1e-6);
        float best = 0.f;
        k_fma_chains<T><<<blocks, 256, 0, s>>>(nullptr, iters, a, b);  // warm-up
        for (int rep = 0; rep < 5 && rc == FHD_OK; ++rep) {
            cudaEventRecord(e0, s);
            k_fma_chains<T><<<blocks, 256, 0, s>>>(nullptr, iters, a, b);
            cudaEventRecord(e1, s);
            float ms = 0.f;
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                rc = FHD_ERR_CUDA;
                break;
            }
            if (best == 0.f || ms < best) best = ms;
        }
        if (rc == FHD_OK) {
            const double flops = 2.0 * 8.0 * 4.0 * (double)iters * (double)blocks * 256.0;
            *tflops = flops / (best * 1e-3) / 1e12;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    if (rc != FHD_OK) cudaGetLastError();
    return rc;
}

}  // namespace

extern "C" int fhd_measure_fma_peak(int device, int fp64, double* tflops) {
    return fp64 ? measure<double>(device, tflops) : measure<float>(device, tflops);
}
