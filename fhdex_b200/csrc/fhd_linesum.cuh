// fhd_linesum.cuh — sums of a field over the planes normal to one direction, in a
// fixed serial order, for the statistics' sumToLine (statsStag.cpp:56-69) and the
// plotfile's WriteHorizontalAverageToMF (ComputeAverages.cpp:96-190).
//
// Entry e of a line is the sum of n1 * n2 source values, inner index fastest, from
// 0.0, divided by n1 * n2: the order of the reference's serial loops, so that one
// entry is one dependent chain and the result is bitwise the reference's.  One
// thread owns one entry; a one-warp block takes 32 consecutive entries of one job
// (one source component).  The chains are few, so every value reaches shared
// memory through an asynchronous 8-byte copy (cp.async) issued kLineStages - 1
// batches of kLineRows values ahead of the additions; each thread reads only the
// shared-memory column its own copies wrote, so cp.async.wait_group alone orders it
// (no block barrier).  With few chains each warp runs alone on its SM sub-partition
// and its per-value instruction count sets the pace: a batch inside one inner run
// takes its 32 addresses as independent base + u * s1 products.
#pragma once
#include "fhd_launch.cuh"

namespace fhd {

constexpr int kMaxLineJobs = 2 * (5 + MAXS) + 2 * (MAXS + 4);
constexpr int kLineRows = 32, kLineStages = 12;   // 96 KiB of dynamic shared memory per one-warp block
constexpr int kLineSmem = kLineStages * kLineRows * 32 * (int)sizeof(double);

struct LineJob {
    const double* src;   // the source component at entry 0's first value
    double* dst;         // line entry 0
    int64_t lstride;     // source offset between consecutive entries
    int64_t s1, s2;      // inner and outer steps of an entry's sum
    int dstride;         // destination stride between consecutive entries
};
struct LineArgs {
    LineJob job[kMaxLineJobs];
    int njobs, lblocks, nlanes;   // jobs; one-warp blocks per job, ceil(nlanes / 32); entries per job
    int n1, n2;                   // inner and outer counts
};

FHD_D void cp_async8(double* dst, const double* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
FHD_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
FHD_D void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

static __global__ void __launch_bounds__(32) k_sum_to_line(const __grid_constant__ LineArgs a) {
    extern __shared__ __align__(16) double line_smem[];
    double(*buf)[kLineRows][32] = reinterpret_cast<double(*)[kLineRows][32]>(line_smem);
    const int lane = threadIdx.x;
    const int c = blockIdx.x / a.lblocks;
    const int e = (blockIdx.x - c * a.lblocks) * 32 + lane;
    if (c >= a.njobs) return;   // uniform over the block
    const bool on = e < a.nlanes;
    const LineJob& J = a.job[c];
    const double* p = J.src + (on ? (int64_t)e * J.lstride : 0);
    const int64_t rows = (int64_t)a.n1 * a.n2, wrap = J.s2 - (int64_t)a.n1 * J.s1;
    // the next value to copy: its index rq = outer * n1 + inner, its inner index and offset
    int64_t rq = 0, offq = 0;
    int jq = 0;
    auto issue = [&](int stage) {   // one group: the next kLineRows values (possibly none)
        if (jq + kLineRows <= a.n1 && rq + kLineRows <= rows) {
            const double* q = p + offq;
            if (on) {
#pragma unroll
                for (int u = 0; u < kLineRows; ++u) cp_async8(&buf[stage][u][lane], q + (int64_t)u * J.s1);
            }
            rq += kLineRows;
            offq += (int64_t)kLineRows * J.s1;
            jq += kLineRows;
            if (jq == a.n1) { jq = 0; offq += wrap; }
        } else {
            for (int u = 0; u < kLineRows; ++u) {
                if (on && rq < rows) cp_async8(&buf[stage][u][lane], p + offq);
                ++rq;
                offq += J.s1;
                if (++jq == a.n1) { jq = 0; offq += wrap; }
            }
        }
        cp_async_commit();
    };
#pragma unroll 1
    for (int st = 0; st < kLineStages - 1; ++st) issue(st);
    double acc = 0.0;
    const int64_t nbatch = (rows + kLineRows - 1) / kLineRows;
#pragma unroll 1
    for (int64_t b = 0; b < nbatch; ++b) {
        issue((int)((b + kLineStages - 1) % kLineStages));   // the stage batch b-1 used
        cp_async_wait<kLineStages - 1>();                    // batch b (group b) has landed
        const int st = (int)(b % kLineStages);
        const int64_t r0 = b * kLineRows;
        if (r0 + kLineRows <= rows) {
#pragma unroll
            for (int u = 0; u < kLineRows; ++u) acc += buf[st][u][lane];
        } else {
            for (int u = 0; r0 + u < rows; ++u) acc += buf[st][u][lane];
        }
    }
    cp_async_wait<0>();
    if (on) J.dst[(int64_t)e * J.dstride] = acc / (double)rows;
}

// The line job of component `comp` of fab f along direction dir: entries along dir,
// each summing its plane with the later of the two other directions outer and the
// earlier inner (the reference's k, j, i loop order restricted to the plane)
static inline LineJob line_job_dir(const fhd_fab& f, int comp, int dir, double* dst, int dstride) {
    const int64_t sx = f.hi[0] - f.lo[0] + 1, sy = sx * (f.hi[1] - f.lo[1] + 1);
    const int64_t sc = sy * (f.hi[2] - f.lo[2] + 1);
    const int64_t st[3] = {1, sx, sy};
    LineJob J;
    J.src = static_cast<const double*>(f.data) + comp * sc - f.lo[2] * sy - f.lo[1] * sx - f.lo[0];
    J.dst = dst;
    J.dstride = dstride;
    J.lstride = st[dir];
    const int inner = dir == 0 ? 1 : 0, outer = dir == 2 ? 1 : 2;
    J.s1 = st[inner];
    J.s2 = st[outer];
    return J;
}

// launches the jobs (all along `dir` of an n-cell box) on stream s
static inline int launch_line_sums(LineArgs& la, const int n[3], int dir, cudaStream_t s) {
    const int inner = dir == 0 ? 1 : 0, outer = dir == 2 ? 1 : 2;
    la.nlanes = n[dir];
    la.lblocks = (la.nlanes + 31) / 32;
    la.n1 = n[inner];
    la.n2 = n[outer];
    // on every call: the attribute belongs to the current device's copy of the kernel
    const cudaError_t e = cudaFuncSetAttribute(k_sum_to_line, cudaFuncAttributeMaxDynamicSharedMemorySize, kLineSmem);
    if (e != cudaSuccess) return cuda_rc(e);
    k_sum_to_line<<<(unsigned)(la.lblocks * la.njobs), 32, kLineSmem, s>>>(la);
    return cuda_rc(cudaGetLastError());
}

}  // namespace fhd
