// fhd_chem.cu — the chemistry source kernel (compute_compressible_chemistry_source_CLE,
// chemistry_functions.cpp:128-193) and its launcher.  Built with -fmad=false: every
// product and sum is rounded on its own, as the host C++ evaluates it.
//
// One thread per valid cell, grid-stride.  Per cell it reads p, T and the NS mole
// fractions, draws (or reads) the nreaction noises and writes the NS species
// components of the source: (2 + NS) + NS doubles of HBM traffic, plus 2 x
// nreaction noise doubles when the A/B fields are injected.
#include "fhd_chem.cuh"
#include "fhd_launch.cuh"

namespace fhd {

struct ChemArgs {
    DevParams P;
    ChemParams C;
    Arr4<const double> pr;   // prim: T comp 4, p comp 5, X comps 6+NS..
    Arr4<double> src;        // species n -> comp 5+n
    Arr4<const double> na, nb;
    int mode;
    double w;                // stage weight of the B field
};

template <int NS>
static __global__ void __launch_bounds__(128) k_chem(ChemArgs a) {
    const int nx = a.P.n[0], ny = a.P.n[1], nz = a.P.n[2];
    const int64_t tot = (int64_t)nx * ny * nz;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % nx), j = (int)((q / nx) % ny), k = (int)(q / ((int64_t)nx * ny));
        double W[MAXR];
#pragma unroll
        for (int m = 0; m < MAXR; ++m) W[m] = 0.0;
        if (a.mode == CN_AB) {
            for (int m = 0; m < a.C.nr; ++m) W[m] = 1.0 * a.na(i, j, k, m) + a.w * a.nb(i, j, k, m);
        } else if (a.mode == CN_W) {
            for (int m = 0; m < a.C.nr; ++m) W[m] = a.na(i, j, k, m);
        } else if (a.mode == CN_PHILOX) {
            // the values fhd_fill_step_noise writes: A = 0.0 + 1.0 * z_A, B = 0.0 + 1.0 * z_B
            const uint32_t pidx = canon(a.P, i, j, k);
            const uint64_t step = noise_step(a.P);
            for (int m = 0; m < a.C.nr; m += 2) {
                float z[4];
                normal_quad(a.P.key0, a.P.key1, pidx, fid_chem(m) >> 1, step, z);
                W[m] = 1.0 * (0.0 + 1.0 * (double)z[0]) + a.w * (0.0 + 1.0 * (double)z[1]);
                if (m + 1 < a.C.nr) W[m + 1] = 1.0 * (0.0 + 1.0 * (double)z[2]) + a.w * (0.0 + 1.0 * (double)z[3]);
            }
        }
        double X[NS], S[NS];
#pragma unroll
        for (int n = 0; n < NS; ++n) X[n] = a.pr(i, j, k, 6 + NS + n);
        chem_point<NS>(a.P, a.C, a.pr(i, j, k, 5), a.pr(i, j, k, 4), X, W, S);
#pragma unroll
        for (int n = 0; n < NS; ++n) a.src(i, j, k, 5 + n) = S[n];
    }
}

template <int NS>
static int chem_launch_t(const ChemArgs& a, cudaStream_t s) {
    const int64_t tot = (int64_t)a.P.n[0] * a.P.n[1] * a.P.n[2];
    k_chem<NS><<<grid_for(tot, 128), 128, 0, s>>>(a);
    return cuda_rc(cudaGetLastError());
}

int chem_launch(const DevParams& P, const ChemParams& C, const fhd_fab& prim, const fhd_fab& source,
                const fhd_fab* na, const fhd_fab* nb, int mode, double w, cudaStream_t s) {
    ChemArgs a;
    std::memset(&a, 0, sizeof(a));
    a.P = P;
    a.C = C;
    a.pr = view<const double>(prim);
    a.src = view<double>(source);
    if (na) a.na = view<const double>(*na);
    if (nb) a.nb = view<const double>(*nb);
    a.mode = mode;
    a.w = w;
    switch (P.ns) {
        case 1: return chem_launch_t<1>(a, s);
        case 2: return chem_launch_t<2>(a, s);
        case 3: return chem_launch_t<3>(a, s);
        case 4: return chem_launch_t<4>(a, s);
        default: return FHD_ERR_UNSUPPORTED;
    }
}

}  // namespace fhd
