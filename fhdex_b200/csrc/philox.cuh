// philox.cuh — counter-based Gaussian noise for the in-kernel stochastic fluxes.
//
// Philox-4x32-10 as published by Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3" (SC'11): 10 rounds of two 32x32->64 multiplies
// with the Weyl key schedule.  One call per (periodic point, noise field) gives
// the pair (z_A, z_B) of standard normals through a Box-Muller transform in FP32
// (CUDA's logf / sincospif), so the A and B white-noise fields of one step are
// regenerated identically in each RK stage and never stored.
//
// Counter layout: c0 = canonical periodic point index (i mod Nx) + Nx*((j mod Ny)
// + Ny*(k mod Nz)), c1 = noise field id, c2/c3 = step (low/high).  Using the
// canonical index reproduces OverrideSync/FillBoundary: periodic duplicates of a
// nodal point and the periodic ghost images of a cell see the same numbers.
#pragma once
#include <cstdint>
#include "fhd_device.cuh"

namespace fhd {

FHD_HD void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]);
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]);
#else
        const uint32_t hi0 = (uint32_t)(((uint64_t)0xD2511F53u * c[0]) >> 32);
        const uint32_t hi1 = (uint32_t)(((uint64_t)0xCD9E8D57u * c[2]) >> 32);
#endif
        const uint32_t lo0 = 0xD2511F53u * c[0];
        const uint32_t lo1 = 0xCD9E8D57u * c[2];
        const uint32_t n0 = hi1 ^ c[1] ^ k0;
        const uint32_t n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// (z_A, z_B) for one (canonical point, field): Box-Muller on two 24-bit uniforms
// in (0,1).
FHD_D void normal_pair(uint32_t key0, uint32_t key1, uint32_t pidx, uint32_t fid, uint64_t step, float& za,
                       float& zb) {
    uint32_t c[4] = {pidx, fid, (uint32_t)step, (uint32_t)(step >> 32)};
    philox4x32_10(c, key0, key1);
    const float u1 = ((float)(c[0] >> 8) + 0.5f) * 5.9604644775390625e-8f;  // 2^-24
    const float u2 = ((float)(c[1] >> 8) + 0.5f) * 5.9604644775390625e-8f;
    const float r = sqrtf(-2.0f * logf(u1));
    float s, co;
    sincospif(2.0f * u2, &s, &co);
    za = r * co;
    zb = r * s;
}

FHD_HD int wrapn(int i, int n) {
    int r = i % n;
    return r < 0 ? r + n : r;
}

FHD_HD uint32_t canon(const DevParams& P, int i, int j, int k) {
    return (uint32_t)wrapn(i, P.n[0]) +
           (uint32_t)P.n[0] * ((uint32_t)wrapn(j, P.n[1]) + (uint32_t)P.n[1] * (uint32_t)wrapn(k, P.n[2]));
}

// Field ids: face d comp c (c = 0 energy, 1.. species) -> d*(MAXS+1)+c;
// edges xy,xz,yz -> 3*(MAXS+1)+e; centres -> 3*(MAXS+1)+3+d.
FHD_HD uint32_t fid_face(int d, int c) { return (uint32_t)(d * (MAXS + 1) + c); }
FHD_HD uint32_t fid_edge(int e) { return (uint32_t)(3 * (MAXS + 1) + e); }
FHD_HD uint32_t fid_cen(int d) { return (uint32_t)(3 * (MAXS + 1) + 3 + d); }

}  // namespace fhd
