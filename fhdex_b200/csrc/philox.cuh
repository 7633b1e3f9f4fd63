// philox.cuh — counter-based Gaussian noise for the in-kernel stochastic fluxes.
//
// Philox-4x32-10 as published by Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3" (SC'11): 10 rounds of two 32x32->64 multiplies
// with the Weyl key schedule.  One call per (periodic point, noise field) gives
// the pairs (z_A, z_B) of standard normals of two noise fields through
// Box-Muller transforms in FP32 (CUDA's logf / __sincosf), so the A and B
// white-noise fields of one step are regenerated identically in each RK stage and
// never stored.
//
// Counter layout: c0 = canonical periodic point index (i mod Nx) + Nx*((j mod Ny)
// + Ny*(k mod Nz)), c1 = noise field id / 2, c2/c3 = step (low/high).  Using the
// canonical index reproduces OverrideSync/FillBoundary: periodic duplicates of a
// nodal point and the periodic ghost images of a cell see the same numbers.
#pragma once
#include <cstdint>
#include "fhd_device.cuh"

namespace fhd {

FHD_HD void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        // one 32x32 -> 64-bit product per multiplier gives both halves
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
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

// Box-Muller pair from two 32-bit words: 24-bit uniforms in (0,1), angle in
// (-pi, pi) (the accuracy range of __sincosf).  log(u1) is the fast intrinsic
// __logf (at most 2^-21.4 absolute error on [0.5, 2], 3 ulp below; u1 >= 2^-25):
// the error reaches the radius only for u1 within ~1e-6 of 1, i.e. for normals of
// magnitude ~1e-3, once per ~1e6 draws.  The radius sqrt(x), x = -2 log(u1) >= 0,
// is formed as x * rsqrt(max(x, 1e-30)) (the hardware reciprocal square root,
// ~1 ulp): the noise needs no correctly rounded square root, and this avoids the
// out-of-line IEEE sqrtf routine.  The clamp keeps x = 0 at r = 0: the largest
// word rounds u1 to exactly 1.0f.
FHD_D void box_muller(uint32_t w0, uint32_t w1, float& za, float& zb) {
    const float u1 = ((float)(w0 >> 8) + 0.5f) * 5.9604644775390625e-8f;  // 2^-24
    const float u2 = ((float)(w1 >> 8) + 0.5f) * 5.9604644775390625e-8f;
    const float x = fmaxf(-2.0f * __logf(u1), 0.0f);
    const float r = x * rsqrtf(fmaxf(x, 1e-30f));
    float s, co;
    __sincosf(6.28318530717958648f * (u2 - 0.5f), &s, &co);
    za = r * co;
    zb = r * s;
}

// One Philox call serves the two noise fields 2q and 2q+1 at a point:
// words (0,1) -> field 2q, words (2,3) -> field 2q+1; each field gets (z_A, z_B).
FHD_D void normal_quad(uint32_t key0, uint32_t key1, uint32_t pidx, uint32_t fpair, uint64_t step, float (&z)[4]) {
    uint32_t c[4] = {pidx, fpair, (uint32_t)step, (uint32_t)(step >> 32)};
    philox4x32_10(c, key0, key1);
    box_muller(c[0], c[1], z[0], z[1]);
    box_muller(c[2], c[3], z[2], z[3]);
}

// (z_A, z_B) of one field
FHD_D void normal_pair(uint32_t key0, uint32_t key1, uint32_t pidx, uint32_t fid, uint64_t step, float& za,
                       float& zb) {
    float z[4];
    normal_quad(key0, key1, pidx, fid >> 1, step, z);
    za = (fid & 1) ? z[2] : z[0];
    zb = (fid & 1) ? z[3] : z[1];
}

// canonical periodic index of a point within one period of the box
FHD_HD int wrap1(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// Directions with walls are not periodic: there a point keeps its own index,
// shifted by one so that the ghost cell -1 and the cell/node n are distinct
// (n + 2 indices: cells -1..n, nodes 0..n), as the reference's wall directions
// neither OverrideSync nor FillBoundary their noise.
FHD_HD uint32_t canon1(const DevParams& P, int d, int i) {
    return P.periodic[d] ? (uint32_t)wrap1(i, P.n[d]) : (uint32_t)(i + 1);
}
FHD_HD uint32_t canon(const DevParams& P, int i, int j, int k) {
    if (!P.walls)
        return (uint32_t)wrap1(i, P.n[0]) +
               (uint32_t)P.n[0] * ((uint32_t)wrap1(j, P.n[1]) + (uint32_t)P.n[1] * (uint32_t)wrap1(k, P.n[2]));
    const uint32_t sx = P.periodic[0] ? P.n[0] : P.n[0] + 2, sy = P.periodic[1] ? P.n[1] : P.n[1] + 2;
    return canon1(P, 0, i) + sx * (canon1(P, 1, j) + sy * canon1(P, 2, k));
}

// Field ids: face d comp c (0 energy, 1.. species) -> 16 d + c; edges xy, xz, yz ->
// 48 + e; centres -> 51 + d.  Fields 2q, 2q+1 share one Philox call, so the six
// stress fields of a point take three calls: (edge xy, xz), (edge yz, centre x),
// (centre y, z).
FHD_HD uint32_t fid_face(int d, int c) { return (uint32_t)(16 * d + c); }
FHD_HD uint32_t fid_edge(int e) { return (uint32_t)(48 + e); }
FHD_HD uint32_t fid_cen(int d) { return (uint32_t)(51 + d); }

}  // namespace fhd
