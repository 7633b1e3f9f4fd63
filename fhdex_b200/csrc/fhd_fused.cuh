// fhd_fused.cuh — one RK stage after the cell kernel in ONE launch: stresses,
// conservative face fluxes, flux divergence, momentum update and the SSP-RK3
// combination (calculateFluxStag + the update of timeStepStag.cpp:439-528,
// 771-861, 1106-1202), marching in z with the intermediates in shared memory.
//
// Each block owns a TX x TY column of cells and a chunk of z-planes.  For output
// plane u it keeps in shared memory:
//   ct, mc   cell stresses (stochastic/deterministic diagonal) and total centre
//            momentum fluxes of planes u and u+1 on the tile grown by one cell
//   e*, m*   edge stresses (s, d) and total edge momentum fluxes of the xy edges
//            of planes u, u+1 and of the xz / yz edges of z-nodes u, u+1
//   ffz      conservative z-face fluxes of z-faces u and u+1
//   ffx, ffy conservative x- and y-face fluxes of plane u
// and per plane runs three phases separated by barriers:
//   A(u+1)  stresses of plane u+1 and edges at z-node u+1 (the k_taus point work)
//   B(u)    z-faces u+1, x- and y-faces of plane u (face_flux), one item list
//   C(u)    cell and face updates of plane u (the k_update point work)
// Nothing but U^{s+1} is written to global memory.  The point functions are the
// same ones the split kernels call, with the same arguments, so the result is
// bit for bit the split pipeline's (and the reference's in FP64).  The operands
// (state, primitives, coefficients, face velocities) are read from global memory
// through L1; the cell kernel (k_cellprep) runs before this one.
#pragma once
#include "fhd_kernels.cuh"

namespace fhd {

template <int TX, int TY>
struct ZmGeom {
    static constexpr int HX = TX + 2, HY = TY + 2;  // cells [-1, TX] x [-1, TY]
    static constexpr int NC = HX * HY;
    static constexpr int NXY = (TX + 1) * (TY + 1);  // xy nodes [0, TX] x [0, TY]
    static constexpr int NXZ = (TX + 1) * TY;        // xz nodes [0, TX] x [0, TY)
    static constexpr int NYZ = TX * (TY + 1);        // yz nodes [0, TX) x [0, TY]
    static constexpr int NT = TX * TY;
    static constexpr int NFX = (TX + 1) * TY;        // x-faces [0, TX] x [0, TY)
    static constexpr int NFY = TX * (TY + 1);        // y-faces [0, TX) x [0, TY]
};

// shared-memory layout (offsets in bytes, every array 16-byte aligned)
template <int NS, class R, int TX, int TY>
struct ZmSmem {
    using G = ZmGeom<TX, TY>;
    static constexpr int NF = 2 + NS;  // conservative face-flux components
    static constexpr size_t al(size_t b) { return (b + 15) & ~(size_t)15; }
    static constexpr size_t ct = 0;                                            // R [2][6][NC]
    static constexpr size_t mc = ct + al(sizeof(R) * 2 * 6 * G::NC);           // double [2][3][NC]
    static constexpr size_t mcz = mc + al(sizeof(double) * 2 * 3 * G::NC);     // double [NT] (plane u-1, z)
    static constexpr size_t exy = mcz + al(sizeof(double) * G::NT);            // R [2][2][NXY]
    static constexpr size_t mxy = exy + al(sizeof(R) * 2 * 2 * G::NXY);        // double [2][2][NXY]
    static constexpr size_t exz = mxy + al(sizeof(double) * 2 * 2 * G::NXY);   // R [2][2][NXZ]
    static constexpr size_t mxz = exz + al(sizeof(R) * 2 * 2 * G::NXZ);        // double [2][2][NXZ]
    static constexpr size_t eyz = mxz + al(sizeof(double) * 2 * 2 * G::NXZ);   // R [2][2][NYZ]
    static constexpr size_t myz = eyz + al(sizeof(R) * 2 * 2 * G::NYZ);        // double [2][2][NYZ]
    static constexpr size_t ffz = myz + al(sizeof(double) * 2 * 2 * G::NYZ);   // double [2][NF][NT]
    static constexpr size_t ffx = ffz + al(sizeof(double) * 2 * NF * G::NT);   // double [NF][NFX]
    static constexpr size_t ffy = ffx + al(sizeof(double) * NF * G::NFX);      // double [NF][NFY]
    static constexpr size_t bytes = ffy + al(sizeof(double) * NF * G::NFY);
};

// views of the shared-memory arrays for one block
template <int NS, class R, int TX, int TY>
struct ZmView {
    using G = ZmGeom<TX, TY>;
    using L = ZmSmem<NS, R, TX, TY>;
    static constexpr int NF = L::NF;
    unsigned char* base;
    int i0, j0;  // global index of the tile's first cell

    FHD_D R* ct(int slot, int c) const { return reinterpret_cast<R*>(base + L::ct) + (slot * 6 + c) * G::NC; }
    FHD_D double* mc(int slot, int c) const { return reinterpret_cast<double*>(base + L::mc) + (slot * 3 + c) * G::NC; }
    FHD_D double* mcz() const { return reinterpret_cast<double*>(base + L::mcz); }
    FHD_D R* exy(int slot, int c) const { return reinterpret_cast<R*>(base + L::exy) + (slot * 2 + c) * G::NXY; }
    FHD_D double* mxy(int slot, int c) const { return reinterpret_cast<double*>(base + L::mxy) + (slot * 2 + c) * G::NXY; }
    FHD_D R* exz(int slot, int c) const { return reinterpret_cast<R*>(base + L::exz) + (slot * 2 + c) * G::NXZ; }
    FHD_D double* mxz(int slot, int c) const { return reinterpret_cast<double*>(base + L::mxz) + (slot * 2 + c) * G::NXZ; }
    FHD_D R* eyz(int slot, int c) const { return reinterpret_cast<R*>(base + L::eyz) + (slot * 2 + c) * G::NYZ; }
    FHD_D double* myz(int slot, int c) const { return reinterpret_cast<double*>(base + L::myz) + (slot * 2 + c) * G::NYZ; }
    FHD_D double* ffz(int slot, int c) const { return reinterpret_cast<double*>(base + L::ffz) + (slot * NF + c) * G::NT; }
    FHD_D double* ffx(int c) const { return reinterpret_cast<double*>(base + L::ffx) + c * G::NFX; }
    FHD_D double* ffy(int c) const { return reinterpret_cast<double*>(base + L::ffy) + c * G::NFY; }

    // local indices (global i, j -> position in each array)
    FHD_D int cell(int i, int j) const { return (i - i0 + 1) + (j - j0 + 1) * G::HX; }
    FHD_D int nxy(int i, int j) const { return (i - i0) + (j - j0) * (TX + 1); }
    FHD_D int nxz(int i, int j) const { return (i - i0) + (j - j0) * (TX + 1); }
    FHD_D int nyz(int i, int j) const { return (i - i0) + (j - j0) * TX; }
    FHD_D int fx(int i, int j) const { return (i - i0) + (j - j0) * (TX + 1); }
    FHD_D int fy(int i, int j) const { return (i - i0) + (j - j0) * TX; }
    static FHD_D int slot(int k) { return k & 1; }  // parity ring (k may be -1)
};

// stresses read back from the rings, for face_flux
template <int NS, class R, int TX, int TY>
struct ZmTaus {
    ZmView<NS, R, TX, TY> v;
    FHD_D CellTaus<R> cell(int i, int j, int k) const {
        const int s = v.slot(k), q = v.cell(i, j);
        CellTaus<R> t;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            t.s[d] = v.ct(s, d)[q];
            t.d[d] = v.ct(s, 3 + d)[q];
        }
        return t;
    }
    template <int E>
    FHD_D Taus<R> edge(int i, int j, int k) const {
        const int s = v.slot(k);
        Taus<R> t;
        if (E == 0) { const int q = v.nxy(i, j); t.s = v.exy(s, 0)[q]; t.d = v.exy(s, 1)[q]; }
        else if (E == 1) { const int q = v.nxz(i, j); t.s = v.exz(s, 0)[q]; t.d = v.exz(s, 1)[q]; }
        else { const int q = v.nyz(i, j); t.s = v.eyz(s, 0)[q]; t.d = v.eyz(s, 1)[q]; }
        return t;
    }
};

// Phase A: the k_taus point work for the cells of plane k on the grown tile and
// the edges of node plane k that the tile uses (taus_point's calls and order).
template <int NS, class R, int NZ, int TX, int TY>
FHD_D void zm_phase_a(const StageArgs<NS, R, NZ>& a, const ZmView<NS, R, TX, TY>& v, int k, bool xy_edges,
                      bool z_edges) {
    using G = ZmGeom<TX, TY>;
    const DevParams& P = a.P;
    const int s = v.slot(k);
    const int hadv = P.advection_type >= 0;
    for (int q = threadIdx.x; q < G::NC; q += blockDim.x) {
        const int li = q % G::HX - 1, lj = q / G::HX - 1;
        const int i = v.i0 + li, j = v.j0 + lj;
        if (i > P.n[0] || j > P.n[1]) continue;  // beyond the box's ghost cell
        const bool edges = i >= 0 && j >= 0 && k >= 0;
        double wc[3] = {0.0, 0.0, 0.0}, we[3] = {0.0, 0.0, 0.0};
        if (NZ != NZ_OFF) a.noise.cen_and_yz_edge(P, i, j, k, edges, wc, we[2]);
        const CellTaus<R> t = cell_taus_w<NS, R, NZ>(P, a.F, wc, i, j, k);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v.ct(s, d)[q] = t.s[d];
            v.ct(s, 3 + d)[q] = t.d[d];
            v.mc(s, d)[q] = cen_total<NS, R>(P, a.F, t, d, i, j, k);
        }
        if (!edges || li < 0 || lj < 0 || !(xy_edges || z_edges)) continue;
        if (NZ != NZ_OFF) a.noise.xy_xz_edges(P, i, j, k, we[0], we[1]);
        double ea, eb;
        if (xy_edges && k < P.n[2]) {
            const Taus<R> e = edge_taus_w<NS, R, NZ, 0>(P, a.F, we[0], i, j, k);
            const int n = v.nxy(i, j);
            v.exy(s, 0)[n] = e.s;
            v.exy(s, 1)[n] = e.d;
            edge_adv<NS, R, 0>(P, a.F, i, j, k, ea, eb);
            v.mxy(s, 0)[n] = edge_total<R>(e, ea, hadv);  // edgey_u
            v.mxy(s, 1)[n] = edge_total<R>(e, eb, hadv);  // edgex_v
        }
        if (z_edges && j < P.n[1] && lj < TY) {
            const Taus<R> e = edge_taus_w<NS, R, NZ, 1>(P, a.F, we[1], i, j, k);
            const int n = v.nxz(i, j);
            v.exz(s, 0)[n] = e.s;
            v.exz(s, 1)[n] = e.d;
            edge_adv<NS, R, 1>(P, a.F, i, j, k, ea, eb);
            v.mxz(s, 0)[n] = edge_total<R>(e, ea, hadv);  // edgez_u
            v.mxz(s, 1)[n] = edge_total<R>(e, eb, hadv);  // edgex_w
        }
        if (z_edges && i < P.n[0] && li < TX) {
            const Taus<R> e = edge_taus_w<NS, R, NZ, 2>(P, a.F, we[2], i, j, k);
            const int n = v.nyz(i, j);
            v.eyz(s, 0)[n] = e.s;
            v.eyz(s, 1)[n] = e.d;
            edge_adv<NS, R, 2>(P, a.F, i, j, k, ea, eb);
            v.myz(s, 0)[n] = edge_total<R>(e, ea, hadv);  // edgez_v
            v.myz(s, 1)[n] = edge_total<R>(e, eb, hadv);  // edgey_w
        }
    }
}

// Phase B: one item list of the z-faces of face plane kz (when kz >= 0) and the
// x/y faces of plane kxy (when kxy >= 0)
template <int NS, class R, int NZ, int TX, int TY>
FHD_D void zm_phase_b(const StageArgs<NS, R, NZ>& a, const ZmView<NS, R, TX, TY>& v, int kz, int kxy) {
    using G = ZmGeom<TX, TY>;
    const DevParams& P = a.P;
    const ZmTaus<NS, R, TX, TY> tg{v};
    constexpr int NF = 2 + NS;
    const int nzi = kz >= 0 ? G::NT : 0;
    const int nxyi = kxy >= 0 ? G::NFX + G::NFY : 0;
    for (int q = threadIdx.x; q < nzi + nxyi; q += blockDim.x) {
        if (q < nzi) {
            const int i = v.i0 + q % TX, j = v.j0 + q / TX;
            if (i >= P.n[0] || j >= P.n[1]) continue;
            const FaceFlux<NS> f = face_flux<NS, R, NZ, 2>(P, a.F, a.noise, tg, i, j, kz);
            const int s = v.slot(kz);
#pragma unroll
            for (int c = 0; c < NF; ++c) v.ffz(s, c)[q] = f.cons[c];
        } else if (q < nzi + G::NFX) {
            const int r = q - nzi;
            const int i = v.i0 + r % (TX + 1), j = v.j0 + r / (TX + 1);
            if (i > P.n[0] || j >= P.n[1]) continue;
            const FaceFlux<NS> f = face_flux<NS, R, NZ, 0>(P, a.F, a.noise, tg, i, j, kxy);
#pragma unroll
            for (int c = 0; c < NF; ++c) v.ffx(c)[r] = f.cons[c];
        } else {
            const int r = q - nzi - G::NFX;
            const int i = v.i0 + r % TX, j = v.j0 + r / TX;
            if (i >= P.n[0] || j > P.n[1]) continue;
            const FaceFlux<NS> f = face_flux<NS, R, NZ, 1>(P, a.F, a.noise, tg, i, j, kxy);
#pragma unroll
            for (int c = 0; c < NF; ++c) v.ffy(c)[r] = f.cons[c];
        }
    }
}

// the face-momentum update of update_point (timeStepStag.cpp:450-489 and the
// stage-2/3 forms), the flux differences t1..t3 given
template <int NS, class R, int NZ>
FHD_D double zm_face_update(const StageArgs<NS, R, NZ>& a, int d, int i, int j, int k, double t1, double t2,
                            double t3) {
    const DevParams& P = a.P;
    const Fields<NS, R>& F = a.F;
    const double dt = P.dt;
    const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
    const double rsum = F.cons(i - e0, j - e1, k - e2, 0) + F.cons(i, j, k, 0);
    const double m0 = a.mom0[d](i, j, k);
    double v;
    if (a.stage == 1) {
        v = m0 - divc(P, dt * t1, P.dx[0], P.rdx[0]) - divc(P, dt * t2, P.dx[1], P.rdx[1]) -
            divc(P, dt * t3, P.dx[2], P.rdx[2]) + 0.5 * dt * P.grav[d] * rsum;
    } else if (a.stage == 2) {
        v = 0.25 * 3.0 * m0 + 0.25 * F.mom[d](i, j, k) - divc(P, 0.25 * dt * t1, P.dx[0], P.rdx[0]) -
            divc(P, 0.25 * dt * t2, P.dx[1], P.rdx[1]) - divc(P, 0.25 * dt * t3, P.dx[2], P.rdx[2]) +
            0.5 * 0.25 * dt * P.grav[d] * rsum;
    } else {
        v = (2. / 3.) * (0.5 * m0 + F.mom[d](i, j, k)) - divc(P, (2. / 3.) * dt * t1, P.dx[0], P.rdx[0]) -
            divc(P, (2. / 3.) * dt * t2, P.dx[1], P.rdx[1]) - divc(P, (2. / 3.) * dt * t3, P.dx[2], P.rdx[2]) +
            0.5 * (2. / 3.) * dt * P.grav[d] * rsum;
    }
    return v;
}

// Phase C: updates of plane k (cells, x/y faces; z-faces of face plane k).  With
// faces_only the plane is the box's top face plane n_z (z-faces only).  Thread
// q always owns tile column q (the mcz array is per column).
template <int NS, class R, int NZ, int TX, int TY>
FHD_D void zm_phase_c(const StageArgs<NS, R, NZ>& a, const ZmView<NS, R, TX, TY>& v, int k, bool faces_only) {
    using G = ZmGeom<TX, TY>;
    const DevParams& P = a.P;
    const Fields<NS, R>& F = a.F;
    const double dt = P.dt;
    const int st = a.stage;
    const int s0 = v.slot(k), s1 = v.slot(k + 1);
    for (int q = threadIdx.x; q < G::NT; q += blockDim.x) {
        const int i = v.i0 + q % TX, j = v.j0 + q / TX;
        if (i >= P.n[0] || j >= P.n[1]) continue;
        if (!faces_only) {
            // cell: flux divergence and the stage combination
            double on[2 + NS];
#pragma unroll
            for (int c = 0; c < 2 + NS; ++c) {
                const int n = (c == 0) ? 0 : 3 + c;
                const double div = divc(P, v.ffx(c)[v.fx(i + 1, j)] - v.ffx(c)[v.fx(i, j)], P.dx[0], P.rdx[0]) +
                                   divc(P, v.ffy(c)[v.fy(i, j + 1)] - v.ffy(c)[v.fy(i, j)], P.dx[1], P.rdx[1]) +
                                   divc(P, v.ffz(s1, c)[q] - v.ffz(s0, c)[q], P.dx[2], P.rdx[2]);
                const double src = a.src.p ? a.src(i, j, k, n) : 0.0;
                const double u0 = a.cons0(i, j, k, n);
                double val;
                if (st == 1) val = u0 - dt * (div) + dt * src;
                else if (st == 2) val = 0.25 * (3.0 * u0 + F.cons(i, j, k, n) - dt * (div) + dt * src);
                else val = (2. / 3.) * (0.5 * u0 + F.cons(i, j, k, n) - dt * (div) + dt * src);
                on[c] = val;
            }
            const double gfac = (st == 1) ? 0.5 * dt : (st == 2) ? 0.5 * 0.25 * dt : 0.5 * (2. / 3.) * dt;
            on[1] += gfac * (P.grav[0] * (F.mom[0](i + 1, j, k) + F.mom[0](i, j, k)) +
                             P.grav[1] * (F.mom[1](i, j + 1, k) + F.mom[1](i, j, k)) +
                             P.grav[2] * (F.mom[2](i, j, k + 1) + F.mom[2](i, j, k)));
#pragma unroll
            for (int c = 0; c < 2 + NS; ++c) a.cons_o(i, j, k, (c == 0) ? 0 : 3 + c) = on[c];
        }
        // z-face of this column at face plane k
        {
            const int c = v.cell(i, j);
            const double t1 = v.mxz(s0, 1)[v.nxz(i + 1, j)] - v.mxz(s0, 1)[v.nxz(i, j)];  // edgex_w
            const double t2 = v.myz(s0, 1)[v.nyz(i, j + 1)] - v.myz(s0, 1)[v.nyz(i, j)];  // edgey_w
            const double t3 = v.mc(s0, 2)[c] - v.mcz()[q];
            a.mom_o[2](i, j, k) = zm_face_update<NS, R, NZ>(a, 2, i, j, k, t1, t2, t3);
            v.mcz()[q] = v.mc(s0, 2)[c];  // centre z flux of plane k, for face plane k + 1
        }
        if (faces_only) continue;
        // x-face (i, j, k), and the box's top x-face n_x (the periodic duplicate of
        // x-face 0, computed as the reference computes it) from the last cell
        const int itop = (i == P.n[0] - 1) ? i + 1 : i;
        for (int ii = i; ii <= itop; ++ii) {
            const double t1 = v.mc(s0, 0)[v.cell(ii, j)] - v.mc(s0, 0)[v.cell(ii - 1, j)];
            const double t2 = v.mxy(s0, 0)[v.nxy(ii, j + 1)] - v.mxy(s0, 0)[v.nxy(ii, j)];  // edgey_u
            const double t3 = v.mxz(s1, 0)[v.nxz(ii, j)] - v.mxz(s0, 0)[v.nxz(ii, j)];      // edgez_u
            a.mom_o[0](ii, j, k) = zm_face_update<NS, R, NZ>(a, 0, ii, j, k, t1, t2, t3);
        }
        // y-face (i, j, k), and the box's top y-face n_y
        const int jtop = (j == P.n[1] - 1) ? j + 1 : j;
        for (int jj = j; jj <= jtop; ++jj) {
            const double t1 = v.mxy(s0, 1)[v.nxy(i + 1, jj)] - v.mxy(s0, 1)[v.nxy(i, jj)];  // edgex_v
            const double t2 = v.mc(s0, 1)[v.cell(i, jj)] - v.mc(s0, 1)[v.cell(i, jj - 1)];
            const double t3 = v.myz(s1, 0)[v.nyz(i, jj)] - v.myz(s0, 0)[v.nyz(i, jj)];      // edgez_v
            a.mom_o[1](i, jj, k) = zm_face_update<NS, R, NZ>(a, 1, i, jj, k, t1, t2, t3);
        }
    }
}

// grid: (tiles in x, tiles in y, z chunks of zc planes); BT threads per block,
// MINB resident blocks requested from the register allocator
template <int NS, class R, int NZ, int TX, int TY, int BT, int MINB>
static __global__ void __launch_bounds__(BT, MINB) k_stage_zm(StageArgs<NS, R, NZ> a, int zc) {
    extern __shared__ __align__(16) unsigned char zm_smem[];
    ZmView<NS, R, TX, TY> v;
    v.base = zm_smem;
    v.i0 = blockIdx.x * TX;
    v.j0 = blockIdx.y * TY;
    const int nz = a.P.n[2];
    const int k0 = blockIdx.z * zc;
    const int k1 = min(k0 + zc, nz);
    // prologue: stresses of planes k0-1 and k0 (edges of z-node k0), z-faces k0
    zm_phase_a<NS, R, NZ, TX, TY>(a, v, k0 - 1, false, false);
    __syncthreads();
    zm_phase_a<NS, R, NZ, TX, TY>(a, v, k0, true, true);
    for (int q = threadIdx.x; q < ZmGeom<TX, TY>::NT; q += blockDim.x)
        v.mcz()[q] = v.mc(v.slot(k0 - 1), 2)[v.cell(v.i0 + q % TX, v.j0 + q / TX)];
    __syncthreads();
    zm_phase_b<NS, R, NZ, TX, TY>(a, v, k0, -1);
    __syncthreads();
    for (int k = k0; k < k1; ++k) {
        zm_phase_a<NS, R, NZ, TX, TY>(a, v, k + 1, k + 1 < nz, true);
        __syncthreads();
        zm_phase_b<NS, R, NZ, TX, TY>(a, v, k + 1, k);
        __syncthreads();
        zm_phase_c<NS, R, NZ, TX, TY>(a, v, k, false);
        __syncthreads();
    }
    // the box's top z-faces n_z (periodic duplicates of z-faces 0, computed as the
    // reference computes them) belong to the last chunk
    if (k1 == nz) zm_phase_c<NS, R, NZ, TX, TY>(a, v, nz, true);
}

}  // namespace fhd
