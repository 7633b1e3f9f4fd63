// fhd_kernels.cuh — sm_100a kernels of the staggered RK3 step.
//
//   k_cellprep  per stage: conservedToPrimitiveStag + calculateTransportCoeffs for
//               every cell once (cells grown by 1, face velocities grown by 1)
//   k_taus      per stage: stochastic + deterministic stresses on cells and edges
//   k_faces<D>  per stage and direction: stochastic + diffusive + hyperbolic
//               conservative face fluxes (one small kernel per direction)
//   k_update    per stage: flux divergence, momentum update and the SSP-RK3
//               combination
//   k_convert   end of step / drop-in conversion (prim, vel, cons 1..3)
//   k_ghosts    periodic FillBoundary of several fabs in one launch
//   k_transport, k_aux_*  drop-in operators (transport coefficients, flux MultiFabs)
//   k_noise_*   Philox noise fills;  k_init_uniform  InitConsVarStag prob_type 1
#pragma once
#include "fhd_flux.cuh"
#include "fhd_transport_alt.cuh"

namespace fhd {

// Every kernel here has internal linkage (static): the FP64 units (built with
// -fmad=false) and the mixed units (-fmad=true) both instantiate the kernels that
// do not depend on the precision (e.g. k_convert_b<NS>) under the same name.
// With external linkage a launch could reach the other unit's device code, and
// which one depends on the order the modules are loaded in.

enum { ST_OK = 0, ST_MASSFRAC = 2, ST_NONFINITE = 3, ST_TIMEOUT = 5 };

FHD_D void flag(int* status, int code) {
    if (status) atomicCAS(status, 0, code);
}

// ===================================================================================
// cellprep: U^s -> (T, p, Y, X), coefficients, face velocities
// ===================================================================================
template <int NS, class R>
struct PrepArgs {
    DevParams P;
    Arr4<const double> cons;
    Arr4<const double> mom[3];
    Arr4<double> vel[3];
    Arr4<double> pr;   // view starting at the T component: T, p, Y[NS], X[NS]
    Arr4<R> eta, zeta, kappa, chi, D;
    int* status;
};

template <int NS, class R>
FHD_D int cellprep_count(const PrepArgs<NS, R>& a) { return (a.P.n[0] + 3) * (a.P.n[1] + 3) * (a.P.n[2] + 3); }

template <int NS, class R>
FHD_D void cellprep_point(const PrepArgs<NS, R>& a, int q) {
    const DevParams& P = a.P;
    const int nx = P.n[0] + 3, ny = P.n[1] + 3;
    const int i = q % nx - 1;
    const int j = (q / nx) % ny - 1;
    const int k = q / (nx * ny) - 1;
    const double rho = a.cons(i, j, k, 0);
    // low face velocities (conservedPrimitiveConversionsStag.cpp:61-67)
    a.vel[0](i, j, k) = 2 * a.mom[0](i, j, k) / (rho + a.cons(i - 1, j, k, 0));
    a.vel[1](i, j, k) = 2 * a.mom[1](i, j, k) / (rho + a.cons(i, j - 1, k, 0));
    a.vel[2](i, j, k) = 2 * a.mom[2](i, j, k) / (rho + a.cons(i, j, k - 1, 0));
    if (i > P.n[0] || j > P.n[1] || k > P.n[2]) return;
    double rY[NS];
#pragma unroll
    for (int n = 0; n < NS; ++n) rY[n] = a.cons(i, j, k, 5 + n);
    Prim<NS> q2;
    const bool fin = cons_to_prim<NS>(P, rho, a.cons(i, j, k, 4), rY, a.mom[0](i, j, k), a.mom[0](i + 1, j, k),
                                      a.mom[1](i, j, k), a.mom[1](i, j + 1, k), a.mom[2](i, j, k),
                                      a.mom[2](i, j, k + 1), q2);
    if (!fin) flag(a.status, ST_NONFINITE);
    a.pr(i, j, k, 0) = q2.T;
    a.pr(i, j, k, 1) = q2.p;
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        a.pr(i, j, k, 2 + n) = q2.Y[n];
        a.pr(i, j, k, 2 + NS + n) = q2.X[n];
    }
    R Yr[NS];
#pragma unroll
    for (int n = 0; n < NS; ++n) Yr[n] = R(q2.Y[n]);
    Coeffs<NS, R> c;
    if (!transport_gio<NS, R>(P, R(rho), R(q2.T), R(q2.p), Yr, c)) flag(a.status, ST_MASSFRAC);
    a.eta(i, j, k) = c.eta;
    a.kappa(i, j, k) = c.kappa;
    a.zeta(i, j, k) = c.zeta;
#pragma unroll
    for (int n = 0; n < NS; ++n) a.chi(i, j, k, n) = c.chi[n];
#pragma unroll
    for (int n = 0; n < NS * NS; ++n) a.D(i, j, k, n) = c.D[n];
}

// Register cap of the cell kernel: 64 registers up to two species (8 blocks of
// 128, no spills); with three or four species the Giovangigli solves need ~164
// registers in FP64 and ~93 in FP32, so cap at 128 (4 blocks, 40 B of spills in
// FP64) and 80 (6 blocks, no spills) to raise occupancy.
template <int NS, class R>
constexpr int cellprep_min_blocks() { return NS <= 2 ? 8 : (sizeof(R) == 8 ? 4 : 6); }

template <int NS, class R>
static __global__ void __launch_bounds__(128, cellprep_min_blocks<NS, R>()) k_cellprep(PrepArgs<NS, R> a) {
    const int tot = cellprep_count(a);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += gridDim.x * blockDim.x) cellprep_point(a, q);
}

// centre momentum flux with the particle reservoir's rule: a ghost cell beyond a
// bc_mass 4 side of direction d takes the stochastic and diffusive part of the cell
// inside it (recomputed here with that cell's own noise)
template <int NS, class R, int NZ, bool WL>
FHD_D double cen_total_res(const DevParams& P, const Fields<NS, R>& F, const Noise<NZ>& nz, const CellTaus<R>& t,
                           int d, int i, int j, int k) {
    if (WL) {
        const int x = d == 0 ? i : (d == 1 ? j : k);
        const int side = x < 0 ? 2 * d : (x > P.n[d] - 1 ? 2 * d + 1 : -1);
        if (side >= 0 && P.bc_mass[side] == 4) {
            int c[3] = {i, j, k};
            c[d] += (side & 1) ? -1 : 1;
            const CellTaus<R> tin = cell_taus<NS, R, NZ, WL>(P, F, nz, c[0], c[1], c[2]);
            return cen_total<NS, R, WL>(P, F, t, d, i, j, k, &tin);
        }
    }
    return cen_total<NS, R, WL>(P, F, t, d, i, j, k);
}

// ===================================================================================
// stage pipeline: k_taus -> k_faces<D> (x3) -> k_update
// ===================================================================================
// Scratch of one stage (owned by the context):
//   ct: cell stresses on the cells grown by 1, comps 0-2 stochastic xx,yy,zz,
//       3-5 deterministic xx,yy,zz
//   et: edge stresses on the points [0, n]^3, comps (s,d) of xy, xz, yz at 0-1, 2-3, 4-5
//   ff[d]: conservative face fluxes (rho, rhoE, rhoY) of direction d on [0, n]^3
//   mc: total centre momentum fluxes (cenflux x, y, z) on the cells grown by 1
//   me: total edge momentum fluxes on [0, n]^3 in the reference's order
//       edgeflux_x[0..1], edgeflux_y[0..1], edgeflux_z[0..1]
template <int NS, class R, int NZ>
struct StageArgs {
    DevParams P;
    Fields<NS, R> F;             // stage-input state U^s + derived fields
    Noise<NZ> noise;
    Arr4<R> ct, et;
    Arr4<double> ff[3];
    Arr4<double> mc, me;
    Arr4<const double> cons0;    // U^0 (for the RK combination)
    Arr4<const double> mom0[3];
    Arr4<double> cons_o;         // U^{s+1}
    Arr4<double> mom_o[3];
    Arr4<const double> src;      // source (nprimvars comps) or p == nullptr
    int stage;                   // 1, 2, 3
};

// stresses on cells (grown by 1) and edges; one thread per point of [-1, n]^3
template <int NS, class R, int NZ>
FHD_D int taus_count(const StageArgs<NS, R, NZ>& a) { return (a.P.n[0] + 2) * (a.P.n[1] + 2) * (a.P.n[2] + 2); }

// WL: walls (the wall variants of the edge stresses, advective edge fluxes and
// StochFluxStag's factors on the edge totals)
template <int NS, class R, int NZ, bool WL = false>
FHD_D void taus_point(const StageArgs<NS, R, NZ>& a, int q) {
    const DevParams& P = a.P;
    const int nx = P.n[0] + 2, ny = P.n[1] + 2;
    {
        const int i = q % nx - 1, j = (q / nx) % ny - 1, k = q / (nx * ny) - 1;
        const bool edges = i >= 0 && j >= 0 && k >= 0;
        double wc[3] = {0.0, 0.0, 0.0}, we[3] = {0.0, 0.0, 0.0};
        if (NZ != NZ_OFF) a.noise.cen_and_yz_edge(P, i, j, k, edges, wc, we[2]);
        const CellTaus<R> t = cell_taus_w<NS, R, NZ, WL>(P, a.F, wc, i, j, k);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            a.ct(i, j, k, d) = t.s[d];
            a.ct(i, j, k, 3 + d) = t.d[d];
            a.mc(i, j, k, d) = cen_total_res<NS, R, NZ, WL>(P, a.F, a.noise, t, d, i, j, k);
        }
        if (!edges) return;
        if (NZ != NZ_OFF) a.noise.xy_xz_edges(P, i, j, k, we[0], we[1]);
        const int hadv = P.advection_type >= 0;
        double ea, eb;
        if (k < P.n[2]) {
            const Taus<R> e = edge_taus_w<NS, R, NZ, 0, WL>(P, a.F, we[0], i, j, k);
            a.et(i, j, k, 0) = e.s;
            a.et(i, j, k, 1) = e.d;
            edge_adv<NS, R, 0, WL>(P, a.F, i, j, k, ea, eb);
            a.me(i, j, k, 2) = WL ? edge_total_w<R, 0>(P, e, ea, hadv, i, j, k) : edge_total<R>(e, ea, hadv);  // edgey_u
            a.me(i, j, k, 0) = WL ? edge_total_w<R, 0>(P, e, eb, hadv, i, j, k) : edge_total<R>(e, eb, hadv);  // edgex_v
        }
        if (j < P.n[1]) {
            const Taus<R> e = edge_taus_w<NS, R, NZ, 1, WL>(P, a.F, we[1], i, j, k);
            a.et(i, j, k, 2) = e.s;
            a.et(i, j, k, 3) = e.d;
            edge_adv<NS, R, 1, WL>(P, a.F, i, j, k, ea, eb);
            a.me(i, j, k, 4) = WL ? edge_total_w<R, 1>(P, e, ea, hadv, i, j, k) : edge_total<R>(e, ea, hadv);  // edgez_u
            a.me(i, j, k, 1) = WL ? edge_total_w<R, 1>(P, e, eb, hadv, i, j, k) : edge_total<R>(e, eb, hadv);  // edgex_w
        }
        if (i < P.n[0]) {
            const Taus<R> e = edge_taus_w<NS, R, NZ, 2, WL>(P, a.F, we[2], i, j, k);
            a.et(i, j, k, 4) = e.s;
            a.et(i, j, k, 5) = e.d;
            edge_adv<NS, R, 2, WL>(P, a.F, i, j, k, ea, eb);
            a.me(i, j, k, 5) = WL ? edge_total_w<R, 2>(P, e, ea, hadv, i, j, k) : edge_total<R>(e, ea, hadv);  // edgez_v
            a.me(i, j, k, 3) = WL ? edge_total_w<R, 2>(P, e, eb, hadv, i, j, k) : edge_total<R>(e, eb, hadv);  // edgey_w
        }
    }
}

template <int NS, class R, int NZ, bool WL = false>
static __global__ void __launch_bounds__(256) k_taus(StageArgs<NS, R, NZ> a) {
    const int tot = taus_count(a);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += gridDim.x * blockDim.x)
        taus_point<NS, R, NZ, WL>(a, q);
}

template <class R>
struct GlobalTaus {
    Arr4<R> ct, et;
    FHD_D CellTaus<R> cell(int i, int j, int k) const {
        CellTaus<R> t;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            t.s[d] = ct(i, j, k, d);
            t.d[d] = ct(i, j, k, 3 + d);
        }
        return t;
    }
    template <int E>
    FHD_D Taus<R> edge(int i, int j, int k) const {
        Taus<R> t;
        t.s = et(i, j, k, 2 * E);
        t.d = et(i, j, k, 2 * E + 1);
        return t;
    }
};

// conservative fluxes of the faces of direction D; one thread per valid face.
template <int NS, class R, int NZ, int D>
FHD_D int faces_count(const StageArgs<NS, R, NZ>& a) {
    return (a.P.n[0] + (D == 0)) * (a.P.n[1] + (D == 1)) * (a.P.n[2] + (D == 2));
}

template <int NS, class R, int NZ, int D, bool WL = false>
FHD_D void faces_point(const StageArgs<NS, R, NZ>& a, int q) {
    const DevParams& P = a.P;
    const int nx = P.n[0] + (D == 0), ny = P.n[1] + (D == 1);
    const GlobalTaus<R> tg{a.ct, a.et};
    const int i = q % nx, j = (q / nx) % ny, k = q / (nx * ny);
    const FaceFlux<NS> f = face_flux<NS, R, NZ, D, GlobalTaus<R>, WL>(P, a.F, a.noise, tg, i, j, k);
#pragma unroll
    for (int c = 0; c < 2 + NS; ++c) a.ff[D](i, j, k, c) = f.cons[c];
}

// MINB = minimum resident blocks requested from the register allocator.
template <int NS, class R, int NZ, int D, int BS, int MINB, bool WL = false>
static __global__ void __launch_bounds__(BS, MINB) k_faces(StageArgs<NS, R, NZ> a) {
    const int tot = faces_count<NS, R, NZ, D>(a);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += gridDim.x * blockDim.x)
        faces_point<NS, R, NZ, D, WL>(a, q);
}

// RK3 stage combination (timeStepStag.cpp:439-528, 771-861, 1106-1202): one thread
// per point of [0, n]^3 updates the cell there (if valid) and the faces there
template <int NS, class R, int NZ>
FHD_D int update_count(const StageArgs<NS, R, NZ>& a) { return (a.P.n[0] + 1) * (a.P.n[1] + 1) * (a.P.n[2] + 1); }

template <int NS, class R, int NZ>
FHD_D void update_point(const StageArgs<NS, R, NZ>& a, int q) {
    const DevParams& P = a.P;
    const Fields<NS, R>& F = a.F;
    const int nx = P.n[0] + 1, ny = P.n[1] + 1;
    const double dt = P.dt;
    const int st = a.stage;
    {
        const int i = q % nx, j = (q / nx) % ny, k = q / (nx * ny);
        const bool cell = i < P.n[0] && j < P.n[1] && k < P.n[2];
        if (cell) {
            double on[2 + NS];
#pragma unroll
            for (int c = 0; c < 2 + NS; ++c) {
                const int n = (c == 0) ? 0 : 3 + c;  // conserved component index
                const double div = divc(P, a.ff[0](i + 1, j, k, c) - a.ff[0](i, j, k, c), P.dx[0], P.rdx[0]) +
                                   divc(P, a.ff[1](i, j + 1, k, c) - a.ff[1](i, j, k, c), P.dx[1], P.rdx[1]) +
                                   divc(P, a.ff[2](i, j, k + 1, c) - a.ff[2](i, j, k, c), P.dx[2], P.rdx[2]);
                const double src = a.src.p ? a.src(i, j, k, n) : 0.0;
                const double u0 = a.cons0(i, j, k, n);
                double v;
                if (st == 1) v = u0 - dt * (div) + dt * src;
                else if (st == 2) v = 0.25 * (3.0 * u0 + F.cons(i, j, k, n) - dt * (div) + dt * src);
                else v = (2. / 3.) * (0.5 * u0 + F.cons(i, j, k, n) - dt * (div) + dt * src);
                on[c] = v;
            }
            // gravity work on the energy with the stage-input momenta
            const double gfac = (st == 1) ? 0.5 * dt : (st == 2) ? 0.5 * 0.25 * dt : 0.5 * (2. / 3.) * dt;
            on[1] += gfac * (P.grav[0] * (F.mom[0](i + 1, j, k) + F.mom[0](i, j, k)) +
                             P.grav[1] * (F.mom[1](i, j + 1, k) + F.mom[1](i, j, k)) +
                             P.grav[2] * (F.mom[2](i, j, k + 1) + F.mom[2](i, j, k)));
#pragma unroll
            for (int c = 0; c < 2 + NS; ++c) a.cons_o(i, j, k, (c == 0) ? 0 : 3 + c) = on[c];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
            if (i >= P.n[0] + e0 || j >= P.n[1] + e1 || k >= P.n[2] + e2) continue;
            // momentum flux differences (timeStepStag.cpp:452-482): centre and edge
            // totals stored by k_taus
            double t1, t2, t3;
            if (d == 0) {
                t1 = a.mc(i, j, k, 0) - a.mc(i - 1, j, k, 0);
                t2 = a.me(i, j + 1, k, 2) - a.me(i, j, k, 2);   // edgey_u
                t3 = a.me(i, j, k + 1, 4) - a.me(i, j, k, 4);   // edgez_u
            } else if (d == 1) {
                t1 = a.me(i + 1, j, k, 0) - a.me(i, j, k, 0);   // edgex_v
                t2 = a.mc(i, j, k, 1) - a.mc(i, j - 1, k, 1);
                t3 = a.me(i, j, k + 1, 5) - a.me(i, j, k, 5);   // edgez_v
            } else {
                t1 = a.me(i + 1, j, k, 1) - a.me(i, j, k, 1);   // edgex_w
                t2 = a.me(i, j + 1, k, 3) - a.me(i, j, k, 3);   // edgey_w
                t3 = a.mc(i, j, k, 2) - a.mc(i, j, k - 1, 2);
            }
            const double rsum = F.cons(i - e0, j - e1, k - e2, 0) + F.cons(i, j, k, 0);
            const double m0 = a.mom0[d](i, j, k);
            double v;
            if (st == 1) {
                v = m0 - divc(P, dt * t1, P.dx[0], P.rdx[0]) - divc(P, dt * t2, P.dx[1], P.rdx[1]) -
                    divc(P, dt * t3, P.dx[2], P.rdx[2]) + 0.5 * dt * P.grav[d] * rsum;
            } else if (st == 2) {
                v = 0.25 * 3.0 * m0 + 0.25 * F.mom[d](i, j, k) - divc(P, 0.25 * dt * t1, P.dx[0], P.rdx[0]) -
                    divc(P, 0.25 * dt * t2, P.dx[1], P.rdx[1]) - divc(P, 0.25 * dt * t3, P.dx[2], P.rdx[2]) +
                    0.5 * 0.25 * dt * P.grav[d] * rsum;
            } else {
                v = (2. / 3.) * (0.5 * m0 + F.mom[d](i, j, k)) - divc(P, (2. / 3.) * dt * t1, P.dx[0], P.rdx[0]) -
                    divc(P, (2. / 3.) * dt * t2, P.dx[1], P.rdx[1]) - divc(P, (2. / 3.) * dt * t3, P.dx[2], P.rdx[2]) +
                    0.5 * (2. / 3.) * dt * P.grav[d] * rsum;
            }
            a.mom_o[d](i, j, k) = v;
        }
    }
}

template <int NS, class R, int NZ>
static __global__ void __launch_bounds__(128, 16) k_update(StageArgs<NS, R, NZ> a) {  // HBM-bound: full occupancy
    const int tot = update_count(a);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += gridDim.x * blockDim.x) update_point(a, q);
}

// ===================================================================================
// conservedToPrimitiveStag on valid cells/faces (conservedPrimitiveConversionsStag.cpp)
// ===================================================================================
template <int NS>
struct ConvArgs {
    DevParams P;
    Arr4<double> prim;   // reference layout (nprimvars comps)
    Arr4<double> vel[3];
    Arr4<double> cons;   // comps 1..3 rewritten
    Arr4<const double> mom[3];
    int* status;
};

template <int NS>
FHD_D int convert_count(const ConvArgs<NS>& a) { return a.P.n[0] * a.P.n[1] * a.P.n[2]; }

template <int NS>
FHD_D void convert_point(const ConvArgs<NS>& a, int q) {
    const DevParams& P = a.P;
    {
        const int i = q % P.n[0];
        const int j = (q / P.n[0]) % P.n[1];
        const int k = q / (P.n[0] * P.n[1]);
        const Arr4<double>& cons = a.cons;
        const double rho = cons(i, j, k, 0);
        const Arr4<const double>&mx = a.mom[0], &my = a.mom[1], &mz = a.mom[2];
        // face velocities (:61-67); the last cell in a direction also owns face n_cells
        const double vxl = 2 * mx(i, j, k) / (rho + cons(i - 1, j, k, 0));
        const double vyl = 2 * my(i, j, k) / (rho + cons(i, j - 1, k, 0));
        const double vzl = 2 * mz(i, j, k) / (rho + cons(i, j, k - 1, 0));
        const double vxh = 2 * mx(i + 1, j, k) / (cons(i + 1, j, k, 0) + rho);
        const double vyh = 2 * my(i, j + 1, k) / (cons(i, j + 1, k, 0) + rho);
        const double vzh = 2 * mz(i, j, k + 1) / (cons(i, j, k + 1, 0) + rho);
        a.vel[0](i, j, k) = vxl;
        a.vel[1](i, j, k) = vyl;
        a.vel[2](i, j, k) = vzl;
        if (i == P.n[0] - 1) a.vel[0](i + 1, j, k) = vxh;
        if (j == P.n[1] - 1) a.vel[1](i, j + 1, k) = vyh;
        if (k == P.n[2] - 1) a.vel[2](i, j, k + 1) = vzh;
        const Arr4<double>& prim = a.prim;
        prim(i, j, k, 0) = rho;
        prim(i, j, k, 1) = 0.5 * (vxl + vxh);
        prim(i, j, k, 2) = 0.5 * (vyl + vyh);
        prim(i, j, k, 3) = 0.5 * (vzl + vzh);
        cons(i, j, k, 1) = 0.5 * (mx(i, j, k) + mx(i + 1, j, k));
        cons(i, j, k, 2) = 0.5 * (my(i, j, k) + my(i, j + 1, k));
        cons(i, j, k, 3) = 0.5 * (mz(i, j, k) + mz(i, j, k + 1));
        double rY[NS];
#pragma unroll
        for (int n = 0; n < NS; ++n) rY[n] = cons(i, j, k, 5 + n);
        Prim<NS> q2;
        if (!cons_to_prim<NS>(P, rho, cons(i, j, k, 4), rY, mx(i, j, k), mx(i + 1, j, k), my(i, j, k), my(i, j + 1, k),
                              mz(i, j, k), mz(i, j, k + 1), q2))
            flag(a.status, ST_NONFINITE);
        prim(i, j, k, 4) = q2.T;
        prim(i, j, k, 5) = q2.p;
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            prim(i, j, k, 6 + n) = q2.Y[n];
            prim(i, j, k, 6 + NS + n) = q2.X[n];
        }
    }
}

template <int NS>
static __global__ void __launch_bounds__(128) k_convert(ConvArgs<NS> a) {
    const int tot = convert_count(a);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += gridDim.x * blockDim.x) convert_point(a, q);
}

// ===================================================================================
// periodic FillBoundary of up to 16 fabs in one launch
// ===================================================================================
struct GhostFab {
    double* p;
    int lo, vhi[3];   // ghost width = -lo; valid upper index per direction
    int64_t sy, sz, sn;
    int c0, nc;       // component range
    int64_t npts;     // ghost points of one component
    int n[3];         // cells of the box (period)
    // periodic directions (walls elsewhere).  mode 0 (FillBoundary): a ghost point
    // is filled only when it lies outside the valid box in periodic directions
    // alone; mode 1 (noise fields whose wall ghosts hold their own values): the
    // periodic coordinates are wrapped and the wall coordinates kept.
    int per[3];
    int mode;
};
struct GhostArgs {
    GhostFab f[16];
    int nf;
    int n[3];
};

FHD_D void ghost_point(const GhostFab& f, int64_t q) {
    const int g = -f.lo;
    const int NX = f.vhi[0] + 1 + 2 * g, NY = f.vhi[1] + 1 + 2 * g;
    const int VX = f.vhi[0] + 1, VY = f.vhi[1] + 1, VZ = f.vhi[2] + 1;
    const int64_t zsl = (int64_t)2 * g * NX * NY;        // two z slabs (all x, y)
    const int64_t ysl = (int64_t)2 * g * NX * VZ;        // two y slabs (valid z)
    {
        const int c = f.c0 + (int)(q / f.npts);
        int64_t r = q % f.npts;
        int i, j, k;
        if (r < zsl) {
            const int kk = (int)(r / ((int64_t)NX * NY));
            r -= (int64_t)kk * NX * NY;
            j = (int)(r / NX) - g; i = (int)(r % NX) - g;
            k = kk < g ? kk - g : VZ + (kk - g);
        } else if (r < zsl + ysl) {
            r -= zsl;
            const int jj = (int)(r / ((int64_t)NX * VZ));
            r -= (int64_t)jj * NX * VZ;
            k = (int)(r / NX); i = (int)(r % NX) - g;
            j = jj < g ? jj - g : VY + (jj - g);
        } else {
            r -= zsl + ysl;
            const int ii = (int)(r / ((int64_t)VY * VZ));
            r -= (int64_t)ii * VY * VZ;
            k = (int)(r / VY); j = (int)(r % VY);
            i = ii < g ? ii - g : VX + (ii - g);
        }
        int s[3] = {i, j, k};
        bool wrapped = false;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (s[d] >= 0 && s[d] <= f.vhi[d]) continue;
            if (!f.per[d]) {
                if (f.mode == 0) return;
                continue;
            }
            wrapped = true;
            while (s[d] < 0) s[d] += f.n[d];
            while (s[d] > f.vhi[d]) s[d] -= f.n[d];
        }
        if (!wrapped) return;
        const int si = s[0], sj = s[1], sk = s[2];
        const int64_t base = (int64_t)c * f.sn;
        f.p[base + (i + g) + (j + g) * f.sy + (k + g) * f.sz] = f.p[base + (si + g) + (sj + g) * f.sy + (sk + g) * f.sz];
    }
}

static __global__ void __launch_bounds__(256) k_ghosts(GhostArgs a) {
    const int fidx = blockIdx.y;
    if (fidx >= a.nf) return;
    const GhostFab& f = a.f[fidx];
    const int64_t tot = f.npts * f.nc;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x)
        ghost_point(f, q);
}

// OverrideSync: nodal point n_cells <- point 0 (per nodal direction)
struct SyncArgs {
    double* p;
    int lo;
    int nodal[3];   // nodal and periodic (a wall direction has no duplicate points)
    int n[3];
    int64_t sy, sz, sn;
    int nc;
};
static __global__ void k_override_sync(SyncArgs a) {
    const int g = -a.lo;
    const int VX = a.n[0] + a.nodal[0], VY = a.n[1] + a.nodal[1], VZ = a.n[2] + a.nodal[2];
    const int64_t tot = (int64_t)VX * VY * VZ * a.nc;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % VX), j = (int)((q / VX) % VY), k = (int)((q / ((int64_t)VX * VY)) % VZ);
        const int c = (int)(q / ((int64_t)VX * VY * VZ));
        int si = i, sj = j, sk = k;
        bool dup = false;
        if (a.nodal[0] && i == a.n[0]) { si = 0; dup = true; }
        if (a.nodal[1] && j == a.n[1]) { sj = 0; dup = true; }
        if (a.nodal[2] && k == a.n[2]) { sk = 0; dup = true; }
        if (!dup) continue;
        const int64_t b = (int64_t)c * a.sn;
        a.p[b + (i + g) + (j + g) * a.sy + (k + g) * a.sz] = a.p[b + (si + g) + (sj + g) * a.sy + (sk + g) * a.sz];
    }
}

// ===================================================================================
// drop-in operators
// ===================================================================================
template <int NS>
struct TransArgs {
    DevParams P;
    Arr4<const double> prim;
    Arr4<double> eta, zeta, kappa, chi, D;
    int ng;
    int* status;
};

template <int NS>
static __global__ void __launch_bounds__(128) k_transport(TransArgs<NS> a) {
    const DevParams& P = a.P;
    const int g = a.ng;
    const int nx = P.n[0] + 2 * g, ny = P.n[1] + 2 * g, nz = P.n[2] + 2 * g;
    const int64_t tot = (int64_t)nx * ny * nz;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % nx) - g, j = (int)((q / nx) % ny) - g, k = (int)(q / ((int64_t)nx * ny)) - g;
        double Y[NS];
#pragma unroll
        for (int n = 0; n < NS; ++n) Y[n] = a.prim(i, j, k, 6 + n);
        Coeffs<NS, double> c;
        if (P.transport_type != 1) {
            // Valk/Waldmann or HCB binary (runs with these models take this kernel)
            const int st = transport_alt<NS>(P, a.prim(i, j, k, 0), a.prim(i, j, k, 4), a.prim(i, j, k, 5), Y, c);
            if (st) flag(a.status, st);
        } else if (!transport_gio<NS, double>(P, a.prim(i, j, k, 0), a.prim(i, j, k, 4), a.prim(i, j, k, 5), Y, c)) {
            flag(a.status, ST_MASSFRAC);
        }
        a.eta(i, j, k) = c.eta;
        a.kappa(i, j, k) = c.kappa;
        a.zeta(i, j, k) = c.zeta;
#pragma unroll
        for (int n = 0; n < NS; ++n) a.chi(i, j, k, n) = c.chi[n];
#pragma unroll
        for (int n = 0; n < NS * NS; ++n) a.D(i, j, k, n) = c.D[n];
    }
}

// stresses recomputed on the fly (operator path)
template <int NS, class R, int NZ, bool WL = false>
struct DirectTaus {
    const DevParams* P;
    const Fields<NS, R>* F;
    const Noise<NZ>* nz;
    FHD_D CellTaus<R> cell(int i, int j, int k) const { return cell_taus<NS, R, NZ, WL>(*P, *F, *nz, i, j, k); }
    template <int E>
    FHD_D Taus<R> edge(int i, int j, int k) const { return edge_taus<NS, R, NZ, E, WL>(*P, *F, *nz, i, j, k); }
};

template <int NS, class R, int NZ>
struct AuxArgs {
    DevParams P;
    Fields<NS, R> F;
    Noise<NZ> noise;
    Arr4<double> ff[3];   // faceflux (nvars+4 comps)
    Arr4<double> ef[6];   // edgeflux_x[0..1], edgeflux_y[0..1], edgeflux_z[0..1]
    Arr4<double> cf[3];   // cenflux (1 ghost)
};

// faceflux[d] on valid faces; items enumerate the three face boxes back to back
template <int NS, class R, int NZ, bool WL = false>
static __global__ void __launch_bounds__(128) k_aux_faces(AuxArgs<NS, R, NZ> a) {
    const DevParams& P = a.P;
    const int* N = P.n;
    const int64_t nxf = (int64_t)(N[0] + 1) * N[1] * N[2], nyf = (int64_t)N[0] * (N[1] + 1) * N[2],
                  nzf = (int64_t)N[0] * N[1] * (N[2] + 1);
    const DirectTaus<NS, R, NZ, WL> tg{&P, &a.F, &a.noise};
    using TG = DirectTaus<NS, R, NZ, WL>;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nxf + nyf + nzf; q += (int64_t)gridDim.x * blockDim.x) {
        int d, i, j, k;
        if (q < nxf) { d = 0; i = (int)(q % (N[0] + 1)); j = (int)((q / (N[0] + 1)) % N[1]); k = (int)(q / ((int64_t)(N[0] + 1) * N[1])); }
        else if (q < nxf + nyf) { const int64_t r = q - nxf; d = 1; i = (int)(r % N[0]); j = (int)((r / N[0]) % (N[1] + 1)); k = (int)(r / ((int64_t)N[0] * (N[1] + 1))); }
        else { const int64_t r = q - nxf - nyf; d = 2; i = (int)(r % N[0]); j = (int)((r / N[0]) % N[1]); k = (int)(r / ((int64_t)N[0] * N[1])); }
        FaceFlux<NS> f;
        if (d == 0) f = face_flux<NS, R, NZ, 0, TG, WL>(P, a.F, a.noise, tg, i, j, k);
        else if (d == 1) f = face_flux<NS, R, NZ, 1, TG, WL>(P, a.F, a.noise, tg, i, j, k);
        else f = face_flux<NS, R, NZ, 2, TG, WL>(P, a.F, a.noise, tg, i, j, k);
        const Arr4<double>& o = a.ff[d];
        o(i, j, k, 0) = f.cons[0];
        o(i, j, k, 1) = 0.0;
        o(i, j, k, 2) = 0.0;
        o(i, j, k, 3) = 0.0;
        o(i, j, k, 4) = f.cons[1];
#pragma unroll
        for (int s = 0; s < NS; ++s) o(i, j, k, 5 + s) = f.cons[2 + s];
#pragma unroll
        for (int c = 0; c < 4; ++c) o(i, j, k, 5 + NS + c) = f.aux[c];
    }
}

// edge fluxes (6 fabs) on valid edges and centre fluxes on cells grown by 1
template <int NS, class R, int NZ, bool WL = false>
static __global__ void __launch_bounds__(128) k_aux_edges_cen(AuxArgs<NS, R, NZ> a) {
    const DevParams& P = a.P;
    const int* N = P.n;
    const int64_t nxy = (int64_t)(N[0] + 1) * (N[1] + 1) * N[2], nxz = (int64_t)(N[0] + 1) * N[1] * (N[2] + 1),
                  nyz = (int64_t)N[0] * (N[1] + 1) * (N[2] + 1), nc = (int64_t)(N[0] + 2) * (N[1] + 2) * (N[2] + 2);
    const int hadv = P.advection_type >= 0;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nxy + nxz + nyz + nc; q += (int64_t)gridDim.x * blockDim.x) {
        double ea, eb;
        if (q < nxy) {
            const int i = (int)(q % (N[0] + 1)), j = (int)((q / (N[0] + 1)) % (N[1] + 1)), k = (int)(q / ((int64_t)(N[0] + 1) * (N[1] + 1)));
            const Taus<R> t = edge_taus<NS, R, NZ, 0, WL>(P, a.F, a.noise, i, j, k);
            edge_adv<NS, R, 0, WL>(P, a.F, i, j, k, ea, eb);
            a.ef[2](i, j, k) = WL ? edge_total_w<R, 0>(P, t, ea, hadv, i, j, k) : edge_total<R>(t, ea, hadv);  // edgey_u
            a.ef[0](i, j, k) = WL ? edge_total_w<R, 0>(P, t, eb, hadv, i, j, k) : edge_total<R>(t, eb, hadv);  // edgex_v
        } else if (q < nxy + nxz) {
            const int64_t r = q - nxy;
            const int i = (int)(r % (N[0] + 1)), j = (int)((r / (N[0] + 1)) % N[1]), k = (int)(r / ((int64_t)(N[0] + 1) * N[1]));
            const Taus<R> t = edge_taus<NS, R, NZ, 1, WL>(P, a.F, a.noise, i, j, k);
            edge_adv<NS, R, 1, WL>(P, a.F, i, j, k, ea, eb);
            a.ef[4](i, j, k) = WL ? edge_total_w<R, 1>(P, t, ea, hadv, i, j, k) : edge_total<R>(t, ea, hadv);  // edgez_u
            a.ef[1](i, j, k) = WL ? edge_total_w<R, 1>(P, t, eb, hadv, i, j, k) : edge_total<R>(t, eb, hadv);  // edgex_w
        } else if (q < nxy + nxz + nyz) {
            const int64_t r = q - nxy - nxz;
            const int i = (int)(r % N[0]), j = (int)((r / N[0]) % (N[1] + 1)), k = (int)(r / ((int64_t)N[0] * (N[1] + 1)));
            const Taus<R> t = edge_taus<NS, R, NZ, 2, WL>(P, a.F, a.noise, i, j, k);
            edge_adv<NS, R, 2, WL>(P, a.F, i, j, k, ea, eb);
            a.ef[5](i, j, k) = WL ? edge_total_w<R, 2>(P, t, ea, hadv, i, j, k) : edge_total<R>(t, ea, hadv);  // edgez_v
            a.ef[3](i, j, k) = WL ? edge_total_w<R, 2>(P, t, eb, hadv, i, j, k) : edge_total<R>(t, eb, hadv);  // edgey_w
        } else {
            const int64_t r = q - nxy - nxz - nyz;
            const int i = (int)(r % (N[0] + 2)) - 1, j = (int)((r / (N[0] + 2)) % (N[1] + 2)) - 1,
                      k = (int)(r / ((int64_t)(N[0] + 2) * (N[1] + 2))) - 1;
            const CellTaus<R> t = cell_taus<NS, R, NZ, WL>(P, a.F, a.noise, i, j, k);
#pragma unroll
            for (int d = 0; d < 3; ++d) a.cf[d](i, j, k) = cen_total_res<NS, R, NZ, WL>(P, a.F, a.noise, t, d, i, j, k);
        }
    }
}

// ===================================================================================
// noise fills and initial state
// ===================================================================================
// MultiFabFillRandomNormal body: value = mean + sd*z on the valid region, with z
// from the counter (canonical point, field = fid0 + comp, stream) -> periodic
// duplicates are equal (OverrideSync); ghosts by k_ghosts afterwards.
// MultiFabFillRandomUniform body (use_b = 2): a uniform in [0, 1) with 53 random
// bits, 27 from the first and 26 from the second word of one Philox call on the
// counter (canonical point, field = fid0 + comp, stream).
struct NoiseFillArgs {
    DevParams P;
    Arr4<double> f;
    int vx, vy, vz;   // extents of the filled box
    int ox, oy, oz;   // its low corner (0, or -1 to take the ghost layer of a wall direction)
    int c0, nc;
    double mean, sd;
    uint32_t fid0;
    int use_b;        // 0: z_A of the field's pair, 1: z_B, 2: the uniform
};

FHD_D double uniform53(uint32_t w0, uint32_t w1) {
    return ((double)(w0 >> 5) * 67108864.0 + (double)(w1 >> 6)) * (1.0 / 9007199254740992.0);
}
static __global__ void k_noise_fill(NoiseFillArgs a) {
    const int64_t tot = (int64_t)a.vx * a.vy * a.vz * a.nc;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % a.vx) + a.ox, j = (int)((q / a.vx) % a.vy) + a.oy,
                  k = (int)((q / ((int64_t)a.vx * a.vy)) % a.vz) + a.oz;
        const int c = (int)(q / ((int64_t)a.vx * a.vy * a.vz));
        if (a.use_b == 2) {
            uint32_t w[4] = {canon(a.P, i, j, k), a.fid0 + (uint32_t)c, (uint32_t)a.P.step, (uint32_t)(a.P.step >> 32)};
            philox4x32_10(w, a.P.key0, a.P.key1);
            a.f(i, j, k, a.c0 + c) = uniform53(w[0], w[1]);
            continue;
        }
        float za, zb;
        normal_pair(a.P.key0, a.P.key1, canon(a.P, i, j, k), a.fid0 + (uint32_t)c, a.P.step, za, zb);
        a.f(i, j, k, a.c0 + c) = a.mean + a.sd * (double)(a.use_b ? zb : za);
    }
}

struct InitArgs {
    Arr4<double> cu;
    int64_t npts;     // points of one component (whole fab incl. ghosts)
    int nvars, ns;
    double rho0, rhoE, rhoY[MAXS];
};
static __global__ void k_init_uniform(InitArgs a) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < a.npts; q += (int64_t)gridDim.x * blockDim.x) {
        double* p = a.cu.p + q;
        p[0] = a.rho0;
        p[a.cu.sn] = 0.0;
        p[2 * a.cu.sn] = 0.0;
        p[3 * a.cu.sn] = 0.0;
        p[4 * a.cu.sn] = a.rhoE;
        for (int s = 0; s < a.ns; ++s) p[(5 + s) * a.cu.sn] = a.rhoY[s];
    }
}

// ===================================================================================
// batched launches: one launch covers the work items of every member of an
// ensemble; block b belongs to the member m with bpref[m] <= b < bpref[m+1]
// ===================================================================================
FHD_D int member_of(const int* __restrict__ bpref, int nmem) {
    int lo = 0, hi = nmem;
    const int b = blockIdx.x;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (bpref[mid] <= b) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The member's argument block, copied once per block into shared memory (every
// thread of a block belongs to the same member): the bodies then read pointers,
// strides and run constants with shared loads on demand instead of holding what
// they read from global memory in registers.
template <class A>
FHD_D const A& member_args(const A* __restrict__ args, int m) {
    static_assert(sizeof(A) % 8 == 0, "argument blocks are copied in 8-byte words");
    __shared__ A sa;
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(args + m);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sa);
    for (int w = threadIdx.x; w < (int)(sizeof(A) / 8); w += blockDim.x) dst[w] = src[w];
    __syncthreads();
    return sa;
}

template <int NS, class R>
static __global__ void __launch_bounds__(128, cellprep_min_blocks<NS, R>()) k_cellprep_b(const PrepArgs<NS, R>* __restrict__ args,
                                                    const int* __restrict__ bpref, int nmem) {
    const int m = member_of(bpref, nmem);
    const PrepArgs<NS, R>& a = member_args(args, m);
    const int q = (blockIdx.x - bpref[m]) * blockDim.x + threadIdx.x;
    if (q < cellprep_count(a)) cellprep_point(a, q);
}

template <int NS, class R, int NZ>
static __global__ void __launch_bounds__(128) k_taus_b(const StageArgs<NS, R, NZ>* __restrict__ args,
                                                const int* __restrict__ bpref, int nmem) {
    const int m = member_of(bpref, nmem);
    const StageArgs<NS, R, NZ>& a = member_args(args, m);
    const int q = (blockIdx.x - bpref[m]) * blockDim.x + threadIdx.x;
    if (q < taus_count(a)) taus_point(a, q);
}

// Register cap of the batched face kernel: MINB resident blocks of 128 threads
// (8: 64 registers, 6: 80, 4: 128), picked per batch by its autotuner.
template <int NS, class R, int NZ, int D, int MINB>
static __global__ void __launch_bounds__(128, MINB) k_faces_b(const StageArgs<NS, R, NZ>* __restrict__ args,
                                                   const int* __restrict__ bpref, int nmem) {
    const int m = member_of(bpref, nmem);
    const StageArgs<NS, R, NZ>& a = member_args(args, m);
    const int q = (blockIdx.x - bpref[m]) * blockDim.x + threadIdx.x;
    if (q < faces_count<NS, R, NZ, D>(a)) faces_point<NS, R, NZ, D>(a, q);
}

template <int NS, class R, int NZ>
static __global__ void __launch_bounds__(128) k_update_b(const StageArgs<NS, R, NZ>* __restrict__ args,
                                                  const int* __restrict__ bpref, int nmem) {
    const int m = member_of(bpref, nmem);
    const StageArgs<NS, R, NZ>& a = member_args(args, m);
    const int q = (blockIdx.x - bpref[m]) * blockDim.x + threadIdx.x;
    if (q < update_count(a)) update_point(a, q);
}

template <int NS>
static __global__ void __launch_bounds__(128) k_convert_b(const ConvArgs<NS>* __restrict__ args,
                                                   const int* __restrict__ bpref, int nmem) {
    const int m = member_of(bpref, nmem);
    const ConvArgs<NS>& a = member_args(args, m);
    const int q = (blockIdx.x - bpref[m]) * blockDim.x + threadIdx.x;
    if (q < convert_count(a)) convert_point(a, q);
}

static __global__ void __launch_bounds__(256) k_ghosts_b(const GhostFab* __restrict__ fabs,
                                                         const int* __restrict__ bpref, int nfab) {
    const int m = member_of(bpref, nfab);
    const GhostFab& f = fabs[m];
    const int64_t q = (int64_t)(blockIdx.x - bpref[m]) * blockDim.x + threadIdx.x;
    if (q < f.npts * f.nc) ghost_point(f, q);
}

// ===================================================================================
// persistent batched step: one launch runs every phase of one RK3 step for every
// member.  Phases per member: for each stage cellprep, stresses, faces x / y / z,
// update, ghost fill; then the conversion, its ghost fill and the step counter.
// Work is cut into chunks of `chunk` items; a unit is one member's (or one ghost
// fab's) part of a phase.  Blocks take chunks in order from one counter (phase-
// major over members) and, before working on a chunk of phase p > 0, wait until
// every chunk of the member's phase p - 1 is done.  A block only ever waits on
// chunks taken before its own, by blocks that are running, so the order cannot
// deadlock; every wait is still bounded in time (limit_ns): on expiry the block
// marks the member FHD_ERR_TIMEOUT, raises the abort flag and all blocks stop
// taking work.
// ===================================================================================
FHD_D unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// bounded wait for every chunk of member m's phase p; 1 when done, 0 on abort or expiry
FHD_D int wait_phase(const PersistArgs& a, int m, int p) {
    volatile const unsigned int* d = a.done + (size_t)m * a.nphase + p;
    const unsigned int target = a.need[(size_t)m * a.nphase + p];
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (*d >= target) {
            __threadfence();
            return 1;
        }
        if (*reinterpret_cast<volatile int*>(a.abort)) return 0;
        if (global_ns() - t0 > a.limit_ns) {
            atomicCAS(a.status + m, 0, ST_TIMEOUT);
            atomicExch(a.abort, 1);
            return 0;
        }
        __nanosleep(256);
    }
}

template <int NS, class R, int NZ>
struct PersistBytes {
    static constexpr size_t a = sizeof(PrepArgs<NS, R>), b = sizeof(StageArgs<NS, R, NZ>), c = sizeof(ConvArgs<NS>),
                            d = sizeof(GhostFab);
    static constexpr size_t m1 = a > b ? a : b, m2 = c > d ? c : d;
    static constexpr size_t value = ((m1 > m2 ? m1 : m2) + 7) / 8 * 8;
};

template <int NS, class R, int NZ, int MINB>
static __global__ void __launch_bounds__(128, MINB) k_batch_persist(PersistArgs a) {
    __shared__ unsigned long long sbuf[PersistBytes<NS, R, NZ>::value / 8];
    __shared__ int s_unit, s_go, s_end;
    __shared__ long long s_chunk;
    for (;;) {
        if (threadIdx.x == 0) {
            long long I = -1;
            if (!*reinterpret_cast<volatile int*>(a.abort)) I = (long long)atomicAdd(a.next, 1u);
            const int end = I < 0 || I >= a.total;
            int u = 0, go = 0;
            if (!end) {
                int lo = 0, hi = a.nunits;
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (a.units[mid].first <= I) lo = mid;
                    else hi = mid;
                }
                u = lo;
                const PUnit& pu = a.units[u];
                go = pu.phase == 0 ? 1 : wait_phase(a, pu.member, pu.phase - 1);
                s_chunk = I - pu.first;
            }
            s_unit = u;
            s_go = go;
            s_end = end;
        }
        __syncthreads();
        if (s_end) break;
        const PUnit& pu = a.units[s_unit];
        const int kind = pu.kind;
        if (s_go) {
            if (kind != PK_STEP) {
                const size_t bytes = kind == PK_PREP ? sizeof(PrepArgs<NS, R>)
                                     : kind == PK_CONVERT ? sizeof(ConvArgs<NS>)
                                     : kind == PK_GHOST ? sizeof(GhostFab) : sizeof(StageArgs<NS, R, NZ>);
                const unsigned long long* src = static_cast<const unsigned long long*>(pu.args);
                for (int w = threadIdx.x; w < (int)((bytes + 7) / 8); w += blockDim.x) sbuf[w] = src[w];
            }
            __syncthreads();
            const int64_t q0 = s_chunk * a.chunk;
            const int64_t q1 = q0 + a.chunk < pu.items ? q0 + a.chunk : pu.items;
            const int64_t q = q0 + threadIdx.x;
            const int st = blockDim.x;
            switch (kind) {
                case PK_PREP: {
                    const auto& A = *reinterpret_cast<const PrepArgs<NS, R>*>(sbuf);
                    for (int64_t x = q; x < q1; x += st) cellprep_point(A, (int)x);
                } break;
                case PK_TAUS: {
                    const auto& A = *reinterpret_cast<const StageArgs<NS, R, NZ>*>(sbuf);
                    for (int64_t x = q; x < q1; x += st) taus_point(A, (int)x);
                } break;
                case PK_FACEX: {
                    const auto& A = *reinterpret_cast<const StageArgs<NS, R, NZ>*>(sbuf);
                    for (int64_t x = q; x < q1; x += st) faces_point<NS, R, NZ, 0>(A, (int)x);
                } break;
                case PK_FACEY: {
                    const auto& A = *reinterpret_cast<const StageArgs<NS, R, NZ>*>(sbuf);
                    for (int64_t x = q; x < q1; x += st) faces_point<NS, R, NZ, 1>(A, (int)x);
                } break;
                case PK_FACEZ: {
                    const auto& A = *reinterpret_cast<const StageArgs<NS, R, NZ>*>(sbuf);
                    for (int64_t x = q; x < q1; x += st) faces_point<NS, R, NZ, 2>(A, (int)x);
                } break;
                case PK_UPDATE: {
                    const auto& A = *reinterpret_cast<const StageArgs<NS, R, NZ>*>(sbuf);
                    for (int64_t x = q; x < q1; x += st) update_point(A, (int)x);
                } break;
                case PK_CONVERT: {
                    const auto& A = *reinterpret_cast<const ConvArgs<NS>*>(sbuf);
                    for (int64_t x = q; x < q1; x += st) convert_point(A, (int)x);
                } break;
                case PK_GHOST: {
                    const auto& G = *reinterpret_cast<const GhostFab*>(sbuf);
                    for (int64_t x = q; x < q1; x += st) ghost_point(G, x);
                } break;
                default:
                    if (threadIdx.x == 0) a.steps[pu.member] += 1;
                    break;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && s_go && pu.phase != a.hold_phase) {
            __threadfence();
            atomicAdd(a.done + (size_t)pu.member * a.nphase + pu.phase, 1u);
        }
    }
}

static __global__ void k_steps_set(uint64_t* step, uint64_t v) { *step = v; }

static __global__ void k_steps_inc(uint64_t* steps, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) steps[i] += 1;
}

}  // namespace fhd
