// fhd_kernels.cuh — sm_100a kernels of the staggered RK3 step.
//
//   k_cellprep  per stage: conservedToPrimitiveStag + calculateTransportCoeffs for
//               every cell once (cells grown by 1, face velocities grown by 1)
//   k_stage     per stage: stochastic + diffusive + hyperbolic fluxes, their
//               divergence and the SSP-RK3 combination, one 3D tile per CTA with
//               the stresses and conservative face fluxes exchanged in shared memory
//   k_convert   end of step / drop-in conversion (prim, vel, cons 1..3)
//   k_ghosts    periodic FillBoundary of several fabs in one launch
//   k_transport, k_aux_*  drop-in operators (transport coefficients, flux MultiFabs)
//   k_noise_*   Philox noise fills;  k_init_uniform  InitConsVarStag prob_type 1
#pragma once
#include "fhd_flux.cuh"

namespace fhd {

enum { ST_OK = 0, ST_MASSFRAC = 2, ST_NONFINITE = 3 };

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
__global__ void __launch_bounds__(128) k_cellprep(PrepArgs<NS, R> a) {
    const DevParams& P = a.P;
    const int nx = P.n[0] + 3, ny = P.n[1] + 3, nz = P.n[2] + 3;
    const int64_t tot = (int64_t)nx * ny * nz;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % nx) - 1;
        const int j = (int)((q / nx) % ny) - 1;
        const int k = (int)(q / ((int64_t)nx * ny)) - 1;
        const double rho = a.cons(i, j, k, 0);
        // low face velocities (conservedPrimitiveConversionsStag.cpp:61-67)
        a.vel[0](i, j, k) = 2 * a.mom[0](i, j, k) / (rho + a.cons(i - 1, j, k, 0));
        a.vel[1](i, j, k) = 2 * a.mom[1](i, j, k) / (rho + a.cons(i, j - 1, k, 0));
        a.vel[2](i, j, k) = 2 * a.mom[2](i, j, k) / (rho + a.cons(i, j, k - 1, 0));
        if (i > P.n[0] || j > P.n[1] || k > P.n[2]) continue;
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
}

// ===================================================================================
// fused stage kernel
// ===================================================================================
template <int NS, class R, int NZ>
struct StageArgs {
    DevParams P;
    Fields<NS, R> F;             // stage-input state U^s + derived fields
    Noise<NZ> noise;
    Arr4<const double> cons0;    // U^0 (for the RK combination)
    Arr4<const double> mom0[3];
    Arr4<double> cons_o;         // U^{s+1}
    Arr4<double> mom_o[3];
    Arr4<const double> src;      // source (nprimvars comps) or p == nullptr
    int stage;                   // 1, 2, 3
};

template <int TX, int TY, int TZ>
struct TileGeom {
    static constexpr int NT = TX * TY * TZ;
    static constexpr int CX = TX + 2, CY = TY + 2, CZ = TZ + 2, NC = CX * CY * CZ;
    static constexpr int NEXY = (TX + 1) * (TY + 1) * TZ;
    static constexpr int NEXZ = (TX + 1) * TY * (TZ + 1);
    static constexpr int NEYZ = TX * (TY + 1) * (TZ + 1);
    static constexpr int NFX = (TX + 1) * TY * TZ;
    static constexpr int NFY = TX * (TY + 1) * TZ;
    static constexpr int NFZ = TX * TY * (TZ + 1);
    FHD_D static int cpos(int ci, int cj, int ck) { return (ci + 1) + CX * ((cj + 1) + CY * (ck + 1)); }
    FHD_D static int exy(int i, int j, int k) { return i + (TX + 1) * (j + (TY + 1) * k); }
    FHD_D static int exz(int i, int j, int k) { return i + (TX + 1) * (j + TY * k); }
    FHD_D static int eyz(int i, int j, int k) { return i + TX * (j + (TY + 1) * k); }
    FHD_D static int fx(int i, int j, int k) { return i + (TX + 1) * (j + TY * k); }
    FHD_D static int fy(int i, int j, int k) { return i + TX * (j + (TY + 1) * k); }
    FHD_D static int fz(int i, int j, int k) { return i + TX * (j + TY * k); }
};

template <int NS, class R, int TX, int TY, int TZ>
struct StageSmem {
    using G = TileGeom<TX, TY, TZ>;
    R ct[6][G::NC];              // cell diag stresses: s xx,yy,zz, d xx,yy,zz
    R exy[2][G::NEXY];           // edge stresses (s, d)
    R exz[2][G::NEXZ];
    R eyz[2][G::NEYZ];
    double fx[2 + NS][G::NFX];   // conservative face fluxes (rho, rhoE, rhoY)
    double fy[2 + NS][G::NFY];
    double fz[2 + NS][G::NFZ];
};

// reads the tile's stresses from shared memory (global indices in, tile-relative inside)
template <int NS, class R, int TX, int TY, int TZ>
struct SmemTaus {
    using G = TileGeom<TX, TY, TZ>;
    const StageSmem<NS, R, TX, TY, TZ>* s;
    int x0, y0, z0;
    FHD_D CellTaus<R> cell(int i, int j, int k) const {
        const int p = G::cpos(i - x0, j - y0, k - z0);
        CellTaus<R> t;
#pragma unroll
        for (int d = 0; d < 3; ++d) { t.s[d] = s->ct[d][p]; t.d[d] = s->ct[3 + d][p]; }
        return t;
    }
    template <int E>
    FHD_D Taus<R> edge(int i, int j, int k) const {
        Taus<R> t;
        if (E == 0) { const int p = G::exy(i - x0, j - y0, k - z0); t.s = s->exy[0][p]; t.d = s->exy[1][p]; }
        if (E == 1) { const int p = G::exz(i - x0, j - y0, k - z0); t.s = s->exz[0][p]; t.d = s->exz[1][p]; }
        if (E == 2) { const int p = G::eyz(i - x0, j - y0, k - z0); t.s = s->eyz[0][p]; t.d = s->eyz[1][p]; }
        return t;
    }
};

template <int NS, class R, int NZ, int TX, int TY, int TZ>
__global__ void __launch_bounds__(TX * TY * TZ) k_stage(StageArgs<NS, R, NZ> a) {
    using G = TileGeom<TX, TY, TZ>;
    using SM = StageSmem<NS, R, TX, TY, TZ>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SM& S = *reinterpret_cast<SM*>(smem_raw);
    const DevParams& P = a.P;
    const Fields<NS, R>& F = a.F;
    const int tid = threadIdx.x;
    const int ntx = (P.n[0] + TX - 1) / TX, nty = (P.n[1] + TY - 1) / TY;
    const int bt = blockIdx.x;
    const int x0 = (bt % ntx) * TX, y0 = ((bt / ntx) % nty) * TY, z0 = (bt / (ntx * nty)) * TZ;
    const int nx = min(TX, P.n[0] - x0), ny = min(TY, P.n[1] - y0), nz = min(TZ, P.n[2] - z0);

    // ---- phase 1: diagonal stresses on the tile and its cross-shaped halo ----
    for (int q = tid; q < G::NC; q += G::NT) {
        const int ci = q % G::CX - 1, cj = (q / G::CX) % G::CY - 1, ck = q / (G::CX * G::CY) - 1;
        const int out = (ci < 0 || ci >= nx) + (cj < 0 || cj >= ny) + (ck < 0 || ck >= nz);
        if (ci > nx || cj > ny || ck > nz || out > 1) continue;
        const CellTaus<R> t = cell_taus<NS, R, NZ>(P, F, a.noise, x0 + ci, y0 + cj, z0 + ck);
#pragma unroll
        for (int d = 0; d < 3; ++d) { S.ct[d][q] = t.s[d]; S.ct[3 + d][q] = t.d[d]; }
    }
    // ---- phase 2: edge stresses ----
    for (int q = tid; q < G::NEXY + G::NEXZ + G::NEYZ; q += G::NT) {
        if (q < G::NEXY) {
            const int ei = q % (TX + 1), ej = (q / (TX + 1)) % (TY + 1), ek = q / ((TX + 1) * (TY + 1));
            if (ei > nx || ej > ny || ek >= nz) continue;
            const Taus<R> t = edge_taus<NS, R, NZ, 0>(P, F, a.noise, x0 + ei, y0 + ej, z0 + ek);
            S.exy[0][q] = t.s; S.exy[1][q] = t.d;
        } else if (q < G::NEXY + G::NEXZ) {
            const int r = q - G::NEXY;
            const int ei = r % (TX + 1), ej = (r / (TX + 1)) % TY, ek = r / ((TX + 1) * TY);
            if (ei > nx || ej >= ny || ek > nz) continue;
            const Taus<R> t = edge_taus<NS, R, NZ, 1>(P, F, a.noise, x0 + ei, y0 + ej, z0 + ek);
            S.exz[0][r] = t.s; S.exz[1][r] = t.d;
        } else {
            const int r = q - G::NEXY - G::NEXZ;
            const int ei = r % TX, ej = (r / TX) % (TY + 1), ek = r / (TX * (TY + 1));
            if (ei >= nx || ej > ny || ek > nz) continue;
            const Taus<R> t = edge_taus<NS, R, NZ, 2>(P, F, a.noise, x0 + ei, y0 + ej, z0 + ek);
            S.eyz[0][r] = t.s; S.eyz[1][r] = t.d;
        }
    }
    __syncthreads();
    // ---- phase 3: conservative face fluxes ----
    const SmemTaus<NS, R, TX, TY, TZ> tg{&S, x0, y0, z0};
    for (int q = tid; q < G::NFX + G::NFY + G::NFZ; q += G::NT) {
        if (q < G::NFX) {
            const int fi = q % (TX + 1), fj = (q / (TX + 1)) % TY, fk = q / ((TX + 1) * TY);
            if (fi > nx || fj >= ny || fk >= nz) continue;
            const FaceFlux<NS> f = face_flux<NS, R, NZ, 0>(P, F, a.noise, tg, x0 + fi, y0 + fj, z0 + fk);
#pragma unroll
            for (int c = 0; c < 2 + NS; ++c) S.fx[c][q] = f.cons[c];
        } else if (q < G::NFX + G::NFY) {
            const int r = q - G::NFX;
            const int fi = r % TX, fj = (r / TX) % (TY + 1), fk = r / (TX * (TY + 1));
            if (fi >= nx || fj > ny || fk >= nz) continue;
            const FaceFlux<NS> f = face_flux<NS, R, NZ, 1>(P, F, a.noise, tg, x0 + fi, y0 + fj, z0 + fk);
#pragma unroll
            for (int c = 0; c < 2 + NS; ++c) S.fy[c][r] = f.cons[c];
        } else {
            const int r = q - G::NFX - G::NFY;
            const int fi = r % TX, fj = (r / TX) % TY, fk = r / (TX * TY);
            if (fi >= nx || fj >= ny || fk > nz) continue;
            const FaceFlux<NS> f = face_flux<NS, R, NZ, 2>(P, F, a.noise, tg, x0 + fi, y0 + fj, z0 + fk);
#pragma unroll
            for (int c = 0; c < 2 + NS; ++c) S.fz[c][r] = f.cons[c];
        }
    }
    __syncthreads();
    // ---- phase 4: RK3 stage combination (timeStepStag.cpp:439-528, 771-861, 1106-1202) ----
    const double dt = P.dt;
    const int st = a.stage;
    {
        const int ci = tid % TX, cj = (tid / TX) % TY, ck = tid / (TX * TY);
        if (ci < nx && cj < ny && ck < nz) {
            const int i = x0 + ci, j = y0 + cj, k = z0 + ck;
            double on[2 + NS];
#pragma unroll
            for (int c = 0; c < 2 + NS; ++c) {
                const int n = (c == 0) ? 0 : 3 + c;  // conserved component index
                const double div = (S.fx[c][G::fx(ci + 1, cj, ck)] - S.fx[c][G::fx(ci, cj, ck)]) / P.dx[0] +
                                   (S.fy[c][G::fy(ci, cj + 1, ck)] - S.fy[c][G::fy(ci, cj, ck)]) / P.dx[1] +
                                   (S.fz[c][G::fz(ci, cj, ck + 1)] - S.fz[c][G::fz(ci, cj, ck)]) / P.dx[2];
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
    }
    // face momenta: faces owned by the tile (low faces of its cells, plus the domain's
    // high face n_cells for the last tile in that direction)
    const int fxn = nx + ((x0 + nx) == P.n[0]), fyn = ny + ((y0 + ny) == P.n[1]), fzn = nz + ((z0 + nz) == P.n[2]);
    const int hadv = P.advection_type >= 0;
    for (int q = tid; q < G::NFX + G::NFY + G::NFZ; q += G::NT) {
        int d, fi, fj, fk;
        if (q < G::NFX) { d = 0; fi = q % (TX + 1); fj = (q / (TX + 1)) % TY; fk = q / ((TX + 1) * TY);
            if (fi >= fxn || fj >= ny || fk >= nz) continue; }
        else if (q < G::NFX + G::NFY) { const int r = q - G::NFX; d = 1; fi = r % TX; fj = (r / TX) % (TY + 1); fk = r / (TX * (TY + 1));
            if (fi >= nx || fj >= fyn || fk >= nz) continue; }
        else { const int r = q - G::NFX - G::NFY; d = 2; fi = r % TX; fj = (r / TX) % TY; fk = r / (TX * TY);
            if (fi >= nx || fj >= ny || fk >= fzn) continue; }
        const int i = x0 + fi, j = y0 + fj, k = z0 + fk;
        double t1, t2, t3, ea, eb;
        if (d == 0) {
            t1 = cen_total<NS, R>(P, F, tg.cell(i, j, k), 0, i, j, k) - cen_total<NS, R>(P, F, tg.cell(i - 1, j, k), 0, i - 1, j, k);
            edge_adv<NS, R, 0>(P, F, i, j + 1, k, ea, eb);
            const double ehi = edge_total<R>(tg.template edge<0>(i, j + 1, k), ea, hadv);
            edge_adv<NS, R, 0>(P, F, i, j, k, ea, eb);
            const double elo = edge_total<R>(tg.template edge<0>(i, j, k), ea, hadv);
            t2 = ehi - elo;
            edge_adv<NS, R, 1>(P, F, i, j, k + 1, ea, eb);
            const double zhi = edge_total<R>(tg.template edge<1>(i, j, k + 1), ea, hadv);
            edge_adv<NS, R, 1>(P, F, i, j, k, ea, eb);
            const double zlo = edge_total<R>(tg.template edge<1>(i, j, k), ea, hadv);
            t3 = zhi - zlo;
        } else if (d == 1) {
            edge_adv<NS, R, 0>(P, F, i + 1, j, k, ea, eb);
            const double xhi = edge_total<R>(tg.template edge<0>(i + 1, j, k), eb, hadv);
            edge_adv<NS, R, 0>(P, F, i, j, k, ea, eb);
            const double xlo = edge_total<R>(tg.template edge<0>(i, j, k), eb, hadv);
            t1 = xhi - xlo;
            t2 = cen_total<NS, R>(P, F, tg.cell(i, j, k), 1, i, j, k) - cen_total<NS, R>(P, F, tg.cell(i, j - 1, k), 1, i, j - 1, k);
            edge_adv<NS, R, 2>(P, F, i, j, k + 1, ea, eb);
            const double zhi = edge_total<R>(tg.template edge<2>(i, j, k + 1), ea, hadv);
            edge_adv<NS, R, 2>(P, F, i, j, k, ea, eb);
            const double zlo = edge_total<R>(tg.template edge<2>(i, j, k), ea, hadv);
            t3 = zhi - zlo;
        } else {
            edge_adv<NS, R, 1>(P, F, i + 1, j, k, ea, eb);
            const double xhi = edge_total<R>(tg.template edge<1>(i + 1, j, k), eb, hadv);
            edge_adv<NS, R, 1>(P, F, i, j, k, ea, eb);
            const double xlo = edge_total<R>(tg.template edge<1>(i, j, k), eb, hadv);
            t1 = xhi - xlo;
            edge_adv<NS, R, 2>(P, F, i, j + 1, k, ea, eb);
            const double yhi = edge_total<R>(tg.template edge<2>(i, j + 1, k), eb, hadv);
            edge_adv<NS, R, 2>(P, F, i, j, k, ea, eb);
            const double ylo = edge_total<R>(tg.template edge<2>(i, j, k), eb, hadv);
            t2 = yhi - ylo;
            t3 = cen_total<NS, R>(P, F, tg.cell(i, j, k), 2, i, j, k) - cen_total<NS, R>(P, F, tg.cell(i, j, k - 1), 2, i, j, k - 1);
        }
        const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
        const double rsum = F.cons(i - e0, j - e1, k - e2, 0) + F.cons(i, j, k, 0);
        const double m0 = a.mom0[d](i, j, k);
        double v;
        if (st == 1) {
            v = m0 - dt * t1 / P.dx[0] - dt * t2 / P.dx[1] - dt * t3 / P.dx[2] + 0.5 * dt * P.grav[d] * rsum;
        } else if (st == 2) {
            v = 0.25 * 3.0 * m0 + 0.25 * F.mom[d](i, j, k) - 0.25 * dt * t1 / P.dx[0] - 0.25 * dt * t2 / P.dx[1] -
                0.25 * dt * t3 / P.dx[2] + 0.5 * 0.25 * dt * P.grav[d] * rsum;
        } else {
            v = (2. / 3.) * (0.5 * m0 + F.mom[d](i, j, k)) - (2. / 3.) * dt * t1 / P.dx[0] -
                (2. / 3.) * dt * t2 / P.dx[1] - (2. / 3.) * dt * t3 / P.dx[2] + 0.5 * (2. / 3.) * dt * P.grav[d] * rsum;
        }
        a.mom_o[d](i, j, k) = v;
    }
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
__global__ void __launch_bounds__(128) k_convert(ConvArgs<NS> a) {
    const DevParams& P = a.P;
    const int64_t tot = (int64_t)P.n[0] * P.n[1] * P.n[2];
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % P.n[0]);
        const int j = (int)((q / P.n[0]) % P.n[1]);
        const int k = (int)(q / ((int64_t)P.n[0] * P.n[1]));
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

// ===================================================================================
// periodic FillBoundary of up to 16 fabs in one launch
// ===================================================================================
struct GhostFab {
    double* p;
    int lo, vhi[3];   // ghost width = -lo; valid upper index per direction
    int64_t sy, sz, sn;
    int c0, nc;       // component range
    int64_t npts;     // ghost points of one component
};
struct GhostArgs {
    GhostFab f[16];
    int nf;
    int n[3];
};

static __global__ void __launch_bounds__(256) k_ghosts(GhostArgs a) {
    const int fidx = blockIdx.y;
    if (fidx >= a.nf) return;
    const GhostFab& f = a.f[fidx];
    const int g = -f.lo;
    const int NX = f.vhi[0] + 1 + 2 * g, NY = f.vhi[1] + 1 + 2 * g;
    const int VX = f.vhi[0] + 1, VY = f.vhi[1] + 1, VZ = f.vhi[2] + 1;
    const int64_t zsl = (int64_t)2 * g * NX * NY;        // two z slabs (all x, y)
    const int64_t ysl = (int64_t)2 * g * NX * VZ;        // two y slabs (valid z)
    const int64_t tot = (f.npts) * f.nc;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
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
        int si = i, sj = j, sk = k;
        while (si < 0) si += a.n[0];
        while (si > f.vhi[0]) si -= a.n[0];
        while (sj < 0) sj += a.n[1];
        while (sj > f.vhi[1]) sj -= a.n[1];
        while (sk < 0) sk += a.n[2];
        while (sk > f.vhi[2]) sk -= a.n[2];
        const int64_t base = (int64_t)c * f.sn;
        f.p[base + (i + g) + (j + g) * f.sy + (k + g) * f.sz] = f.p[base + (si + g) + (sj + g) * f.sy + (sk + g) * f.sz];
    }
}

// OverrideSync: nodal point n_cells <- point 0 (per nodal direction)
struct SyncArgs {
    double* p;
    int lo;
    int nodal[3];
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
__global__ void __launch_bounds__(128) k_transport(TransArgs<NS> a) {
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
        if (!transport_gio<NS, double>(P, a.prim(i, j, k, 0), a.prim(i, j, k, 4), a.prim(i, j, k, 5), Y, c))
            flag(a.status, ST_MASSFRAC);
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
template <int NS, class R, int NZ>
struct DirectTaus {
    const DevParams* P;
    const Fields<NS, R>* F;
    const Noise<NZ>* nz;
    FHD_D CellTaus<R> cell(int i, int j, int k) const { return cell_taus<NS, R, NZ>(*P, *F, *nz, i, j, k); }
    template <int E>
    FHD_D Taus<R> edge(int i, int j, int k) const { return edge_taus<NS, R, NZ, E>(*P, *F, *nz, i, j, k); }
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
template <int NS, class R, int NZ>
__global__ void __launch_bounds__(128) k_aux_faces(AuxArgs<NS, R, NZ> a) {
    const DevParams& P = a.P;
    const int* N = P.n;
    const int64_t nxf = (int64_t)(N[0] + 1) * N[1] * N[2], nyf = (int64_t)N[0] * (N[1] + 1) * N[2],
                  nzf = (int64_t)N[0] * N[1] * (N[2] + 1);
    const DirectTaus<NS, R, NZ> tg{&P, &a.F, &a.noise};
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nxf + nyf + nzf; q += (int64_t)gridDim.x * blockDim.x) {
        int d, i, j, k;
        if (q < nxf) { d = 0; i = (int)(q % (N[0] + 1)); j = (int)((q / (N[0] + 1)) % N[1]); k = (int)(q / ((int64_t)(N[0] + 1) * N[1])); }
        else if (q < nxf + nyf) { const int64_t r = q - nxf; d = 1; i = (int)(r % N[0]); j = (int)((r / N[0]) % (N[1] + 1)); k = (int)(r / ((int64_t)N[0] * (N[1] + 1))); }
        else { const int64_t r = q - nxf - nyf; d = 2; i = (int)(r % N[0]); j = (int)((r / N[0]) % N[1]); k = (int)(r / ((int64_t)N[0] * N[1])); }
        FaceFlux<NS> f;
        if (d == 0) f = face_flux<NS, R, NZ, 0>(P, a.F, a.noise, tg, i, j, k);
        else if (d == 1) f = face_flux<NS, R, NZ, 1>(P, a.F, a.noise, tg, i, j, k);
        else f = face_flux<NS, R, NZ, 2>(P, a.F, a.noise, tg, i, j, k);
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
template <int NS, class R, int NZ>
__global__ void __launch_bounds__(128) k_aux_edges_cen(AuxArgs<NS, R, NZ> a) {
    const DevParams& P = a.P;
    const int* N = P.n;
    const int64_t nxy = (int64_t)(N[0] + 1) * (N[1] + 1) * N[2], nxz = (int64_t)(N[0] + 1) * N[1] * (N[2] + 1),
                  nyz = (int64_t)N[0] * (N[1] + 1) * (N[2] + 1), nc = (int64_t)(N[0] + 2) * (N[1] + 2) * (N[2] + 2);
    const int hadv = P.advection_type >= 0;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nxy + nxz + nyz + nc; q += (int64_t)gridDim.x * blockDim.x) {
        double ea, eb;
        if (q < nxy) {
            const int i = (int)(q % (N[0] + 1)), j = (int)((q / (N[0] + 1)) % (N[1] + 1)), k = (int)(q / ((int64_t)(N[0] + 1) * (N[1] + 1)));
            const Taus<R> t = edge_taus<NS, R, NZ, 0>(P, a.F, a.noise, i, j, k);
            edge_adv<NS, R, 0>(P, a.F, i, j, k, ea, eb);
            a.ef[2](i, j, k) = edge_total<R>(t, ea, hadv);  // edgey_u
            a.ef[0](i, j, k) = edge_total<R>(t, eb, hadv);  // edgex_v
        } else if (q < nxy + nxz) {
            const int64_t r = q - nxy;
            const int i = (int)(r % (N[0] + 1)), j = (int)((r / (N[0] + 1)) % N[1]), k = (int)(r / ((int64_t)(N[0] + 1) * N[1]));
            const Taus<R> t = edge_taus<NS, R, NZ, 1>(P, a.F, a.noise, i, j, k);
            edge_adv<NS, R, 1>(P, a.F, i, j, k, ea, eb);
            a.ef[4](i, j, k) = edge_total<R>(t, ea, hadv);  // edgez_u
            a.ef[1](i, j, k) = edge_total<R>(t, eb, hadv);  // edgex_w
        } else if (q < nxy + nxz + nyz) {
            const int64_t r = q - nxy - nxz;
            const int i = (int)(r % N[0]), j = (int)((r / N[0]) % (N[1] + 1)), k = (int)(r / ((int64_t)N[0] * (N[1] + 1)));
            const Taus<R> t = edge_taus<NS, R, NZ, 2>(P, a.F, a.noise, i, j, k);
            edge_adv<NS, R, 2>(P, a.F, i, j, k, ea, eb);
            a.ef[5](i, j, k) = edge_total<R>(t, ea, hadv);  // edgez_v
            a.ef[3](i, j, k) = edge_total<R>(t, eb, hadv);  // edgey_w
        } else {
            const int64_t r = q - nxy - nxz - nyz;
            const int i = (int)(r % (N[0] + 2)) - 1, j = (int)((r / (N[0] + 2)) % (N[1] + 2)) - 1,
                      k = (int)(r / ((int64_t)(N[0] + 2) * (N[1] + 2))) - 1;
            const CellTaus<R> t = cell_taus<NS, R, NZ>(P, a.F, a.noise, i, j, k);
#pragma unroll
            for (int d = 0; d < 3; ++d) a.cf[d](i, j, k) = cen_total<NS, R>(P, a.F, t, d, i, j, k);
        }
    }
}

// ===================================================================================
// noise fills and initial state
// ===================================================================================
// MultiFabFillRandomNormal body: value = mean + sd*z on the valid region, with z
// from the counter (canonical point, field = fid0 + comp, stream) -> periodic
// duplicates are equal (OverrideSync); ghosts by k_ghosts afterwards.
struct NoiseFillArgs {
    DevParams P;
    Arr4<double> f;
    int vx, vy, vz;   // valid extents
    int c0, nc;
    double mean, sd;
    uint32_t fid0;
    int use_b;        // take z_B of the pair instead of z_A
};
static __global__ void k_noise_fill(NoiseFillArgs a) {
    const int64_t tot = (int64_t)a.vx * a.vy * a.vz * a.nc;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % a.vx), j = (int)((q / a.vx) % a.vy), k = (int)((q / ((int64_t)a.vx * a.vy)) % a.vz);
        const int c = (int)(q / ((int64_t)a.vx * a.vy * a.vz));
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

}  // namespace fhd
