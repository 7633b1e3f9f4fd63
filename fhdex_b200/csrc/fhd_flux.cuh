// fhd_flux.cuh — point flux functions of calculateFluxStag (fluxStag.cpp:5-1868)
// for a fully periodic box, shared by the fused stage kernel and the drop-in
// operator kernels.
//
// Accumulation order per flux component is the reference's: stochastic part
// assigned (fluxStag.cpp:298-803), diffusive part added (:872-1448), hyperbolic
// part added (:1508-1866), and the energy flux finally gets heat + viscous
// heating + Dufour (:1592).  R is the compute type of the stochastic/diffusive
// terms (double: reference order; float: mixed precision); hyperbolic terms and
// all state sums stay in double.
#pragma once
#include "fhd_device.cuh"
#include "philox.cuh"

namespace fhd {

// ---- field accessors ------------------------------------------------------------
template <int NS, class R>
struct Fields {
    Arr4<const double> cons;     // comp 0 rho, 4 rhoE, 5.. rhoY
    Arr4<const double> mom[3];   // face momenta
    Arr4<const double> vel[3];   // face velocities
    Arr4<const double> pr;       // T at comp pT, p pT+1, Y pT+2.., X pT+2+NS..
    int pT;
    Arr4<const R> eta, zeta, kappa, chi, D;

    FHD_D double T(int i, int j, int k) const { return pr(i, j, k, pT); }
    FHD_D double p(int i, int j, int k) const { return pr(i, j, k, pT + 1); }
    FHD_D double Y(int i, int j, int k, int n) const { return pr(i, j, k, pT + 2 + n); }
    FHD_D double X(int i, int j, int k, int n) const { return pr(i, j, k, pT + 2 + NS + n); }
};

// ---- noise sources --------------------------------------------------------------
enum { NZ_OFF = 0, NZ_W = 1, NZ_AB = 2, NZ_PHILOX = 3 };

struct NoiseArrays {
    Arr4<const double> fa[3], fb[3];   // face noise (W or A, B); energy at comp foff
    int foa[3], fob[3];
    Arr4<const double> ea[3], eb[3];   // xy, xz, yz
    Arr4<const double> ca[3], cb[3];   // centres (1 ghost)
};

// W = 1.0*A + w*B (MultiFab::LinComb, timeStepStag.cpp:258-326).  The *_all
// accessors fetch every noise field needed at one point at once, so that the
// in-kernel generator runs one Philox call per pair of fields.
template <int MODE>
struct Noise {
    NoiseArrays a;
    double w;

    FHD_D double comb(double A, double B) const { return 1.0 * A + w * B; }
    // fields fid0 and fid0+1 (fid0 even) at one point, each W = A + w B
    FHD_D void gauss2(const DevParams& P, uint32_t fid0, int i, int j, int k, double sd, double& w0,
                      double& w1) const {
        float z[4];
        normal_quad(P.key0, P.key1, canon(P, i, j, k), fid0 >> 1, noise_step(P), z);
        w0 = comb(0.0 + sd * (double)z[0], 0.0 + sd * (double)z[1]);
        w1 = comb(0.0 + sd * (double)z[2], 0.0 + sd * (double)z[3]);
    }
    // fields fid0 and fid0+1 with their own standard deviations
    FHD_D void gauss2sd(const DevParams& P, uint32_t fid0, int i, int j, int k, double sd0, double sd1, double& w0,
                        double& w1) const {
        float z[4];
        normal_quad(P.key0, P.key1, canon(P, i, j, k), fid0 >> 1, noise_step(P), z);
        w0 = comb(0.0 + sd0 * (double)z[0], 0.0 + sd0 * (double)z[1]);
        w1 = comb(0.0 + sd1 * (double)z[2], 0.0 + sd1 * (double)z[3]);
    }
    FHD_D double gauss1(const DevParams& P, uint32_t fid, int i, int j, int k, double sd) const {
        float za, zb;
        normal_pair(P.key0, P.key1, canon(P, i, j, k), fid, noise_step(P), za, zb);
        return comb(0.0 + sd * (double)za, 0.0 + sd * (double)zb);
    }
    template <int NC>
    FHD_D void face_all(const DevParams& P, int d, int i, int j, int k, double (&out)[NC]) const {
        if (MODE == NZ_PHILOX) {
#pragma unroll
            for (int c = 0; c < NC; c += 2) {
                if (c + 1 < NC) gauss2(P, fid_face(d, c), i, j, k, 1.0, out[c], out[c + 1]);
                else out[c] = gauss1(P, fid_face(d, c), i, j, k, 1.0);
            }
        } else {
#pragma unroll
            for (int c = 0; c < NC; ++c) out[c] = face(P, d, c, i, j, k);
        }
    }
    FHD_D void cen_all(const DevParams& P, int i, int j, int k, double (&out)[3]) const {
        if (MODE == NZ_PHILOX) {
            out[0] = gauss1(P, fid_cen(0), i, j, k, P.csd0);
            gauss2(P, fid_cen(1), i, j, k, P.sqrt2, out[1], out[2]);
        } else {
#pragma unroll
            for (int d = 0; d < 3; ++d) out[d] = cen(P, d, i, j, k);
        }
    }
    // The six stress fields of point (i,j,k) in three Philox calls: the centre
    // fields of cell (i,j,k) with, when `edges`, the yz edge field of node (i,j,k)
    // (cen_and_yz_edge), then the xy and xz edge fields (xy_xz_edges)
    FHD_D void cen_and_yz_edge(const DevParams& P, int i, int j, int k, bool edges, double (&wc)[3],
                               double& we2) const {
        if (MODE == NZ_PHILOX) {
            gauss2sd(P, fid_edge(2), i, j, k, 1.0, P.csd0, we2, wc[0]);
            gauss2(P, fid_cen(1), i, j, k, P.sqrt2, wc[1], wc[2]);
        } else {
            cen_all(P, i, j, k, wc);
            if (edges) we2 = edge(P, 2, i, j, k);
        }
    }
    FHD_D void xy_xz_edges(const DevParams& P, int i, int j, int k, double& we0, double& we1) const {
        if (MODE == NZ_PHILOX) {
            gauss2(P, fid_edge(0), i, j, k, 1.0, we0, we1);
        } else {
            we0 = edge(P, 0, i, j, k);
            we1 = edge(P, 1, i, j, k);
        }
    }
    FHD_D void edge_all(const DevParams& P, int i, int j, int k, double (&out)[3]) const {
        if (MODE == NZ_PHILOX) {
            gauss2(P, fid_edge(0), i, j, k, 1.0, out[0], out[1]);
            out[2] = gauss1(P, fid_edge(2), i, j, k, 1.0);  // (shares its call with centre x)
        } else {
#pragma unroll
            for (int e = 0; e < 3; ++e) out[e] = edge(P, e, i, j, k);
        }
    }
    FHD_D double face(const DevParams& P, int d, int c, int i, int j, int k) const {
        if (MODE == NZ_W) return a.fa[d](i, j, k, a.foa[d] + c);
        if (MODE == NZ_AB) return comb(a.fa[d](i, j, k, a.foa[d] + c), a.fb[d](i, j, k, a.fob[d] + c));
        if (MODE == NZ_PHILOX) return gauss1(P, fid_face(d, c), i, j, k, 1.0);
        return 0.0;
    }
    FHD_D double edge(const DevParams& P, int e, int i, int j, int k) const {
        if (MODE == NZ_W) return a.ea[e](i, j, k);
        if (MODE == NZ_AB) return comb(a.ea[e](i, j, k), a.eb[e](i, j, k));
        if (MODE == NZ_PHILOX) return gauss1(P, fid_edge(e), i, j, k, 1.0);
        return 0.0;
    }
    FHD_D double cen(const DevParams& P, int d, int i, int j, int k) const {
        if (MODE == NZ_W) return a.ca[d](i, j, k);
        if (MODE == NZ_AB) return comb(a.ca[d](i, j, k), a.cb[d](i, j, k));
        if (MODE == NZ_PHILOX) return gauss1(P, fid_cen(d), i, j, k, d == 0 ? P.csd0 : P.sqrt2);
        return 0.0;
    }
};

// ---- stresses --------------------------------------------------------------------
template <class R>
struct Taus {  // stochastic (s) and deterministic (d) parts
    R s, d;
};

template <class R>
struct CellTaus {
    R s[3], d[3];
};

// diagonal stresses at a cell: stochastic fluxStag.cpp:163-206, deterministic :872-924;
// wc: the three centre noise values W of the cell.  WL: the reference-ordered
// pipeline, which also carries the quasi-1-D / 2-D runs (P.dim 1 / 2): only the
// x (x and y) stresses, the 1-D amplitudes scaled by sqrt(3) and the 2-D trace
// factor by (3+sqrt(3))/2 (fluxStag.cpp:171-192, 875-904)
template <int NS, class R, int NZ, bool WL = false>
FHD_D CellTaus<R> cell_taus_w(const DevParams& P, const Fields<NS, R>& F, const double (&wc)[3], int i, int j, int k) {
    CellTaus<R> t;
    const R eta = F.eta(i, j, k);
    const bool visc3 = (P.visc_type == 3 || P.visc_type == -3);
    if (WL && P.dim < 3) {
        if (NZ != NZ_OFF) {
            const R etaT = eta * R(F.T(i, j, k));
            R fac1 = dsqrt(R(2.0) * R(P.k_B) * etaT * R(P.volinv) * R(P.dtinv));
            R fac2 = R(-1.0 / 3.0) * dsqrt(R(2.0) * R(P.k_B) * etaT * R(P.volinv) * R(P.dtinv));
            const R w0 = R(wc[0]), w1 = R(wc[1]);
            if (P.dim == 1) {
                fac1 *= R(P.sqrt3);
                fac2 *= R(P.sqrt3);
                const R traceZ = w0;
                t.s[0] = (fac1 * w0) + (fac2 * traceZ);
                t.s[1] = R(0.0);
            } else {
                fac2 *= R(P.fac2d);
                const R traceZ = w0 + w1;
                t.s[0] = (fac1 * w0) + (fac2 * traceZ);
                t.s[1] = (fac1 * w1) + (fac2 * traceZ);
            }
            t.s[2] = R(0.0);
        } else {
            t.s[0] = t.s[1] = t.s[2] = R(0.);
        }
        const R u_x = divc(P, R(F.vel[0](i + 1, j, k)) - R(F.vel[0](i, j, k)), R(P.dx[0]), R(P.rdx[0]));
        const R eta23 = divc(P, R(2) * eta, R(3.), R(P.r3));
        if (P.dim == 1) {
            const R div = u_x;
            t.d[0] = R(2) * eta * u_x + (R(0.0) - eta23) * div;
            t.d[1] = R(0.0);
        } else {
            const R v_y = divc(P, R(F.vel[1](i, j + 1, k)) - R(F.vel[1](i, j, k)), R(P.dx[1]), R(P.rdx[1]));
            const R div = u_x + v_y;
            t.d[0] = R(2) * eta * u_x + (R(0.0) - eta23) * div;
            t.d[1] = R(2) * eta * v_y + (R(0.0) - eta23) * div;
        }
        t.d[2] = R(0.0);
        return t;
    }
    if (NZ != NZ_OFF) {
        const R Tc = R(F.T(i, j, k));
        const R etaT = eta * Tc;
        const R zetaT = F.zeta(i, j, k) * Tc;
        const R fac1 = dsqrt(R(2.0) * R(P.k_B) * etaT * R(P.volinv) * R(P.dtinv));
        R fac2 = R(-1.0 / 3.0) * dsqrt(R(2.0) * R(P.k_B) * etaT * R(P.volinv) * R(P.dtinv));
        if (visc3)
            fac2 = dsqrt(divc(P, R(P.k_B) * zetaT * R(P.volinv) * R(P.dtinv), R(3.0), R(P.r3))) -
                   divc(P, dsqrt(R(2.0) * R(P.k_B) * etaT * R(P.volinv) * R(P.dtinv)), R(3.0), R(P.r3));
        const R w0 = R(wc[0]), w1 = R(wc[1]), w2 = R(wc[2]);
        const R traceZ = w0 + w1 + w2;
        t.s[0] = (fac1 * w0) + (fac2 * traceZ);
        t.s[1] = (fac1 * w1) + (fac2 * traceZ);
        t.s[2] = (fac1 * w2) + (fac2 * traceZ);
    } else {
        t.s[0] = t.s[1] = t.s[2] = R(0.);
    }
    const R u_x = divc(P, R(F.vel[0](i + 1, j, k)) - R(F.vel[0](i, j, k)), R(P.dx[0]), R(P.rdx[0]));
    const R v_y = divc(P, R(F.vel[1](i, j + 1, k)) - R(F.vel[1](i, j, k)), R(P.dx[1]), R(P.rdx[1]));
    const R w_z = divc(P, R(F.vel[2](i, j, k + 1)) - R(F.vel[2](i, j, k)), R(P.dx[2]), R(P.rdx[2]));
    const R div = u_x + v_y + w_z;
    const R zc = visc3 ? R(F.zeta(i, j, k)) : R(0.0);
    const R eta23 = divc(P, R(2) * eta, R(3.), R(P.r3));
    t.d[0] = R(2) * eta * u_x + (zc - eta23) * div;
    t.d[1] = R(2) * eta * v_y + (zc - eta23) * div;
    t.d[2] = R(2) * eta * w_z + (zc - eta23) * div;
    return t;
}

// off-diagonal stress at an edge E (0 xy, 1 xz, 2 yz): stochastic fluxStag.cpp:209-295,
// deterministic :927-1023.  The four cells around the edge are c00, c01, c10, c11
// in the reference's summation order.
// WL: walls; an edge on a wall plane averages only the two cells on the wall's
// ghost side for its stochastic amplitude and its viscosity, and differences the
// velocity across the wall over the half cell (fluxStag.cpp:221-232, 250-261,
// 279-290, 939-1019: the first direction's wall is tested last and wins a corner).
template <int NS, class R, int NZ, int E, bool WL = false>
FHD_D Taus<R> edge_taus_w(const DevParams& P, const Fields<NS, R>& F, double wnoise, int i, int j, int k) {
    // quasi-1-D: no shear stress; quasi-2-D: only xy (fluxStag.cpp:212-214, 241-243,
    // 270-272, 930-932, 962-964, 995-997)
    if (WL && (P.dim == 1 || (P.dim == 2 && E != 0))) {
        Taus<R> z;
        z.s = R(0.0);
        z.d = R(0.0);
        return z;
    }
    // cells: (a) low-low, (b) low-high, (c) high-low, (d) high-high in the edge's two directions
    int ai, aj, ak, bi, bj, bk, ci, cj, ck;
    if (E == 0) { ai = i - 1; aj = j - 1; ak = k; bi = i - 1; bj = j; bk = k; ci = i; cj = j - 1; ck = k; }
    else if (E == 1) { ai = i - 1; aj = j; ak = k - 1; bi = i - 1; bj = j; bk = k; ci = i; cj = j; ck = k - 1; }
    else { ai = i; aj = j - 1; ak = k - 1; bi = i; bj = j - 1; bk = k; ci = i; cj = j; ck = k - 1; }
    Taus<R> t;
    if (NZ != NZ_OFF) {
        R etaT = R(0.25) * (F.eta(ai, aj, ak) * R(F.T(ai, aj, ak)) + F.eta(bi, bj, bk) * R(F.T(bi, bj, bk)) +
                            F.eta(ci, cj, ck) * R(F.T(ci, cj, ck)) + F.eta(i, j, k) * R(F.T(i, j, k)));
        if (WL) {
            // cells a (lo, lo), b (lo, hi), c (hi, lo), d = (i, j, k) in the edge's
            // (first, second) directions; the wall of the second direction is tested first
            const int d1 = E == 2 ? 1 : 0, d2 = E == 0 ? 1 : 2;
            const int x1 = d1 == 0 ? i : j, x2 = d2 == 1 ? j : k;
            const R ta = F.eta(ai, aj, ak) * R(F.T(ai, aj, ak)), tb = F.eta(bi, bj, bk) * R(F.T(bi, bj, bk));
            const R tc = F.eta(ci, cj, ck) * R(F.T(ci, cj, ck)), td = F.eta(i, j, k) * R(F.T(i, j, k));
            if (x2 == 0 && dirichlet_side(P, 2 * d2)) etaT = R(0.5) * (ta + tc);
            if (x2 == P.n[d2] && dirichlet_side(P, 2 * d2 + 1)) etaT = R(0.5) * (tb + td);
            if (x1 == 0 && dirichlet_side(P, 2 * d1)) etaT = R(0.5) * (ta + tb);
            if (x1 == P.n[d1] && dirichlet_side(P, 2 * d1 + 1)) etaT = R(0.5) * (tc + td);
        }
        const R fac = dsqrt(R(2.0) * R(P.k_B) * etaT * R(P.volinv) * R(P.dtinv));
        t.s = fac * R(wnoise);
    } else {
        t.s = R(0.);
    }
    R g1, g2;
    if (E == 0) {
        g1 = divc(P, R(F.vel[0](i, j, k)) - R(F.vel[0](i, j - 1, k)), R(P.dx[1]), R(P.rdx[1]));  // u_y
        g2 = divc(P, R(F.vel[1](i, j, k)) - R(F.vel[1](i - 1, j, k)), R(P.dx[0]), R(P.rdx[0]));  // v_x
    } else if (E == 1) {
        g1 = divc(P, R(F.vel[0](i, j, k)) - R(F.vel[0](i, j, k - 1)), R(P.dx[2]), R(P.rdx[2]));  // u_z
        g2 = divc(P, R(F.vel[2](i, j, k)) - R(F.vel[2](i - 1, j, k)), R(P.dx[0]), R(P.rdx[0]));  // w_x
    } else {
        g1 = divc(P, R(F.vel[1](i, j, k)) - R(F.vel[1](i, j, k - 1)), R(P.dx[2]), R(P.rdx[2]));  // v_z
        g2 = divc(P, R(F.vel[2](i, j, k)) - R(F.vel[2](i, j - 1, k)), R(P.dx[1]), R(P.rdx[1]));  // w_y
    }
    R ei = R(0.25) * (F.eta(ai, aj, ak) + F.eta(bi, bj, bk) + F.eta(ci, cj, ck) + F.eta(i, j, k));
    if (WL) {
        // a wall plane: the gradient across it over the half cell to the wall value,
        // eta from the two ghost-side cells (fluxStag.cpp:939-954, 971-986, 1004-1019);
        // g1 is the gradient across the second direction, g2 across the first
        const int d1 = E == 2 ? 1 : 0, d2 = E == 0 ? 1 : 2;
        const int x1 = d1 == 0 ? i : j, x2 = d2 == 1 ? j : k;
        const R ea = F.eta(ai, aj, ak), eb = F.eta(bi, bj, bk), ec = F.eta(ci, cj, ck), ed = F.eta(i, j, k);
        R n1, n2;  // numerators of g1, g2
        if (E == 0) {
            n1 = R(F.vel[0](i, j, k)) - R(F.vel[0](i, j - 1, k));
            n2 = R(F.vel[1](i, j, k)) - R(F.vel[1](i - 1, j, k));
        } else if (E == 1) {
            n1 = R(F.vel[0](i, j, k)) - R(F.vel[0](i, j, k - 1));
            n2 = R(F.vel[2](i, j, k)) - R(F.vel[2](i - 1, j, k));
        } else {
            n1 = R(F.vel[1](i, j, k)) - R(F.vel[1](i, j, k - 1));
            n2 = R(F.vel[2](i, j, k)) - R(F.vel[2](i, j - 1, k));
        }
        if (x2 == 0 && dirichlet_side(P, 2 * d2)) {
            g1 = divc(P, n1, R(P.hdx[d2]), R(P.rhdx[d2]));
            ei = R(0.5) * (ea + ec);
        }
        if (x2 == P.n[d2] && dirichlet_side(P, 2 * d2 + 1)) {
            g1 = divc(P, n1, R(P.hdx[d2]), R(P.rhdx[d2]));
            ei = R(0.5) * (eb + ed);
        }
        if (x1 == 0 && dirichlet_side(P, 2 * d1)) {
            g2 = divc(P, n2, R(P.hdx[d1]), R(P.rhdx[d1]));
            ei = R(0.5) * (ea + eb);
        }
        if (x1 == P.n[d1] && dirichlet_side(P, 2 * d1 + 1)) {
            g2 = divc(P, n2, R(P.hdx[d1]), R(P.rhdx[d1]));
            ei = R(0.5) * (ec + ed);
        }
    }
    t.d = ei * (g1 + g2);
    return t;
}

template <int NS, class R, int NZ, bool WL = false>
FHD_D CellTaus<R> cell_taus(const DevParams& P, const Fields<NS, R>& F, const Noise<NZ>& nz, int i, int j, int k) {
    double wc[3] = {0.0, 0.0, 0.0};
    if (NZ != NZ_OFF) nz.cen_all(P, i, j, k, wc);
    return cell_taus_w<NS, R, NZ, WL>(P, F, wc, i, j, k);
}

template <int NS, class R, int NZ, int E, bool WL = false>
FHD_D Taus<R> edge_taus(const DevParams& P, const Fields<NS, R>& F, const Noise<NZ>& nz, int i, int j, int k) {
    return edge_taus_w<NS, R, NZ, E, WL>(P, F, NZ != NZ_OFF ? nz.edge(P, E, i, j, k) : 0.0, i, j, k);
}

// ---- face fluxes ---------------------------------------------------------------------
template <int NS>
struct FaceFlux {
    double cons[2 + NS];  // comps 0 (rho), 4 (rhoE), 5.. (rhoY)
    double aux[4];        // comps nvars .. nvars+3 (heat, visc. heating diag/shear, Dufour)
};

// TauGet: .cell(i,j,k) -> CellTaus, .edge<E>(i,j,k) -> Taus.
// WL: the box has physical walls.  A face on a wall plane (the reference's
// "(i == 0) and is_lo_x_dirichlet_mass" faces) then takes the wall values from the
// cell on the wall's ghost side with half-cell differences (fluxStag.cpp's
// Dirichlet branches), StochFluxStag's factors on its stochastic heat, species,
// Dufour and shear-heating parts (boundaryStag.cpp:2086-3009),
// BCWallReservoirFluxStag's zero species / Dufour fluxes on impermeable walls
// (boundaryStag.cpp:300-580) and no advective flux (fluxStag.cpp:1511-1529).
template <int NS, class R, int NZ, int D, class TauGet, bool WL = false>
FHD_D FaceFlux<NS> face_flux(const DevParams& P, const Fields<NS, R>& F, const Noise<NZ>& nz, const TauGet& tg,
                             int i, int j, int k) {
    constexpr int e0 = D == 0, e1 = D == 1, e2 = D == 2;
    const int im = i - e0, jm = j - e1, km = k - e2;
    const Arr4<const double>& velx = F.vel[0];
    const Arr4<const double>& vely = F.vel[1];
    const Arr4<const double>& velz = F.vel[2];
    // wall side of this face (0 lo, 1 hi, -1 none) and the cell holding the wall values
    const int ws = WL ? wall_face(P, D, D == 0 ? i : (D == 1 ? j : k)) : -1;
    const int gi = ws == 0 ? im : i, gj = ws == 0 ? jm : j, gk = ws == 0 ? km : k;
    const int wside = 2 * D + (ws == 1 ? 1 : 0);
    // a transverse face of a quasi-1-D (y, z) or 2-D (z) run carries no heat,
    // species or Dufour flux, stochastic or diffusive (fluxStag.cpp:504-510,
    // 666-672, 1185-1191, 1324-1330)
    const bool transverse = WL && ((D == 1 && P.dim == 1) || (D == 2 && P.dim < 3));
    // flux components in the reference's accumulation order
    R heat = R(0.0), vdiag = R(0.0), vshear = R(0.0), duf = R(0.0);
    R spec[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) spec[s] = R(0.0);

    const R un = R(F.vel[D](i, j, k));

    // ---- viscous heating terms, complete (stochastic part assigned,
    // fluxStag.cpp:298-781, then the deterministic part added, :1026-1426).  Each
    // flux variable keeps the reference's own sequence of operations; finishing
    // these two first only shortens the live ranges of their operands.
    {
    const CellTaus<R> tl = tg.cell(im, jm, km);
    const CellTaus<R> th = tg.cell(i, j, k);
    // the two transverse edge families touching this face and their (lo, hi) positions
    Taus<R> ea0, ea1, eb0, eb1;  // ea: first transverse dir, eb: second
    R va0l, va0h, va1l, va1h, vb0l, vb0h, vb1l, vb1h;  // transverse velocities (lo/hi sides of the face)
    if (D == 0) {
        ea0 = tg.template edge<0>(i, j, k);  ea1 = tg.template edge<0>(i, j + 1, k);
        eb0 = tg.template edge<1>(i, j, k);  eb1 = tg.template edge<1>(i, j, k + 1);
        va1h = R(vely(i, j + 1, k)); va1l = R(vely(i - 1, j + 1, k));
        va0h = R(vely(i, j, k));     va0l = R(vely(i - 1, j, k));
        vb1h = R(velz(i, j, k + 1)); vb1l = R(velz(i - 1, j, k + 1));
        vb0h = R(velz(i, j, k));     vb0l = R(velz(i - 1, j, k));
    } else if (D == 1) {
        ea0 = tg.template edge<0>(i, j, k);  ea1 = tg.template edge<0>(i + 1, j, k);
        eb0 = tg.template edge<2>(i, j, k);  eb1 = tg.template edge<2>(i, j, k + 1);
        va1h = R(velx(i + 1, j, k)); va1l = R(velx(i + 1, j - 1, k));
        va0h = R(velx(i, j, k));     va0l = R(velx(i, j - 1, k));
        vb1h = R(velz(i, j, k + 1)); vb1l = R(velz(i, j - 1, k + 1));
        vb0h = R(velz(i, j, k));     vb0l = R(velz(i, j - 1, k));
    } else {
        ea0 = tg.template edge<1>(i, j, k);  ea1 = tg.template edge<1>(i + 1, j, k);
        eb0 = tg.template edge<2>(i, j, k);  eb1 = tg.template edge<2>(i, j + 1, k);
        va1h = R(velx(i + 1, j, k)); va1l = R(velx(i + 1, j, k - 1));
        va0h = R(velx(i, j, k));     va0l = R(velx(i, j, k - 1));
        vb1h = R(vely(i, j + 1, k)); vb1l = R(vely(i, j + 1, k - 1));
        vb0h = R(vely(i, j, k));     vb0l = R(vely(i, j, k - 1));
    }
    if (NZ != NZ_OFF) {
        vdiag = R(0.5) * un * (tl.s[D] + th.s[D]);
        R vsh = R(0.0);
        if (WL && ws == 0) {
            vsh += R(0.5) * (va1l * ea1.s + va0l * ea0.s);
            vsh += R(0.5) * (vb1l * eb1.s + vb0l * eb0.s);
        } else if (WL && ws == 1) {
            vsh += R(0.5) * (va1h * ea1.s + va0h * ea0.s);
            vsh += R(0.5) * (vb1h * eb1.s + vb0h * eb0.s);
        } else {
            vsh += R(0.25) * ((va1h + va1l) * ea1.s + (va0h + va0l) * ea0.s);
            vsh += R(0.25) * ((vb1h + vb1l) * eb1.s + (vb0h + vb0l) * eb0.s);
        }
        vshear = vsh;
        // StochFluxStag: velocity walls scale the stochastic shear heating (a
        // reservoir side keeps the factor 1)
        if (WL && ws >= 0 && (P.bc_vel[wside] == 1 || P.bc_vel[wside] == 2) && P.bc_mass[wside] < 3)
            vshear *= R(stoch_factor(P, P.bc_vel[wside]));
    }
    vdiag -= R(0.5) * un * (tl.d[D] + th.d[D]);
    R vsh = R(0.0);
    if (WL && ws == 0) {
        vsh -= R(0.5) * (va1l * ea1.d + va0l * ea0.d);
        vsh -= R(0.5) * (vb1l * eb1.d + vb0l * eb0.d);
    } else if (WL && ws == 1) {
        vsh -= R(0.5) * (va1h * ea1.d + va0h * ea0.d);
        vsh -= R(0.5) * (vb1h * eb1.d + vb0h * eb0.d);
    } else {
        vsh -= R(0.25) * ((va1h + va1l) * ea1.d + (va0h + va0l) * ea0.d);
        vsh -= R(0.25) * ((vb1h + vb1l) * eb1.d + (vb0h + vb0l) * eb0.d);
    }
    vshear += vsh;
    }

    // ---- stochastic part (fluxStag.cpp:298-781) ----
    if (NZ != NZ_OFF && !transverse) {
        const R Th = R(F.T(i, j, k)), Tl = R(F.T(im, jm, km));
        R kp = (F.kappa(i, j, k) * Th * Th + F.kappa(im, jm, km) * Tl * Tl);
        R meanT = R(0.5) * (Th + Tl);
        if (WL && ws >= 0) {
            const R Tg = R(F.T(gi, gj, gk));
            kp = R(2.0) * F.kappa(gi, gj, gk) * Tg * Tg;
            meanT = Tg;
        }
        double wf[NS + 1];
        nz.template face_all<NS + 1>(P, D, i, j, k, wf);
        const R fw0 = dsqrt(R(P.k_B) * kp * R(P.volinv) * R(P.dtinv));
        heat = fw0 * R(wf[0]);
        // StochFluxStag: thermal walls scale the stochastic heat flux (a reservoir
        // side keeps the factor 1)
        if (WL && ws >= 0 && (P.bc_therm[wside] == 1 || P.bc_therm[wside] == 2) && P.bc_mass[wside] < 3)
            heat *= R(stoch_factor(P, P.bc_therm[wside]));
        // species noise, Soret: mixtures only (a single gas has no species flux)
        if constexpr (NS > 1) {
        R yy[NS], yyp[NS], DY[NS * NS], sqD[NS * NS], hk[NS], wien[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            wien[s] = R(0.);
            yy[s] = clamp01(R(F.Y(im, jm, km, s)));
            yyp[s] = clamp01(R(F.Y(i, j, k, s)));
            if (WL && ws == 0) yyp[s] = clamp01(R(F.Y(im, jm, km, s)));
            if (WL && ws == 1) yy[s] = clamp01(R(F.Y(i, j, k, s)));
        }
        R sumy = R(0.), sumyp = R(0.);
#pragma unroll
        for (int n = 0; n < NS; ++n) { sumy += yy[n]; sumyp += yyp[n]; }
#pragma unroll
        for (int n = 0; n < NS; ++n) { yy[n] = rdiv(yy[n], sumy); yyp[n] = rdiv(yyp[n], sumyp); }
        R MWmix = R(0.);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            MWmix = MWmix + divc(P, R(0.5) * (yy[s] + yyp[s]), R(P.molmass[s]), R(P.rmolmass[s]));
#pragma unroll
            for (int ll = 0; ll < NS; ++ll) {
                if (WL && ws >= 0)
                    DY[s * NS + ll] = R(0.5) * (F.D(gi, gj, gk, ll * NS + s) * yy[ll] + F.D(gi, gj, gk, ll * NS + s) * yyp[ll] +
                                                (F.D(gi, gj, gk, s * NS + ll) * yy[s] + F.D(gi, gj, gk, s * NS + ll) * yyp[s]));
                else
                    DY[s * NS + ll] = R(0.5) * (F.D(im, jm, km, ll * NS + s) * yy[ll] + F.D(i, j, k, ll * NS + s) * yyp[ll] +
                                                (F.D(im, jm, km, s * NS + ll) * yy[s] + F.D(i, j, k, s * NS + ll) * yyp[s]));
            }
        }
#pragma unroll
        for (int s = 0; s < NS; ++s)
            if (fabs(yy[s]) + fabs(yyp[s]) <= R(1.e-12)) {
#pragma unroll
                for (int n = 0; n < NS; ++n) { DY[s * NS + n] = R(0.); DY[n * NS + s] = R(0.); }
            }
        MWmix = rdiv(R(1.), MWmix);
        CholeskyDecomp<NS, R>(DY, sqD);
        const R fwc = dsqrt(divc(P, R(P.k_B) * MWmix * R(P.volinv), R(P.Runiv) * R(P.dt), R(P.rRdt)));
        R zs[NS];
#pragma unroll
        for (int ll = 0; ll < NS; ++ll) zs[ll] = R(wf[1 + ll]);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
#pragma unroll
            for (int ll = 0; ll <= s; ++ll) wien[s] = wien[s] + fwc * sqD[s * NS + ll] * zs[ll];
            spec[s] = wien[s];
        }
        GetEnthalpies<NS, R>(P, meanT, hk);
        R soret = R(0.);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            R soret_s;
            if (WL && ws >= 0)
                soret_s = (hk[s] + divc(P, R(P.Runiv) * meanT, R(P.molmass[s]), R(P.rmolmass[s])) *
                                       F.chi(gi, gj, gk, s)) * wien[s];
            else
                soret_s = (hk[s] + divc(P, R(P.Runiv) * meanT, R(P.molmass[s]), R(P.rmolmass[s])) * R(0.5) *
                                       (F.chi(im, jm, km, s) + F.chi(i, j, k, s))) * wien[s];
            soret += soret_s;
        }
        duf = soret;
        // StochFluxStag: mass walls scale the stochastic species and Dufour fluxes
        if (WL && ws >= 0 && (P.bc_mass[wside] == 1 || P.bc_mass[wside] == 2)) {
            const R f = R(stoch_factor(P, P.bc_mass[wside]));
#pragma unroll
            for (int s = 0; s < NS; ++s) spec[s] *= f;
            duf *= f;
        }
        }
    }

    // ---- diffusive part (fluxStag.cpp:1026-1426) ----
    if (!transverse) {
        // wall faces difference over the half cell to the wall value
        const R h = (WL && ws >= 0) ? R(P.hdx[D]) : R(P.dx[D]);
        const R rh = (WL && ws >= 0) ? R(P.rhdx[D]) : R(P.rdx[D]);
        const R Tl = R(F.T(im, jm, km)), Th = R(F.T(i, j, k));
        const R pl = R(F.p(im, jm, km)), ph = R(F.p(i, j, k));
        R kp = R(0.5) * (F.kappa(im, jm, km) + F.kappa(i, j, k));
        R meanT = R(0.5) * (Tl + Th);
        R meanP = R(0.5) * (pl + ph);
        if (WL && ws >= 0) {
            kp = F.kappa(gi, gj, gk);
            meanT = R(F.T(gi, gj, gk));
            meanP = R(F.p(gi, gj, gk));
        }
        heat -= divc(P, kp * (Th - Tl), h, rh);
        // species diffusion, Dufour: mixtures only
        if constexpr (NS > 1) {
        R dk[NS], sor[NS], Fk[NS], hk[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const R Xl = R(F.X(im, jm, km, s)), Xh = R(F.X(i, j, k, s));
            const R term1 = divc(P, Xh - Xl, h, rh);
            R mX = R(0.5) * (Xl + Xh);
            R mY = R(0.5) * (R(F.Y(im, jm, km, s)) + R(F.Y(i, j, k, s)));
            if (WL && ws >= 0) {
                mX = R(F.X(gi, gj, gk, s));
                mY = R(F.Y(gi, gj, gk, s));
            }
            const R term2 = divz(divc0(P, (mX - mY) * (ph - pl), h, rh), meanP);
            dk[s] = term1 + term2;
            R ChiX = R(0.5) * (F.chi(im, jm, km, s) * Xl + F.chi(i, j, k, s) * Xh);
            if (WL && ws >= 0) ChiX = F.chi(gi, gj, gk, s) * R(F.X(gi, gj, gk, s));
            sor[s] = divz(divc0(P, ChiX * (Th - Tl), h, rh), meanT);
        }
#pragma unroll
        for (int kk = 0; kk < NS; ++kk) {
            R f = R(0.);
#pragma unroll
            for (int ll = 0; ll < NS; ++ll) {
                R Fks;
                if (WL && ws >= 0) Fks = F.D(gi, gj, gk, ll * NS + kk) * (dk[ll] + sor[ll]);
                else Fks = R(0.5) * (F.D(im, jm, km, ll * NS + kk) + F.D(i, j, k, ll * NS + kk)) * (dk[ll] + sor[ll]);
                f -= Fks;
            }
            Fk[kk] = f;
        }
        GetEnthalpies<NS, R>(P, meanT, hk);
        R Q5 = R(0.);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            if (WL && ws >= 0) {
                Q5 += (hk[s] + divc0(P, R(P.Runiv) * meanT * F.chi(gi, gj, gk, s), R(P.molmass[s]), R(P.rmolmass[s]))) *
                      Fk[s];
            } else {
                // z faces use chi(i,j,k)+chi(i,j,k), fluxStag.cpp:1407 (kept from the reference)
                const R chs = (D == 2) ? (F.chi(i, j, k, s) + F.chi(i, j, k, s)) : (F.chi(im, jm, km, s) + F.chi(i, j, k, s));
                Q5 += (hk[s] + divc0(P, R(0.5) * R(P.Runiv) * meanT * chs, R(P.molmass[s]), R(P.rmolmass[s]))) * Fk[s];
            }
        }
        duf += Q5;
#pragma unroll
        for (int s = 0; s < NS; ++s) spec[s] += Fk[s];
        }
        // BCWallReservoirFluxStag: impermeable walls carry no species or Dufour flux
        if (WL && ws >= 0 && P.bc_mass[wside] == 1) {
#pragma unroll
            for (int s = 0; s < NS; ++s) spec[s] = R(0.);
            duf = R(0.);
        }
    }

    // ---- hyperbolic part (fluxStag.cpp:1508-1764), in double ----
    FaceFlux<NS> out;
    double f0 = 0.0, f4 = 0.0;
    double fs[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) fs[s] = (double)spec[s];
    const int adv = P.advection_type;
    if (WL && ws >= 0) {
        // no advection through a wall face (fluxStag.cpp:1511-1529)
        f0 += 0.0;
        f4 += 0.0;
#pragma unroll
        for (int s = 0; s < NS; ++s) fs[s] += 0.0;
    } else if (adv >= 0) {
        const double m = F.mom[D](i, j, k);
        const double u = F.vel[D](i, j, k);
        f0 += m;
        const double pl = F.p(im, jm, km), ph = F.p(i, j, k);
        if (adv == 2) {
            f4 += 0.5 * (F.cons(im, jm, km, 4) + F.cons(i, j, k, 4)) * u + 0.5 * (pl + ph) * u;
#pragma unroll
            for (int s = 0; s < NS; ++s) fs[s] += 0.5 * (F.cons(im, jm, km, 5 + s) + F.cons(i, j, k, 5 + s)) * u;
        } else {
            const double meanT = 0.5 * (F.T(im, jm, km) + F.T(i, j, k));
            const double meanRho = 0.5 * (F.cons(im, jm, km, 0) + F.cons(i, j, k, 0));
            double hk[NS];
            GetEnthalpies<NS, double>(P, meanT, hk);
            if (adv == 1) {
                const double meanE = 0.5 * (F.cons(im, jm, km, 4) + F.cons(i, j, k, 4)) / meanRho;
                const double meanP = 0.5 * (pl + ph);
                f4 += m * (meanE + (meanP / meanRho));
            }
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const double Yk = 0.5 * (F.Y(im, jm, km, s) + F.Y(i, j, k, s));
                fs[s] += Yk * m;
                if (adv == 0) f4 += m * Yk * hk[s];
            }
            if (adv == 0) {
                const Arr4<const double>& mx = F.mom[0];
                const Arr4<const double>& my = F.mom[1];
                const Arr4<const double>& mz = F.mom[2];
                double keP = 0., keM = 0.;
                keP += (mx(i + 1, j, k) + mx(i, j, k)) * (mx(i + 1, j, k) + mx(i, j, k));
                keP += (my(i, j + 1, k) + my(i, j, k)) * (my(i, j + 1, k) + my(i, j, k));
                keP += (mz(i, j, k + 1) + mz(i, j, k)) * (mz(i, j, k + 1) + mz(i, j, k));
                keP *= (0.125 / F.cons(i, j, k, 0) / F.cons(i, j, k, 0));
                keM += (mx(im + 1, jm, km) + mx(im, jm, km)) * (mx(im + 1, jm, km) + mx(im, jm, km));
                keM += (my(im, jm + 1, km) + my(im, jm, km)) * (my(im, jm + 1, km) + my(im, jm, km));
                keM += (mz(im, jm, km + 1) + mz(im, jm, km)) * (mz(im, jm, km + 1) + mz(im, jm, km));
                // z faces divide by cons(i,j-1,k,0), fluxStag.cpp:1755 (kept from the reference)
                const double rm = (D == 2) ? F.cons(i, j - 1, k, 0) : F.cons(im, jm, km, 0);
                keM *= (0.125 / rm / rm);
                f4 += m * 0.5 * (keP + keM);
            }
        }
    }
    out.aux[0] = (double)heat;
    out.aux[1] = (double)vdiag;
    out.aux[2] = (double)vshear;
    out.aux[3] = (double)duf;
    f4 += out.aux[0] + out.aux[1] + out.aux[2] + out.aux[3];
    // a single gas: its species density is the density, so its flux is the mass
    // flux exactly (rhoY stays bitwise equal to rho through the RK update)
    if constexpr (NS == 1) fs[0] = f0;
    out.cons[0] = f0;
    out.cons[1] = f4;
#pragma unroll
    for (int s = 0; s < NS; ++s) out.cons[2 + s] = fs[s];
    return out;
}

// ---- momentum fluxes --------------------------------------------------------------
// advective edge terms (fluxStag.cpp:1767-1845): returns the two fluxes of edge E:
// E=0 xy: (edgey_u, edgex_v); E=1 xz: (edgez_u, edgex_w); E=2 yz: (edgez_v, edgey_w)
// WL: walls; an edge on a wall plane takes the momentum / velocity of its wall
// side only (fluxStag.cpp:1774-1789, 1797-1812, 1820-1835: the second
// direction's wall is tested first, the first direction's wins a corner).
template <int NS, class R, int E, bool WL = false>
FHD_D void edge_adv(const DevParams& P, const Fields<NS, R>& F, int i, int j, int k, double& a, double& b) {
    const Arr4<const double>&mx = F.mom[0], &my = F.mom[1], &mz = F.mom[2];
    const Arr4<const double>&vx = F.vel[0], &vy = F.vel[1], &vz = F.vel[2];
    if (P.advection_type < 0) { a = b = 0.0; return; }
    // edge of directions (p, q) = xy, xz or yz: a carries the p-momentum along q
    // (m0, m1 the p-face momenta on the q-1 / q sides, u0, u1 the q-face velocities
    // on the p-1 / p sides), b the q-momentum along p (n0, n1 on the p sides, w0,
    // w1 the p-face velocities on the q sides)
    double m0, m1, u0, u1, n0, n1, w0, w1;
    if (E == 0) {
        m0 = mx(i, j - 1, k); m1 = mx(i, j, k); u0 = vy(i - 1, j, k); u1 = vy(i, j, k);
        n0 = my(i - 1, j, k); n1 = my(i, j, k); w0 = vx(i, j - 1, k); w1 = vx(i, j, k);
    } else if (E == 1) {
        m0 = mx(i, j, k - 1); m1 = mx(i, j, k); u0 = vz(i - 1, j, k); u1 = vz(i, j, k);
        n0 = mz(i - 1, j, k); n1 = mz(i, j, k); w0 = vx(i, j, k - 1); w1 = vx(i, j, k);
    } else {
        m0 = my(i, j, k - 1); m1 = my(i, j, k); u0 = vz(i, j - 1, k); u1 = vz(i, j, k);
        n0 = mz(i, j - 1, k); n1 = mz(i, j, k); w0 = vy(i, j, k - 1); w1 = vy(i, j, k);
    }
    a = 0.25 * (m0 + m1) * (u0 + u1);
    b = 0.25 * (n0 + n1) * (w0 + w1);
    if (WL) {
        const int dp = E == 2 ? 1 : 0, dq = E == 0 ? 1 : 2;
        const int xp = dp == 0 ? i : j, xq = dq == 1 ? j : k;
        if (xq == 0 && dirichlet_side(P, 2 * dq)) { a = 0.5 * (m0) * (u0 + u1); b = 0.5 * (n0 + n1) * (w0); }
        if (xq == P.n[dq] && dirichlet_side(P, 2 * dq + 1)) { a = 0.5 * (m1) * (u0 + u1); b = 0.5 * (n0 + n1) * (w1); }
        if (xp == 0 && dirichlet_side(P, 2 * dp)) { a = 0.5 * (m0 + m1) * (u0); b = 0.5 * (n0) * (w0 + w1); }
        if (xp == P.n[dp] && dirichlet_side(P, 2 * dp + 1)) { a = 0.5 * (m0 + m1) * (u1); b = 0.5 * (n1) * (w0 + w1); }
    }
}

// edge momentum flux = tau_s - tau_d + advective (fluxStag.cpp:784-796, 1429-1441, 1767-1845)
template <class R>
FHD_D double edge_total(const Taus<R>& t, double adv, int has_adv) {
    double v = (double)t.s;
    v -= (double)t.d;
    if (has_adv) v += adv;
    return v;
}

// the same with walls: StochFluxStag's velocity-wall factors on the stochastic part
// of an edge of type E lying on wall planes, in its order (lo x, hi x, lo y, hi y,
// lo z, hi z; boundaryStag.cpp:2456-3009)
template <class R, int E>
FHD_D double edge_total_w(const DevParams& P, const Taus<R>& t, double adv, int has_adv, int i, int j, int k) {
    double v = (double)t.s;
    const int x[3] = {i, j, k};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const bool along = (E == 0) ? (d != 2) : (E == 1) ? (d != 1) : (d != 0);  // the edge is nodal in d
        if (!along) continue;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int side = 2 * d + h, b = P.bc_vel[side];
            // a reservoir side keeps the factor 1
            if ((b == 1 || b == 2) && P.bc_mass[side] < 3 && x[d] == (h ? P.n[d] : 0)) v *= stoch_factor(P, b);
        }
    }
    v -= (double)t.d;
    if (has_adv) v += adv;
    return v;
}

// centre momentum flux in direction d at a cell (fluxStag.cpp:799-803, 1444-1448, 1848-1866).
// WL: the stochastic and diffusive part of a ghost cell beyond a reservoir side of
// direction d is 0 (bc_mass 3) or, given as `inner` (bc_mass 4), that of the cell
// inside it (BCWallReservoirFluxStag, boundaryStag.cpp:482-577).
template <int NS, class R, bool WL = false>
FHD_D double cen_total(const DevParams& P, const Fields<NS, R>& F, const CellTaus<R>& t, int d, int i, int j, int k,
                       const CellTaus<R>* inner = nullptr) {
    double v = (double)t.s[d];
    v -= (double)t.d[d];
    if (WL) {
        const int x = d == 0 ? i : (d == 1 ? j : k);
        const int side = x < 0 ? 2 * d : (x > P.n[d] - 1 ? 2 * d + 1 : -1);
        if (side >= 0 && P.bc_mass[side] == 3) v = 0.0;
        if (side >= 0 && P.bc_mass[side] == 4 && inner) {
            v = (double)inner->s[d];
            v -= (double)inner->d[d];
        }
    }
    if (P.advection_type >= 0) {
        if (WL && d >= P.dim) {
            v += 0.0;   // no transverse pressure / advection term in 1-D and 2-D (fluxStag.cpp:1850-1860)
        } else {
            const Arr4<const double>& m = F.mom[d];
            const Arr4<const double>& u = F.vel[d];
            const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
            v += 0.25 * (m(i, j, k) + m(i + e0, j + e1, k + e2)) * (u(i, j, k) + u(i + e0, j + e1, k + e2)) +
                 F.p(i, j, k);
        }
    }
    return v;
}

}  // namespace fhd
