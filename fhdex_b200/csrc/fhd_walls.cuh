// fhd_walls.cuh — physical boundaries of the staggered step (boundaryStag.cpp):
// the ghost-cell and wall-face conditions that setBCStag applies after each
// stage's conversion, as two kernels:
//
//   k_bc_mom       BCMomNormal + BCMomTrans of the three face-momentum / face-
//                  velocity pairs (boundaryStag.cpp:1289-1661)
//   k_bc_prim<NS>  BCMassTempPress of the three directions followed by BCRhoRhoE
//                  (boundaryStag.cpp:840-1287, 1663-2084)
//
// The reference applies these as one pass per direction and side, each over the
// whole grown box, so that a corner ghost is written several times and the last
// direction's pass wins.  Here every ghost point is written once, by a thread that
// composes the passes it would have seen: the value a reflecting pass copies from
// its mirror point is itself the result of the earlier passes at that point, so a
// point that is a ghost in several wall directions walks its mirror chain from the
// last direction back to the first (a constant wall value ends the walk) and reads
// the stored value at the end of the chain, which is always a point no pass
// writes.  Factors (slip 1, no-slip 0) multiply in the passes' order.
#pragma once
#include "fhd_device.cuh"

namespace fhd {

// the points of box B = [blo, bhi] outside its core C = [clo, chi]
struct Shell {
    int blo[3], bhi[3], clo[3], chi[3];
    int64_t n;
};

FHD_HD int64_t span(int a, int b) { return b >= a ? (int64_t)(b - a + 1) : 0; }

inline Shell make_shell(const int blo[3], const int bhi[3], const int clo[3], const int chi[3]) {
    Shell s;
    int64_t nb = 1, nc = 1;
    for (int d = 0; d < 3; ++d) {
        s.blo[d] = blo[d];
        s.bhi[d] = bhi[d];
        s.clo[d] = clo[d];
        s.chi[d] = chi[d];
        nb *= span(blo[d], bhi[d]);
        nc *= span(clo[d], chi[d]);
    }
    s.n = nb - nc;
    return s;
}

// q-th point of the shell: the z slabs below and above the core (whole x-y
// planes), then the y slabs beside it (core z), then the x slabs (core y and z)
FHD_D void shell_point(const Shell& s, int64_t q, int& i, int& j, int& k) {
    const int64_t BX = span(s.blo[0], s.bhi[0]), BY = span(s.blo[1], s.bhi[1]);
    const int64_t CX = span(s.clo[0], s.chi[0]), CY = span(s.clo[1], s.chi[1]), CZ = span(s.clo[2], s.chi[2]);
    if (CX == 0 || CY == 0 || CZ == 0) {
        i = s.blo[0] + (int)(q % BX);
        j = s.blo[1] + (int)((q / BX) % BY);
        k = s.blo[2] + (int)(q / (BX * BY));
        return;
    }
    const int64_t zb = span(s.blo[2], s.clo[2] - 1), za = span(s.chi[2] + 1, s.bhi[2]);
    const int64_t nz = (zb + za) * BX * BY;
    if (q < nz) {
        const int64_t kk = q / (BX * BY), r = q % (BX * BY);
        i = s.blo[0] + (int)(r % BX);
        j = s.blo[1] + (int)(r / BX);
        k = kk < zb ? s.blo[2] + (int)kk : s.chi[2] + 1 + (int)(kk - zb);
        return;
    }
    q -= nz;
    const int64_t yb = span(s.blo[1], s.clo[1] - 1), ya = span(s.chi[1] + 1, s.bhi[1]);
    const int64_t ny = (yb + ya) * BX * CZ;
    if (q < ny) {
        const int64_t kk = q / ((yb + ya) * BX), r = q % ((yb + ya) * BX), jj = r / BX;
        i = s.blo[0] + (int)(r % BX);
        j = jj < yb ? s.blo[1] + (int)jj : s.chi[1] + 1 + (int)(jj - yb);
        k = s.clo[2] + (int)kk;
        return;
    }
    q -= ny;
    const int64_t xb = span(s.blo[0], s.clo[0] - 1), xa = span(s.chi[0] + 1, s.bhi[0]);
    const int64_t ii = q % (xb + xa), r = q / (xb + xa);
    i = ii < xb ? s.blo[0] + (int)ii : s.chi[0] + 1 + (int)(ii - xb);
    j = s.clo[1] + (int)(r % CY);
    k = s.clo[2] + (int)(r / CY);
}

FHD_HD bool wall_dir(const DevParams& P, int d) { return P.walls && !P.periodic[d]; }

// ---- face momentum and velocity --------------------------------------------------
// For mom[d] / vel[d] (nodal in d): BCMomNormal zeroes the wall faces and the
// ghosts beyond them in d; BCMomTrans then sets the ghosts of every other wall
// direction e to fac * (the value at the mirror point -x-1 / 2n-1-x), fac = 1 on a
// slip and 0 on a no-slip wall, directions in the order x, y, z.
struct BcMomArgs {
    DevParams P;
    Arr4<double> mom[3], vel[3];
    Shell sh[3];
};

static __global__ void __launch_bounds__(256) k_bc_mom(BcMomArgs a) {
    const int d = blockIdx.y;
    const DevParams& P = a.P;
    const Shell& sh = a.sh[d];
    const Arr4<double>& mom = a.mom[d];
    const Arr4<double>& vel = a.vel[d];
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < sh.n; q += (int64_t)gridDim.x * blockDim.x) {
        int p[3];
        shell_point(sh, q, p[0], p[1], p[2]);
        int m[3] = {p[0], p[1], p[2]};
        int side[3] = {-1, -1, -1};
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            if (e == d || !wall_dir(P, e)) continue;
            if (p[e] < 0) { side[e] = 2 * e; m[e] = -p[e] - 1; }
            else if (p[e] > P.n[e] - 1) { side[e] = 2 * e + 1; m[e] = 2 * P.n[e] - 1 - p[e]; }
        }
        const bool normal = wall_dir(P, d) && (p[d] <= 0 || p[d] >= P.n[d]);
        double vm = 0.0, vv = 0.0;
        if (!normal) {
            vm = mom(m[0], m[1], m[2]);
            vv = vel(m[0], m[1], m[2]);
        }
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            if (side[e] < 0) continue;
            const double fac = P.bc_vel[side[e]] == 1 ? 1.0 : 0.0;
            vm = fac * vm;
            vv = fac * vv;
        }
        mom(p[0], p[1], p[2]) = vm;
        vel(p[0], p[1], p[2]) = vv;
    }
}

// ---- ghost-cell state ------------------------------------------------------------
// BCMassTempPress per wall side: an impermeable wall (bc_mass 1) mirrors Y and X,
// a concentration wall (2) sets them to the wall composition; an adiabatic wall
// (bc_therm 1) mirrors T and p, an isothermal one (2) sets T to the wall
// temperature and mirrors p.  BCRhoRhoE then sets rho = GetDensity(p, T, Y) in
// prim and cons, rho Y, and rho E = rho e(T, Y) + the kinetic energy of the
// ghost's face momenta.
template <int NS>
struct BcPrimArgs {
    DevParams P;
    WallParams W;
    Arr4<double> prim, cons;
    Arr4<const double> mom[3];
    Shell sh;
};

template <int NS>
static __global__ void __launch_bounds__(128) k_bc_prim(BcPrimArgs<NS> a) {
    const DevParams& P = a.P;
    const WallParams& W = a.W;
    const Arr4<double>& prim = a.prim;
    constexpr int NPRIM = 6 + 2 * NS;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < a.sh.n; q += (int64_t)gridDim.x * blockDim.x) {
        int p[3];
        shell_point(a.sh, q, p[0], p[1], p[2]);
        int side[3] = {-1, -1, -1}, mir[3] = {p[0], p[1], p[2]};
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            if (!wall_dir(P, e)) continue;
            if (p[e] < 0) { side[e] = 2 * e; mir[e] = -p[e] - 1; }
            else if (p[e] > P.n[e] - 1) { side[e] = 2 * e + 1; mir[e] = 2 * P.n[e] - 1 - p[e]; }
        }
        double v[NPRIM];
#pragma unroll
        for (int c = 4; c < NPRIM; ++c) {
            int m[3] = {p[0], p[1], p[2]};
            bool set = false;
            for (int e = 2; e >= 0 && !set; --e) {
                const int s = side[e];
                if (s < 0) continue;
                if (c == 4 && P.bc_therm[s] == 2) { v[c] = W.t[s]; set = true; }
                else if (c >= 6 && P.bc_mass[s] == 2) {
                    v[c] = c < 6 + NS ? W.Yk[s][c - 6] : W.Xk[s][c - 6 - NS];
                    set = true;
                } else {
                    m[e] = mir[e];
                }
            }
            if (!set) v[c] = prim(m[0], m[1], m[2], c);
        }
#pragma unroll
        for (int c = 4; c < NPRIM; ++c) prim(p[0], p[1], p[2], c) = v[c];
        // BCRhoRhoE (GetDensity, GetEnergy: compressible_functions.H:1481-1511)
        const double T = v[4], pt = v[5];
        double molmix = 0.;
#pragma unroll
        for (int n = 0; n < NS; ++n) molmix += v[6 + n] / P.molmass[n];
        molmix = 1. / molmix;
        const double rho = pt / (P.Runiv / molmix) / T;
        double cvmix = 0., e0mix = 0.;
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            cvmix += v[6 + n] * P.hcv[n];
            e0mix += v[6 + n] * P.e0[n];
        }
        const double intenergy = e0mix + T * cvmix;
        const int i = p[0], j = p[1], k = p[2];
        prim(i, j, k, 0) = rho;
        a.cons(i, j, k, 0) = rho;
#pragma unroll
        for (int n = 0; n < NS; ++n) a.cons(i, j, k, 5 + n) = rho * v[6 + n];
        const Arr4<const double>&mx = a.mom[0], &my = a.mom[1], &mz = a.mom[2];
        double kin = 0.;
        kin += (mx(i + 1, j, k) + mx(i, j, k)) * (mx(i + 1, j, k) + mx(i, j, k));
        kin += (my(i, j + 1, k) + my(i, j, k)) * (my(i, j + 1, k) + my(i, j, k));
        kin += (mz(i, j, k + 1) + mz(i, j, k)) * (mz(i, j, k + 1) + mz(i, j, k));
        kin *= (0.125 / rho);
        a.cons(i, j, k, 4) = rho * intenergy + kin;
    }
}

// ---- one pass of the reference's boundary routines ---------------------------------
// With reservoirs (bc_mass 3: ghost cells held at the reservoir's state, flow through
// the interface) the reference's passes read values that earlier passes of the same
// call left at ghost corners, some of them through the density in cons, so they run
// here one launch per pass, in the reference's order, each over the slab of the grown
// box beyond one side:
//   BC_MTP   BCMassTempPress of side s     (prim; cons rho on reservoir sides)
//   BC_MOMN  BCMomNormal of side s         (mom[d], vel[d]; d = the side's direction)
//   BC_MOMT  BCMomTrans of side s on mom[c], vel[c] (c != d)
//   BC_RRE   BCRhoRhoE of side s           (prim rho, cons rho, rho E, rho Y)
enum { BC_MTP = 0, BC_MOMN = 1, BC_MOMT = 2, BC_RRE = 3 };

template <int NS>
struct BcPassArgs {
    DevParams P;
    WallParams W;
    Arr4<double> prim, cons, mom, vel;   // mom, vel: component c (BC_MOMN: c = d)
    Arr4<const double> mx, my, mz;       // face momenta (BC_RRE)
    int fn, side, c;
    int blo[3], bhi[3];                  // the slab
};

template <int NS>
static __global__ void __launch_bounds__(128) k_bc_pass(BcPassArgs<NS> a) {
    const DevParams& P = a.P;
    const WallParams& W = a.W;
    const int s = a.side, d = s >> 1, hi = s & 1;
    const int64_t nx = a.bhi[0] - a.blo[0] + 1, ny = a.bhi[1] - a.blo[1] + 1, nz = a.bhi[2] - a.blo[2] + 1;
    const int64_t tot = nx * ny * nz;
    const int bm = P.bc_mass[s], bt = P.bc_therm[s], bv = P.bc_vel[s];
    constexpr int NPRIM = 6 + 2 * NS;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
        int p[3] = {a.blo[0] + (int)(q % nx), a.blo[1] + (int)((q / nx) % ny), a.blo[2] + (int)(q / (nx * ny))};
        const int i = p[0], j = p[1], k = p[2];
        const int n = P.n[d];
        int m[3] = {i, j, k};
        m[d] = hi ? 2 * n - 1 - p[d] : -p[d] - 1;   // mirror across the side (cell-centred direction d)
        if (a.fn == BC_MTP) {
            const Arr4<double>& pr = a.prim;
            if (bm == 1)
                for (int c = 6; c < NPRIM; ++c) pr(i, j, k, c) = pr(m[0], m[1], m[2], c);
            if (bm == 2)
                for (int c = 0; c < NS; ++c) {
                    pr(i, j, k, 6 + c) = W.Yk[s][c];
                    pr(i, j, k, 6 + NS + c) = W.Xk[s][c];
                }
            if (bm >= 3) {
                for (int c = 0; c < NS; ++c) {
                    pr(i, j, k, 6 + c) = W.Yk[s][c];
                    pr(i, j, k, 6 + NS + c) = W.Xk[s][c];
                    pr(i, j, k, 0) = W.rho[s];
                    a.cons(i, j, k, 0) = W.rho[s];
                    pr(i, j, k, 4) = W.t[s];
                    pr(i, j, k, 5) = W.p[s];
                }
            } else if (bt == 1) {
                for (int c = 4; c < 6; ++c) pr(i, j, k, c) = pr(m[0], m[1], m[2], c);
            } else if (bt == 2) {
                pr(i, j, k, 4) = W.t[s];
                pr(i, j, k, 5) = pr(m[0], m[1], m[2], 5);
            }
        } else if (a.fn == BC_MOMN) {
            // mom[d], vel[d] are nodal in d: the interface face is n_d * hi
            const int f = hi ? n : 0;
            const bool ghost = hi ? p[d] > f : p[d] < f;
            int fi[3] = {i, j, k}, gi[3] = {i, j, k};
            fi[d] = f;            // the interface face / the cell inside it
            gi[d] = f - 1;        // the cell before it
            if (bm >= 3) {
                if (ghost) {
                    a.vel(i, j, k) = -2 * a.mom(fi[0], fi[1], fi[2]) /
                                     (a.cons(fi[0], fi[1], fi[2], 0) + a.cons(gi[0], gi[1], gi[2], 0));
                    a.mom(i, j, k) = -1 * a.mom(fi[0], fi[1], fi[2]);
                } else if (p[d] == f) {
                    a.vel(i, j, k) = 2 * a.mom(i, j, k) / (a.cons(fi[0], fi[1], fi[2], 0) + a.cons(gi[0], gi[1], gi[2], 0));
                }
            } else if (bv == 1 || bv == 2) {
                if (ghost) {
                    a.vel(i, j, k) = 0.0;
                    a.mom(i, j, k) = 0.0;
                } else if (p[d] == f) {
                    a.vel(i, j, k) = 0.;
                    a.mom(i, j, k) = 0.;
                }
            }
        } else if (a.fn == BC_MOMT) {
            if (bv == 1 || bv == 2) {
                const double fac = bm >= 3 ? 0.0 : (bv == 1 ? 1.0 : 0.0);
                a.vel(i, j, k) = fac * a.vel(m[0], m[1], m[2]);
                a.mom(i, j, k) = fac * a.mom(m[0], m[1], m[2]);
            }
        } else {
            const Arr4<double>& pr = a.prim;
            if (bm >= 3) {
                const double temp = pr(i, j, k, 4), rho = pr(i, j, k, 0);
                double cvmix = 0., e0mix = 0.;
                for (int c = 0; c < NS; ++c) {
                    cvmix += pr(i, j, k, 6 + c) * P.hcv[c];
                    e0mix += pr(i, j, k, 6 + c) * P.e0[c];
                }
                const double intenergy = e0mix + temp * cvmix;
                for (int c = 0; c < NS; ++c) a.cons(i, j, k, 5 + c) = rho * pr(i, j, k, 6 + c);
                const double kinenergy = 0.;
                a.cons(i, j, k, 4) = rho * intenergy + kinenergy;
            } else if (bv == 1 || bv == 2) {
                const double temp = pr(i, j, k, 4), pt = pr(i, j, k, 5);
                double molmix = 0.;
                for (int c = 0; c < NS; ++c) molmix += pr(i, j, k, 6 + c) / P.molmass[c];
                molmix = 1. / molmix;
                const double rho = pt / (P.Runiv / molmix) / temp;
                double cvmix = 0., e0mix = 0.;
                for (int c = 0; c < NS; ++c) {
                    cvmix += pr(i, j, k, 6 + c) * P.hcv[c];
                    e0mix += pr(i, j, k, 6 + c) * P.e0[c];
                }
                const double intenergy = e0mix + temp * cvmix;
                pr(i, j, k, 0) = rho;
                a.cons(i, j, k, 0) = rho;
                for (int c = 0; c < NS; ++c) a.cons(i, j, k, 5 + c) = rho * pr(i, j, k, 6 + c);
                double kin = 0.;
                kin += (a.mx(i + 1, j, k) + a.mx(i, j, k)) * (a.mx(i + 1, j, k) + a.mx(i, j, k));
                kin += (a.my(i, j + 1, k) + a.my(i, j, k)) * (a.my(i, j + 1, k) + a.my(i, j, k));
                kin += (a.mz(i, j, k + 1) + a.mz(i, j, k)) * (a.mz(i, j, k + 1) + a.mz(i, j, k));
                kin *= (0.125 / rho);
                a.cons(i, j, k, 4) = rho * intenergy + kin;
            }
        }
    }
}

}  // namespace fhd
