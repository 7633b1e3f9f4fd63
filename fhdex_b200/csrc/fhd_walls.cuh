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
#include "philox.cuh"

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
// With reservoirs (bc_mass 3 / 4: ghost cells held at the reservoir's state, flow
// through the interface) the reference's passes read values that earlier passes of the same
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
                    if (bm == 3) {
                        a.vel(i, j, k) = -2 * a.mom(fi[0], fi[1], fi[2]) /
                                         (a.cons(fi[0], fi[1], fi[2], 0) + a.cons(gi[0], gi[1], gi[2], 0));
                        a.mom(i, j, k) = -1 * a.mom(fi[0], fi[1], fi[2]);
                    } else if (bm == 4) {
                        a.vel(i, j, k) = -1 * a.vel(fi[0], fi[1], fi[2]);
                        a.mom(i, j, k) = -1 * a.mom(fi[0], fi[1], fi[2]);
                    }
                } else if (p[d] == f && bm == 3) {
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

// ---- the particle reservoir (bc_mass 4): ComputeFluxMomReservoir ---------------------
// (reservoirStag.cpp:11-869, reservoirStag_K.H).  Per face of a reservoir interface two
// Poisson processes of particles crossing in a stage's dt: from the reservoir (the ghost
// cell's temperature and rho Y, at rest) and to it (the inside cell's temperature, rho Y
// and velocity), each particle with a random normal velocity (rejection sampling of the
// flux-weighted Maxwellian) and two tangential ones; their mass, species mass, energy and
// momenta become the face's flux (faceflux_res) and normal momentum (cumom_res).  The
// random numbers come from Philox per (face, stage, side, draw); a test can record every
// draw to replay them into the reference.
struct ResArgs {
    DevParams P;
    Arr4<const double> cons0, prim0, vel[3];
    double* fres[3];          // faceflux_res[d]: the reference's layout (no ghosts, nvars comps)
    double* mres[3];          // cumom_res[d]
    int fsy[3], fsz[3], fsn[3];
    double mass[MAXS];
    double dt;                // the stage's dt (dt, dt / 4, 2 dt / 3)
    int stage;
    int sides[6], nsides;
    int64_t face_pref[7];     // faces of the listed sides, prefix sums
    double* rec;              // test hook: draws of (stage, listed side, face), rec_cap each, or nullptr
    int rec_cap;
    int* status;
};

struct ResRng {
    uint32_t k0, k1, c0, c1, c3;
    uint32_t n;
    double* rec;
    int cap;
    FHD_D uint64_t bits() {
        uint32_t w[4] = {c0, c1, n, c3};
        philox4x32_10(w, k0, k1);
        return ((uint64_t)w[0] << 32) | w[1];
    }
    FHD_D void keep(double v) {
        if (rec && (int)n < cap) rec[n] = v;
        ++n;
    }
    // uniform in (0, 1]: the top 53 bits + 1, over 2^53
    FHD_D double U() {
        const double v = (double)((bits() >> 11) + 1) * (1.0 / 9007199254740992.0);
        keep(v);
        return v;
    }
    // standard normal (Box-Muller on two such uniforms of one Philox call)
    FHD_D double Z() {
        uint32_t w[4] = {c0, c1, n, c3};
        philox4x32_10(w, k0, k1);
        const double u1 = (double)(((((uint64_t)w[0] << 32) | w[1]) >> 11) + 1) * (1.0 / 9007199254740992.0);
        const double u2 = (double)(((((uint64_t)w[2] << 32) | w[3]) >> 11) + 1) * (1.0 / 9007199254740992.0);
        const double v = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
        keep(v);
        return v;
    }
};

constexpr int kResMaxTries = 1 << 16;      // rejection-sampling attempts per velocity
constexpr int kResMaxParticles = 1 << 22;  // particles per process

// random_cross_vel (reservoirStag_K.H:10-57); ok = 0 when the attempts run out
FHD_D double res_cross_vel(double a, double vT, bool tangential, double Vt, ResRng& g, int& ok) {
    const double sqrtPI = 1.77245385091;
    const double small_number = 1.0e-13;
    double v = 0.0;
    if (!tangential) {
        double z = 0.0;
        if (a > small_number) {
            bool stop = false;
            for (int t = 0; !stop; ++t) {
                if (t >= kResMaxTries) { ok = 0; break; }
                const double u = g.U();
                if ((a * sqrtPI) / (a * sqrtPI + 1.0 + a * a) > u) {
                    z = -1.0 * fabs(0.0 + sqrt(0.5) * g.Z());
                    stop = true;
                } else if ((a * sqrtPI + 1.0) / (a * sqrtPI + 1.0 + a * a) > u) {
                    z = -1.0 * sqrt(-1.0 * log(g.U()));
                    stop = true;
                } else {
                    z = a * (1.0 - sqrt(g.U()));
                    if (exp(1.0 * z * z) > g.U()) stop = true;
                }
            }
            v = (a - z) * vT;
        } else if (a < -1.0 * small_number) {
            bool stop = false;
            for (int t = 0; !stop; ++t) {
                if (t >= kResMaxTries) { ok = 0; break; }
                z = -1.0 * sqrt(a * a - log(g.U()));
                if (a > z * (1.0 - g.U())) stop = true;
            }
            v = (a - z) * vT;
        } else {
            v = vT * sqrt(-1.0 * log(g.U()));
        }
    } else {
        v = Vt + vT * (0.0 + sqrt(0.5) * g.Z());
    }
    return v;
}

// poisson_process_reservoir (reservoirStag_K.H:59-166), three dimensions
template <int NS>
FHD_D int res_poisson(const ResArgs& a, const double (&rhoYk)[NS], double T, double Vn, double area, double VT1,
                      double VT2, ResRng& g, double& mass_cross, double (&mom_cross)[3], double& en_cross,
                      double (&spec)[NS]) {
    const double sqrtPI = 1.77245385091;
    const double small_number = 1.0e-13;
    const double kB = a.P.k_B;
    mass_cross = 0.0;
    en_cross = 0.0;
    for (int c = 0; c < 3; ++c) mom_cross[c] = 0.0;
    for (int n = 0; n < NS; ++n) spec[n] = 0.0;
    double rate[NS], timer[NS], vth[NS], ratio[NS];
    bool stopf[NS];
    for (int n = 0; n < NS; ++n) {
        vth[n] = sqrt(2.0 * kB * T / a.mass[n]);
        ratio[n] = Vn / vth[n];
        const double num_density = rhoYk[n] / a.mass[n];
        if (fabs(ratio[n]) > small_number)
            rate[n] = (1.0 / (2.0 * sqrtPI)) * num_density * area * vth[n] *
                      (exp(-1.0 * ratio[n] * ratio[n]) + ratio[n] * sqrtPI * (1.0 + erf(ratio[n])));
        else
            rate[n] = (1.0 / (2.0 * sqrtPI)) * num_density * area * vth[n];
        timer[n] = 0.0;
        stopf[n] = false;
    }
    int ok = 1;
    bool stop = false;
    for (int it = 0; !stop; ++it) {
        if (it >= kResMaxParticles) return 0;
        for (int n = 0; n < NS; ++n) {
            if (stopf[n]) continue;
            mass_cross += a.mass[n];
            spec[n] += a.mass[n];
            double v = res_cross_vel(ratio[n], vth[n], false, 0.0, g, ok);
            mom_cross[0] += a.mass[n] * v;
            en_cross += 0.5 * a.mass[n] * (v) * (v);
            v = res_cross_vel(ratio[n], vth[n], true, VT1, g, ok);
            mom_cross[1] += a.mass[n] * v;
            en_cross += 0.5 * a.mass[n] * (v) * (v);
            v = res_cross_vel(ratio[n], vth[n], true, VT2, g, ok);
            mom_cross[2] += a.mass[n] * v;
            en_cross += 0.5 * a.mass[n] * (v) * (v);
        }
        stop = true;
        for (int n = 0; n < NS; ++n) {
            if (!stopf[n]) {
                const double rn = g.U();
                timer[n] = timer[n] - log(rn) / (rate[n]);
                if (timer[n] >= a.dt) stopf[n] = true;
            }
            stop = stop && stopf[n];
        }
        if (!ok) return 0;
    }
    return ok;
}

// one thread per face of a reservoir interface: both processes, into faceflux_res / cumom_res
template <int NS>
static __global__ void __launch_bounds__(128) k_reservoir(ResArgs a) {
    const DevParams& P = a.P;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < a.face_pref[a.nsides];
         q += (int64_t)gridDim.x * blockDim.x) {
        int li = 0;
        while (q >= a.face_pref[li + 1]) ++li;
        const int s = a.sides[li], d = s >> 1, hi = s & 1;
        const int64_t f = q - a.face_pref[li];
        const int e1 = d == 0 ? 1 : 0, e2 = d == 2 ? 1 : 2;  // the tangential directions, in order
        int x[3];
        x[d] = hi ? P.n[d] : 0;
        x[e1] = (int)(f % P.n[e1]);
        x[e2] = (int)(f / P.n[e1]);
        int in[3] = {x[0], x[1], x[2]}, gh[3] = {x[0], x[1], x[2]};
        in[d] = hi ? P.n[d] - 1 : 0;       // the cell inside the interface
        gh[d] = hi ? P.n[d] : -1;          // the reservoir's ghost cell
        const double area = P.dx[e1] * P.dx[e2];
        const double vol = P.dx[0] * P.dx[1] * P.dx[2];
        ResRng g;
        g.k0 = P.key0;
        g.k1 = P.key1;
        g.c0 = (uint32_t)f;
        g.c1 = 0x40000000u | ((uint32_t)a.stage << 8) | (uint32_t)s;
        g.c3 = (uint32_t)noise_step(P);
        g.n = 0;
        g.rec = a.rec ? a.rec + ((int64_t)a.stage * a.face_pref[a.nsides] + q) * a.rec_cap : nullptr;
        g.cap = a.rec_cap;
        double* fl = a.fres[d];
        const int64_t fidx = x[0] + (int64_t)x[1] * a.fsy[d] + (int64_t)x[2] * a.fsz[d];
        const int64_t fsn = a.fsn[d];
        double& mom = a.mres[d][fidx];
        // particles in the inside cell (for the correction of the incoming fluxes)
        double N = 0.0;
        for (int n = 0; n < NS; ++n) N += vol * (a.cons0(in[0], in[1], in[2], 5 + n) / a.mass[n]);
        double rhoYk[NS], spec[NS], mc[3], mass_cross, en_cross;
        // from the reservoir (at rest, at the ghost cell's state)
        for (int n = 0; n < NS; ++n) rhoYk[n] = a.cons0(gh[0], gh[1], gh[2], 5 + n);
        int ok = res_poisson<NS>(a, rhoYk, a.prim0(gh[0], gh[1], gh[2], 4), 0.0, area, 0.0, 0.0, g, mass_cross, mc,
                                 en_cross, spec);
        if (!hi) {
            fl[fidx] += (1.0 - (1.0 / (12.0 * N))) * mass_cross / (a.dt * area);
            fl[fidx + 4 * fsn] += (1.0 + (1.0 / (4.0 * N))) * en_cross / (a.dt * area);
            for (int n = 0; n < NS; ++n) fl[fidx + (5 + n) * fsn] += (1.0 - (1.0 / (12.0 * N))) * spec[n] / (a.dt * area);
            mom += mc[0] / vol;
            fl[fidx + fsn] += mc[1] / a.dt / area;
            fl[fidx + 2 * fsn] += mc[2] / a.dt / area;
        } else {
            fl[fidx] -= (1.0 - (1.0 / (12.0 * N))) * mass_cross / (a.dt * area);
            fl[fidx + 4 * fsn] -= (1.0 + (1.0 / (4.0 * N))) * en_cross / (a.dt * area);
            for (int n = 0; n < NS; ++n) fl[fidx + (5 + n) * fsn] -= (1.0 - (1.0 / (12.0 * N))) * spec[n] / (a.dt * area);
            mom -= mc[0] / vol;
            fl[fidx + fsn] -= mc[1] / a.dt / area;
            fl[fidx + 2 * fsn] -= mc[2] / a.dt / area;
        }
        // to the reservoir (the inside cell's state and velocity)
        const Arr4<const double>& vx = a.vel[0];
        const Arr4<const double>& vy = a.vel[1];
        const Arr4<const double>& vz = a.vel[2];
        const int i = in[0], j = in[1], k = in[2];
        double V[3];
        V[0] = 0.5 * (vx(i, j, k) + vx(i + 1, j, k));
        V[1] = 0.5 * (vy(i, j, k) + vy(i, j + 1, k));
        V[2] = 0.5 * (vz(i, j, k) + vz(i, j, k + 1));
        if (!hi) V[d] = -0.5 * (a.vel[d](i, j, k) + a.vel[d](i + (d == 0), j + (d == 1), k + (d == 2)));
        for (int n = 0; n < NS; ++n) rhoYk[n] = a.cons0(i, j, k, 5 + n);
        ok &= res_poisson<NS>(a, rhoYk, a.prim0(i, j, k, 4), V[d], area, V[e1], V[e2], g, mass_cross, mc, en_cross,
                              spec);
        if (!hi) {
            fl[fidx] -= mass_cross / (a.dt * area);
            fl[fidx + 4 * fsn] -= en_cross / (a.dt * area);
            for (int n = 0; n < NS; ++n) fl[fidx + (5 + n) * fsn] -= spec[n] / (a.dt * area);
            mom -= mc[0] / vol;
            fl[fidx + fsn] -= mc[1] / a.dt / area;
            fl[fidx + 2 * fsn] -= mc[2] / a.dt / area;
        } else {
            fl[fidx] += mass_cross / (a.dt * area);
            fl[fidx + 4 * fsn] += en_cross / (a.dt * area);
            for (int n = 0; n < NS; ++n) fl[fidx + (5 + n) * fsn] += spec[n] / (a.dt * area);
            mom += mc[0] / vol;
            fl[fidx + fsn] += mc[1] / a.dt / area;
            fl[fidx + 2 * fsn] += mc[2] / a.dt / area;
        }
        if (!ok && a.status) atomicCAS(a.status, 0, 5);  // FHD_ERR_TIMEOUT: a sampling loop ran out of attempts
    }
}

// ResetReservoirFluxes (reservoirStag.cpp:871-1394) on the stage's flux scratch (or on
// the caller's flux MultiFabs): the interface faces take the reservoir's mass, energy and
// species fluxes, the interface edges the average of two tangential reservoir fluxes.
// The reference reads those pairs from faceflux_res, which has no ghost cells, at index
// -1 and n of the edge's other direction as well; Array4 then addresses the neighbouring
// row, plane or component of the same allocation, and so does the flat index here.
struct ResResetArgs {
    DevParams P;
    const double* fres[3];
    int fsy[3], fsz[3], fsn[3];
    Arr4<double> ff[3];       // face fluxes: comps cons 0, 4, 5.. at fcomp[0], [1], [2]..
    int fc_rho, fc_rhoE, fc_Y;
    Arr4<double> ef[6];       // edge fluxes: edgex_v, edgex_w, edgey_u, edgey_w, edgez_u, edgez_v
    int side;
};

template <int NS>
static __global__ void __launch_bounds__(128) k_res_reset(ResResetArgs a) {
    const DevParams& P = a.P;
    const int s = a.side, d = s >> 1, hi = s & 1;
    const int e1 = d == 0 ? 1 : 0, e2 = d == 2 ? 1 : 2;
    const int plane = hi ? P.n[d] : 0;
    // items: the interface faces, then the (e1-nodal) edges, then the (e2-nodal) edges
    const int64_t nf = (int64_t)P.n[e1] * P.n[e2];
    const int64_t ne1 = (int64_t)(P.n[e1] + 1) * P.n[e2], ne2 = (int64_t)P.n[e1] * (P.n[e2] + 1);
    const double* fr = a.fres[d];
    const int64_t sy = a.fsy[d], sz = a.fsz[d], sn = a.fsn[d];
    auto flat = [&](int i, int j, int k, int c) { return (int64_t)i + j * sy + k * sz + c * sn; };
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nf + ne1 + ne2;
         q += (int64_t)gridDim.x * blockDim.x) {
        int x[3];
        x[d] = plane;
        if (q < nf) {
            x[e1] = (int)(q % P.n[e1]);
            x[e2] = (int)(q / P.n[e1]);
            const Arr4<double>& f = a.ff[d];
            if (!f.p) continue;
            f(x[0], x[1], x[2], a.fc_rho) = fr[flat(x[0], x[1], x[2], 0)];
            f(x[0], x[1], x[2], a.fc_rhoE) = fr[flat(x[0], x[1], x[2], 4)];
            for (int n = 0; n < NS; ++n) f(x[0], x[1], x[2], a.fc_Y + n) = fr[flat(x[0], x[1], x[2], 5 + n)];
            continue;
        }
        // an edge nodal in d and in e (e1: the first tangential direction, comp 1 of
        // faceflux_res; e2: the second, comp 2), averaged over the two faces beside it in e
        const bool first = q < nf + ne1;
        const int64_t r = first ? q - nf : q - nf - ne1;
        const int e = first ? e1 : e2, o = first ? e2 : e1;
        const int ce = first ? 1 : 2;
        x[e] = (int)(r % (P.n[e] + 1));
        x[o] = (int)(r / (P.n[e] + 1));
        int y[3] = {x[0], x[1], x[2]};
        y[e] -= 1;
        const double v = 0.5 * (fr[flat(x[0], x[1], x[2], ce)] + fr[flat(y[0], y[1], y[2], ce)]);
        // which edge flux: the momentum component e carried in direction d
        int slot;
        if (d == 0) slot = e == 1 ? 0 : 1;        // edgex_v (xy), edgex_w (xz)
        else if (d == 1) slot = e == 0 ? 2 : 3;   // edgey_u (xy), edgey_w (yz)
        else slot = e == 0 ? 4 : 5;               // edgez_u (xz), edgez_v (yz)
        const Arr4<double>& ef = a.ef[slot];
        if (ef.p) ef(x[0], x[1], x[2]) = v;
    }
}

// ResetReservoirMom (reservoirStag.cpp:1396-1625): the interface faces' normal momentum
struct ResMomArgs {
    DevParams P;
    const double* mres[3];
    int fsy[3], fsz[3];
    Arr4<double> mom[3];
    int side;
};

static __global__ void __launch_bounds__(128) k_res_mom(ResMomArgs a) {
    const DevParams& P = a.P;
    const int s = a.side, d = s >> 1, hi = s & 1;
    const int e1 = d == 0 ? 1 : 0, e2 = d == 2 ? 1 : 2;
    const int64_t nf = (int64_t)P.n[e1] * P.n[e2];
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nf; q += (int64_t)gridDim.x * blockDim.x) {
        int x[3];
        x[d] = hi ? P.n[d] : 0;
        x[e1] = (int)(q % P.n[e1]);
        x[e2] = (int)(q / P.n[e1]);
        a.mom[d](x[0], x[1], x[2]) = a.mres[d][x[0] + (int64_t)x[1] * a.fsy[d] + (int64_t)x[2] * a.fsz[d]];
    }
}

}  // namespace fhd
