// fhd_device.cuh — device data views and point physics of the staggered FHD step.
//
// Point physics restated from FHDeX src_compressible/compressible_functions.H for
// sm_100a: compile-time species count NS (fully unrolled, register resident), a
// compute type R (double for the reference-order FP64 path, float for the mixed
// path).  With R = double and -fmad=false every expression below evaluates in the
// reference's operation order, so results are bitwise those of the CPU path.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "fhd_div.h"

#define FHD_HD __host__ __device__ __forceinline__
#define FHD_D __device__ __forceinline__

namespace fhd {

constexpr int MAXS = 8;

// AMReX Array4 view: (i,j,k,n) at p[(i-lo0) + (j-lo1)*sy + (k-lo2)*sz + n*sn].
// 32-bit offsets: the host rejects fabs with 2^31 or more elements.
template <class T>
struct Arr4 {
    T* p;
    int lo0, lo1, lo2;
    int sy, sz, sn;
    FHD_HD T& operator()(int i, int j, int k, int n = 0) const {
        return p[(i - lo0) + (j - lo1) * sy + (k - lo2) * sz + n * sn];
    }
};

// Parameters as the kernels see them (by value in the kernel parameter bank).
// Cell-independent sub-expressions of the transport model are precomputed on the
// host in the reference's own operation order (host IEEE double arithmetic gives
// the identical values the reference computes inside its loops).
struct DevParams {
    int ns, nvars, nprim;
    int n[3];
    double dx[3];
    double dt;
    double volinv, dtinv;            // 1./(dx0*dx1*dx2), 1./dt   (fluxStag.cpp:97-98)
    double k_B, Runiv;
    double grav[3];
    double zeta_ratio;
    int visc_type, advection_type, stoch;
    // physical boundaries; side s = 2 d + (0 lo, 1 hi); -1 on periodic sides
    int walls;                       // any wall
    int periodic[3];
    int bc_vel[6], bc_mass[6], bc_therm[6];
    double hdx[3], rhdx[3];          // 0.5*dx and RN(1/(0.5*dx)) (the wall faces' half-cell divisor)
    double molmass[MAXS], hcv[MAXS], hcp[MAXS], e0[MAXS];
    // Giovangigli model constants (compressible_functions.H:1180-1222)
    double mm[MAXS];                 // molmass*(k_B/Runiv)
    double mmkB[MAXS];               // mm*k_B (first product of the eta1 sqrt argument)
    double eta1pre[MAXS];            // 5.0/(16.0*diam(i,i)*diam(i,i))
    double diam[MAXS][MAXS];         // 0.5*(d_i+d_j)
    double mu[MAXS][MAXS];           // m_i*m_j/(m_i+m_j)
    double msum[MAXS][MAXS];         // m_i+m_j
    double vfac[MAXS][MAXS];         // 1.0+0.6*m_k/m_i*AKL
    double kfac[MAXS][MAXS];         // 7.5 m_i/m_k + 6.25 m_k/m_i - 3.0 m_k/m_i BKL + 4.0 AKL
    double koff;                     // 55.0/4.0-3.0*BKL-4.0*AKL
    double voff;                     // 0.6*AKL-1.0
    double cfac;                     // 6.0*CKL-5.0
    double sqrt2, sqrt3;
    // quasi-1-D / 2-D runs (do_1D / do_2D): dim 1 or 2, else 3; fac2d = (3+sqrt(3))/2,
    // the 2-D trace factor (fluxStag.cpp:185); csd0 the deviation of the x centre
    // noise (1 in 1-D, sqrt(2) otherwise: timeStepStag.cpp:208-222)
    int dim;
    double fac2d, csd0;
    // transport model (transCoeffs.cpp:58-73): 1 Giovangigli, 2 Valk/Waldmann (pair
    // constants in the device table vwt), 3 HCB binary
    int transport_type;
    const struct VWTable* vwt;
    // noise
    uint32_t key0, key1;             // Philox key
    uint64_t step;                   // Philox counter words 2-3
    const uint64_t* step_ptr;        // when set, the step is read here (batched graph replay)
    // correctly rounded reciprocals (host 1.0 / x) of the constant divisors, for
    // div_rcp; the dividend window is empty (div_span 0: plain divisions) when a
    // divisor lies outside div_rcp's divisor window
    double rdx[3];
    double rmolmass[MAXS], rmm[MAXS];
    double rmu[MAXS][MAXS], rmsum[MAXS][MAXS];
    double rRdt;                     // 1/(Runiv*dt)
    double rpi, r3;                  // 1/pi (the transport model's pi), 1/3
    uint32_t div_lo, div_span;
};

// a / b in the compute type: FP64 the correctly rounded division (the reference's
// arithmetic); FP32 (the mixed path, held to a tolerance against FP64) the fast
// division __fdividef (about 2 ulp; physical divisors stay far below 2^126).
FHD_D double rdiv(double a, double b) { return a / b; }
FHD_D float rdiv(float a, float b) { return __fdividef(a, b); }

// a / b for a constant divisor b with y = RN(1/b) from DevParams: bitwise a / b
// (fhd_div.h).  In single precision (the mixed path, held to a tolerance against
// FP64, not to bitwise parity) the product a * y: within about one FP32 ulp of a / b.
FHD_D double divc(const DevParams& P, double a, double b, double y) { return div_rcp(a, b, y, P.div_lo, P.div_span); }
FHD_D float divc(const DevParams&, float a, float, float y) { return a * y; }
// divc for call sites whose dividend is often exactly zero (zero handled inline)
FHD_D double divc0(const DevParams& P, double a, double b, double y) {
    return div_rcp_z(a, b, y, P.div_lo, P.div_span);
}
FHD_D float divc0(const DevParams&, float a, float, float y) { return a * y; }
// a / b for a cell value b used as a divisor several times, y = 1.0 / b
FHD_D double divv(const DevParams& P, double a, double b, double y) {
    return div_rcp_any(a, b, y, P.div_lo, P.div_span);
}
FHD_D float divv(const DevParams&, float a, float, float y) { return a * y; }
// a / Dbin with the reciprocal path for up to two species (see transport_gio)
template <int NS, class R>
FHD_D R div_dbin(const DevParams& P, R a, R b, R y) {
    if constexpr (NS <= 2) return divv(P, a, b, y);
    else return rdiv(a, b);
}
// a / b for a cell value b where the dividend is often exactly zero (the Soret
// terms of identical species, whose thermal diffusion ratios vanish)
FHD_D double divz(double a, double b) { return div_zero_short(a, b); }
FHD_D float divz(float a, float b) { return rdiv(a, b); }

FHD_D uint64_t noise_step(const DevParams& P) { return P.step_ptr ? *P.step_ptr : P.step; }

// ---- persistent batched step: work units and run descriptor (k_batch_persist) -----------
enum { PK_PREP = 0, PK_TAUS = 1, PK_FACEX = 2, PK_FACEY = 3, PK_FACEZ = 4, PK_UPDATE = 5, PK_CONVERT = 6,
       PK_GHOST = 7, PK_STEP = 8 };

struct PUnit {
    const void* args;   // the unit's argument block (PrepArgs, StageArgs, ConvArgs or GhostFab)
    int64_t first;      // global index of the unit's first chunk
    int64_t items;      // work items (points; points x components for a ghost fab)
    int member, phase, kind, pad;
};

struct PersistArgs {
    const PUnit* units;
    int nunits, nphase;
    int64_t total;              // chunks of the step
    int chunk;                  // items per chunk
    unsigned int* next;         // chunk dispenser
    unsigned int* done;         // [member][phase] finished chunks
    const unsigned int* need;   // [member][phase] chunks
    int* status;                // per member
    int* abort;
    uint64_t* steps;            // per-member step counters
    unsigned long long limit_ns;
    int hold_phase;             // failure-injection hook: this phase's completions are never published (-1: none)
};

// ---- physical boundaries ---------------------------------------------------------------
// wall values per side s = 2 d + (0 lo, 1 hi) (after SetupCWallStag): wall or
// reservoir temperature, reservoir pressure and density, wall / reservoir Y and X
struct WallParams {
    double t[6], p[6], rho[6];
    double Yk[6][MAXS], Xk[6][MAXS];
};

// the reference's is_<lo|hi>_<d>_dirichlet_mass (fluxStag.cpp:84-89): a side whose
// bc_mass is neither -1 (periodic) nor 3
FHD_HD bool dirichlet_side(const DevParams& P, int side) {
    const int b = P.bc_mass[side];
    return b != -1 && b != 3;
}
// the wall side (0 lo, 1 hi) of the face plane idx of direction d, or -1: the
// reference's (i == 0 and is_lo_x_dirichlet_mass) / (i == n_cells[0] and
// is_hi_x_dirichlet_mass) tests
FHD_HD int wall_face(const DevParams& P, int d, int idx) {
    if (idx == 0 && dirichlet_side(P, 2 * d)) return 0;
    if (idx == P.n[d] && dirichlet_side(P, 2 * d + 1)) return 1;
    return -1;
}
// StochFluxStag's factors (boundaryStag.cpp:2086-3009) on a wall side: 0 for an
// impermeable / adiabatic / slip wall (type 1), sqrt(2) for a concentration /
// isothermal / no-slip wall (type 2), 1 otherwise
FHD_HD double stoch_factor(const DevParams& P, int type) {
    return type == 1 ? 0. : (type == 2 ? P.sqrt2 : 1.0);
}

// ---- EOS helpers (compressible_functions.H:138-219, 1497-1520) ----------------------
// Products summed in double go through mul_rn / add_rn, which are never fused into
// an FMA: the conversion then gives the same bits in the FP64 units (built without
// contraction) and in the mixed units (built with it), where the persistent batched
// step converts the state.  FP32 code keeps the compiler's contraction.
FHD_D double mul_rn(double a, double b) { return __dmul_rn(a, b); }
FHD_D double add_rn(double a, double b) { return __dadd_rn(a, b); }
FHD_D float mul_rn(float a, float b) { return a * b; }
FHD_D float add_rn(float a, float b) { return a + b; }

template <int NS, class R>
FHD_D void GetMolfrac(const DevParams& P, const R (&Y)[NS], R (&X)[NS]) {
    R molmix = R(0.);
#pragma unroll
    for (int n = 0; n < NS; ++n) molmix += divc(P, Y[n], R(P.molmass[n]), R(P.rmolmass[n]));
    molmix = rdiv(R(1.), molmix);
#pragma unroll
    for (int n = 0; n < NS; ++n) X[n] = divc(P, Y[n] * molmix, R(P.molmass[n]), R(P.rmolmass[n]));
}

template <int NS, class R>
FHD_D R GetTemperature(const DevParams& P, R energy, const R (&Y)[NS]) {
    R cvmix = R(0.), e0mix = R(0.);
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        cvmix = add_rn(cvmix, mul_rn(Y[n], R(P.hcv[n])));
        e0mix = add_rn(e0mix, mul_rn(Y[n], R(P.e0[n])));
    }
    return rdiv(energy - e0mix, cvmix);
}

template <int NS, class R>
FHD_D R GetPressureGas(const DevParams& P, const R (&Y)[NS], R density, R temp) {
    R molmix = R(0.);
#pragma unroll
    for (int n = 0; n < NS; ++n) molmix += divc(P, Y[n], R(P.molmass[n]), R(P.rmolmass[n]));
    molmix = rdiv(R(1.), molmix);
    return density * rdiv(R(P.Runiv), molmix) * temp;
}

template <int NS, class R>
FHD_D void GetEnthalpies(const DevParams& P, R T, R (&hk)[NS]) {
#pragma unroll
    for (int i = 0; i < NS; ++i) hk[i] = R(P.e0[i]) + R(P.hcp[i]) * T;
}

template <class R>
FHD_D R clamp01(R y) { return fmax(R(0.), fmin(R(1.), y)); }
template <>
FHD_D float clamp01<float>(float y) { return fmaxf(0.f, fminf(1.f, y)); }

template <class R> FHD_D R dsqrt(R x);
template <> FHD_D double dsqrt<double>(double x) { return sqrt(x); }
template <> FHD_D float dsqrt<float>(float x) { return sqrtf(x); }

// CholeskyDecomp (compressible_functions.H:460-511): lower factor of a symmetric
// NS x NS matrix with the reference's "sum <= 0 -> zero pivot, zero column" guard.
// Only the lower triangle reaches the result.
template <int NS, class R>
FHD_D void CholeskyDecomp(R (&a)[NS * NS], R (&sqda)[NS * NS]) {
    R p[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        int ising = 0;
#pragma unroll
        for (int j = i; j < NS; ++j) {
            R sum1 = a[i * NS + j];
#pragma unroll
            for (int k = i - 1; k >= 0; --k) sum1 = sum1 - a[i * NS + k] * a[j * NS + k];
            if (i == j) {
                if (sum1 <= R(0.)) { p[i] = R(0.); ising = 1; }
                else p[i] = dsqrt(sum1);
            }
            if (ising == 0) a[j * NS + i] = rdiv(sum1, p[i]);
            else a[j * NS + i] = R(0.);
        }
    }
#pragma unroll
    for (int i = 0; i < NS; ++i)
#pragma unroll
        for (int j = 0; j < NS; ++j) sqda[i * NS + j] = (j < i) ? a[i * NS + j] : (j == i ? p[i] : R(0.));
}

// D_GIO1 (compressible_functions.H:647-778).  Dout[j*NS+i] = Diff_ij(i,j)*Ykp[i].
// rDbin: 1.0 / Dbin off the diagonal (only off-diagonal entries divide here)
template <int NS, class R>
FHD_D void D_GIO1(const DevParams& P, const R (&Dbin)[NS][NS], const R (&rDbin)[NS][NS], const R (&Ykp)[NS],
                  const R (&Xkp)[NS], R (&Dout)[NS * NS]) {
    R Diff[NS * NS], PJ[NS * NS], M2[NS * NS], Pmat[NS * NS], Jmat[NS * NS];
    R Di[NS], Minv[NS], Mmat[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        R term2 = R(0.);
#pragma unroll
        for (int j = 0; j < NS; ++j)
            if (j != i) term2 = term2 + div_dbin<NS, R>(P, Xkp[j], Dbin[i][j], rDbin[i][j]);
        Di[i] = rdiv(R(1.) - Ykp[i], term2);
    }
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        Mmat[i] = rdiv(Xkp[i], Di[i]);
        Minv[i] = rdiv(Di[i], Xkp[i]);
    }
#pragma unroll
    for (int i = 0; i < NS; ++i)
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            R v = -Ykp[j];
            if (i == j) v = v + R(1.);
            Pmat[i * NS + j] = v;
        }
    // Zmat = -Deltamat (+ Mmat on the diagonal); Jmat = Minv*Zmat
#pragma unroll
    for (int i = 0; i < NS; ++i)
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            R Deltamat;
            if (i == j) {
                R term1 = R(0.);
#pragma unroll
                for (int k = 0; k < NS; ++k)
                    if (k != i) term1 = term1 + div_dbin<NS, R>(P, Xkp[i] * Xkp[k], Dbin[i][k], rDbin[i][k]);
                Deltamat = term1;
            } else {
                Deltamat = div_dbin<NS, R>(P, -Xkp[i] * Xkp[j], Dbin[i][j], rDbin[i][j]);
            }
            R z = -Deltamat;
            if (i == j) z = z + Mmat[i];
            Jmat[i * NS + j] = Minv[i] * z;
        }
#pragma unroll
    for (int i = 0; i < NS; ++i)
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            R s = R(0.);
#pragma unroll
            for (int k = 0; k < NS; ++k) s = s + Pmat[i * NS + k] * Jmat[k * NS + j];
            PJ[i * NS + j] = s;
        }
#pragma unroll
    for (int i = 0; i < NS; ++i)
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            R scr = R(0.);
#pragma unroll
            for (int k = 0; k < NS; ++k) scr = scr + Pmat[i * NS + k] * Minv[k] * Pmat[j * NS + k];
            M2[i * NS + j] = scr;
            Diff[i * NS + j] = scr;
        }
#pragma unroll
    for (int ll = 0; ll < 3; ++ll) {
        R M1[NS * NS];
#pragma unroll
        for (int i = 0; i < NS; ++i)
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                R scr = R(0.);
#pragma unroll
                for (int k = 0; k < NS; ++k) scr = scr + PJ[i * NS + k] * Diff[k * NS + j];
                M1[i * NS + j] = scr + M2[i * NS + j];
            }
#pragma unroll
        for (int q = 0; q < NS * NS; ++q) Diff[q] = M1[q];
    }
#pragma unroll
    for (int i = 0; i < NS; ++i)
#pragma unroll
        for (int j = 0; j < NS; ++j) Dout[j * NS + i] = Diff[i * NS + j] * Ykp[i];
}

// Per-cell transport coefficients: calculateTransportCoeffs body (transCoeffs.cpp:37-89)
// with IdealMixtureTransportGIO (compressible_functions.H:1153-1352).
// Yraw: prim(6+n) (unclamped).  Returns false when a mass fraction is outside (0,1)
// (the reference aborts there).
template <int NS, class R>
struct Coeffs {
    R eta, kappa, zeta;
    R chi[NS];
    R D[NS * NS];
};

template <int NS, class R>
FHD_D bool transport_gio(const DevParams& P, R rho, R temperature, R pressure, const R (&Yraw)[NS],
                         Coeffs<NS, R>& c) {
    bool ok = true;
    R Yk[NS];
    R sumYk = R(0.);
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        // a single gas has Y = 1 by construction: the range check (transCoeffs.cpp:45-46)
        // applies to mixtures only
        if (NS > 1 && (Yraw[n] <= R(0.) || Yraw[n] >= R(1.))) ok = false;
        Yk[n] = clamp01(Yraw[n]);
        sumYk += Yk[n];
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) Yk[n] = rdiv(Yk[n], sumYk);

    const R pi = R(3.1415926535897932);
    R mbar = R(0.0);
#pragma unroll
    for (int n = 0; n < NS; ++n) mbar += divc(P, Yk[n], R(P.mm[n]), R(P.rmm[n]));
    mbar = rdiv(R(1.0), mbar);
    R Xk[NS], Xkp[NS], Ykp[NS];
    R Xksum = R(0.0);
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        Xk[n] = divc(P, Yk[n] * mbar, R(P.mm[n]), R(P.rmm[n]));
        Xksum += Xk[n];
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) Xkp[n] = Xk[n] + R(1.0e-16) * (divc(P, Xksum, R(double(NS)), R(1.0 / double(NS))) - Xk[n]);
#pragma unroll
    for (int n = 0; n < NS; ++n) Ykp[n] = rdiv(Xkp[n] * R(P.mm[n]), mbar);

    const R kT = R(P.k_B) * temperature;
    R Dbin[NS][NS];
#pragma unroll
    for (int i = 0; i < NS; ++i)
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            if (j < i) { Dbin[i][j] = Dbin[j][i]; continue; }  // symmetric: bitwise equal
            const R dij = R(P.diam[i][j]);
            Dbin[i][j] = rdiv((R(3.0) / R(16.0)) * dsqrt(divc(P, R(2.0) * pi * kT * kT * kT, R(P.mu[i][j]), R(P.rmu[i][j]))),
                              pressure * pi * dij * dij);
        }
    // reciprocals of the off-diagonal binary diffusivities, each a divisor ~7 times below
    // (up to two species: one reciprocal for 14 divisions; with more species the
    // reciprocals held across the solves cost more in spills than they save)
    R rDbin[NS][NS];
#pragma unroll
    for (int i = 0; i < NS; ++i)
#pragma unroll
        for (int j = 0; j < NS; ++j)
            rDbin[i][j] = (i == j || NS > 2) ? R(0.) : (j < i ? rDbin[j][i] : rdiv(R(1.), Dbin[i][j]));
    // viscosity
    R amat[NS][NS], Bi[NS], rhs[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        const R eta1 = R(P.eta1pre[i]) * dsqrt(divc(P, R(P.mmkB[i]) * temperature, pi, R(P.rpi)));
        rhs[i] = Xkp[i];
        Bi[i] = rhs[i];
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            if (i == j) {
                R a = rdiv(Xkp[i] * Xkp[i], eta1);
#pragma unroll
                for (int k = 0; k < NS; ++k)
                    if (k != i)
                        a += rdiv(R(2.0) * kT * Xkp[i] * Xkp[k], pressure * Dbin[i][k] * R(P.msum[i][k])) *
                             R(P.vfac[i][k]);
                amat[i][i] = a;
            } else {
                amat[i][j] = rdiv(R(2.0) * kT * Xkp[i] * Xkp[j], pressure * Dbin[i][j] * R(P.msum[i][j])) *
                             R(P.voff);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < NS - 1; ++j)
#pragma unroll
        for (int i = j + 1; i < NS; ++i) {
            const R fact1 = rdiv(amat[i][j], amat[j][j]);
#pragma unroll
            for (int k = 0; k < NS; ++k) amat[i][k] -= fact1 * amat[j][k];
            Bi[i] -= fact1 * Bi[j];
        }
    Bi[NS - 1] = rdiv(Bi[NS - 1], amat[NS - 1][NS - 1]);
#pragma unroll
    for (int i = NS - 2; i > -1; --i) {
        R sum1 = R(0.0);
#pragma unroll
        for (int j = NS - 1; j > i; --j) sum1 += amat[i][j] * Bi[j];
        Bi[i] = rdiv(Bi[i] - sum1, amat[i][i]);
    }
    R eta = R(0.0);
#pragma unroll
    for (int i = 0; i < NS; ++i) eta += Xkp[i] * Bi[i];
    c.eta = eta;
    c.zeta = R(0.);
    // thermal conductivity
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        rhs[i] = R(2.5) * Xkp[i];
        Bi[i] = rhs[i];
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            if (i == j) {
                R a = rdiv(Xkp[i] * Xkp[i], Dbin[i][j]) * R(2.0) * R(1.0);
#pragma unroll
                for (int k = 0; k < NS; ++k)
                    if (k != i)
                        a += divc(P, div_dbin<NS, R>(P, Xkp[i] * Xkp[k], Dbin[i][k], rDbin[i][k]) * R(P.mu[i][k]), R(P.msum[i][k]),
                                  R(P.rmsum[i][k])) * R(P.kfac[i][k]);
                amat[i][i] = a;
            } else {
                amat[i][j] = divc(P, div_dbin<NS, R>(P, R(-1.0) * Xkp[i] * Xkp[j], Dbin[i][j], rDbin[i][j]) * R(P.mu[i][j]),
                                  R(P.msum[i][j]), R(P.rmsum[i][j])) * R(P.koff);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < NS - 1; ++j)
#pragma unroll
        for (int i = j + 1; i < NS; ++i) {
            const R fact1 = rdiv(amat[i][j], amat[j][j]);
#pragma unroll
            for (int k = 0; k < NS; ++k) amat[i][k] -= fact1 * amat[j][k];
            Bi[i] -= fact1 * Bi[j];
        }
    Bi[NS - 1] = rdiv(Bi[NS - 1], amat[NS - 1][NS - 1]);
#pragma unroll
    for (int i = NS - 2; i > -1; --i) {
        R sum1 = R(0.0);
#pragma unroll
        for (int j = NS - 1; j > i; --j) sum1 += amat[i][j] * Bi[j];
        Bi[i] = rdiv(Bi[i] - sum1, amat[i][i]);
    }
    R kappa = R(0.0);
#pragma unroll
    for (int i = 0; i < NS; ++i) kappa += rhs[i] * Bi[i];
    kappa *= rdiv(pressure, temperature);
    c.kappa = kappa;
    // thermal diffusion ratios
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        R ch = R(0.0);
        R row[NS];
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            if (i == j) {
                R a = R(0.0);
#pragma unroll
                for (int k = 0; k < NS; ++k)
                    if (k != i)
                        a -= divc(P, div_dbin<NS, R>(P, R(0.5) * Xkp[k], Dbin[i][k], rDbin[i][k]) * R(P.mm[k]), R(P.msum[i][k]),
                                  R(P.rmsum[i][k])) * R(P.cfac);
                row[j] = a;
            } else {
                row[j] = divc(P, div_dbin<NS, R>(P, R(0.5) * Xkp[j], Dbin[i][j], rDbin[i][j]) * R(P.mm[i]), R(P.msum[i][j]),
                              R(P.rmsum[i][j])) * R(P.cfac);
            }
        }
#pragma unroll
        for (int j = 0; j < NS; ++j) ch += row[j] * Bi[j];
        c.chi[i] = ch;
    }
    if constexpr (NS == 1) {
        c.D[0] = R(0.);  // a single gas has no species diffusion
    } else {
        R Dl[NS * NS];
        D_GIO1<NS, R>(P, Dbin, rDbin, Ykp, Xkp, Dl);
#pragma unroll
        for (int q = 0; q < NS * NS; ++q) c.D[q] = Dl[q] * rho;
    }
    if (P.visc_type == 3 || P.visc_type == -3) c.zeta = R(P.zeta_ratio) * c.eta;
    return ok;
}

// conservedToPrimitiveStag cell body (conservedPrimitiveConversionsStag.cpp:97-140):
// from rho, rhoE, rhoY and the six face momenta around the cell.
template <int NS>
struct Prim {
    double T, p;
    double Y[NS], X[NS];
};

template <int NS>
FHD_D bool cons_to_prim(const DevParams& P, double rho, double rhoE, const double (&rhoY)[NS], double mxl,
                        double mxh, double myl, double myh, double mzl, double mzh, Prim<NS>& q) {
    double kin = 0.;
    kin = add_rn(kin, mul_rn(mxh + mxl, mxh + mxl));
    kin = add_rn(kin, mul_rn(myh + myl, myh + myl));
    kin = add_rn(kin, mul_rn(mzh + mzl, mzh + mzl));
    kin *= (0.125 / rho);
    const double intenergy = (rhoE - kin) / rho;
    double Yf[NS];
    double sumYk = 0.;
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        q.Y[n] = rhoY[n] / rho;
        Yf[n] = clamp01(q.Y[n]);
        sumYk += Yf[n];
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) Yf[n] /= sumYk;
    q.T = GetTemperature<NS, double>(P, intenergy, Yf);
    GetMolfrac<NS, double>(P, q.Y, q.X);
    q.p = GetPressureGas<NS, double>(P, q.Y, rho, q.T);
    return isfinite(q.T) && isfinite(q.p);
}

}  // namespace fhd
