// fhd_oracle.cpp — CPU ORACLE (test infrastructure only; never shipped, never on the
// product path).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
// reference arm may load it.
//
// A plain C++17 restatement of FHDeX's compressible staggered-grid RK3 step for a
// single fully periodic box, following the reference operator by operator and
// keeping its floating-point operation order (build with -ffp-contract=off so
// a*b+c is never fused).  Every function cites the reference lines it follows.
// The reference application needs AMReX (not vendored, no network), but its
// hot-path sources compile unmodified against the host-only AMReX stand-in in
// oracle/amrex_host (oracle/_ref, recipe in oracle/Makefile); tests/
// test_reference_pin.py holds this restatement bit for bit to that build, and
// tests/ also check it against the reference's known-answer formulas
// (closed-form hard-sphere transport, exact conservation, equilibrium variances).
//
// Scope: periodic boundaries (every physical-BC routine on the path is then a
// no-op: boundaryStag.cpp:5-14, 1555-1557), 3D, algorithm_type 2,
// transport_type 1 (Giovangigli), stoch_stress_form 0/1, advection_type 0/1/2,
// visc_type 1/2/3, the compressible chemistry source (reaction_type 0/1), no
// reservoir/membrane/turbulence forcing.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/fhd_capi.h"

namespace {

constexpr int MAXS = FHD_MAX_SPECIES;
const int kCellNodal[3] = {0, 0, 0};

// ---- global parameters (the reference's common::/compressible:: namespaces) ----
struct P {
    int ns = 2, nvars = 7, nprimvars = 10;
    int n[3] = {1, 1, 1};
    double dx[3] = {1, 1, 1};
    double molmass[MAXS], diameter[MAXS], dof[MAXS], e0[MAXS], hcv[MAXS], hcp[MAXS];
    double k_B = 1.38064852e-16, Runiv = 8.314462175e7;
    double grav[3] = {0, 0, 0};
    double zeta_ratio = -1;
    int visc_type = 1, advection_type = 0, algorithm_type = 2, stoch_stress_form = 1;
    // chemistry (chemistry_namespace.H; common::avogadro)
    int nreaction = 0, reaction_type = 0;
    int stoich_R[FHD_MAX_REACTIONS][MAXS], stoich_PR[FHD_MAX_REACTIONS][MAXS];
    double rate_const[FHD_MAX_REACTIONS], alpha_param[FHD_MAX_REACTIONS], beta_param[FHD_MAX_REACTIONS];
    double T0_chem = 0, avogadro = 0;
    int cross_cell = 0;   // plot_cross's x* (common::cross_cell)
} g;

struct Fab {
    double* p;
    int lo[3], hi[3], nc, nodal[3];
    long sy, sz, sn;
    Fab() : p(nullptr), nc(0), sy(0), sz(0), sn(0) {
        for (int d = 0; d < 3; ++d) { lo[d] = hi[d] = 0; nodal[d] = 0; }
    }
    explicit Fab(const fhd_fab& f) {
        p = static_cast<double*>(f.data);
        for (int d = 0; d < 3; ++d) { lo[d] = f.lo[d]; hi[d] = f.hi[d]; nodal[d] = f.nodal[d]; }
        nc = f.ncomp;
        long nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
        sy = nx; sz = nx * ny; sn = nx * ny * nz;
    }
    double& operator()(int i, int j, int k, int n = 0) const {
        return p[(i - lo[0]) + (j - lo[1]) * sy + (k - lo[2]) * sz + n * sn];
    }
    int ngrow() const { return -lo[0]; }
};

// Owned temporary fab (cell or nodal box grown by ng), zero-initialised.
struct OwnedFab {
    std::vector<double> v;
    Fab f;
    OwnedFab(int nx, int ny, int nz, const int nodal[3], int ng, int nc) {
        fhd_fab d;
        int nn[3] = {nx, ny, nz};
        for (int k = 0; k < 3; ++k) {
            d.lo[k] = -ng;
            d.hi[k] = nn[k] - 1 + nodal[k] + ng;
            d.nodal[k] = nodal[k];
        }
        d.ncomp = nc;
        d.dtype = FHD_F64;
        long n = 1;
        for (int k = 0; k < 3; ++k) n *= (d.hi[k] - d.lo[k] + 1);
        v.assign(n * nc, 0.0);
        d.data = v.data();
        f = Fab(d);
    }
};

inline int wrapi(int i, int n) { int r = i % n; return r < 0 ? r + n : r; }

// ---- AMReX semantics restated ---------------------------------------------------

// MultiFab::FillBoundary(periodicity), one periodic box: every ghost point takes
// the value of its periodic image in the valid region; valid points untouched.
void fill_boundary(const Fab& f) {
    const int* N = g.n;
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = f.lo[2]; k <= f.hi[2]; ++k)
        for (int j = f.lo[1]; j <= f.hi[1]; ++j)
            for (int i = f.lo[0]; i <= f.hi[0]; ++i) {
                int idx[3] = {i, j, k}, src[3];
                bool ghost = false;
                for (int d = 0; d < 3; ++d) {
                    int vhi = N[d] - 1 + f.nodal[d];
                    if (idx[d] < 0 || idx[d] > vhi) ghost = true;
                    src[d] = idx[d];
                    while (src[d] < 0) src[d] += N[d];
                    while (src[d] > vhi) src[d] -= N[d];
                }
                if (!ghost) continue;
                for (int n = 0; n < f.nc; ++n) f(i, j, k, n) = f(src[0], src[1], src[2], n);
            }
}

// MultiFab::OverrideSync(periodicity): for a nodal direction the point n_cells
// duplicates point 0; the low-side point owns it.
void override_sync(const Fab& f) {
    const int* N = g.n;
    for (int k = 0; k <= N[2] - 1 + f.nodal[2]; ++k)
        for (int j = 0; j <= N[1] - 1 + f.nodal[1]; ++j)
            for (int i = 0; i <= N[0] - 1 + f.nodal[0]; ++i) {
                int s[3] = {i, j, k};
                bool dup = false;
                for (int d = 0; d < 3; ++d)
                    if (f.nodal[d] && s[d] == N[d]) { s[d] = 0; dup = true; }
                if (!dup) continue;
                for (int n = 0; n < f.nc; ++n) f(i, j, k, n) = f(s[0], s[1], s[2], n);
            }
}

// ---- point physics: compressible_functions.H ------------------------------------

// GetMolfrac, compressible_functions.H:138-151
inline void GetMolfrac(const double* Yk, double* Xk) {
    double molmix = 0.;
    for (int n = 0; n < g.ns; ++n) molmix += Yk[n] / g.molmass[n];
    molmix = 1. / molmix;
    for (int n = 0; n < g.ns; ++n) Xk[n] = Yk[n] * molmix / g.molmass[n];
}
// GetTemperature, compressible_functions.H:168-182
inline void GetTemperature(double energy, const double* Yk, double& temp) {
    double cvmix = 0., e0mix = 0.;
    for (int n = 0; n < g.ns; ++n) { cvmix += Yk[n] * g.hcv[n]; e0mix += Yk[n] * g.e0[n]; }
    temp = (energy - e0mix) / cvmix;
}
// GetPressureGas, compressible_functions.H:184-199
inline void GetPressureGas(double& pressure, const double* Yk, double density, double temp) {
    double molmix = 0.;
    for (int n = 0; n < g.ns; ++n) molmix += Yk[n] / g.molmass[n];
    molmix = 1. / molmix;
    pressure = density * (g.Runiv / molmix) * temp;
}
// GetEnergy, compressible_functions.H:1497-1510
inline void GetEnergy(double& energy, const double* massvec, double temp) {
    double cvmix = 0., e0mix = 0.;
    for (int i = 0; i < g.ns; ++i) { cvmix += massvec[i] * g.hcv[i]; e0mix += massvec[i] * g.e0[i]; }
    energy = e0mix + temp * cvmix;
}
// GetEnthalpies, compressible_functions.H:1512-1519
inline void GetEnthalpies(double T, double* hk) {
    for (int i = 0; i < g.ns; ++i) hk[i] = g.e0[i] + g.hcp[i] * T;
}

// CholeskyDecomp, compressible_functions.H:460-511.  Only the lower triangle and
// the diagonal reach the result; the reference's writes above the diagonal use a
// not-yet-set pivot and are never read back, so they are not restated.
inline void CholeskyDecomp(double* a, int ns, double* sqda) {
    double p[MAXS];
    for (int i = 0; i < ns; ++i) {
        int ising = 0;
        for (int j = i; j < ns; ++j) {
            double sum1 = a[i * ns + j];
            for (int k = i - 1; k >= 0; --k) sum1 = sum1 - a[i * ns + k] * a[j * ns + k];
            if (i == j) {
                if (sum1 <= 0.) { p[i] = 0.; ising = 1; }
                else p[i] = std::sqrt(sum1);
            }
            if (ising == 0) a[j * ns + i] = sum1 / p[i];
            else a[j * ns + i] = 0.;
        }
    }
    for (int i = 0; i < ns; ++i) for (int j = 0; j < ns; ++j) sqda[i * ns + j] = 0.;
    for (int i = 0; i < ns; ++i) {
        for (int j = i - 1; j >= 0; --j) sqda[i * ns + j] = a[i * ns + j];
        sqda[i * ns + i] = p[i];
    }
}

// D_GIO1, compressible_functions.H:647-778; writes D_tilde comp j*ns+i.
void D_GIO1(const double Dbin[MAXS][MAXS], const double* Ykp, const double* Xkp,
            double* Dout /* ns*ns, component order */) {
    const int ns = g.ns;
    double Diff_ij[MAXS * MAXS], Zmat[MAXS * MAXS], Pmat[MAXS * MAXS], Jmat[MAXS * MAXS],
        PJ[MAXS * MAXS], matrix1[MAXS * MAXS], matrix2[MAXS * MAXS];
    double Di[MAXS], Minv[MAXS], Mmat[MAXS];
    const int jmax = 3;
    for (int i = 0; i < ns; ++i) {
        double term2 = 0.;
        for (int j = 0; j < ns; ++j) if (j != i) term2 = term2 + Xkp[j] / Dbin[i][j];
        Di[i] = (1. - Ykp[i]) / term2;
    }
    for (int i = 0; i < ns; ++i) { Mmat[i] = Xkp[i] / Di[i]; Minv[i] = Di[i] / Xkp[i]; }
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j < ns; ++j) {
            Pmat[i * ns + j] = -Ykp[j];
            if (i == j) Pmat[i * ns + j] = Pmat[i * ns + j] + 1.;
        }
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j < ns; ++j) {
            double Deltamat;
            if (i == j) {
                double term1 = 0.;
                for (int k = 0; k < ns; ++k) if (k != i) term1 = term1 + Xkp[i] * Xkp[k] / Dbin[i][k];
                Deltamat = term1;
            } else {
                Deltamat = -Xkp[i] * Xkp[j] / Dbin[i][j];
            }
            Zmat[i * ns + j] = -Deltamat;
        }
    for (int i = 0; i < ns; ++i) Zmat[i * ns + i] = Zmat[i * ns + i] + Mmat[i];
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j < ns; ++j) Jmat[i * ns + j] = Minv[i] * Zmat[i * ns + j];
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j < ns; ++j) {
            PJ[i * ns + j] = 0.;
            for (int k = 0; k < ns; ++k) PJ[i * ns + j] = PJ[i * ns + j] + Pmat[i * ns + k] * Jmat[k * ns + j];
        }
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j < ns; ++j) {
            double scr = 0.;
            for (int k = 0; k < ns; ++k) scr = scr + Pmat[i * ns + k] * Minv[k] * Pmat[j * ns + k];
            matrix2[i * ns + j] = scr;
            Diff_ij[i * ns + j] = scr;
        }
    for (int ll = 0; ll < jmax; ++ll) {
        for (int i = 0; i < ns; ++i)
            for (int j = 0; j < ns; ++j) {
                double scr = 0.;
                for (int k = 0; k < ns; ++k) scr = scr + PJ[i * ns + k] * Diff_ij[k * ns + j];
                matrix1[i * ns + j] = scr + matrix2[i * ns + j];
            }
        for (int i = 0; i < ns * ns; ++i) Diff_ij[i] = matrix1[i];
    }
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j < ns; ++j) Dout[j * ns + i] = Diff_ij[i * ns + j] * Ykp[i];
}

// IdealMixtureTransportGIO, compressible_functions.H:1153-1352.
void IdealMixtureTransportGIO(double temperature, double pressure, const double* Yk,
                              double& eta, double& kappa, double& zeta, double* Dout,
                              double* chitil) {
    const int ns = g.ns;
    double mu[MAXS][MAXS], diam[MAXS][MAXS], Dbin[MAXS][MAXS], amat[MAXS][MAXS];
    double molecular_mass[MAXS], Xk[MAXS], Xkp[MAXS], Ykp[MAXS], eta1[MAXS], rhs[MAXS], Bi[MAXS];
    const double pi = 3.1415926535897932;
    for (int n = 0; n < ns; ++n) molecular_mass[n] = g.molmass[n] * (g.k_B / g.Runiv);
    double mbar = 0.0;
    for (int n = 0; n < ns; ++n) mbar += Yk[n] / molecular_mass[n];
    mbar = 1.0 / mbar;
    double Xksum = 0.0;
    for (int n = 0; n < ns; ++n) { Xk[n] = Yk[n] * mbar / molecular_mass[n]; Xksum += Xk[n]; }
    for (int n = 0; n < ns; ++n) Xkp[n] = Xk[n] + 1.0e-16 * (Xksum / double(ns) - Xk[n]);
    for (int n = 0; n < ns; ++n) Ykp[n] = Xkp[n] * molecular_mass[n] / mbar;
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j < ns; ++j) {
            diam[i][j] = 0.5 * (g.diameter[i] + g.diameter[j]);
            mu[i][j] = molecular_mass[i] * molecular_mass[j] / (molecular_mass[i] + molecular_mass[j]);
        }
    const double kT = g.k_B * temperature;
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j < ns; ++j)
            Dbin[i][j] = (3.0 / 16.0) * std::sqrt(2.0 * pi * kT * kT * kT / mu[i][j]) /
                         (pressure * pi * diam[i][j] * diam[i][j]);
    const double AKL = 1.0, BKL = 1.0, CKL = 1.0;
    // viscosity
    for (int i = 0; i < ns; ++i)
        eta1[i] = 5.0 / (16.0 * diam[i][i] * diam[i][i]) * std::sqrt(molecular_mass[i] * g.k_B * temperature / pi);
    for (int i = 0; i < ns; ++i) {
        rhs[i] = Xkp[i];
        Bi[i] = rhs[i];
        for (int j = 0; j < ns; ++j) {
            if (i == j) {
                amat[i][i] = Xkp[i] * Xkp[i] / eta1[i];
                for (int k = 0; k < ns; ++k)
                    if (k != i)
                        amat[i][i] += 2.0 * kT * Xkp[i] * Xkp[k] /
                                      (pressure * Dbin[i][k] * (molecular_mass[i] + molecular_mass[k])) *
                                      (1.0 + 0.6 * molecular_mass[k] / molecular_mass[i] * AKL);
            } else {
                amat[i][j] = 2.0 * kT * Xkp[i] * Xkp[j] /
                             (pressure * Dbin[i][j] * (molecular_mass[i] + molecular_mass[j])) * (0.6 * AKL - 1.0);
            }
        }
    }
    for (int j = 0; j < ns - 1; ++j)
        for (int i = j + 1; i < ns; ++i) {
            double fact1 = amat[i][j] / amat[j][j];
            for (int k = 0; k < ns; ++k) amat[i][k] -= fact1 * amat[j][k];
            Bi[i] -= fact1 * Bi[j];
        }
    Bi[ns - 1] /= amat[ns - 1][ns - 1];
    for (int i = ns - 2; i > -1; --i) {
        double sum1 = 0.0;
        for (int j = ns - 1; j > i; --j) sum1 += amat[i][j] * Bi[j];
        Bi[i] = (Bi[i] - sum1) / amat[i][i];
    }
    eta = 0.0;
    for (int i = 0; i < ns; ++i) eta += Xkp[i] * Bi[i];
    zeta = 0.;
    // thermal conductivity
    for (int i = 0; i < ns; ++i) {
        rhs[i] = 2.5 * Xkp[i];
        Bi[i] = rhs[i];
        for (int j = 0; j < ns; ++j) {
            if (i == j) {
                amat[i][i] = Xkp[i] * Xkp[i] / Dbin[i][j] * 2.0 * AKL;
                for (int k = 0; k < ns; ++k)
                    if (k != i)
                        amat[i][i] += Xkp[i] * Xkp[k] / Dbin[i][k] * mu[i][k] /
                                      (molecular_mass[i] + molecular_mass[k]) *
                                      (7.5 * molecular_mass[i] / molecular_mass[k] +
                                       6.25 * molecular_mass[k] / molecular_mass[i] -
                                       3.0 * molecular_mass[k] / molecular_mass[i] * BKL + 4.0 * AKL);
            } else {
                amat[i][j] = -1.0 * Xkp[i] * Xkp[j] / Dbin[i][j] * mu[i][j] /
                             (molecular_mass[i] + molecular_mass[j]) * (55.0 / 4.0 - 3.0 * BKL - 4.0 * AKL);
            }
        }
    }
    for (int j = 0; j < ns - 1; ++j)
        for (int i = j + 1; i < ns; ++i) {
            double fact1 = amat[i][j] / amat[j][j];
            for (int k = 0; k < ns; ++k) amat[i][k] -= fact1 * amat[j][k];
            Bi[i] -= fact1 * Bi[j];
        }
    Bi[ns - 1] /= amat[ns - 1][ns - 1];
    for (int i = ns - 2; i > -1; --i) {
        double sum1 = 0.0;
        for (int j = ns - 1; j > i; --j) sum1 += amat[i][j] * Bi[j];
        Bi[i] = (Bi[i] - sum1) / amat[i][i];
    }
    kappa = 0.0;
    for (int i = 0; i < ns; ++i) kappa += rhs[i] * Bi[i];
    kappa *= pressure / temperature;
    // thermal diffusion ratios
    for (int i = 0; i < ns; ++i) {
        chitil[i] = 0.0;
        for (int j = 0; j < ns; ++j) {
            if (i == j) {
                amat[i][i] = 0.0;
                for (int k = 0; k < ns; ++k)
                    if (k != i)
                        amat[i][i] -= 0.5 * Xkp[k] / Dbin[i][k] * molecular_mass[k] /
                                      (molecular_mass[i] + molecular_mass[k]) * (6.0 * CKL - 5.0);
            } else {
                amat[i][j] = 0.5 * Xkp[j] / Dbin[i][j] * molecular_mass[i] /
                             (molecular_mass[i] + molecular_mass[j]) * (6.0 * CKL - 5.0);
            }
        }
    }
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j < ns; ++j) chitil[i] += amat[i][j] * Bi[j];
    D_GIO1(Dbin, Ykp, Xkp, Dout);
}

// ---- operators ------------------------------------------------------------------

int g_status = 0;

// calculateTransportCoeffs, transCoeffs.cpp:7-90, on the cell box grown by the
// ghost width of prim (ngc).
void transport_coeffs(const Fab& prim, const Fab& eta, const Fab& zeta, const Fab& kappa,
                      const Fab& chi, const Fab& D) {
    const int ns = g.ns, ng = prim.ngrow();
    int bad = 0;
    #pragma omp parallel for collapse(2) schedule(static) reduction(|:bad)
    for (int k = -ng; k < g.n[2] + ng; ++k)
        for (int j = -ng; j < g.n[1] + ng; ++j)
            for (int i = -ng; i < g.n[0] + ng; ++i) {
                double Yk_fixed[MAXS], Xk_fixed[MAXS];
                double sumYk = 0.;
                for (int n = 0; n < ns; ++n) {
                    double y = prim(i, j, k, 6 + n);
                    if (y <= 0.0 || y >= 1.0) bad = 1;   // amrex::Abort in the reference
                    Yk_fixed[n] = std::max(0., std::min(1., y));
                    sumYk += Yk_fixed[n];
                }
                for (int n = 0; n < ns; ++n) Yk_fixed[n] /= sumYk;
                GetMolfrac(Yk_fixed, Xk_fixed);
                double e, kp, z, Dl[MAXS * MAXS], ch[MAXS];
                IdealMixtureTransportGIO(prim(i, j, k, 4), prim(i, j, k, 5), Yk_fixed, e, kp, z, Dl, ch);
                eta(i, j, k) = e;
                kappa(i, j, k) = kp;
                zeta(i, j, k) = z;
                for (int n = 0; n < ns; ++n) chi(i, j, k, n) = ch[n];
                for (int kk = 0; kk < ns; ++kk)
                    for (int ll = 0; ll < ns; ++ll) {
                        int n = kk * ns + ll;
                        D(i, j, k, n) = Dl[n] * prim(i, j, k, 0);
                    }
                if (std::abs(g.visc_type) == 3) zeta(i, j, k) = g.zeta_ratio * eta(i, j, k);
            }
    if (bad) g_status = g_status ? g_status : FHD_ERR_MASSFRAC;
}

// conservedToPrimitiveStag, conservedPrimitiveConversionsStag.cpp:5-144.
void conserved_to_primitive(const Fab& prim, const Fab vel[3], const Fab& cons, const Fab mom[3]) {
    const int ns = g.ns;
    const int* N = g.n;
    // face velocities on valid faces (:59-68)
    for (int d = 0; d < 3; ++d) {
        const Fab& v = vel[d];
        const Fab& m = mom[d];
        int e[3] = {d == 0, d == 1, d == 2};
        #pragma omp parallel for collapse(2) schedule(static)
        for (int k = 0; k < N[2] + e[2]; ++k)
            for (int j = 0; j < N[1] + e[1]; ++j)
                for (int i = 0; i < N[0] + e[0]; ++i)
                    v(i, j, k) = 2 * m(i, j, k) / (cons(i, j, k, 0) + cons(i - e[0], j - e[1], k - e[2], 0));
    }
    const Fab &velx = vel[0], &vely = vel[1], &velz = vel[2];
    const Fab &momx = mom[0], &momy = mom[1], &momz = mom[2];
    int bad = 0;
    #pragma omp parallel for collapse(2) schedule(static) reduction(|:bad)
    for (int k = 0; k < N[2]; ++k)
        for (int j = 0; j < N[1]; ++j)
            for (int i = 0; i < N[0]; ++i) {
                double Xk[MAXS], Yk[MAXS], Yk_fixed[MAXS];
                prim(i, j, k, 0) = cons(i, j, k, 0);
                prim(i, j, k, 1) = 0.5 * (velx(i, j, k) + velx(i + 1, j, k));
                prim(i, j, k, 2) = 0.5 * (vely(i, j, k) + vely(i, j + 1, k));
                prim(i, j, k, 3) = 0.5 * (velz(i, j, k) + velz(i, j, k + 1));
                cons(i, j, k, 1) = 0.5 * (momx(i, j, k) + momx(i + 1, j, k));
                cons(i, j, k, 2) = 0.5 * (momy(i, j, k) + momy(i, j + 1, k));
                cons(i, j, k, 3) = 0.5 * (momz(i, j, k) + momz(i, j, k + 1));
                double kinenergy = 0.;
                kinenergy += (momx(i + 1, j, k) + momx(i, j, k)) * (momx(i + 1, j, k) + momx(i, j, k));
                kinenergy += (momy(i, j + 1, k) + momy(i, j, k)) * (momy(i, j + 1, k) + momy(i, j, k));
                kinenergy += (momz(i, j, k + 1) + momz(i, j, k)) * (momz(i, j, k + 1) + momz(i, j, k));
                kinenergy *= (0.125 / cons(i, j, k, 0));
                double intenergy = (cons(i, j, k, 4) - kinenergy) / cons(i, j, k, 0);
                double sumYk = 0.;
                for (int n = 0; n < ns; ++n) {
                    Yk[n] = cons(i, j, k, 5 + n) / cons(i, j, k, 0);
                    Yk_fixed[n] = std::max(0., std::min(1., Yk[n]));
                    sumYk += Yk_fixed[n];
                }
                for (int n = 0; n < ns; ++n) Yk_fixed[n] /= sumYk;
                double T;
                GetTemperature(intenergy, Yk_fixed, T);
                prim(i, j, k, 4) = T;
                GetMolfrac(Yk, Xk);
                for (int n = 0; n < ns; ++n) {
                    prim(i, j, k, 6 + n) = Yk[n];
                    prim(i, j, k, 6 + ns + n) = Xk[n];
                }
                double p;
                GetPressureGas(p, Yk, cons(i, j, k, 0), T);
                prim(i, j, k, 5) = p;
                if (!std::isfinite(T) || !std::isfinite(p)) bad = 1;
            }
    if (bad) g_status = g_status ? g_status : FHD_ERR_NONFINITE;
}

// calculateFluxStag, fluxStag.cpp:5-1868, periodic (no Dirichlet branches taken).
// ef[6] = edgeflux_x[0] (xy, v), edgeflux_x[1] (xz, w), edgeflux_y[0] (xy, u),
//         edgeflux_y[1] (yz, w), edgeflux_z[0] (xz, u), edgeflux_z[1] (yz, v).
// se[3] = combined xy, xz, yz edge noise (stochedge_x[0], stochedge_x[1], stochedge_y[1]).
// sf[3] face noise (energy at comp sf_off, species after), sc[3] centre noise (1 ghost).
void flux_stag(const Fab& cons, const Fab mom[3], const Fab& prim, const Fab vel[3],
               const Fab& eta, const Fab& zeta, const Fab& kappa, const Fab& chi, const Fab& Dij,
               const Fab ff[3], const Fab ef[6], const Fab cf[3], const Fab sf[3], const Fab se[3],
               const Fab sc[3], double dt) {
    const int ns = g.ns, nvars = g.nvars;
    const int* N = g.n;
    const double* dx = g.dx;
    const double k_B = g.k_B, Runiv = g.Runiv;

    const Fab &edgex_v = ef[0], &edgex_w = ef[1], &edgey_u = ef[2], &edgey_w = ef[3], &edgez_u = ef[4],
              &edgez_v = ef[5];
    const Fab &cenx_u = cf[0], &ceny_v = cf[1], &cenz_w = cf[2];
    const Fab &velx = vel[0], &vely = vel[1], &velz = vel[2];
    const Fab &momx = mom[0], &momy = mom[1], &momz = mom[2];
    const int ngc = 2;

    // :30-45 zero every flux (valid + ghosts)
    for (int d = 0; d < 3; ++d) {
        std::fill(ff[d].p, ff[d].p + ff[d].sn * ff[d].nc, 0.0);
        std::fill(cf[d].p, cf[d].p + cf[d].sn * cf[d].nc, 0.0);
    }
    for (int e = 0; e < 6; ++e) std::fill(ef[e].p, ef[e].p + ef[e].sn * ef[e].nc, 0.0);

    // :47-81 stress temporaries (cells and edges, ngc ghosts), zeroed
    const int cnod[3] = {0, 0, 0}, nxy[3] = {1, 1, 0}, nyz[3] = {0, 1, 1}, nxz[3] = {1, 0, 1};
    OwnedFab tdx(N[0], N[1], N[2], cnod, ngc, 1), tdy(N[0], N[1], N[2], cnod, ngc, 1),
        tdz(N[0], N[1], N[2], cnod, ngc, 1);
    OwnedFab tsx(N[0], N[1], N[2], cnod, ngc, 1), tsy(N[0], N[1], N[2], cnod, ngc, 1),
        tsz(N[0], N[1], N[2], cnod, ngc, 1);
    OwnedFab txy(N[0], N[1], N[2], nxy, ngc, 1), tyz(N[0], N[1], N[2], nyz, ngc, 1),
        txz(N[0], N[1], N[2], nxz, ngc, 1);
    OwnedFab sxy(N[0], N[1], N[2], nxy, ngc, 1), syz(N[0], N[1], N[2], nyz, ngc, 1),
        sxz(N[0], N[1], N[2], nxz, ngc, 1);
    const Fab &tauxx = tdx.f, &tauyy = tdy.f, &tauzz = tdz.f;
    const Fab &tauxx_s = tsx.f, &tauyy_s = tsy.f, &tauzz_s = tsz.f;
    const Fab &tauxy = txy.f, &tauyz = tyz.f, &tauxz = txz.f;
    const Fab &tauxy_s = sxy.f, &tauyz_s = syz.f, &tauxz_s = sxz.f;

    const int sfo[3] = {sf[0].nc - (ns + 1), sf[1].nc - (ns + 1), sf[2].nc - (ns + 1)};

    if (g.stoch_stress_form == 1) {
        const double volinv = 1. / (dx[0] * dx[1] * dx[2]);
        const double dtinv = 1. / dt;
        // :163-206 diagonal stochastic stress on cells grown by 1
        #pragma omp parallel for collapse(2) schedule(static)
        for (int k = -1; k <= N[2]; ++k)
            for (int j = -1; j <= N[1]; ++j)
                for (int i = -1; i <= N[0]; ++i) {
                    double etaT = eta(i, j, k) * prim(i, j, k, 4);
                    double zetaT = zeta(i, j, k) * prim(i, j, k, 4);
                    double fac1 = std::sqrt(2.0 * k_B * etaT * volinv * dtinv);
                    double fac2 = (-1.0 / 3.0) * std::sqrt(2.0 * k_B * etaT * volinv * dtinv);
                    if (std::abs(g.visc_type) == 3)
                        fac2 = std::sqrt(k_B * zetaT * volinv * dtinv / 3.0) -
                               std::sqrt(2.0 * k_B * etaT * volinv * dtinv) / 3.0;
                    double traceZ = sc[0](i, j, k) + sc[1](i, j, k) + sc[2](i, j, k);
                    tauxx_s(i, j, k) = (fac1 * sc[0](i, j, k)) + (fac2 * traceZ);
                    tauyy_s(i, j, k) = (fac1 * sc[1](i, j, k)) + (fac2 * traceZ);
                    tauzz_s(i, j, k) = (fac1 * sc[2](i, j, k)) + (fac2 * traceZ);
                }
        // :209-295 off-diagonal stochastic stress on edges
        #pragma omp parallel for collapse(2) schedule(static)
        for (int k = 0; k <= N[2]; ++k)
            for (int j = 0; j <= N[1]; ++j)
                for (int i = 0; i <= N[0]; ++i) {
                    if (k < N[2]) {  // xy edge (nodal x,y)
                        double etaT = 0.25 * (eta(i - 1, j - 1, k) * prim(i - 1, j - 1, k, 4) +
                                              eta(i - 1, j, k) * prim(i - 1, j, k, 4) +
                                              eta(i, j - 1, k) * prim(i, j - 1, k, 4) +
                                              eta(i, j, k) * prim(i, j, k, 4));
                        double fac = std::sqrt(2.0 * k_B * etaT * volinv * dtinv);
                        tauxy_s(i, j, k) = fac * se[0](i, j, k);
                    }
                    if (j < N[1]) {  // xz edge
                        double etaT = 0.25 * (eta(i - 1, j, k - 1) * prim(i - 1, j, k - 1, 4) +
                                              eta(i - 1, j, k) * prim(i - 1, j, k, 4) +
                                              eta(i, j, k - 1) * prim(i, j, k - 1, 4) +
                                              eta(i, j, k) * prim(i, j, k, 4));
                        double fac = std::sqrt(2.0 * k_B * etaT * volinv * dtinv);
                        tauxz_s(i, j, k) = fac * se[1](i, j, k);
                    }
                    if (i < N[0]) {  // yz edge
                        double etaT = 0.25 * (eta(i, j - 1, k - 1) * prim(i, j - 1, k - 1, 4) +
                                              eta(i, j - 1, k) * prim(i, j - 1, k, 4) +
                                              eta(i, j, k - 1) * prim(i, j, k - 1, 4) +
                                              eta(i, j, k) * prim(i, j, k, 4));
                        double fac = std::sqrt(2.0 * k_B * etaT * volinv * dtinv);
                        tauyz_s(i, j, k) = fac * se[2](i, j, k);
                    }
                }
        // :298-781 stochastic face fluxes (heat, viscous heating, species, Dufour)
        for (int d = 0; d < 3; ++d) {
            const Fab& fl = ff[d];
            const Fab& sfd = sf[d];
            const int o = sfo[d];
            const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
            #pragma omp parallel for collapse(2) schedule(static)
            for (int k = 0; k < N[2] + e2; ++k)
                for (int j = 0; j < N[1] + e1; ++j)
                    for (int i = 0; i < N[0] + e0; ++i) {
                        const int im = i - e0, jm = j - e1, km = k - e2;  // lower cell
                        double kp = (kappa(i, j, k) * prim(i, j, k, 4) * prim(i, j, k, 4) +
                                     kappa(im, jm, km) * prim(im, jm, km, 4) * prim(im, jm, km, 4));
                        double meanT = 0.5 * (prim(i, j, k, 4) + prim(im, jm, km, 4));
                        double wiener[MAXS + 1];
                        // heat flux
                        double fw0 = std::sqrt(k_B * kp * volinv * dtinv);
                        wiener[0] = fw0 * sfd(i, j, k, o);
                        fl(i, j, k, nvars) = wiener[0];
                        // viscous heating: diagonal and shear
                        double vsh = 0.0;
                        if (d == 0) {
                            fl(i, j, k, nvars + 1) = 0.5 * velx(i, j, k) * (tauxx_s(i - 1, j, k) + tauxx_s(i, j, k));
                            vsh += 0.25 * ((vely(i, j + 1, k) + vely(i - 1, j + 1, k)) * tauxy_s(i, j + 1, k) +
                                           (vely(i, j, k) + vely(i - 1, j, k)) * tauxy_s(i, j, k));
                            vsh += 0.25 * ((velz(i, j, k + 1) + velz(i - 1, j, k + 1)) * tauxz_s(i, j, k + 1) +
                                           (velz(i, j, k) + velz(i - 1, j, k)) * tauxz_s(i, j, k));
                        } else if (d == 1) {
                            fl(i, j, k, nvars + 1) = 0.5 * vely(i, j, k) * (tauyy_s(i, j - 1, k) + tauyy_s(i, j, k));
                            vsh += 0.25 * ((velx(i + 1, j, k) + velx(i + 1, j - 1, k)) * tauxy_s(i + 1, j, k) +
                                           (velx(i, j, k) + velx(i, j - 1, k)) * tauxy_s(i, j, k));
                            vsh += 0.25 * ((velz(i, j, k + 1) + velz(i, j - 1, k + 1)) * tauyz_s(i, j, k + 1) +
                                           (velz(i, j, k) + velz(i, j - 1, k)) * tauyz_s(i, j, k));
                        } else {
                            fl(i, j, k, nvars + 1) = 0.5 * velz(i, j, k) * (tauzz_s(i, j, k - 1) + tauzz_s(i, j, k));
                            vsh += 0.25 * ((velx(i + 1, j, k - 1) + velx(i + 1, j, k)) * tauxz_s(i + 1, j, k) +
                                           (velx(i, j, k) + velx(i, j, k - 1)) * tauxz_s(i, j, k));
                            vsh += 0.25 * ((vely(i, j + 1, k - 1) + vely(i, j + 1, k)) * tauyz_s(i, j + 1, k) +
                                           (vely(i, j, k) + vely(i, j, k - 1)) * tauyz_s(i, j, k));
                        }
                        fl(i, j, k, nvars + 2) = vsh;
                        // species noise (algorithm_type 2)
                        double yy[MAXS], yyp[MAXS], DijY_edge[MAXS * MAXS], sqD[MAXS * MAXS], hk[MAXS];
                        for (int n = 1; n < 1 + ns; ++n) wiener[n] = 0.;
                        for (int s = 0; s < ns; ++s) {
                            yy[s] = std::max(0., std::min(1., prim(im, jm, km, 6 + s)));
                            yyp[s] = std::max(0., std::min(1., prim(i, j, k, 6 + s)));
                        }
                        double sumy = 0., sumyp = 0.;
                        for (int n = 0; n < ns; ++n) { sumy += yy[n]; sumyp += yyp[n]; }
                        for (int n = 0; n < ns; ++n) { yy[n] /= sumy; yyp[n] /= sumyp; }
                        double MWmix = 0.;
                        for (int s = 0; s < ns; ++s) {
                            MWmix = MWmix + 0.5 * (yy[s] + yyp[s]) / g.molmass[s];
                            for (int ll = 0; ll < ns; ++ll)
                                DijY_edge[s * ns + ll] =
                                    0.5 * (Dij(im, jm, km, ll * ns + s) * yy[ll] + Dij(i, j, k, ll * ns + s) * yyp[ll] +
                                           (Dij(im, jm, km, s * ns + ll) * yy[s] + Dij(i, j, k, s * ns + ll) * yyp[s]));
                        }
                        for (int s = 0; s < ns; ++s)
                            if (std::abs(yy[s]) + std::abs(yyp[s]) <= 1.e-12)
                                for (int n = 0; n < ns; ++n) { DijY_edge[s * ns + n] = 0.; DijY_edge[n * ns + s] = 0.; }
                        MWmix = 1. / MWmix;
                        CholeskyDecomp(DijY_edge, ns, sqD);
                        for (int s = 0; s < ns; ++s) {
                            for (int ll = 0; ll <= s; ++ll) {
                                double fw = std::sqrt(k_B * MWmix * volinv / (Runiv * dt)) * sqD[s * ns + ll];
                                wiener[1 + s] = wiener[1 + s] + fw * sfd(i, j, k, o + 1 + ll);
                            }
                            fl(i, j, k, 5 + s) = wiener[1 + s];
                        }
                        GetEnthalpies(meanT, hk);
                        double soret = 0.;
                        for (int s = 0; s < ns; ++s) {
                            double soret_s = (hk[s] + Runiv * meanT / g.molmass[s] * 0.5 *
                                                          (chi(im, jm, km, s) + chi(i, j, k, s))) * wiener[1 + s];
                            soret += soret_s;
                        }
                        fl(i, j, k, nvars + 3) = soret;
                    }
        }
        // :784-803 momentum fluxes <- stochastic stresses
        for (int k = 0; k <= N[2]; ++k)
            for (int j = 0; j <= N[1]; ++j)
                for (int i = 0; i <= N[0]; ++i) {
                    if (k < N[2]) { edgey_u(i, j, k) = tauxy_s(i, j, k); edgex_v(i, j, k) = tauxy_s(i, j, k); }
                    if (j < N[1]) { edgez_u(i, j, k) = tauxz_s(i, j, k); edgex_w(i, j, k) = tauxz_s(i, j, k); }
                    if (i < N[0]) { edgez_v(i, j, k) = tauyz_s(i, j, k); edgey_w(i, j, k) = tauyz_s(i, j, k); }
                }
        for (int k = -1; k <= N[2]; ++k)
            for (int j = -1; j <= N[1]; ++j)
                for (int i = -1; i <= N[0]; ++i) {
                    cenx_u(i, j, k) = tauxx_s(i, j, k);
                    ceny_v(i, j, k) = tauyy_s(i, j, k);
                    cenz_w(i, j, k) = tauzz_s(i, j, k);
                }
    }

    // ---- diffusive fluxes :819-1449 ----
    // :872-924 diagonal stress on cells grown by 1
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = -1; k <= N[2]; ++k)
        for (int j = -1; j <= N[1]; ++j)
            for (int i = -1; i <= N[0]; ++i) {
                double u_x = (velx(i + 1, j, k) - velx(i, j, k)) / dx[0];
                double v_y = (vely(i, j + 1, k) - vely(i, j, k)) / dx[1];
                double w_z = (velz(i, j, k + 1) - velz(i, j, k)) / dx[2];
                double div = u_x + v_y + w_z;
                double e = eta(i, j, k);
                if (std::abs(g.visc_type) == 3) {
                    double z = zeta(i, j, k);
                    tauxx(i, j, k) = 2 * e * u_x + (z - 2 * e / 3.) * div;
                    tauyy(i, j, k) = 2 * e * v_y + (z - 2 * e / 3.) * div;
                    tauzz(i, j, k) = 2 * e * w_z + (z - 2 * e / 3.) * div;
                } else {
                    tauxx(i, j, k) = 2 * e * u_x + (0.0 - 2 * e / 3.) * div;
                    tauyy(i, j, k) = 2 * e * v_y + (0.0 - 2 * e / 3.) * div;
                    tauzz(i, j, k) = 2 * e * w_z + (0.0 - 2 * e / 3.) * div;
                }
            }
    // :927-1023 off-diagonal stress on edges
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k <= N[2]; ++k)
        for (int j = 0; j <= N[1]; ++j)
            for (int i = 0; i <= N[0]; ++i) {
                if (k < N[2]) {
                    double u_y = (velx(i, j, k) - velx(i, j - 1, k)) / dx[1];
                    double v_x = (vely(i, j, k) - vely(i - 1, j, k)) / dx[0];
                    double ei = 0.25 * (eta(i - 1, j - 1, k) + eta(i - 1, j, k) + eta(i, j - 1, k) + eta(i, j, k));
                    tauxy(i, j, k) = ei * (u_y + v_x);
                }
                if (j < N[1]) {
                    double u_z = (velx(i, j, k) - velx(i, j, k - 1)) / dx[2];
                    double w_x = (velz(i, j, k) - velz(i - 1, j, k)) / dx[0];
                    double ei = 0.25 * (eta(i - 1, j, k - 1) + eta(i - 1, j, k) + eta(i, j, k - 1) + eta(i, j, k));
                    tauxz(i, j, k) = ei * (u_z + w_x);
                }
                if (i < N[0]) {
                    double v_z = (vely(i, j, k) - vely(i, j, k - 1)) / dx[2];
                    double w_y = (velz(i, j, k) - velz(i, j - 1, k)) / dx[1];
                    double ei = 0.25 * (eta(i, j - 1, k - 1) + eta(i, j - 1, k) + eta(i, j, k - 1) + eta(i, j, k));
                    tauyz(i, j, k) = ei * (v_z + w_y);
                }
            }
    // :1026-1426 diffusive face fluxes
    for (int d = 0; d < 3; ++d) {
        const Fab& fl = ff[d];
        const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
        const double h = dx[d];
        #pragma omp parallel for collapse(2) schedule(static)
        for (int k = 0; k < N[2] + e2; ++k)
            for (int j = 0; j < N[1] + e1; ++j)
                for (int i = 0; i < N[0] + e0; ++i) {
                    const int im = i - e0, jm = j - e1, km = k - e2;
                    double vsh = 0.0;
                    if (d == 0) {
                        fl(i, j, k, nvars + 1) -= 0.5 * velx(i, j, k) * (tauxx(i - 1, j, k) + tauxx(i, j, k));
                        vsh -= 0.25 * ((vely(i, j + 1, k) + vely(i - 1, j + 1, k)) * tauxy(i, j + 1, k) +
                                       (vely(i, j, k) + vely(i - 1, j, k)) * tauxy(i, j, k));
                        vsh -= 0.25 * ((velz(i, j, k + 1) + velz(i - 1, j, k + 1)) * tauxz(i, j, k + 1) +
                                       (velz(i, j, k) + velz(i - 1, j, k)) * tauxz(i, j, k));
                    } else if (d == 1) {
                        fl(i, j, k, nvars + 1) -= 0.5 * vely(i, j, k) * (tauyy(i, j - 1, k) + tauyy(i, j, k));
                        vsh -= 0.25 * ((velx(i + 1, j, k) + velx(i + 1, j - 1, k)) * tauxy(i + 1, j, k) +
                                       (velx(i, j, k) + velx(i, j - 1, k)) * tauxy(i, j, k));
                        vsh -= 0.25 * ((velz(i, j, k + 1) + velz(i, j - 1, k + 1)) * tauyz(i, j, k + 1) +
                                       (velz(i, j, k) + velz(i, j - 1, k)) * tauyz(i, j, k));
                    } else {
                        fl(i, j, k, nvars + 1) -= 0.5 * velz(i, j, k) * (tauzz(i, j, k - 1) + tauzz(i, j, k));
                        vsh -= 0.25 * ((velx(i + 1, j, k - 1) + velx(i + 1, j, k)) * tauxz(i + 1, j, k) +
                                       (velx(i, j, k) + velx(i, j, k - 1)) * tauxz(i, j, k));
                        vsh -= 0.25 * ((vely(i, j + 1, k - 1) + vely(i, j + 1, k)) * tauyz(i, j + 1, k) +
                                       (vely(i, j, k) + vely(i, j, k - 1)) * tauyz(i, j, k));
                    }
                    fl(i, j, k, nvars + 2) += vsh;
                    const double kp = 0.5 * (kappa(im, jm, km) + kappa(i, j, k));
                    const double meanT = 0.5 * (prim(im, jm, km, 4) + prim(i, j, k, 4));
                    const double meanP = 0.5 * (prim(im, jm, km, 5) + prim(i, j, k, 5));
                    fl(i, j, k, nvars) -= kp * (prim(i, j, k, 4) - prim(im, jm, km, 4)) / h;
                    double meanXk[MAXS], meanYk[MAXS], dk[MAXS], Fk[MAXS], hk[MAXS], soret[MAXS];
                    for (int s = 0; s < ns; ++s) {
                        double term1 = (prim(i, j, k, 6 + ns + s) - prim(im, jm, km, 6 + ns + s)) / h;
                        meanXk[s] = 0.5 * (prim(im, jm, km, 6 + ns + s) + prim(i, j, k, 6 + ns + s));
                        meanYk[s] = 0.5 * (prim(im, jm, km, 6 + s) + prim(i, j, k, 6 + s));
                        double term2 = (meanXk[s] - meanYk[s]) * (prim(i, j, k, 5) - prim(im, jm, km, 5)) / h / meanP;
                        dk[s] = term1 + term2;
                        double ChiX = 0.5 * (chi(im, jm, km, s) * prim(im, jm, km, 6 + ns + s) +
                                             chi(i, j, k, s) * prim(i, j, k, 6 + ns + s));
                        soret[s] = ChiX * (prim(i, j, k, 4) - prim(im, jm, km, 4)) / h / meanT;
                    }
                    for (int kk = 0; kk < ns; ++kk) {
                        Fk[kk] = 0.;
                        for (int ll = 0; ll < ns; ++ll) {
                            double Fks = 0.5 * (Dij(im, jm, km, ll * ns + kk) + Dij(i, j, k, ll * ns + kk)) *
                                         (dk[ll] + soret[ll]);
                            Fk[kk] -= Fks;
                        }
                    }
                    GetEnthalpies(meanT, hk);
                    double Q5 = 0.;
                    for (int s = 0; s < ns; ++s) {
                        // z faces: chi(i,j,k)+chi(i,j,k) as at fluxStag.cpp:1407 (reference quirk)
                        const double chs = (d == 2) ? (chi(i, j, k, s) + chi(i, j, k, s))
                                                    : (chi(im, jm, km, s) + chi(i, j, k, s));
                        double Q5s = (hk[s] + 0.5 * Runiv * meanT * chs / g.molmass[s]) * Fk[s];
                        Q5 += Q5s;
                    }
                    fl(i, j, k, nvars + 3) += Q5;
                    for (int s = 0; s < ns; ++s) fl(i, j, k, 5 + s) += Fk[s];
                }
    }
    // :1429-1448 momentum fluxes -= deterministic stresses
    for (int k = 0; k <= N[2]; ++k)
        for (int j = 0; j <= N[1]; ++j)
            for (int i = 0; i <= N[0]; ++i) {
                if (k < N[2]) { edgey_u(i, j, k) -= tauxy(i, j, k); edgex_v(i, j, k) -= tauxy(i, j, k); }
                if (j < N[1]) { edgez_u(i, j, k) -= tauxz(i, j, k); edgex_w(i, j, k) -= tauxz(i, j, k); }
                if (i < N[0]) { edgez_v(i, j, k) -= tauyz(i, j, k); edgey_w(i, j, k) -= tauyz(i, j, k); }
            }
    for (int k = -1; k <= N[2]; ++k)
        for (int j = -1; j <= N[1]; ++j)
            for (int i = -1; i <= N[0]; ++i) {
                cenx_u(i, j, k) -= tauxx(i, j, k);
                ceny_v(i, j, k) -= tauyy(i, j, k);
                cenz_w(i, j, k) -= tauzz(i, j, k);
            }

    // ---- hyperbolic fluxes :1459-1866 ----
    const int adv = g.advection_type;
    for (int d = 0; d < 3; ++d) {
        const Fab& fl = ff[d];
        const Fab& md = mom[d];
        const Fab& vd = vel[d];
        const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
        #pragma omp parallel for collapse(2) schedule(static)
        for (int k = 0; k < N[2] + e2; ++k)
            for (int j = 0; j < N[1] + e1; ++j)
                for (int i = 0; i < N[0] + e0; ++i) {
                    const int im = i - e0, jm = j - e1, km = k - e2;
                    if (adv >= 0) {
                        fl(i, j, k, 0) += md(i, j, k);
                        double meanT = 0.5 * (prim(im, jm, km, 4) + prim(i, j, k, 4));
                        double meanRho = 0.5 * (prim(im, jm, km, 0) + prim(i, j, k, 0));
                        double meanP = 0.5 * (prim(im, jm, km, 5) + prim(i, j, k, 5));
                        double hk[MAXS];
                        GetEnthalpies(meanT, hk);
                        double meanE = 0.5 * (cons(im, jm, km, 4) + cons(i, j, k, 4)) / meanRho;
                        if (adv == 1) {
                            fl(i, j, k, 4) += md(i, j, k) * (meanE + (meanP / meanRho));
                        } else if (adv == 2) {
                            fl(i, j, k, 4) += 0.5 * (cons(im, jm, km, 4) + cons(i, j, k, 4)) * vd(i, j, k) +
                                              0.5 * (prim(im, jm, km, 5) + prim(i, j, k, 5)) * vd(i, j, k);
                        }
                        for (int n = 0; n < ns; ++n) {
                            double Yk = 0.5 * (prim(im, jm, km, 6 + n) + prim(i, j, k, 6 + n));
                            if (adv == 0 || adv == 1) fl(i, j, k, 5 + n) += Yk * md(i, j, k);
                            else if (adv == 2)
                                fl(i, j, k, 5 + n) += 0.5 * (cons(im, jm, km, 5 + n) + cons(i, j, k, 5 + n)) * vd(i, j, k);
                            if (adv == 0) fl(i, j, k, 4) += md(i, j, k) * Yk * hk[n];
                        }
                        if (adv == 0) {
                            double keP = 0., keM = 0.;
                            keP += (momx(i + 1, j, k) + momx(i, j, k)) * (momx(i + 1, j, k) + momx(i, j, k));
                            keP += (momy(i, j + 1, k) + momy(i, j, k)) * (momy(i, j + 1, k) + momy(i, j, k));
                            keP += (momz(i, j, k + 1) + momz(i, j, k)) * (momz(i, j, k + 1) + momz(i, j, k));
                            keP *= (0.125 / cons(i, j, k, 0) / cons(i, j, k, 0));
                            keM += (momx(im + 1, jm, km) + momx(im, jm, km)) * (momx(im + 1, jm, km) + momx(im, jm, km));
                            keM += (momy(im, jm + 1, km) + momy(im, jm, km)) * (momy(im, jm + 1, km) + momy(im, jm, km));
                            keM += (momz(im, jm, km + 1) + momz(im, jm, km)) * (momz(im, jm, km + 1) + momz(im, jm, km));
                            // z faces divide by cons(i,j-1,k,0), fluxStag.cpp:1755 (reference quirk)
                            double rm = (d == 2) ? cons(i, j - 1, k, 0) : cons(im, jm, km, 0);
                            keM *= (0.125 / rm / rm);
                            fl(i, j, k, 4) += md(i, j, k) * 0.5 * (keP + keM);
                        }
                    }
                    fl(i, j, k, 4) += fl(i, j, k, nvars) + fl(i, j, k, nvars + 1) + fl(i, j, k, nvars + 2) +
                                      fl(i, j, k, nvars + 3);
                }
    }
    // :1767-1845 advective momentum fluxes on edges
    if (adv >= 0) {
        #pragma omp parallel for collapse(2) schedule(static)
        for (int k = 0; k <= N[2]; ++k)
            for (int j = 0; j <= N[1]; ++j)
                for (int i = 0; i <= N[0]; ++i) {
                    if (k < N[2]) {
                        double y_u = 0.25 * (momx(i, j - 1, k) + momx(i, j, k)) * (vely(i - 1, j, k) + vely(i, j, k));
                        double x_v = 0.25 * (momy(i - 1, j, k) + momy(i, j, k)) * (velx(i, j - 1, k) + velx(i, j, k));
                        edgey_u(i, j, k) += y_u;
                        edgex_v(i, j, k) += x_v;
                    }
                    if (j < N[1]) {
                        double z_u = 0.25 * (momx(i, j, k - 1) + momx(i, j, k)) * (velz(i - 1, j, k) + velz(i, j, k));
                        double x_w = 0.25 * (momz(i - 1, j, k) + momz(i, j, k)) * (velx(i, j, k - 1) + velx(i, j, k));
                        edgez_u(i, j, k) += z_u;
                        edgex_w(i, j, k) += x_w;
                    }
                    if (i < N[0]) {
                        double z_v = 0.25 * (momy(i, j, k - 1) + momy(i, j, k)) * (velz(i, j - 1, k) + velz(i, j, k));
                        double y_w = 0.25 * (momz(i, j - 1, k) + momz(i, j, k)) * (vely(i, j, k - 1) + vely(i, j, k));
                        edgez_v(i, j, k) += z_v;
                        edgey_w(i, j, k) += y_w;
                    }
                }
        // :1848-1866 advective centre momentum fluxes + pressure
        #pragma omp parallel for collapse(2) schedule(static)
        for (int k = -1; k <= N[2]; ++k)
            for (int j = -1; j <= N[1]; ++j)
                for (int i = -1; i <= N[0]; ++i) {
                    cenx_u(i, j, k) += 0.25 * (momx(i, j, k) + momx(i + 1, j, k)) * (velx(i, j, k) + velx(i + 1, j, k)) + prim(i, j, k, 5);
                    ceny_v(i, j, k) += 0.25 * (momy(i, j, k) + momy(i, j + 1, k)) * (vely(i, j, k) + vely(i, j + 1, k)) + prim(i, j, k, 5);
                    cenz_w(i, j, k) += 0.25 * (momz(i, j, k) + momz(i, j, k + 1)) * (velz(i, j, k) + velz(i, j, k + 1)) + prim(i, j, k, 5);
                }
    }
}

// MultiFab::LinComb(dst, a, x, xc, b, y, yc, dc, nc, ng): dst = a*x + b*y
void lincomb(const Fab& dst, double a, const Fab& x, int xc, double b, const Fab& y, int yc, int dc,
             int nc, int ng) {
    const int* N = g.n;
    for (int n = 0; n < nc; ++n)
        for (int k = -ng; k <= N[2] - 1 + dst.nodal[2] + ng; ++k)
            for (int j = -ng; j <= N[1] - 1 + dst.nodal[1] + ng; ++j)
                for (int i = -ng; i <= N[0] - 1 + dst.nodal[0] + ng; ++i)
                    dst(i, j, k, dc + n) = a * x(i, j, k, xc + n) + b * y(i, j, k, yc + n);
}

// compute_compressible_chemistry_source_CLE, chemistry_functions.cpp:128-193: per
// valid cell, the law-of-mass-action rates and (reaction_type 1) their Langevin
// terms into source comps 5..5+ns-1
void chem_source_cle(double dt, double dV, const Fab& prim, const Fab& source, const Fab& ranchem) {
    const int* N = g.n;
    const int ns = g.ns, nr = g.nreaction;
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < N[2]; ++k)
        for (int j = 0; j < N[1]; ++j)
            for (int i = 0; i < N[0]; ++i) {
                double pres = prim(i, j, k, 5);
                double T = prim(i, j, k, 4);
                double T0 = g.T0_chem;
                double ctot = pres / g.Runiv / T;
                double Navo = g.avogadro;
                double ck[MAXS];
                for (int n = 0; n < ns; n++) ck[n] = prim(i, j, k, 6 + ns + n) * ctot;
                double avg_react_rate[FHD_MAX_REACTIONS];
                for (int m = 0; m < nr; m++) {
                    avg_react_rate[m] = g.rate_const[m];
                    avg_react_rate[m] *= std::exp(-g.alpha_param[m] / g.Runiv * (1 / T - 1 / T0));
                    avg_react_rate[m] *= std::pow(T / T0, g.beta_param[m]);
                    for (int n = 0; n < ns; n++) avg_react_rate[m] *= std::pow(ck[n], g.stoich_R[m][n]);
                }
                double sourceArr[MAXS];
                for (int n = 0; n < ns; n++) sourceArr[n] = 0.;
                for (int m = 0; m < nr; m++) {
                    avg_react_rate[m] = std::max(0., avg_react_rate[m]);
                    double W = (g.reaction_type == 1 ? ranchem(i, j, k, m) : 0.0) / std::sqrt(dt * dV);
                    for (int n = 0; n < ns; n++) {
                        sourceArr[n] += g.molmass[n] * g.stoich_PR[m][n] * avg_react_rate[m];
                        if (g.reaction_type == 1)
                            sourceArr[n] += g.molmass[n] * g.stoich_PR[m][n] * std::sqrt(avg_react_rate[m] / Navo) * W;
                    }
                }
                for (int n = 0; n < ns; n++) source(i, j, k, 5 + n) = sourceArr[n];
            }
}

// The RK3 stage update of cons and face momenta, timeStepStag.cpp:439-528 (stage 1),
// :771-861 (stage 2), :1106-1202 (stage 3).
void stage_update(int stage, const Fab& cu, const Fab mom[3], const Fab& cin, const Fab min_[3],
                  const Fab& cout, const Fab mout[3], const Fab& source, const Fab ff[3],
                  const Fab ef[6], const Fab cf[3], double dt) {
    const int* N = g.n;
    const double* dx = g.dx;
    const double* grav = g.grav;
    const int nvars = g.nvars;
    const Fab &xf = ff[0], &yf = ff[1], &zf = ff[2];
    const Fab &edgex_v = ef[0], &edgex_w = ef[1], &edgey_u = ef[2], &edgey_w = ef[3], &edgez_u = ef[4],
              &edgez_v = ef[5];
    const Fab &cenx_u = cf[0], &ceny_v = cf[1], &cenz_w = cf[2];
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < N[2]; ++k)
        for (int j = 0; j < N[1]; ++j)
            for (int i = 0; i < N[0]; ++i)
                for (int n = 0; n < nvars; ++n) {
                    double div = (xf(i + 1, j, k, n) - xf(i, j, k, n)) / dx[0] +
                                 (yf(i, j + 1, k, n) - yf(i, j, k, n)) / dx[1] +
                                 (zf(i, j, k + 1, n) - zf(i, j, k, n)) / dx[2];
                    double src = source.p ? source(i, j, k, n) : 0.0;
                    if (stage == 1)
                        cout(i, j, k, n) = cu(i, j, k, n) - dt * (div) + dt * src;
                    else if (stage == 2)
                        cout(i, j, k, n) = 0.25 * (3.0 * cu(i, j, k, n) + cin(i, j, k, n) - dt * (div) + dt * src);
                    else
                        cout(i, j, k, n) = (2. / 3.) * (0.5 * cu(i, j, k, n) + cin(i, j, k, n) - dt * (div) + dt * src);
                }
    // face momenta: tbx/tby/tbz (valid faces)
    for (int d = 0; d < 3; ++d) {
        const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
        const Fab& m0 = mom[d];
        const Fab& mi = min_[d];
        const Fab& mo = mout[d];
        // density used in the gravity term: cu (stage 1), cup (stage 2), cup2 (stage 3)
        const Fab& rho = (stage == 1) ? cu : cin;
        #pragma omp parallel for collapse(2) schedule(static)
        for (int k = 0; k < N[2] + e2; ++k)
            for (int j = 0; j < N[1] + e1; ++j)
                for (int i = 0; i < N[0] + e0; ++i) {
                    double t1, t2, t3;  // the three flux differences
                    if (d == 0) {
                        t1 = cenx_u(i, j, k) - cenx_u(i - 1, j, k);
                        t2 = edgey_u(i, j + 1, k) - edgey_u(i, j, k);
                        t3 = edgez_u(i, j, k + 1) - edgez_u(i, j, k);
                    } else if (d == 1) {
                        t1 = edgex_v(i + 1, j, k) - edgex_v(i, j, k);
                        t2 = ceny_v(i, j, k) - ceny_v(i, j - 1, k);
                        t3 = edgez_v(i, j, k + 1) - edgez_v(i, j, k);
                    } else {
                        t1 = edgex_w(i + 1, j, k) - edgex_w(i, j, k);
                        t2 = edgey_w(i, j + 1, k) - edgey_w(i, j, k);
                        t3 = cenz_w(i, j, k) - cenz_w(i, j, k - 1);
                    }
                    const double rsum = rho(i - e0, j - e1, k - e2, 0) + rho(i, j, k, 0);
                    if (stage == 1) {
                        mo(i, j, k) = m0(i, j, k) - dt * t1 / dx[0] - dt * t2 / dx[1] - dt * t3 / dx[2] +
                                      0.5 * dt * grav[d] * rsum;
                    } else if (stage == 2) {
                        mo(i, j, k) = 0.25 * 3.0 * m0(i, j, k) + 0.25 * mi(i, j, k) - 0.25 * dt * t1 / dx[0] -
                                      0.25 * dt * t2 / dx[1] - 0.25 * dt * t3 / dx[2] +
                                      0.5 * 0.25 * dt * grav[d] * rsum;
                    } else {
                        mo(i, j, k) = (2. / 3.) * (0.5 * m0(i, j, k) + mi(i, j, k)) - (2. / 3.) * dt * t1 / dx[0] -
                                      (2. / 3.) * dt * t2 / dx[1] - (2. / 3.) * dt * t3 / dx[2] +
                                      0.5 * (2. / 3.) * dt * grav[d] * rsum;
                    }
                }
    }
    // gravity work on the energy, :508-528 / :841-861 / :1181-1202 (momenta of the
    // stage input: cumom, cupmom, cup2mom)
    const Fab* mg = (stage == 1) ? mom : min_;
    const double fac = (stage == 1) ? 0.5 * dt : (stage == 2) ? 0.5 * 0.25 * dt : 0.5 * (2. / 3.) * dt;
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < N[2]; ++k)
        for (int j = 0; j < N[1]; ++j)
            for (int i = 0; i < N[0]; ++i)
                cout(i, j, k, 4) += fac * (grav[0] * (mg[0](i + 1, j, k) + mg[0](i, j, k)) +
                                           grav[1] * (mg[1](i, j + 1, k) + mg[1](i, j, k)) +
                                           grav[2] * (mg[2](i, j, k + 1) + mg[2](i, j, k)));
}


}  // namespace

// =============================== C API ===========================================
extern "C" {

int orc_set_params(const fhd_params* p) {
    if (!p || p->nspecies < 1 || p->nspecies > MAXS) return FHD_ERR_BAD_ARG;
    // the quasi-1-D / 2-D runs are held to the reference's own code (oracle/_ref), not restated here
    if (p->do_1D || p->do_2D) return FHD_ERR_UNSUPPORTED;
    g.ns = p->nspecies;
    g.nvars = 5 + g.ns;
    g.nprimvars = 6 + 2 * g.ns;
    for (int d = 0; d < 3; ++d) {
        g.n[d] = p->n_cells[d];
        g.dx[d] = (p->prob_hi[d] - p->prob_lo[d]) / p->n_cells[d];
        g.cross_cell = p->cross_cell;
        g.grav[d] = p->grav[d];
    }
    g.k_B = p->k_B;
    g.Runiv = p->Runiv;
    for (int i = 0; i < MAXS; ++i) {
        g.molmass[i] = p->molmass[i];
        g.diameter[i] = p->diameter[i];
        g.dof[i] = p->dof[i];
        g.e0[i] = p->e0[i];
        g.hcv[i] = p->hcv[i];
        g.hcp[i] = p->hcp[i];
    }
    // GetHcGas, compressible_functions.cpp:91-100
    for (int i = 0; i < g.ns; ++i) {
        if (g.hcv[i] < 0.) g.hcv[i] = 0.5 * g.dof[i] * g.Runiv / g.molmass[i];
        if (g.hcp[i] < 0.) g.hcp[i] = 0.5 * (2. + g.dof[i]) * g.Runiv / g.molmass[i];
    }
    g.visc_type = p->visc_type;
    g.advection_type = p->advection_type;
    g.algorithm_type = p->algorithm_type;
    g.stoch_stress_form = p->stoch_stress_form;
    g.zeta_ratio = p->zeta_ratio;
    if (g.algorithm_type != 2 || p->transport_type != 1) return FHD_ERR_UNSUPPORTED;
    // chemistry_functions.cpp:45-124; avogadro = Runiv / k_B unless given (common_functions.cpp:775)
    if (p->nreaction < 0 || p->nreaction > FHD_MAX_REACTIONS) return FHD_ERR_BAD_ARG;
    g.nreaction = p->nreaction;
    g.reaction_type = p->reaction_type;
    if (g.nreaction > 0 && g.reaction_type != 0 && g.reaction_type != 1) return FHD_ERR_UNSUPPORTED;
    if (g.nreaction > 0 && !(p->T0_chem > 0.)) return FHD_ERR_BAD_ARG;
    for (int m = 0; m < FHD_MAX_REACTIONS; ++m) {
        for (int n = 0; n < MAXS; ++n) {
            g.stoich_R[m][n] = p->stoich_R[m][n];
            g.stoich_PR[m][n] = p->stoich_P[m][n] - p->stoich_R[m][n];
        }
        g.rate_const[m] = p->rate_const[m];
        g.alpha_param[m] = p->alpha_param[m];
        g.beta_param[m] = p->beta_param[m];
    }
    g.T0_chem = p->T0_chem;
    g.avogadro = p->avogadro > 0 ? p->avogadro : g.Runiv / g.k_B;
    return FHD_OK;
}

int orc_get_hc(double* hcv, double* hcp) {
    for (int i = 0; i < g.ns; ++i) { hcv[i] = g.hcv[i]; hcp[i] = g.hcp[i]; }
    return FHD_OK;
}

int orc_take_status() { int s = g_status; g_status = 0; return s; }

// OpenMP thread count of the oracle's parallel loops (<= 0: all host cores);
// returns the count in effect.  Lets the CPU baseline be timed at 1 thread and
// at all cores.
int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n <= 0) n = omp_get_num_procs();
    omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int orc_fill_boundary(fhd_fab f) { fill_boundary(Fab(f)); return FHD_OK; }
int orc_override_sync(fhd_fab f) { override_sync(Fab(f)); return FHD_OK; }

// InitConsVarStag, prob_type 1: compressible_functions_stag.cpp:36-56
int orc_init_cons_var_stag(fhd_fab cu_, const fhd_fab* mom_, double rho0, double T_init,
                           const double* rhobar) {
    Fab cu(cu_);
    double intEnergy, massvec[MAXS];
    for (int i = 0; i < g.ns; ++i) massvec[i] = rhobar[i];
    GetEnergy(intEnergy, massvec, T_init);
    std::fill(cu.p, cu.p + cu.sn * cu.nc, 0.0);
    for (long q = 0; q < cu.sn; ++q) {
        cu.p[q] = rho0;
        cu.p[q + 1 * cu.sn] = 0;
        cu.p[q + 2 * cu.sn] = 0;
        cu.p[q + 3 * cu.sn] = 0;
        cu.p[q + 4 * cu.sn] = rho0 * intEnergy;
        for (int i = 0; i < g.ns; ++i) cu.p[q + (5 + i) * cu.sn] = rho0 * rhobar[i];
    }
    for (int d = 0; d < 3; ++d) {
        Fab m(mom_[d]);
        std::fill(m.p, m.p + m.sn * m.nc, 0.0);
    }
    return FHD_OK;
}

int orc_conserved_to_primitive_stag(fhd_fab prim, const fhd_fab* vel, fhd_fab cu, const fhd_fab* mom) {
    Fab v[3] = {Fab(vel[0]), Fab(vel[1]), Fab(vel[2])};
    Fab m[3] = {Fab(mom[0]), Fab(mom[1]), Fab(mom[2])};
    conserved_to_primitive(Fab(prim), v, Fab(cu), m);
    return orc_take_status();
}

int orc_transport_coeffs(fhd_fab prim, fhd_fab eta, fhd_fab zeta, fhd_fab kappa, fhd_fab chi, fhd_fab D) {
    transport_coeffs(Fab(prim), Fab(eta), Fab(zeta), Fab(kappa), Fab(chi), Fab(D));
    return orc_take_status();
}

int orc_chemistry_source_cle(double dt, double dV, fhd_fab prim, fhd_fab source, fhd_fab ranchem) {
    if (g.nreaction < 1 || !prim.data || !source.data) return FHD_ERR_BAD_ARG;
    if (g.reaction_type == 1 && !ranchem.data) return FHD_ERR_BAD_ARG;
    Fab r;
    if (ranchem.data) r = Fab(ranchem);
    chem_source_cle(dt, dV, Fab(prim), Fab(source), r);
    return FHD_OK;
}

int orc_flux_stag(fhd_fab cu, const fhd_fab* mom, fhd_fab prim, const fhd_fab* vel, fhd_fab eta,
                  fhd_fab zeta, fhd_fab kappa, fhd_fab chi, fhd_fab D, const fhd_fab* faceflux,
                  const fhd_fab* edgeflux, const fhd_fab* cenflux, const fhd_fab* stochface,
                  const fhd_fab* stochedge, const fhd_fab* stochcen, double dt) {
    Fab m[3], v[3], ff[3], cf[3], sf[3], se[3], sc[3], ef[6];
    for (int d = 0; d < 3; ++d) {
        m[d] = Fab(mom[d]); v[d] = Fab(vel[d]); ff[d] = Fab(faceflux[d]); cf[d] = Fab(cenflux[d]);
        sf[d] = Fab(stochface[d]); se[d] = Fab(stochedge[d]); sc[d] = Fab(stochcen[d]);
    }
    for (int e = 0; e < 6; ++e) ef[e] = Fab(edgeflux[e]);
    flux_stag(Fab(cu), m, Fab(prim), v, Fab(eta), Fab(zeta), Fab(kappa), Fab(chi), Fab(D), ff, ef, cf, sf, se,
              sc, dt);
    return FHD_OK;
}

// RK3stepStag, timeStepStag.cpp:13-1245, with the A/B noise fields injected.
// fluxes/coefficients: caller-owned (they hold stage-3 values on return, as in the
// reference).  noise: A/B fields as documented for fhd_noise.
int orc_rk3_step_stag(fhd_fab cu_, const fhd_fab* mom_, fhd_fab prim_, const fhd_fab* vel_,
                      fhd_fab source_, fhd_fab eta_, fhd_fab zeta_, fhd_fab kappa_, fhd_fab chi_,
                      fhd_fab D_, const fhd_fab* faceflux, const fhd_fab* edgeflux, const fhd_fab* cenflux,
                      const fhd_noise* noise, double dt) {
    const int* N = g.n;
    const int nvars = g.nvars, ns = g.ns;
    Fab cu(cu_), prim(prim_), eta(eta_), zeta(zeta_), kappa(kappa_), chi(chi_), D(D_);
    Fab source;
    if (source_.data) source = Fab(source_);
    // the reference's driver always passes a (zeroed) source; chemistry writes into it
    OwnedFab own_source(N[0], N[1], N[2], kCellNodal, 0, g.nreaction > 0 && !source_.data ? nvars : 1);
    if (g.nreaction > 0 && !source_.data) source = own_source.f;
    // ranchem = 1.0*ranchem_A + w*ranchem_B per stage (timeStepStag.cpp:354-361)
    const bool cle = g.nreaction > 0 && g.reaction_type == 1;
    if (cle && (!noise || !noise->chem[0].data || !noise->chem[1].data)) return FHD_ERR_BAD_ARG;
    OwnedFab ranchem(N[0], N[1], N[2], kCellNodal, 0, cle ? g.nreaction : 1);
    Fab mom[3], vel[3], ff[3], cf[3], ef[6];
    for (int d = 0; d < 3; ++d) {
        mom[d] = Fab(mom_[d]); vel[d] = Fab(vel_[d]); ff[d] = Fab(faceflux[d]); cf[d] = Fab(cenflux[d]);
    }
    for (int e = 0; e < 6; ++e) ef[e] = Fab(edgeflux[e]);
    const int ngc = cu.ngrow();
    const int cn[3] = {0, 0, 0};
    const int fn[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    const int en[3][3] = {{1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
    // :30-62 stage temporaries, zeroed
    OwnedFab cup(N[0], N[1], N[2], cn, ngc, nvars), cup2(N[0], N[1], N[2], cn, ngc, nvars);
    OwnedFab cupm0(N[0], N[1], N[2], fn[0], ngc, 1), cupm1(N[0], N[1], N[2], fn[1], ngc, 1),
        cupm2(N[0], N[1], N[2], fn[2], ngc, 1);
    OwnedFab cup2m0(N[0], N[1], N[2], fn[0], ngc, 1), cup2m1(N[0], N[1], N[2], fn[1], ngc, 1),
        cup2m2(N[0], N[1], N[2], fn[2], ngc, 1);
    Fab cupmom[3] = {cupm0.f, cupm1.f, cupm2.f};
    Fab cup2mom[3] = {cup2m0.f, cup2m1.f, cup2m2.f};
    // :68-89 combined noise fields: faces nvars comps (0 ghosts), edges, centres (1 ghost)
    OwnedFab sf0(N[0], N[1], N[2], fn[0], 0, ns + 1), sf1(N[0], N[1], N[2], fn[1], 0, ns + 1),
        sf2(N[0], N[1], N[2], fn[2], 0, ns + 1);
    OwnedFab se0(N[0], N[1], N[2], en[0], 0, 1), se1(N[0], N[1], N[2], en[1], 0, 1),
        se2(N[0], N[1], N[2], en[2], 0, 1);
    OwnedFab sc0(N[0], N[1], N[2], cn, 1, 1), sc1(N[0], N[1], N[2], cn, 1, 1), sc2(N[0], N[1], N[2], cn, 1, 1);
    Fab sf[3] = {sf0.f, sf1.f, sf2.f}, se[3] = {se0.f, se1.f, se2.f}, sc[3] = {sc0.f, sc1.f, sc2.f};

    const double swgt1 = 1.0;
    const double w[3] = {(2.0 * std::sqrt(2.0) + 1.0 * std::sqrt(3.0)) / 5.0,
                         (-4.0 * std::sqrt(2.0) + 3.0 * std::sqrt(3.0)) / 5.0,
                         (1.0 * std::sqrt(2.0) - 2.0 * std::sqrt(3.0)) / 10.0};

    auto weigh_noise = [&](double w2) {
        if (g.stoch_stress_form != 1 || !noise) return;
        for (int d = 0; d < 3; ++d) {
            Fab A(noise->face[0][d]), B(noise->face[1][d]);
            int oa = A.nc - (ns + 1), ob = B.nc - (ns + 1);
            lincomb(sf[d], swgt1, A, oa, w2, B, ob, 0, ns + 1, 0);
            lincomb(se[d], swgt1, Fab(noise->edge[0][d]), 0, w2, Fab(noise->edge[1][d]), 0, 0, 1, 0);
            lincomb(sc[d], swgt1, Fab(noise->cen[0][d]), 0, w2, Fab(noise->cen[1][d]), 0, 0, 1, 1);
        }
    };

    const Fab* cins[3] = {&cu, &cup.f, &cup2.f};
    const Fab* mins[3] = {mom, cupmom, cup2mom};
    const Fab* couts[3] = {&cup.f, &cup2.f, &cu};
    const Fab* mouts[3] = {cupmom, cup2mom, mom};
    for (int s = 0; s < 3; ++s) {
        transport_coeffs(prim, eta, zeta, kappa, chi, D);
        weigh_noise(w[s]);
        flux_stag(*cins[s], mins[s], prim, vel, eta, zeta, kappa, chi, D, ff, ef, cf, sf, se, sc, dt);
        if (g.nreaction > 0) {
            if (cle) lincomb(ranchem.f, swgt1, Fab(noise->chem[0]), 0, w[s], Fab(noise->chem[1]), 0, 0, g.nreaction, 0);
            chem_source_cle(dt, g.dx[0] * g.dx[1] * g.dx[2], prim, source, ranchem.f);
        }
        stage_update(s + 1, cu, mom, *cins[s], mins[s], *couts[s], mouts[s], source, ff, ef, cf, dt);
        for (int d = 0; d < 3; ++d) fill_boundary(mouts[s][d]);
        fill_boundary(*couts[s]);
        conserved_to_primitive(prim, vel, *couts[s], mouts[s]);
        for (int d = 0; d < 3; ++d) fill_boundary(vel[d]);
        fill_boundary(prim);
        fill_boundary(*couts[s]);
    }
    return orc_take_status();
}

// Standard normals for the self-contained oracle runs: Philox-4x32-10 (Salmon et
// al., SC'11) counters + Box-Muller in FP64.  Statistics only; the in-kernel GPU
// noise is a different transform and is compared through injection.
static inline void philox_round(uint32_t c[4], const uint32_t k[2]) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t r0 = hi1 ^ c[1] ^ k[0];
    uint32_t r1 = lo1;
    uint32_t r2 = hi0 ^ c[3] ^ k[1];
    uint32_t r3 = lo0;
    c[0] = r0; c[1] = r1; c[2] = r2; c[3] = r3;
}
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    uint32_t k[2] = {key[0], key[1]};
    for (int r = 0; r < 10; ++r) {
        if (r > 0) { k[0] += 0x9E3779B9u; k[1] += 0xBB67AE85u; }
        philox_round(c, k);
    }
    for (int i = 0; i < 4; ++i) out[i] = c[i];
}

// MultiFabFillRandomNormal (MultiFabFillRandom.cpp:34-50) for the oracle's own
// runs: normals(mean, sqrt(variance)) on the valid region, then OverrideSync and
// FillBoundary.
int orc_fill_random_normal(fhd_fab mf_, int scomp, int ncomp, double mean, double variance,
                           uint64_t seed, uint64_t stream_id) {
    Fab mf(mf_);
    const int* N = g.n;
    const double sd = std::sqrt(variance);
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    const int nx = N[0] + mf.nodal[0], ny = N[1] + mf.nodal[1], nz = N[2] + mf.nodal[2];
    #pragma omp parallel for collapse(2) schedule(static)
    for (int n = 0; n < ncomp; ++n)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; i += 2) {
                    uint32_t ctr[4] = {(uint32_t)(i + nx * (j + ny * k)), (uint32_t)n, (uint32_t)stream_id,
                                       (uint32_t)(stream_id >> 32)};
                    uint32_t o[4];
                    orc_philox4x32_10(ctr, key, o);
                    // 53-bit uniforms in (0,1]
                    double u1 = ((double)(((uint64_t)o[0] << 21) ^ (o[1] >> 11)) + 1.0) * (1.0 / 9007199254740992.0);
                    double u2 = ((double)(((uint64_t)o[2] << 21) ^ (o[3] >> 11)) + 0.5) * (1.0 / 9007199254740992.0);
                    double r = std::sqrt(-2.0 * std::log(u1));
                    double z0 = r * std::cos(2.0 * 3.14159265358979323846 * u2);
                    double z1 = r * std::sin(2.0 * 3.14159265358979323846 * u2);
                    mf(i, j, k, scomp + n) = mean + sd * z0;
                    if (i + 1 < nx) mf(i + 1, j, k, scomp + n) = mean + sd * z1;
                }
    override_sync(mf);
    fill_boundary(mf);
    return FHD_OK;
}

// sumToLine(mf, icomp, ncomp, domain, 0): for every x index i and component n the
// sum of mf(i, j, k, icomp + n) over the y-z plane, from 0.0 with k outer and j
// inner (a serial one-box AMReX sumToLine), in entry i*ncomp + n, then divided by
// n_cells[1]*n_cells[2] as evaluateStatsStag3D does (statsStag.cpp:56-69).
static std::vector<double> line_average(const Fab& f, int icomp, int ncomp) {
    const int* N = g.n;
    std::vector<double> hv((size_t)N[0] * ncomp, 0.0);
    for (int n = 0; n < ncomp; ++n)
        for (int k = 0; k < N[2]; ++k)
            for (int j = 0; j < N[1]; ++j)
                for (int i = 0; i < N[0]; ++i) hv[(size_t)i * ncomp + n] += f(i, j, k, icomp + n);
    for (double& v : hv) v /= N[1] * N[2];
    return hv;
}

// EvaluateSpatialCorrelations3D (statsStag.cpp:868-1105) on the line averages of
// cu, cuMeans (components 0..nvars-1) and prim, primMeans (1..nspecies+4): the
// x* quantities from the lines at cross_cell, then every x cell's running
// averages and derived correlations in the reference's statement order.  As in
// the reference, the lines' "Y_k" are prim components 5+k (pressure for k = 0),
// and entries 37+nspecies+1 and +2 re-apply the update of entries 37 and
// 37+nspecies-1.
static void spatial_cross(const Fab& cu, const Fab& cumeans, const Fab& prim, const Fab& primmeans, double* S_,
                          double* xcross, int64_t steps) {
    const int ns = g.ns, nvars = 5 + ns, nprims = ns + 4, ncross = 37 + ns + 3, H = ns - 1;
    const std::vector<double> cu_avg = line_average(cu, 0, nvars), cumeans_avg = line_average(cumeans, 0, nvars);
    const std::vector<double> prim_avg = line_average(prim, 1, nprims), primmeans_avg = line_average(primmeans, 1, nprims);
    const double stepsminusone = steps - 1.;
    const double stepsinv = 1. / steps;
    const int cc = g.cross_cell;
    double* dx = xcross;
    dx[0] = cu_avg[0 + nvars * cc];
    dx[1] = cumeans_avg[0 + nvars * cc];
    dx[2] = cu_avg[4 + nvars * cc];
    dx[3] = cumeans_avg[4 + nvars * cc];
    for (int d = 0; d < 3; ++d) {
        dx[4 + 2 * d] = cu_avg[1 + d + nvars * cc];
        dx[5 + 2 * d] = cumeans_avg[1 + d + nvars * cc];
    }
    for (int q = 0; q < 4; ++q) {
        dx[10 + 2 * q] = prim_avg[q + nprims * cc];
        dx[11 + 2 * q] = primmeans_avg[q + nprims * cc];
    }
    for (int n = 0; n < ns; ++n) {
        dx[18 + 4 * n + 0] = cu_avg[5 + n + nvars * cc];
        dx[18 + 4 * n + 1] = cumeans_avg[5 + n + nvars * cc];
        dx[18 + 4 * n + 2] = prim_avg[4 + n + nprims * cc];
        dx[18 + 4 * n + 3] = primmeans_avg[4 + n + nprims * cc];
    }
    const double meanrhocross = dx[1], meanuxcross = dx[11];
    double meanYkcross[MAXS], delrhoYkcross[MAXS], delYkcross[MAXS];
    for (int n = 0; n < ns; ++n) {
        meanYkcross[n] = dx[18 + 4 * n + 3];
        delrhoYkcross[n] = dx[18 + 4 * n + 0] - dx[18 + 4 * n + 1];
        delYkcross[n] = dx[18 + 4 * n + 2] - dx[18 + 4 * n + 3];
    }
    const double delrhocross = dx[0] - dx[1], delKcross = dx[2] - dx[3];
    const double deljxcross = dx[4] - dx[5], deljycross = dx[6] - dx[7], deljzcross = dx[8] - dx[9];
    const double delTcross = dx[16] - dx[17], delvxcross = dx[10] - dx[11];
    double cvcross = 0.;
    for (int l = 0; l < ns; ++l) cvcross = cvcross + g.hcv[l] * dx[18 + 4 * l + 1] / dx[1];
    const double cvinvcross = 1.0 / cvcross;
    const double qmeancross = cvcross * dx[17] - 0.5 * (dx[11] * dx[11] + dx[13] * dx[13] + dx[15] * dx[15]);
    const double delGcross = dx[11] * (dx[4] - dx[5]) + dx[13] * (dx[6] - dx[7]) + dx[15] * (dx[8] - dx[9]);
    for (int i = 0; i < g.n[0]; ++i) {
        const double* c = &cu_avg[(size_t)nvars * i];
        const double* cm = &cumeans_avg[(size_t)nvars * i];
        const double* pr = &prim_avg[(size_t)nprims * i];
        const double* pm = &primmeans_avg[(size_t)nprims * i];
        const double meanrho = cm[0];
        double meanYk[MAXS], delrhoYk[MAXS], delYk[MAXS];
        for (int n = 0; n < ns; ++n) {
            meanYk[n] = pm[4 + n];
            delrhoYk[n] = c[5 + n] - cm[5 + n];
            delYk[n] = pr[4 + n] - pm[4 + n];
        }
        const double delrho = c[0] - cm[0], delK = c[4] - cm[4];
        const double deljx = c[1] - cm[1], deljy = c[2] - cm[2], deljz = c[3] - cm[3];
        const double delT = pr[3] - pm[3], delvx = pr[0] - pm[0];
        double cv = 0.;
        for (int l = 0; l < ns; ++l) cv = cv + g.hcv[l] * cm[5 + l] / cm[0];
        const double cvinv = 1.0 / cv;
        const double qmean = cv * pm[3] - 0.5 * (pm[0] * pm[0] + pm[1] * pm[1] + pm[2] * pm[2]);
        const double delG = pm[0] * deljx + pm[1] * deljy + pm[2] * deljz;
        double* S = S_ + (size_t)ncross * i;
        auto upd = [&](int q, double x) { S[q] = (S[q] * stepsminusone + x) * stepsinv; };
        const double pairs[19] = {delrhocross * delrho, delKcross * delK, deljxcross * deljx, deljycross * deljy,
                                  deljzcross * deljz, deljxcross * delrho, deljxcross * delrhoYk[0],
                                  deljxcross * delrhoYk[H], delrhocross * delrhoYk[0], delrhocross * delrhoYk[H],
                                  delrhoYkcross[0] * delrho, delrhoYkcross[H] * delrho, delGcross * delG,
                                  delGcross * delK, delKcross * delG, delrhocross * delK, delKcross * delrho,
                                  delrhocross * delG, delGcross * delrho};
        for (int q = 0; q < 19; ++q) upd(q, pairs[q]);
        S[19] = (cvinvcross * cvinv / (meanrhocross * meanrho)) *
                (S[1] + S[12] - S[13] - S[14] + qmean * qmeancross * S[0] - qmeancross * S[15] - qmean * S[16] +
                 qmeancross * S[17] + qmean * S[18]);
        S[20] = (cvinvcross / meanrhocross) * (S[16] - S[18] - qmeancross * S[0]);
        S[21] = (1.0 / meanrhocross) * (S[5] - meanuxcross * S[0]);
        S[22] = (1.0 / meanrhocross) * (S[6] - meanuxcross * S[8]);
        S[23] = (1.0 / meanrhocross) * (S[7] - meanuxcross * S[9]);
        S[24] = (1.0 / (meanrho * meanrhocross)) *
                (S[6] - meanuxcross * S[8] - meanYk[0] * S[5] + meanuxcross * meanYk[0] * S[0]);
        S[25] = (1.0 / (meanrho * meanrhocross)) *
                (S[7] - meanuxcross * S[9] - meanYk[H] * S[5] + meanuxcross * meanYk[H] * S[0]);
        const double direct[11] = {delTcross * delT, delTcross * delrho, delTcross * delvx, delvxcross * delrho,
                                   delvxcross * delYk[0], delvxcross * delYk[H], delvxcross * delrhoYk[0],
                                   delvxcross * delrhoYk[H], delYkcross[0] * delYk[0], delYkcross[H] * delYk[H],
                                   delYkcross[0] * delYk[H]};
        for (int q = 0; q < 11; ++q) upd(26 + q, direct[q]);
        for (int n = 0; n < ns; ++n) upd(37 + n, delrhoYkcross[n] * delrhoYk[n]);
        upd(37 + ns, delrhoYkcross[H] * delrhoYk[0]);
        double dd = (S[37] * stepsminusone + delrhoYkcross[0] * delrhoYk[0]) * stepsinv;
        S[37 + ns + 1] = (1.0 / (meanrho * meanrhocross)) *
                         (dd - meanYkcross[0] * S[8] - meanYk[0] * S[10] + meanYkcross[0] * meanYk[0] * S[0]);
        dd = (S[37 + H] * stepsminusone + delrhoYkcross[H] * delrhoYk[H]) * stepsinv;
        S[37 + ns + 2] = (1.0 / (meanrho * meanrhocross)) *
                         (dd - meanYkcross[H] * S[9] - meanYk[H] * S[11] + meanYkcross[H] * meanYk[H] * S[0]);
    }
}

// evaluateStatsStag3D's statistics (statsStag.cpp:10-77) without surface
// coverage: EvaluateStatsMeans (:200-365) then
// FillBoundary of the cell means, EvaluateVarsCoVarsMom3 (:367-691) then
// FillBoundary of the cell variances, each loop in the reference's order, then
// with FHD_STATS_CROSS the spatial cross-correlations (:46-76).
// flags as fhd_stats_stag.
int orc_stats_stag(fhd_fab cu_, fhd_fab prim_, const fhd_fab* mom_, const fhd_stats* st, int64_t steps, int flags) {
    const int* N = g.n;
    const int ns = g.ns, nvars = 5 + ns, nprimvars = 6 + 2 * ns;
    Fab cu(cu_), prim(prim_), cumeans(st->cuMeans), primmeans(st->primMeans);
    Fab mom[3] = {Fab(mom_[0]), Fab(mom_[1]), Fab(mom_[2])};
    Fab mm[3] = {Fab(st->cumomMeans[0]), Fab(st->cumomMeans[1]), Fab(st->cumomMeans[2])};
    Fab vm[3] = {Fab(st->velMeans[0]), Fab(st->velMeans[1]), Fab(st->velMeans[2])};
    const double stepsminusone = steps - 1.;
    const double stepsinv = 1. / steps;
    const bool means = flags & FHD_STATS_MEANS, vars = flags & FHD_STATS_VARS;
    if (vars && !means) return FHD_ERR_BAD_ARG;
    if (means) {
        // mean momentum on faces (:215-243)
        for (int d = 0; d < 3; ++d)
            for (int k = 0; k < N[2] + (d == 2); ++k)
                for (int j = 0; j < N[1] + (d == 1); ++j)
                    for (int i = 0; i < N[0] + (d == 0); ++i)
                        mm[d](i, j, k) = (mm[d](i, j, k) * stepsminusone + mom[d](i, j, k)) * stepsinv;
        // mean density on the cells grown by ngc = 2 (:245-256)
        for (int k = -2; k < N[2] + 2; ++k)
            for (int j = -2; j < N[1] + 2; ++j)
                for (int i = -2; i < N[0] + 2; ++i)
                    cumeans(i, j, k, 0) = (cumeans(i, j, k, 0) * stepsminusone + cu(i, j, k, 0)) * stepsinv;
        // other means (:258-317)
        for (int k = 0; k < N[2]; ++k)
            for (int j = 0; j < N[1]; ++j)
                for (int i = 0; i < N[0]; ++i) {
                    double fracvec[MAXS];
                    const Fab &mxm = mm[0], &mym = mm[1], &mzm = mm[2];
                    cumeans(i, j, k, 1) = 0.5 * (mxm(i, j, k) + mxm(i + 1, j, k));
                    cumeans(i, j, k, 2) = 0.5 * (mym(i, j, k) + mym(i, j + 1, k));
                    cumeans(i, j, k, 3) = 0.5 * (mzm(i, j, k) + mzm(i, j, k + 1));
                    cumeans(i, j, k, 4) = (cumeans(i, j, k, 4) * stepsminusone + cu(i, j, k, 4)) * stepsinv;
                    for (int l = 5; l < nvars; ++l) {
                        cumeans(i, j, k, l) = (cumeans(i, j, k, l) * stepsminusone + cu(i, j, k, l)) * stepsinv;
                        fracvec[l - 5] = cumeans(i, j, k, l) / cumeans(i, j, k, 0);
                        primmeans(i, j, k, l + 1) = fracvec[l - 5];
                    }
                    for (int l = 0; l < ns; ++l)
                        primmeans(i, j, k, 6 + ns + l) =
                            (primmeans(i, j, k, 6 + ns + l) * stepsminusone + prim(i, j, k, 6 + ns + l)) * stepsinv;
                    double densitymeaninv = 1.0 / cumeans(i, j, k, 0);
                    primmeans(i, j, k, 1) = densitymeaninv * 0.5 * (mxm(i, j, k) + mxm(i + 1, j, k));
                    primmeans(i, j, k, 2) = densitymeaninv * 0.5 * (mym(i, j, k) + mym(i, j + 1, k));
                    primmeans(i, j, k, 3) = densitymeaninv * 0.5 * (mzm(i, j, k) + mzm(i, j, k + 1));
                    for (int c = 0; c < 3; ++c)
                        primmeans(i, j, k, nprimvars + c) =
                            (primmeans(i, j, k, nprimvars + c) * stepsminusone + prim(i, j, k, 1 + c)) * stepsinv;
                    primmeans(i, j, k, 0) = cumeans(i, j, k, 0);
                    primmeans(i, j, k, 4) = (primmeans(i, j, k, 4) * stepsminusone + prim(i, j, k, 4)) * stepsinv;
                    GetPressureGas(primmeans(i, j, k, 5), fracvec, cumeans(i, j, k, 0), primmeans(i, j, k, 4));
                }
        // mean face velocities (:320-363)
        for (int d = 0; d < 3; ++d) {
            const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
            for (int k = 0; k < N[2] + e2; ++k)
                for (int j = 0; j < N[1] + e1; ++j)
                    for (int i = 0; i < N[0] + e0; ++i) {
                        double densitymeaninv = 2.0 / (cumeans(i - e0, j - e1, k - e2, 0) + cumeans(i, j, k, 0));
                        vm[d](i, j, k) = mm[d](i, j, k) * densitymeaninv;
                    }
        }
        fill_boundary(cumeans);
        fill_boundary(primmeans);
    }
    if (vars) {
        Fab cuvars(st->cuVars), primvars(st->primVars), covars(st->coVars);
        Fab mv[3] = {Fab(st->cumomVars[0]), Fab(st->cumomVars[1]), Fab(st->cumomVars[2])};
        Fab vv[3] = {Fab(st->velVars[0]), Fab(st->velVars[1]), Fab(st->velVars[2])};
        // momentum and velocity variances (:387-435)
        for (int d = 0; d < 3; ++d) {
            const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
            for (int k = 0; k < N[2] + e2; ++k)
                for (int j = 0; j < N[1] + e1; ++j)
                    for (int i = 0; i < N[0] + e0; ++i) {
                        double delj = mom[d](i, j, k) - mm[d](i, j, k);
                        mv[d](i, j, k) = (mv[d](i, j, k) * stepsminusone + delj * delj) * stepsinv;
                        double densitymeaninv = 2.0 / (cumeans(i - e0, j - e1, k - e2, 0) + cumeans(i, j, k, 0));
                        double delrho = 0.5 * (cu(i - e0, j - e1, k - e2, 0) + cu(i, j, k, 0)) -
                                        0.5 * (cumeans(i - e0, j - e1, k - e2, 0) + cumeans(i, j, k, 0));
                        double delvel = (delj - vm[d](i, j, k) * delrho) * densitymeaninv;
                        vv[d](i, j, k) = (vv[d](i, j, k) * stepsminusone + delvel * delvel) * stepsinv;
                    }
        }
        // cell variances and covariances (:438-613)
        for (int k = 0; k < N[2]; ++k)
            for (int j = 0; j < N[1]; ++j)
                for (int i = 0; i < N[0]; ++i) {
                    const Fab &momx = mom[0], &momy = mom[1], &momz = mom[2];
                    const Fab &momxmeans = mm[0], &momymeans = mm[1], &momzmeans = mm[2];
                    double delrho = cu(i, j, k, 0) - cumeans(i, j, k, 0);
                    cuvars(i, j, k, 0) = (cuvars(i, j, k, 0) * stepsminusone + delrho * delrho) * stepsinv;
                    double delenergy = cu(i, j, k, 4) - cumeans(i, j, k, 4);
                    cuvars(i, j, k, 4) = (cuvars(i, j, k, 4) * stepsminusone + delenergy * delenergy) * stepsinv;
                    for (int l = 5; l < nvars; ++l) {
                        double delmassvec = cu(i, j, k, l) - cumeans(i, j, k, l);
                        cuvars(i, j, k, l) = (cuvars(i, j, k, l) * stepsminusone + delmassvec * delmassvec) * stepsinv;
                    }
                    double delrhoYk[MAXS], Ykmean[MAXS], delYk[MAXS];
                    for (int s = 0; s < ns; ++s) {
                        delrhoYk[s] = cu(i, j, k, 5 + s) - cumeans(i, j, k, 5 + s);
                        Ykmean[s] = primmeans(i, j, k, 6 + s);
                        delYk[s] = (delrhoYk[s] - Ykmean[s] * delrho) / cumeans(i, j, k, 0);
                        primvars(i, j, k, 6 + s) = (primvars(i, j, k, 6 + s) * stepsminusone + delYk[s] * delYk[s]) * stepsinv;
                    }
                    primvars(i, j, k, 0) = cuvars(i, j, k, 0);
                    double vx = 0.5 * (vm[0](i, j, k) + vm[0](i + 1, j, k));
                    double vy = 0.5 * (vm[1](i, j, k) + vm[1](i, j + 1, k));
                    double vz = 0.5 * (vm[2](i, j, k) + vm[2](i, j, k + 1));
                    double T = primmeans(i, j, k, 4);
                    double densitymeaninv = 1.0 / cumeans(i, j, k, 0);
                    double cv = 0.;
                    for (int l = 0; l < ns; ++l) cv = cv + g.hcv[l] * cumeans(i, j, k, 5 + l) / cumeans(i, j, k, 0);
                    double cvinv = 1.0 / cv;
                    double qmean = cv * T - 0.5 * (vx * vx + vy * vy + vz * vz);
                    double deljx = 0.5 * (momx(i, j, k) + momx(i + 1, j, k)) - 0.5 * (momxmeans(i, j, k) + momxmeans(i + 1, j, k));
                    double deljy = 0.5 * (momy(i, j, k) + momy(i, j + 1, k)) - 0.5 * (momymeans(i, j, k) + momymeans(i, j + 1, k));
                    double deljz = 0.5 * (momz(i, j, k) + momz(i, j, k + 1)) - 0.5 * (momzmeans(i, j, k) + momzmeans(i, j, k + 1));
                    cuvars(i, j, k, 1) = (cuvars(i, j, k, 1) * stepsminusone + deljx * deljx) * stepsinv;
                    cuvars(i, j, k, 2) = (cuvars(i, j, k, 2) * stepsminusone + deljy * deljy) * stepsinv;
                    cuvars(i, j, k, 3) = (cuvars(i, j, k, 3) * stepsminusone + deljz * deljz) * stepsinv;
                    double delvelx = (deljx - vx * delrho) * densitymeaninv;
                    double delvely = (deljy - vy * delrho) * densitymeaninv;
                    double delvelz = (deljz - vz * delrho) * densitymeaninv;
                    primvars(i, j, k, 1) = (primvars(i, j, k, 1) * stepsminusone + delvelx * delvelx) * stepsinv;
                    primvars(i, j, k, 2) = (primvars(i, j, k, 2) * stepsminusone + delvely * delvely) * stepsinv;
                    primvars(i, j, k, 3) = (primvars(i, j, k, 3) * stepsminusone + delvelz * delvelz) * stepsinv;
                    double delg = vx * deljx + vy * deljy + vz * deljz;
                    const int np = nprimvars;
                    primvars(i, j, k, np + 0) = (primvars(i, j, k, np + 0) * stepsminusone + delg * delg) * stepsinv;
                    primvars(i, j, k, np + 1) = (primvars(i, j, k, np + 1) * stepsminusone + delg * delenergy) * stepsinv;
                    primvars(i, j, k, np + 2) = (primvars(i, j, k, np + 2) * stepsminusone + delrho * delenergy) * stepsinv;
                    primvars(i, j, k, np + 3) = (primvars(i, j, k, np + 3) * stepsminusone + delrho * delg) * stepsinv;
                    primvars(i, j, k, np + 4) =
                        (primvars(i, j, k, np + 4) * stepsminusone +
                         cvinv * cvinv * densitymeaninv * densitymeaninv *
                             (cuvars(i, j, k, 4) + primvars(i, j, k, np + 0) - 2 * primvars(i, j, k, np + 1) +
                              qmean * (qmean * cuvars(i, j, k, 0) - 2 * primvars(i, j, k, np + 2) +
                                       2 * primvars(i, j, k, np + 3)))) *
                        stepsinv;
                    double delT = prim(i, j, k, 4) - primmeans(i, j, k, 4);
                    primvars(i, j, k, 4) = (primvars(i, j, k, 4) * stepsminusone + delT * delT) * stepsinv;
                    double deltemp = delT;
                    const double terms[26] = {
                        delrho * deljx, delrho * deljy, delrho * deljz, deljx * deljy, deljy * deljz, deljx * deljz,
                        delrho * delenergy, deljx * delenergy, deljy * delenergy, deljz * delenergy,
                        delrhoYk[0] * delrhoYk[ns - 1], delrho * delvelx, delrho * delvely, delrho * delvelz,
                        delvelx * delvely, delvely * delvelz, delvelx * delvelz, delrho * deltemp, delvelx * deltemp,
                        delvely * deltemp, delvelz * deltemp, delYk[0] * delYk[ns - 1], delYk[0] * delvelx,
                        delYk[ns - 1] * delvelx, delrhoYk[0] * delvelx, delrhoYk[ns - 1] * delvelx};
                    for (int c = 0; c < 26; ++c)
                        covars(i, j, k, c) = (covars(i, j, k, c) * stepsminusone + terms[c]) * stepsinv;
                }
        // third and fourth moments (:616-689)
        const bool m3on = flags & FHD_STATS_MOM3, m4on = flags & FHD_STATS_MOM4;
        if (m3on || m4on) {
            Fab m3(st->mom3), m4(st->mom4);
            for (int k = 0; k < N[2]; ++k)
                for (int j = 0; j < N[1]; ++j)
                    for (int i = 0; i < N[0]; ++i) {
                        double delrho = cu(i, j, k, 0) - cumeans(i, j, k, 0);
                        if (m3on) m3(i, j, k, 0) = (m3(i, j, k, 0) * stepsminusone + delrho * delrho * delrho) * stepsinv;
                        if (m4on) m4(i, j, k, 0) = (m4(i, j, k, 0) * stepsminusone + delrho * delrho * delrho * delrho) * stepsinv;
                        double delenergy = cu(i, j, k, 4) - cumeans(i, j, k, 4);
                        if (m3on) m3(i, j, k, 4) = (m3(i, j, k, 4) * stepsminusone + delenergy * delenergy * delenergy) * stepsinv;
                        if (m4on)
                            m4(i, j, k, 4) =
                                (m4(i, j, k, 4) * stepsminusone + delenergy * delenergy * delenergy * delenergy) * stepsinv;
                        double delrhoYk[MAXS], delYk[MAXS];
                        for (int s = 0; s < ns; ++s) {
                            delrhoYk[s] = cu(i, j, k, 5 + s) - cumeans(i, j, k, 5 + s);
                            double Ykmean = primmeans(i, j, k, 6 + s);
                            delYk[s] = (delrhoYk[s] - Ykmean * delrho) / cumeans(i, j, k, 0);
                            if (m3on) m3(i, j, k, 5 + s) = (m3(i, j, k, 5 + s) * stepsminusone + delYk[s] * delYk[s] * delYk[s]) * stepsinv;
                            if (m4on)
                                m4(i, j, k, 5 + s) =
                                    (m4(i, j, k, 5 + s) * stepsminusone + delYk[s] * delYk[s] * delYk[s] * delYk[s]) * stepsinv;
                        }
                        double vx = 0.5 * (vm[0](i, j, k) + vm[0](i + 1, j, k));
                        double vy = 0.5 * (vm[1](i, j, k) + vm[1](i, j + 1, k));
                        double vz = 0.5 * (vm[2](i, j, k) + vm[2](i, j, k + 1));
                        double densitymeaninv = 1.0 / cumeans(i, j, k, 0);
                        double deljx = 0.5 * (mom[0](i, j, k) + mom[0](i + 1, j, k)) - 0.5 * (mm[0](i, j, k) + mm[0](i + 1, j, k));
                        double deljy = 0.5 * (mom[1](i, j, k) + mom[1](i, j + 1, k)) - 0.5 * (mm[1](i, j, k) + mm[1](i, j + 1, k));
                        double deljz = 0.5 * (mom[2](i, j, k) + mom[2](i, j, k + 1)) - 0.5 * (mm[2](i, j, k) + mm[2](i, j, k + 1));
                        double dv[3] = {(deljx - vx * delrho) * densitymeaninv, (deljy - vy * delrho) * densitymeaninv,
                                        (deljz - vz * delrho) * densitymeaninv};
                        for (int c = 0; c < 3; ++c) {
                            if (m3on) m3(i, j, k, 1 + c) = (m3(i, j, k, 1 + c) * stepsminusone + dv[c] * dv[c] * dv[c]) * stepsinv;
                            if (m4on)
                                m4(i, j, k, 1 + c) = (m4(i, j, k, 1 + c) * stepsminusone + dv[c] * dv[c] * dv[c] * dv[c]) * stepsinv;
                        }
                        double delT = prim(i, j, k, 4) - primmeans(i, j, k, 4);
                        if (m3on) m3(i, j, k, 5 + ns) = (m3(i, j, k, 5 + ns) * stepsminusone + delT * delT * delT) * stepsinv;
                        if (m4on) m4(i, j, k, 5 + ns) = (m4(i, j, k, 5 + ns) * stepsminusone + delT * delT * delT * delT) * stepsinv;
                    }
        }
        fill_boundary(cuvars);
        fill_boundary(primvars);
    }
    if (flags & FHD_STATS_CROSS) {
        if (g.cross_cell < 0 || g.cross_cell > N[0] - 1 || !st->spatialCross || !st->dataSliceMeans_xcross)
            return FHD_ERR_BAD_ARG;
        spatial_cross(cu, cumeans, prim, primmeans, st->spatialCross, st->dataSliceMeans_xcross, steps);
    }
    return FHD_OK;
}

// Host-drawn noise for injected-noise runs: one std::mt19937_64(seed) engine
// (the generator the C++ standard specifies), Box-Muller on 53-bit uniforms,
// filling in a fixed order: for A then B, for d = 0..2: face[d] (all its
// components, variance 1), edge[d] (variance 1), cen[d] (variance 2, the 3D
// centre-noise variance of timeStepStag.cpp:219-222); valid points only, i
// fastest, component slowest.  Each field is then OverrideSync'ed and
// FillBoundary'ed, as MultiFabFillRandomNormal leaves it.  Deterministic and
// serial: fixtures made from it are reproducible on any host with this libm.
int orc_fill_noise_mt64(const fhd_noise* nz, uint64_t seed) {
    std::mt19937_64 eng(seed);
    bool have = false;
    double spare = 0.0;
    auto normal = [&]() {
        if (have) { have = false; return spare; }
        double u1 = ((double)(eng() >> 11) + 1.0) * (1.0 / 9007199254740992.0);  // (0,1]
        double u2 = (double)(eng() >> 11) * (1.0 / 9007199254740992.0);          // [0,1)
        double r = std::sqrt(-2.0 * std::log(u1));
        double a = 2.0 * 3.14159265358979323846 * u2;
        spare = r * std::sin(a);
        have = true;
        return r * std::cos(a);
    };
    auto fill = [&](const fhd_fab& f_, double variance) {
        Fab f(f_);
        const double sd = std::sqrt(variance);
        const int* N = g.n;
        for (int n = 0; n < f.nc; ++n)
            for (int k = 0; k < N[2] + f.nodal[2]; ++k)
                for (int j = 0; j < N[1] + f.nodal[1]; ++j)
                    for (int i = 0; i < N[0] + f.nodal[0]; ++i) f(i, j, k, n) = sd * normal();
        override_sync(f);
        fill_boundary(f);
    };
    for (int s = 0; s < 2; ++s)
        for (int d = 0; d < 3; ++d) {
            fill(nz->face[s][d], 1.0);
            fill(nz->edge[s][d], 1.0);
            fill(nz->cen[s][d], 2.0);
        }
    for (int s = 0; s < 2; ++s)
        if (nz->chem[s].data) fill(nz->chem[s], 1.0);  // ranchem_A/B, variance 1
    return FHD_OK;
}

// The acoustic CFL diagnostic, compressible_functions_stag.cpp:691-776 (max over faces).
double orc_max_acoustic_cfl(fhd_fab prim_, const fhd_fab* vel_, double dt) {
    Fab prim(prim_);
    const int* N = g.n;
    double cmax = 0.0;
    for (int d = 0; d < 3; ++d) {
        Fab v(vel_[d]);
        const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
        for (int k = 0; k < N[2] + e2; ++k)
            for (int j = 0; j < N[1] + e1; ++j)
                for (int i = 0; i < N[0] + e0; ++i) {
                    double temp = 0.5 * (prim(i - e0, j - e1, k - e2, 4) + prim(i, j, k, 4));
                    double Yk[MAXS];
                    for (int s = 0; s < g.ns; ++s) Yk[s] = 0.5 * (prim(i - e0, j - e1, k - e2, 6 + s) + prim(i, j, k, 6 + s));
                    double molmix = 0., cvmix = 0., cpmix = 0.;
                    for (int s = 0; s < g.ns; ++s) { molmix += Yk[s] / g.molmass[s]; cvmix += Yk[s] * g.hcv[s]; cpmix += Yk[s] * g.hcp[s]; }
                    molmix = 1. / molmix;
                    double gamma = cpmix / cvmix;
                    double c = std::sqrt(gamma * (g.Runiv / molmix) * temp);
                    cmax = std::max(cmax, (c + std::abs(v(i, j, k))) * dt / g.dx[d]);
                }
    }
    return cmax;
}

}  // extern "C"
