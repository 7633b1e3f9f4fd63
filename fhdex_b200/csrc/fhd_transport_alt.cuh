// fhd_transport_alt.cuh — the other two transport models of calculateTransportCoeffs
// (transCoeffs.cpp:58-73): Valk/Waldmann (transport_type 2,
// IdealMixtureTransportVW, compressible_functions.H:1047-1152, with ViscLin :968-1043,
// LambdaLin :781-911, D_GIO :512-645 and ThermalDiff :913-966) and the
// Hirschfelder-Curtiss-Bird binary hard-sphere model (transport_type 3,
// IdealMixtureTransportHCBBin :1355-1478).  FP64, each expression in the reference's
// operation order (the units that include this are built with -fmad=false).
//
// The Valk/Waldmann pair constants that do not depend on the cell (the parts of
// Dbin, omega11, a_ij1, a_ij2 and alphabar before their temperature factors, and the
// powers of the molecular masses) come from the host in a VWTable, computed there by
// the reference's own expressions with the host's pow; a cell then applies only its
// temperature and pressure.  One power depends on the cell (LambdaLin's
// pow(D_T[i]/(n_i m_i) - D_T[j]/(n_j m_j), 2.)); it is taken as the rounded product,
// which the host libm's pow can miss by one ulp (measured: about one value in 1200),
// so this model follows the reference to rounding, not bit for bit.
#pragma once
#include "fhd_device.cuh"

namespace fhd {

struct VWTable {
    double DbinC[MAXS * MAXS];     // 3/16 sqrt(2 pi kB^3 (mi+mj)/mi/mj) / (pi d^2): Dbin = DbinC T sqrtT / p
    double omegaC[MAXS * MAXS];    // sqrt(pi kB / (2 mu)) d^2: omega11 = omegaC sqrtT
    double a1C[MAXS * MAXS];       // a_ij1 = a1C / sqrtT
    double a2C[MAXS * MAXS];       // a_ij2 = a2C / sqrtT
    double alphabar[MAXS * MAXS];
    double ps2[MAXS * MAXS];       // pow(mi + mj, 2.)
    double ps3[MAXS * MAXS];       // pow(mi + mj, 3.)
    double pm2[MAXS];              // pow(mi, 2.)
};

// Decomp / Solve (compressible_functions.H:222-268, 323-361) on an n x n system held in
// rows of stride ld, with the reference's partial pivoting through ip (1-based).
// Returns false where the reference aborts ("singular matrix in decomp").
FHD_D bool vw_decomp(int neq, double* a, int* ip, int ld) {
    const double eps = 1.e-30, eps2 = 1.e-60;
    bool ok = true;
    for (int n = 0; n < neq; ++n) ip[n] = n + 1;
    for (int i = 0; i < neq - 1; ++i) {
        const int ip1 = i + 2;
        int k = i + 1;
        double apm = fabs(a[(ip[i] - 1) * ld + i]);
        for (int j = ip1 - 1; j < neq; ++j) {
            const double apn = fabs(a[(ip[j] - 1) * ld + i]);
            if (apm >= apn) continue;
            apm = apn;
            k = j + 1;
        }
        const int j = ip[k - 1];
        ip[k - 1] = ip[i];
        ip[i] = j;
        if (apm < eps) ok = false;
        for (int l = ip1 - 1; l < neq; ++l) {
            const int n = ip[l];
            const double amult = a[(n - 1) * ld + i] / a[(j - 1) * ld + i];
            a[(n - 1) * ld + i] = amult;
            if (fabs(amult) < eps2) continue;
            for (int kk = ip1 - 1; kk < neq; ++kk) a[(n - 1) * ld + kk] = a[(n - 1) * ld + kk] - amult * a[(j - 1) * ld + kk];
        }
    }
    if (fabs(a[(ip[neq - 1] - 1) * ld + neq - 1]) < eps) ok = false;
    return ok;
}

FHD_D void vw_solve(int neq, const double* a, double* b, int* ip, int ld) {
    for (int l = 1; l < neq; ++l) {
        const int n = ip[l];
        for (int k = 0; k < l; ++k) b[n - 1] = b[n - 1] - a[(n - 1) * ld + k] * b[ip[k] - 1];
    }
    b[ip[neq - 1] - 1] = b[ip[neq - 1] - 1] / a[(ip[neq - 1] - 1) * ld + neq - 1];
    for (int l = 0; l < neq - 1; ++l) {
        const int j = neq - (l + 1);
        const int n = ip[j - 1];
        for (int k = j; k < neq; ++k) b[n - 1] = b[n - 1] - a[(n - 1) * ld + k] * b[ip[k] - 1];
        b[n - 1] = b[n - 1] / a[(n - 1) * ld + j - 1];
    }
    for (int n = 0; n < neq; ++n) {
        while (ip[n] != n + 1) {
            const int j = ip[n];
            const double scr = b[j - 1];
            ip[n] = ip[j - 1];
            b[j - 1] = b[ip[j - 1] - 1];
            b[ip[j - 1] - 1] = scr;
            ip[j - 1] = j;
        }
    }
}

// Decompnp / Solvenp (:405-459): no pivoting
template <int NS>
FHD_D bool vw_decompnp(double (&a)[NS * NS]) {
    const double eps = 1.e-30, eps2 = 1.e-60;
    for (int i = 0; i < NS - 1; ++i)
        for (int l = i + 1; l < NS; ++l) {
            const double amult = a[l * NS + i] / a[i * NS + i];
            a[l * NS + i] = amult;
            if (fabs(amult) < eps2) continue;
            for (int k = i + 1; k < NS; ++k) a[l * NS + k] = a[l * NS + k] - amult * a[i * NS + k];
        }
    return !(fabs(a[(NS - 1) * NS + NS - 1]) < eps);
}

template <int NS>
FHD_D void vw_solvenp(const double (&a)[NS * NS], double (&b)[NS]) {
    for (int l = 1; l < NS; ++l)
        for (int k = 0; k < l; ++k) b[l] = b[l] - a[l * NS + k] * b[k];
    b[NS - 1] = b[NS - 1] / a[(NS - 1) * NS + NS - 1];
    for (int l = 0; l < NS - 1; ++l) {
        const int j = NS - (l + 1);
        for (int k = j; k < NS; ++k) b[j - 1] = b[j - 1] - a[(j - 1) * NS + k] * b[k];
        b[j - 1] = b[j - 1] / a[(j - 1) * NS + j - 1];
    }
}

// IdealMixtureTransportVW for one cell: eta, kappa (zeta 0), chi and D (not yet
// multiplied by rho); Xk from GetMolfrac of the clamped, renormalised Y.  Returns false
// where a decomposition is singular (the reference aborts).
template <int NS>
FHD_D bool transport_vw(const DevParams& P, double density, double temperature, double pressure,
                        const double (&Xk)[NS], Coeffs<NS, double>& c) {
    const VWTable& V = *P.vwt;
    double xxtr[NS], yytr[NS], mk[NS];
#pragma unroll
    for (int n = 0; n < NS; ++n) mk[n] = P.mm[n];
#pragma unroll
    for (int ii = 0; ii < NS; ++ii) {
        double sumXk = 0.;
#pragma unroll
        for (int jj = 0; jj < NS; ++jj) sumXk += Xk[jj];
        xxtr[ii] = Xk[ii] + 1.e-15 * (sumXk / (double)NS - Xk[ii]);
    }
    double MWmix = 0.;
#pragma unroll
    for (int ii = 0; ii < NS; ++ii) MWmix += xxtr[ii] * P.molmass[ii];
#pragma unroll
    for (int ii = 0; ii < NS; ++ii) yytr[ii] = P.molmass[ii] / MWmix * xxtr[ii];
    const double sqrtT = sqrt(temperature);
    double Dbin[NS][NS], om[NS * NS];
#pragma unroll
    for (int i = 0; i < NS; ++i)
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            Dbin[i][j] = V.DbinC[i * MAXS + j] * temperature * sqrtT / pressure;
            om[i * NS + j] = V.omegaC[i * MAXS + j] * sqrtT;
        }
    bool ok = true;
    // ViscLin (:968-1043)
    {
        double nk[NS], diag[NS], QoR[NS * NS], b[NS];
        int ip[NS];
#pragma unroll
        for (int ii = 0; ii < NS; ++ii) nk[ii] = density * yytr[ii] / mk[ii];
#pragma unroll
        for (int ii = 0; ii < NS; ++ii) {
            diag[ii] = 0.;
#pragma unroll
            for (int kk = 0; kk < NS; ++kk)
                diag[ii] = diag[ii] + nk[kk] * mk[kk] / V.ps2[ii * MAXS + kk] *
                                          (5. * mk[ii] * om[ii * NS + kk] + 3. * mk[kk] * om[ii * NS + kk]);
        }
#pragma unroll
        for (int ii = 0; ii < NS; ++ii) {
#pragma unroll
            for (int jj = 0; jj < NS; ++jj) {
                double sum1 = -nk[jj] * mk[jj] / V.ps2[ii * MAXS + jj] * 2. * mk[jj] * om[ii * NS + jj];
                if (ii == jj) sum1 = sum1 + diag[ii];
                QoR[ii * NS + jj] = -(16. / 15.) * (mk[ii] / mk[jj]) * sum1;
            }
            b[ii] = -1.;
        }
        ok = vw_decomp(NS, QoR, ip, NS) && ok;
        vw_solve(NS, QoR, b, ip, NS);
        double sum1 = 0.;
#pragma unroll
        for (int ii = 0; ii < NS; ++ii) sum1 = sum1 + nk[ii] * b[ii];
        c.eta = 0.5 * P.k_B * temperature * sum1;
    }
    c.zeta = 0.;
    // LambdaLin (:781-911)
    {
        double nk[NS], beta[NS], d1[NS], d2[NS], d3[NS], d4[NS], DT[NS];
        double QQ[4 * NS * NS], aS[2 * NS];
        int ip[2 * NS];
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            nk[i] = density * yytr[i] / mk[i];
            d1[i] = 0.;
            d2[i] = 0.;
            d3[i] = 0.;
            d4[i] = 0.;
        }
#pragma unroll
        for (int i = 0; i < NS; ++i)
#pragma unroll
            for (int k = 0; k < NS; ++k) {
                const double o = om[i * NS + k];
                d1[i] = d1[i] + nk[k] * mk[k] / (mk[i] + mk[k]) * nk[i] * mk[i] * o;
                if (k != i) d2[i] = d2[i] + nk[k] * mk[k] / (mk[i] + mk[k]) * o;
                d3[i] = d3[i] + nk[i] * nk[k] * V.pm2[k] / V.ps2[i * MAXS + k] * .5 * o;
                d4[i] = d4[i] + nk[i] * nk[k] * mk[k] / V.ps3[i * MAXS + k] *
                                    ((5. / 4. * (6. * V.pm2[i] + 5. * V.pm2[k]) * o - 3. * V.pm2[k] * o) +
                                     4. * mk[i] * mk[k] * o);
            }
#pragma unroll
        for (int i = 0; i < NS; ++i)
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                const double o = om[i * NS + j];
                double s00 = -nk[j] * mk[j] * d2[i] - nk[j] * mk[j] / (mk[i] + mk[j]) * nk[i] * mk[i] * o;
                double s01 = -nk[i] * nk[j] * V.pm2[j] / V.ps2[i * MAXS + j] * .5 * o;
                // the reference's sum11 takes mk[j] in both Sonine terms (kept)
                double s11 = nk[i] * nk[j] * mk[j] / V.ps3[i * MAXS + j] *
                             (-(5. / 4. * (6. * V.pm2[j] + 5. * V.pm2[j]) * o - 3. * V.pm2[j] * o) +
                              4. * mk[j] * mk[j] * o);
                if (i == j) {
                    s00 = s00 + d1[i];
                    s01 = s01 + d3[i];
                    s11 = s11 + d4[i];
                }
                const double ratm = mk[i] / mk[j];
                const double sqratm = sqrt(ratm);
                const double scr = ratm * sqratm;
                QQ[i * 2 * NS + j] = 8. * sqratm / mk[i] * s00;
                QQ[i * 2 * NS + j + NS] = -8. * scr * s01;
                QQ[(i + NS) * 2 * NS + j] = -8. * sqratm * s01;
                QQ[(i + NS) * 2 * NS + j + NS] = 8. * ratm * sqratm * s11;
            }
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            aS[i] = 0.;
            beta[i] = sqrt(2. * P.k_B * temperature / mk[i]);
            aS[i + NS] = -(15. / 4.) * nk[i] * beta[i];
        }
        ok = vw_decomp(2 * NS, QQ, ip, 2 * NS) && ok;
        vw_solve(2 * NS, QQ, aS, ip, 2 * NS);
#pragma unroll
        for (int i = 0; i < NS; ++i) DT[i] = 0.5 * nk[i] * beta[i] * mk[i] * aS[i];
        double sum1 = 0;
#pragma unroll
        for (int i = 0; i < NS; ++i) sum1 = sum1 + nk[i] * beta[i] * aS[NS + i];
        const double lamdaprime = -5. / 4. * P.k_B * sum1;
        sum1 = 0;
#pragma unroll
        for (int i = 0; i < NS; ++i)
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                const double dd = DT[i] / (nk[i] * mk[i]) - DT[j] / (nk[j] * mk[j]);
                sum1 = sum1 + nk[i] * nk[j] / Dbin[i][j] * (dd * dd);
            }
        double ntotal = 0;
#pragma unroll
        for (int i = 0; i < NS; ++i) ntotal += nk[i];
        c.kappa = lamdaprime - 0.5 * P.k_B / ntotal * sum1;
    }
    // D_GIO (:512-645) is D_GIO1 on a flat Dbin
    {
        double rDbin[NS][NS], Dout[NS * NS];
#pragma unroll
        for (int i = 0; i < NS; ++i)
#pragma unroll
            for (int j = 0; j < NS; ++j) rDbin[i][j] = (i == j || NS > 2) ? 0. : rdiv(1., Dbin[i][j]);
        D_GIO1<NS, double>(P, Dbin, rDbin, yytr, xxtr, Dout);
#pragma unroll
        for (int q = 0; q < NS * NS; ++q) c.D[q] = Dout[q];
    }
    // ThermalDiff (:913-966)
    {
        double Aij[NS * NS], AA[NS];
#pragma unroll
        for (int i = 0; i < NS; ++i) {
#pragma unroll
            for (int j = 0; j < NS; ++j) Aij[i * NS + j] = xxtr[j] * (V.a2C[i * MAXS + j] / sqrtT);
            AA[i] = 15. / 4.;
        }
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            double sumTemp = 0.;
#pragma unroll
            for (int k = 0; k < NS; ++k) sumTemp = sumTemp + xxtr[k] * (V.a1C[i * MAXS + k] / sqrtT);
            Aij[i * NS + i] = Aij[i * NS + i] + sumTemp;
        }
        ok = vw_decompnp<NS>(Aij) && ok;
        vw_solvenp<NS>(Aij, AA);
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            double sumTemp = 0.;
#pragma unroll
            for (int j = 0; j < NS; ++j)
                sumTemp = sumTemp + xxtr[j] * (V.alphabar[k * MAXS + j] * (AA[k] / mk[k] - AA[j] / mk[j]) / sqrtT);
            c.chi[k] = sumTemp;
        }
    }
    return ok;
}

// IdealMixtureTransportHCBBin for one cell of a binary mixture (NS == 2)
FHD_D void transport_hcb(const DevParams& P, double density, double temperature, const double (&Xk)[2],
                         Coeffs<2, double>& c) {
    const double pi = 3.1415926535897932;
    const double k_B = P.k_B;
    double xxtr[2], yytr[2];
    for (int ii = 0; ii < 2; ++ii) {
        double sumXk = 0.;
        for (int jj = 0; jj < 2; ++jj) sumXk += Xk[jj];
        xxtr[ii] = Xk[ii] + 1.e-15 * (sumXk / 2.0 - Xk[ii]);
    }
    double MWmix = 0.;
    for (int ii = 0; ii < 2; ++ii) MWmix += xxtr[ii] * P.molmass[ii];
    for (int ii = 0; ii < 2; ++ii) yytr[ii] = P.molmass[ii] / MWmix * xxtr[ii];
    const double m0 = P.mm[0], m1 = P.mm[1];
    const double d0 = P.diam[0][0], d1 = P.diam[1][1];   // 0.5 * (d + d) == d
    const double mx = 2.0 * m0 * m1 / (m0 + m1);
    const double dx = P.diam[0][1];                       // 0.5 * (d0 + d1), formed on the host
    const double conc = xxtr[1], onc = xxtr[0];
    const double eta0 = (5.0 / (16.0 * d0 * d0)) * sqrt(m0 * k_B * temperature / pi);
    const double eta1 = (5.0 / (16.0 * d1 * d1)) * sqrt(m1 * k_B * temperature / pi);
    const double etax = (5.0 / (16.0 * dx * dx)) * sqrt(mx * k_B * temperature / pi);
    const double Xeta = (onc * onc / eta0) + (2.0 * conc * onc / etax) + (conc * conc / eta1);
    const double Yeta = (3.0 / 5.0) * ((onc * onc * m0) / (eta0 * m1) +
                                       (2.0 * conc * onc * etax * (m0 + m1) * (m0 + m1)) / (4.0 * eta0 * eta1 * m0 * m1) +
                                       (conc * conc * m1) / (eta1 * m0));
    const double Zeta = (3.0 / 5.0) * ((onc * onc * m0 / m1) +
                                       2.0 * conc * onc *
                                           (((m0 + m1) * (m0 + m1) / (4.0 * m0 * m1)) * ((etax / eta0) + (etax / eta1)) - 1.0) +
                                       conc * conc * m1 / m0);
    c.eta = 1.016 * (1.0 + Zeta) / (Xeta + Yeta);
    const double kappa0 = 15.0 * k_B * eta0 / (4.0 * m0);
    const double kappa1 = 15.0 * k_B * eta1 / (4.0 * m1);
    const double kappax = 15.0 * k_B * etax / (4.0 * mx);
    const double U0 = 4.0 / 15.0 - 17.0 * m0 / (60.0 * m1) + (m0 - m1) * (m0 - m1) / (2.0 * m0 * m1);
    const double U1 = 4.0 / 15.0 - 17.0 * m1 / (60.0 * m0) + (m0 - m1) * (m0 - m1) / (2.0 * m0 * m1);
    const double UY = 4.0 * (m0 + m1) * (m0 + m1) * kappax * kappax / (15.0 * 4.0 * m0 * m1 * kappa0 * kappa1) -
                      17.0 / 60.0 + 13.0 * (m0 - m1) * (m0 - m1) / (32.0 * m0 * m1);
    const double UZ = (4.0 / 15.0) * (((m0 + m1) * (m0 + m1) / (4.0 * m0 * m1)) * ((kappax / kappa0) + (kappax / kappa1)) -
                                      1.0) -
                      17.0 / 60.0;
    const double Xkappa = onc * onc / kappa0 + 2.0 * conc * onc / kappax + conc * conc / kappa1;
    const double Ykappa = onc * onc * U0 / kappa0 + 2.0 * conc * onc * UY / kappax + conc * conc * U1 / kappa1;
    const double Zkappa = onc * onc * U0 + 2.0 * conc * onc * UZ + conc * conc * U1;
    c.kappa = 1.025 * (1.0 + Zkappa) / (Xkappa + Ykappa);
    c.zeta = 0.0;
    const double diff = 6.0 * 1.133 * etax / (5.0 * density);
    const double S0 = (m0 + m1) * kappax / (2.0 * m1 * kappa0) - 15 * (m1 - m0) / (8.0 * m0) - 1.0;
    const double S1 = (m0 + m1) * kappax / (2.0 * m0 * kappa1) - 15 * (m0 - m1) / (8.0 * m1) - 1.0;
    double thermal_diff = 1.299 * conc * onc * (S1 * conc - S0 * onc) / (6.0 * kappax * (Xkappa + Ykappa));
    const double mR = m0 / m1;
    const double diffO = mR * diff * yytr[1] * yytr[1] * yytr[1] / (yytr[0] * xxtr[1] * xxtr[1]);
    const double diff1 = mR * diff * yytr[1] * yytr[1] / (xxtr[1] * xxtr[1]);
    c.D[0] = 1.0 * yytr[0] * diffO;
    c.D[1] = -1.0 * yytr[0] * diffO;
    c.D[2] = -1.0 * yytr[0] * diff1;
    c.D[3] = 1.0 * yytr[0] * diff1;
    thermal_diff = thermal_diff * mR * yytr[1] * yytr[1] / (xxtr[1] * xxtr[1]);
    c.chi[0] = -1.0 * xxtr[1] * xxtr[1] * thermal_diff / (mR * xxtr[0] * yytr[1] * yytr[1]);
    c.chi[1] = 1.0 * xxtr[1] * thermal_diff / (mR * yytr[1] * yytr[1]);
}

// calculateTransportCoeffs for one cell with transport_type 2 or 3 (transCoeffs.cpp:37-89):
// the mass-fraction check and clamp, GetMolfrac, the model, D *= rho and the bulk
// viscosity.  Returns 0, 2 (FHD_ERR_MASSFRAC: a mass fraction outside (0,1)) or 9
// (FHD_ERR_SINGULAR: a singular Valk/Waldmann system).
template <int NS>
FHD_D int transport_alt(const DevParams& P, double rho, double T, double p, const double (&Yraw)[NS],
                        Coeffs<NS, double>& c) {
    int st = 0;
    double Yk[NS], Xk[NS];
    double sumYk = 0.;
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        if (Yraw[n] <= 0.0 || Yraw[n] >= 1.0) st = 2;
        Yk[n] = fmax(0., fmin(1., Yraw[n]));
        sumYk += Yk[n];
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) Yk[n] /= sumYk;
    // GetMolfrac (compressible_functions.H:139-153)
    double molmix = 0.;
#pragma unroll
    for (int n = 0; n < NS; ++n) molmix += Yk[n] / P.molmass[n];
    molmix = 1. / molmix;
#pragma unroll
    for (int n = 0; n < NS; ++n) Xk[n] = Yk[n] * molmix / P.molmass[n];
    if constexpr (NS == 2) {
        if (P.transport_type == 3) transport_hcb(P, rho, T, Xk, c);
        else if (!transport_vw<NS>(P, rho, T, p, Xk, c)) st = st ? st : 9;
    } else {
        if (!transport_vw<NS>(P, rho, T, p, Xk, c)) st = st ? st : 9;
    }
#pragma unroll
    for (int q = 0; q < NS * NS; ++q) c.D[q] *= rho;
    if (P.visc_type == 3 || P.visc_type == -3) c.zeta = P.zeta_ratio * c.eta;
    return st;
}

}  // namespace fhd
