// fhd_chem.cuh — chemistry source of the compressible staggered step:
// compute_compressible_chemistry_source_CLE (chemistry_functions.cpp:128-193),
// called once per RK stage with the stage's primitive state
// (timeStepStag.cpp:354-361, 681-688, 1014-1021).
//
// Per valid cell, with c_k = X_k p / (Runiv T) the molar concentrations, reaction
// m has the law-of-mass-action rate
//     a_m = max(0, k_m exp(-alpha_m/Runiv (1/T - 1/T0)) (T/T0)^beta_m prod_n c_n^R_mn)
// and species n gets
//     S_n = sum_m M_n (P_mn - R_mn) (a_m + [CLE] sqrt(a_m / N_A) W_m / sqrt(dt dV)).
// Operation order is the reference's: the rate is built as successive products,
// S_n accumulates reaction by reaction, mean term before Langevin term.  Fusing
// the reference's two reaction loops into one changes no arithmetic: each rate
// depends only on its own reaction.
//
// Divisions by the run's constants (Runiv, T0, sqrt(dt dV), N_A) and the second
// division by the cell's T (whose reciprocal the rate needs anyway) use the
// correctly rounded reciprocal-and-correction division of fhd_div.h: the same
// quotients as a / b, in a few instructions instead of an iterative division.
//
// c_n^R for the integer stoichiometric coefficients is R-1 multiplications: 1 for
// R = 0 and c for R = 1 as pow returns them, c*c (correctly rounded, as a correctly
// rounded pow gives) for R = 2, within an ulp of pow for R >= 3.  exp and the real
// power (T/T0)^beta are the CUDA library functions: their last-ulp rounding can
// differ from the host C library's.
#pragma once
#include <cmath>
#include <cstring>
#include "../../include/fhd_capi.h"
#include "fhd_device.cuh"
#include "philox.cuh"

namespace fhd {

constexpr int MAXR = FHD_MAX_REACTIONS;

struct ChemParams {
    int nr;                 // reactions
    int type;               // 0 deterministic, 1 CLE
    int sR[MAXR][MAXS];     // reactant coefficients
    int sPR[MAXR][MAXS];    // products - reactants
    double rate[MAXR];      // k_m
    double nar[MAXR];       // -alpha_m / Runiv
    double beta[MAXR];
    double T0, rT0;         // T0 and 1/T0
    double navo;            // Avogadro's number
    double sq;              // sqrt(dt * dV)
    double rR, rnavo, rsq;  // 1/Runiv, 1/navo, 1/sq
    uint32_t div_lo, div_span;  // dividend window of div_rcp (span 0: plain divisions)
};

// Noise of the chemistry source: none (deterministic), the per-step A/B fields
// (W = 1.0*A + w*B, MultiFab::LinComb at timeStepStag.cpp:355-358), W given
// directly (the drop-in operator's ranchem), or A/B generated in-kernel.
enum ChemNoise { CN_OFF = 0, CN_AB = 1, CN_W = 2, CN_PHILOX = 3 };

// Philox field ids of the reaction noises: 56 + m (two reactions per call),
// apart from the face (16 d + c), edge (48 + e) and centre (51 + d) fields.
FHD_HD uint32_t fid_chem(int m) { return (uint32_t)(56 + m); }

// host: the constants of one step (the reference derives them per cell in the
// same order: -alpha/Runiv, 1/T0, sqrt(dt*dV))
inline ChemParams chem_params(const fhd_params& p, double dt, double dV) {
    ChemParams C;
    std::memset(&C, 0, sizeof(C));
    C.nr = p.nreaction;
    C.type = p.reaction_type;
    for (int m = 0; m < MAXR; ++m) {
        for (int n = 0; n < MAXS; ++n) {
            C.sR[m][n] = p.stoich_R[m][n];
            C.sPR[m][n] = p.stoich_P[m][n] - p.stoich_R[m][n];
        }
        C.rate[m] = p.rate_const[m];
        C.nar[m] = -p.alpha_param[m] / p.Runiv;
        C.beta[m] = p.beta_param[m];
    }
    C.T0 = p.T0_chem;
    C.rT0 = 1 / p.T0_chem;
    C.navo = p.avogadro > 0 ? p.avogadro : p.Runiv / p.k_B;
    C.sq = std::sqrt(dt * dV);
    C.rR = 1.0 / p.Runiv;
    C.rnavo = 1.0 / C.navo;
    C.rsq = 1.0 / C.sq;
    const bool ok = div_divisor_ok(p.Runiv) && div_divisor_ok(C.T0) && div_divisor_ok(C.navo) && div_divisor_ok(C.sq);
    C.div_lo = kDivAlo;
    C.div_span = ok ? kDivAspan : 0u;
    return C;
}

FHD_D double chem_ipow(double c, int r) {
    if (r <= 0) return 1.0;
    double v = c;
    for (int q = 1; q < r; ++q) v = v * c;
    return v;
}

// source S_0..S_{NS-1} of one cell from p, T, X and the reaction noises W[m]
// (chemistry_functions.cpp:147-190)
template <int NS>
FHD_D void chem_point(const DevParams& P, const ChemParams& C, double pres, double T, const double (&X)[NS],
                      const double* W, double (&S)[NS]) {
    const double rT = 1 / T;
    const double ctot = div_rcp_any(div_rcp(pres, P.Runiv, C.rR, C.div_lo, C.div_span), T, rT);
    double ck[NS];
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        ck[n] = X[n] * ctot;
        S[n] = 0.;
    }
#pragma unroll 1
    for (int m = 0; m < C.nr; ++m) {
        double a = C.rate[m];
        a *= exp(C.nar[m] * (rT - C.rT0));
        a *= pow(div_rcp(T, C.T0, C.rT0, C.div_lo, C.div_span), C.beta[m]);
#pragma unroll
        for (int n = 0; n < NS; ++n) a *= chem_ipow(ck[n], C.sR[m][n]);
        a = (0. < a) ? a : 0.;  // std::max(0., a)
        const double Wm = div_rcp_z(W[m], C.sq, C.rsq, C.div_lo, C.div_span);
        const double fl = C.type == 1 ? sqrt(div_rcp_z(a, C.navo, C.rnavo, C.div_lo, C.div_span)) : 0.0;
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            S[n] += P.molmass[n] * (double)C.sPR[m][n] * a;
            if (C.type == 1) S[n] += P.molmass[n] * (double)C.sPR[m][n] * fl * Wm;
        }
    }
}

}  // namespace fhd
