// fhd_stats.cu — running statistics of the staggered state: the per-cell part of
// evaluateStatsStag3D (statsStag.cpp:10-77), i.e. EvaluateStatsMeans
// (statsStag.cpp:200-365) and EvaluateVarsCoVarsMom3 (:367-691) without surface
// coverage.  FP64 in the reference's operation order (this unit is built with
// -fmad=false), so the results equal the CPU restatement bit for bit.
//
// The reference's passes depend on neighbours' freshly updated means, so the
// update runs as three data-parallel passes, each writing only its own point:
//   k_stats_means_a: momentum means on valid faces, density mean on the cells
//                    grown by 2 (statsStag.cpp:215-256)
//   k_stats_means_b: the other cell means (:258-317) and the face-velocity
//                    means (:320-363), which read the new momentum/density means
//   [FillBoundary of cuMeans and primMeans]
//   k_stats_vars:    momentum/velocity variances on faces (:387-435), the cell
//                    variances and covariances (:438-613) and the third/fourth
//                    moments (:616-689)
//   [FillBoundary of cuVars and primVars]
//   k_sum_to_line, k_spatial_cross (FHD_STATS_CROSS): the yz-averaged spatial
//                    cross-correlations (statsStag.cpp:46-76)
// Every pass reads and writes each operand once per point: it is bound by HBM.
#include "fhd_launch.cuh"
#include "fhd_linesum.cuh"

namespace fhd {

struct StatsArgs {
    DevParams P;
    Arr4<const double> cu, prim, mom[3];
    Arr4<double> cum, cuv, pm, pv, cov, m3, m4;
    Arr4<double> vm[3], vv[3], mm[3], mv[3];
    double sm1, sinv;   // stepsminusone, stepsinv
    int mom3, mom4;     // plot_mom3 / plot_mom4
};

// pass A: one thread per point of the cell box grown by 2
static __global__ void __launch_bounds__(256) k_stats_means_a(StatsArgs a) {
    const int* n = a.P.n;
    const int gx = n[0] + 4, gy = n[1] + 4, gz = n[2] + 4;
    const int64_t tot = (int64_t)gx * gy * gz;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = int(q % gx) - 2, j = int((q / gx) % gy) - 2, k = int(q / ((int64_t)gx * gy)) - 2;
        // loads first, then the updates, then the stores (see pass B)
        const double r0 = a.cum(i, j, k, 0), u0 = a.cu(i, j, k, 0);
        bool on[3];
        double om[3], um[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            on[d] = !(i < 0 || j < 0 || k < 0 || i > n[0] - 1 + (d == 0) || j > n[1] - 1 + (d == 1) ||
                      k > n[2] - 1 + (d == 2));
            if (!on[d]) continue;
            om[d] = a.mm[d](i, j, k);
            um[d] = a.mom[d](i, j, k);
        }
        // mean density, also on the ghost cells (statsStag.cpp:245-256)
        a.cum(i, j, k, 0) = (r0 * a.sm1 + u0) * a.sinv;
        // mean momentum on valid faces (statsStag.cpp:228-241)
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (on[d]) a.mm[d](i, j, k) = (om[d] * a.sm1 + um[d]) * a.sinv;
    }
}

// pass B: one thread per point of [0, n]^3
template <int NS>
static __global__ void __launch_bounds__(256) k_stats_means_b(StatsArgs a) {
    const DevParams& P = a.P;
    const int* n = P.n;
    const int gx = n[0] + 1, gy = n[1] + 1, gz = n[2] + 1;
    const int nprim = 6 + 2 * NS;
    const int64_t tot = (int64_t)gx * gy * gz;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = int(q % gx), j = int((q / gx) % gy), k = int(q / ((int64_t)gx * gy));
        if (i < n[0] && j < n[1] && k < n[2]) {
            // cell means (statsStag.cpp:275-316).  Every operand is loaded before
            // the first store (the statistics are distinct arrays the compiler
            // cannot prove unaliased, so a load after a store would wait for it),
            // then the reference's arithmetic runs in its order, then all stores.
            const Arr4<double>& cm = a.cum;
            const Arr4<double>& pm = a.pm;
            const Arr4<double>&mxm = a.mm[0], &mym = a.mm[1], &mzm = a.mm[2];
            const double mx0 = mxm(i, j, k), mx1 = mxm(i + 1, j, k);
            const double my0 = mym(i, j, k), my1 = mym(i, j + 1, k);
            const double mz0 = mzm(i, j, k), mz1 = mzm(i, j, k + 1);
            const double rho = cm(i, j, k, 0);
            double c4 = cm(i, j, k, 4);
            const double u4 = a.cu(i, j, k, 4);
            double cs[NS], us[NS], px[NS], ux[NS], pc[3], uc[3];
#pragma unroll
            for (int l = 0; l < NS; ++l) {
                cs[l] = cm(i, j, k, 5 + l);
                us[l] = a.cu(i, j, k, 5 + l);
                px[l] = pm(i, j, k, 6 + NS + l);
                ux[l] = a.prim(i, j, k, 6 + NS + l);
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                pc[c] = pm(i, j, k, nprim + c);
                uc[c] = a.prim(i, j, k, 1 + c);
            }
            double pT = pm(i, j, k, 4);
            const double uT = a.prim(i, j, k, 4);
            // arithmetic, in the reference's order
            double fracvec[NS];
            const double c1 = 0.5 * (mx0 + mx1);
            const double c2 = 0.5 * (my0 + my1);
            const double c3 = 0.5 * (mz0 + mz1);
            c4 = (c4 * a.sm1 + u4) * a.sinv;
#pragma unroll
            for (int l = 0; l < NS; ++l) {
                cs[l] = (cs[l] * a.sm1 + us[l]) * a.sinv;
                fracvec[l] = cs[l] / rho;
            }
#pragma unroll
            for (int l = 0; l < NS; ++l) px[l] = (px[l] * a.sm1 + ux[l]) * a.sinv;
            const double densitymeaninv = 1.0 / rho;
            const double p1 = densitymeaninv * 0.5 * (mx0 + mx1);
            const double p2 = densitymeaninv * 0.5 * (my0 + my1);
            const double p3 = densitymeaninv * 0.5 * (mz0 + mz1);
#pragma unroll
            for (int c = 0; c < 3; ++c) pc[c] = (pc[c] * a.sm1 + uc[c]) * a.sinv;
            pT = (pT * a.sm1 + uT) * a.sinv;
            const double pp = GetPressureGas<NS, double>(P, fracvec, rho, pT);
            // stores
            cm(i, j, k, 1) = c1;
            cm(i, j, k, 2) = c2;
            cm(i, j, k, 3) = c3;
            cm(i, j, k, 4) = c4;
#pragma unroll
            for (int l = 0; l < NS; ++l) {
                cm(i, j, k, 5 + l) = cs[l];
                pm(i, j, k, 6 + l) = fracvec[l];
                pm(i, j, k, 6 + NS + l) = px[l];
            }
            pm(i, j, k, 1) = p1;
            pm(i, j, k, 2) = p2;
            pm(i, j, k, 3) = p3;
#pragma unroll
            for (int c = 0; c < 3; ++c) pm(i, j, k, nprim + c) = pc[c];
            pm(i, j, k, 0) = rho;
            pm(i, j, k, 4) = pT;
            pm(i, j, k, 5) = pp;
        }
        // face-velocity means (statsStag.cpp:343-362)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
            if (i > n[0] - 1 + e0 || j > n[1] - 1 + e1 || k > n[2] - 1 + e2) continue;
            const double densitymeaninv = 2.0 / (a.cum(i - e0, j - e1, k - e2, 0) + a.cum(i, j, k, 0));
            a.vm[d](i, j, k) = a.mm[d](i, j, k) * densitymeaninv;
        }
    }
}

// pass C: one thread per point of [0, n]^3.  As in pass B, operands are loaded in
// groups before the stores they feed, so each thread keeps many loads in flight.
template <int NS>
static __global__ void __launch_bounds__(256) k_stats_vars(StatsArgs a) {
    const DevParams& P = a.P;
    const int* n = P.n;
    const int gx = n[0] + 1, gy = n[1] + 1, gz = n[2] + 1;
    const int nvars = 5 + NS, nprim = 6 + 2 * NS;
    const int64_t tot = (int64_t)gx * gy * gz;
    const double sm1 = a.sm1, sinv = a.sinv;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = int(q % gx), j = int((q / gx) % gy), k = int(q / ((int64_t)gx * gy));
        const Arr4<const double>& cu = a.cu;
        const Arr4<double>& cm = a.cum;
        // momentum and velocity variances on faces (statsStag.cpp:416-435)
        {
            bool on[3];
            double fm[3], fmm[3], fmv[3], fvm[3], fvv[3], crl[3], crh[3], url[3], urh[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
                on[d] = !(i > n[0] - 1 + e0 || j > n[1] - 1 + e1 || k > n[2] - 1 + e2);
                if (!on[d]) continue;
                fm[d] = a.mom[d](i, j, k);
                fmm[d] = a.mm[d](i, j, k);
                fmv[d] = a.mv[d](i, j, k);
                fvm[d] = a.vm[d](i, j, k);
                fvv[d] = a.vv[d](i, j, k);
                crl[d] = cm(i - e0, j - e1, k - e2, 0);
                crh[d] = cm(i, j, k, 0);
                url[d] = cu(i - e0, j - e1, k - e2, 0);
                urh[d] = cu(i, j, k, 0);
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (!on[d]) continue;
                const double delj = fm[d] - fmm[d];
                fmv[d] = (fmv[d] * sm1 + delj * delj) * sinv;
                const double densitymeaninv = 2.0 / (crl[d] + crh[d]);
                const double delrho = 0.5 * (url[d] + urh[d]) - 0.5 * (crl[d] + crh[d]);
                const double delvel = (delj - fvm[d] * delrho) * densitymeaninv;
                fvv[d] = (fvv[d] * sm1 + delvel * delvel) * sinv;
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (!on[d]) continue;
                a.mv[d](i, j, k) = fmv[d];
                a.vv[d](i, j, k) = fvv[d];
            }
        }
        if (i >= n[0] || j >= n[1] || k >= n[2]) continue;
        // cell variances and covariances (statsStag.cpp:474-613)
        const Arr4<double>&cv = a.cuv, &pv = a.pv, &co = a.cov;
        const Arr4<double>& pm = a.pm;
        // group 1: the state and the means
        const double cu0 = cu(i, j, k, 0), cm0 = cm(i, j, k, 0), cu4 = cu(i, j, k, 4), cm4 = cm(i, j, k, 4);
        double cus[NS], cms[NS], pmY[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            cus[s] = cu(i, j, k, 5 + s);
            cms[s] = cm(i, j, k, 5 + s);
            pmY[s] = pm(i, j, k, 6 + s);
        }
        const double vxm0 = a.vm[0](i, j, k), vxm1 = a.vm[0](i + 1, j, k);
        const double vym0 = a.vm[1](i, j, k), vym1 = a.vm[1](i, j + 1, k);
        const double vzm0 = a.vm[2](i, j, k), vzm1 = a.vm[2](i, j, k + 1);
        const double mx0 = a.mom[0](i, j, k), mx1 = a.mom[0](i + 1, j, k);
        const double my0 = a.mom[1](i, j, k), my1 = a.mom[1](i, j + 1, k);
        const double mz0 = a.mom[2](i, j, k), mz1 = a.mom[2](i, j, k + 1);
        const double mxm0 = a.mm[0](i, j, k), mxm1 = a.mm[0](i + 1, j, k);
        const double mym0 = a.mm[1](i, j, k), mym1 = a.mm[1](i, j + 1, k);
        const double mzm0 = a.mm[2](i, j, k), mzm1 = a.mm[2](i, j, k + 1);
        const double T = pm(i, j, k, 4);
        const double pT = a.prim(i, j, k, 4);
        // the fluctuations (statsStag.cpp:474-541)
        const double delrho = cu0 - cm0;
        const double delenergy = cu4 - cm4;
        double delrhoYk[NS], delYk[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            delrhoYk[s] = cus[s] - cms[s];
            delYk[s] = (delrhoYk[s] - pmY[s] * delrho) / cm0;
        }
        const double vx = 0.5 * (vxm0 + vxm1);
        const double vy = 0.5 * (vym0 + vym1);
        const double vz = 0.5 * (vzm0 + vzm1);
        const double densitymeaninv = 1.0 / cm0;
        double cvm = 0.;
#pragma unroll
        for (int l = 0; l < NS; ++l) cvm = cvm + P.hcv[l] * cms[l] / cm0;
        const double cvinv = 1.0 / cvm;
        const double qmean = cvm * T - 0.5 * (vx * vx + vy * vy + vz * vz);
        const double deljx = 0.5 * (mx0 + mx1) - 0.5 * (mxm0 + mxm1);
        const double deljy = 0.5 * (my0 + my1) - 0.5 * (mym0 + mym1);
        const double deljz = 0.5 * (mz0 + mz1) - 0.5 * (mzm0 + mzm1);
        const double delvelx = (deljx - vx * delrho) * densitymeaninv;
        const double delvely = (deljy - vy * delrho) * densitymeaninv;
        const double delvelz = (deljz - vz * delrho) * densitymeaninv;
        const double delg = vx * deljx + vy * deljy + vz * deljz;
        const double delT = pT - T;
        const double deltemp = delT;
        // group 2: the variances
        {
            double ocv[5 + NS], opv[5], opY[NS], opn[5];
#pragma unroll
            for (int c = 0; c < nvars; ++c) ocv[c] = cv(i, j, k, c);
#pragma unroll
            for (int c = 1; c < 5; ++c) opv[c] = pv(i, j, k, c);
#pragma unroll
            for (int s = 0; s < NS; ++s) opY[s] = pv(i, j, k, 6 + s);
#pragma unroll
            for (int c = 0; c < 5; ++c) opn[c] = pv(i, j, k, nprim + c);
            ocv[0] = (ocv[0] * sm1 + delrho * delrho) * sinv;
            ocv[4] = (ocv[4] * sm1 + delenergy * delenergy) * sinv;
#pragma unroll
            for (int l = 5; l < nvars; ++l) {
                const double delmassvec = cus[l - 5] - cms[l - 5];
                ocv[l] = (ocv[l] * sm1 + delmassvec * delmassvec) * sinv;
            }
#pragma unroll
            for (int s = 0; s < NS; ++s) opY[s] = (opY[s] * sm1 + delYk[s] * delYk[s]) * sinv;
            ocv[1] = (ocv[1] * sm1 + deljx * deljx) * sinv;
            ocv[2] = (ocv[2] * sm1 + deljy * deljy) * sinv;
            ocv[3] = (ocv[3] * sm1 + deljz * deljz) * sinv;
            opv[1] = (opv[1] * sm1 + delvelx * delvelx) * sinv;
            opv[2] = (opv[2] * sm1 + delvely * delvely) * sinv;
            opv[3] = (opv[3] * sm1 + delvelz * delvelz) * sinv;
            opn[0] = (opn[0] * sm1 + delg * delg) * sinv;
            opn[1] = (opn[1] * sm1 + delg * delenergy) * sinv;
            opn[2] = (opn[2] * sm1 + delrho * delenergy) * sinv;
            opn[3] = (opn[3] * sm1 + delrho * delg) * sinv;
            opn[4] = (opn[4] * sm1 + cvinv * cvinv * densitymeaninv * densitymeaninv *
                                         (ocv[4] + opn[0] - 2 * opn[1] +
                                          qmean * (qmean * ocv[0] - 2 * opn[2] + 2 * opn[3]))) *
                     sinv;
            opv[4] = (opv[4] * sm1 + delT * delT) * sinv;
#pragma unroll
            for (int c = 0; c < nvars; ++c) cv(i, j, k, c) = ocv[c];
            pv(i, j, k, 0) = ocv[0];
#pragma unroll
            for (int c = 1; c < 5; ++c) pv(i, j, k, c) = opv[c];
#pragma unroll
            for (int s = 0; s < NS; ++s) pv(i, j, k, 6 + s) = opY[s];
#pragma unroll
            for (int c = 0; c < 5; ++c) pv(i, j, k, nprim + c) = opn[c];
        }
        // group 3: the covariances (statsStag.cpp:560-585)
        {
            const double cterm[26] = {delrho * deljx, delrho * deljy, delrho * deljz, deljx * deljy, deljy * deljz,
                                      deljx * deljz, delrho * delenergy, deljx * delenergy, deljy * delenergy,
                                      deljz * delenergy, delrhoYk[0] * delrhoYk[NS - 1], delrho * delvelx,
                                      delrho * delvely, delrho * delvelz, delvelx * delvely, delvely * delvelz,
                                      delvelx * delvelz, delrho * deltemp, delvelx * deltemp, delvely * deltemp,
                                      delvelz * deltemp, delYk[0] * delYk[NS - 1], delYk[0] * delvelx,
                                      delYk[NS - 1] * delvelx, delrhoYk[0] * delvelx, delrhoYk[NS - 1] * delvelx};
            double oco[26];
#pragma unroll
            for (int c = 0; c < 26; ++c) oco[c] = co(i, j, k, c);
#pragma unroll
            for (int c = 0; c < 26; ++c) co(i, j, k, c) = (oco[c] * sm1 + cterm[c]) * sinv;
        }
        // group 4: third and fourth moments (statsStag.cpp:639-688); their recomputed
        // inputs equal the values above
        if (a.mom3 || a.mom4) {
            const double dv[3] = {delvelx, delvely, delvelz};
            double o3[6 + NS], o4[6 + NS];
#pragma unroll
            for (int c = 0; c < 6 + NS; ++c) {
                if (a.mom3) o3[c] = a.m3(i, j, k, c);
                if (a.mom4) o4[c] = a.m4(i, j, k, c);
            }
            if (a.mom3) {
                o3[0] = (o3[0] * sm1 + delrho * delrho * delrho) * sinv;
                o3[4] = (o3[4] * sm1 + delenergy * delenergy * delenergy) * sinv;
#pragma unroll
                for (int s = 0; s < NS; ++s) o3[5 + s] = (o3[5 + s] * sm1 + delYk[s] * delYk[s] * delYk[s]) * sinv;
#pragma unroll
                for (int c = 0; c < 3; ++c) o3[1 + c] = (o3[1 + c] * sm1 + dv[c] * dv[c] * dv[c]) * sinv;
                o3[5 + NS] = (o3[5 + NS] * sm1 + delT * delT * delT) * sinv;
#pragma unroll
                for (int c = 0; c < 6 + NS; ++c) a.m3(i, j, k, c) = o3[c];
            }
            if (a.mom4) {
                o4[0] = (o4[0] * sm1 + delrho * delrho * delrho * delrho) * sinv;
                o4[4] = (o4[4] * sm1 + delenergy * delenergy * delenergy * delenergy) * sinv;
#pragma unroll
                for (int s = 0; s < NS; ++s)
                    o4[5 + s] = (o4[5 + s] * sm1 + delYk[s] * delYk[s] * delYk[s] * delYk[s]) * sinv;
#pragma unroll
                for (int c = 0; c < 3; ++c) o4[1 + c] = (o4[1 + c] * sm1 + dv[c] * dv[c] * dv[c] * dv[c]) * sinv;
                o4[5 + NS] = (o4[5 + NS] * sm1 + delT * delT * delT * delT) * sinv;
#pragma unroll
                for (int c = 0; c < 6 + NS; ++c) a.m4(i, j, k, c) = o4[c];
            }
        }
    }
}

template <int NS>
static int stats_launch(const StatsArgs& a, bool means, bool vars, const fhd_fab& cuMeans,
                        const fhd_fab& primMeans, const fhd_fab& cuVars, const fhd_fab& primVars, cudaStream_t s) {
    const int* n = a.P.n;
    const int64_t ga = (int64_t)(n[0] + 4) * (n[1] + 4) * (n[2] + 4);
    const int64_t gb = (int64_t)(n[0] + 1) * (n[1] + 1) * (n[2] + 1);
    if (means) {
        k_stats_means_a<<<grid_for(ga, 256), 256, 0, s>>>(a);
        k_stats_means_b<NS><<<grid_for(gb, 256), 256, 0, s>>>(a);
        const GhostReq g[2] = {{cuMeans, 0, cuMeans.ncomp}, {primMeans, 0, primMeans.ncomp}};
        const int rc = fill_ghosts(g, 2, n, s, a.P.periodic, 0);
        if (rc) return rc;
    }
    if (vars) {
        k_stats_vars<NS><<<grid_for(gb, 256), 256, 0, s>>>(a);
        const GhostReq g[2] = {{cuVars, 0, cuVars.ncomp}, {primVars, 0, primVars.ncomp}};
        const int rc = fill_ghosts(g, 2, n, s, a.P.periodic, 0);
        if (rc) return rc;
    }
    return cuda_rc(cudaGetLastError());
}

// ---- plot_cross: the yz-averaged spatial cross-correlations ------------------------------
// evaluateStatsStag3D's x-line averages (statsStag.cpp:46-74) and
// EvaluateSpatialCorrelations3D (:868-1105), after the means and variances.
//
// The four sumToLine results (cu and cuMeans components 0..nvars-1, prim and
// primMeans components 1..nspecies+4) along x, each entry (i, n) its y-z plane summed
// with k outer and j inner and divided by n_cells[1]*n_cells[2]: k_sum_to_line
// (fhd_linesum.cuh).

// k_spatial_cross: one thread per x cell i updates spatialCross(i, 0..ncross-1) in
// the reference's statement order (a later entry reads the earlier entries' new
// values); every thread derives the x* quantities from the same line entries, and
// thread 0 also stores them as dataSliceMeans_xcross.  The reference's "Y_k" of the
// lines is entry 4+k of the prim line, i.e. prim component 5+k (pressure for k = 0);
// the update of entries 37+nspecies+1 and +2 re-applies the running-average update
// to entries 37 and 37+nspecies-1 that were already updated this step.  Both kept.
struct CrossArgs {
    const double *cu, *cum, *pr, *pm;   // lines: cu/cuMeans nvars per i, prim/primMeans nspecies+4 per i
    double* S;                          // spatialCross, ncross per i
    double* xcross;                     // dataSliceMeans_xcross (nstats)
    double hcv[MAXS];
    int nx, cc, ncross;
    double sm1, sinv;                   // stepsminusone, stepsinv
};

// The x* quantities and this cell's (or x line's) fluctuations that every
// correlation update reads (statsStag.cpp:913-1004 in 3-D, :1363-1437 in 1-D).
template <int NS>
struct CrossStar {
    double meanrho, meanux, meanYk[NS], delrhoYk[NS], delYk[NS];
    double delrho, delK, deljx, deljy, deljz, delT, delvx, cvinv, qmean, delG;
};
template <int NS>
struct CrossHere {
    double meanrho, meanYk[NS], delrhoYk[NS], delYk[NS];
    double delrho, delK, deljx, deljy, deljz, delT, delvx, cvinv, qmean, delG;
};

// the x* quantities from the 18 + 4 nspecies entries of data_xcross
template <int NS>
FHD_D CrossStar<NS> cross_star(const double* dx, const double* hcv) {
    CrossStar<NS> c;
    c.meanrho = dx[1];
    c.meanux = dx[11];
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        c.meanYk[n] = dx[18 + 4 * n + 3];
        c.delrhoYk[n] = dx[18 + 4 * n + 0] - dx[18 + 4 * n + 1];
        c.delYk[n] = dx[18 + 4 * n + 2] - dx[18 + 4 * n + 3];
    }
    c.delrho = dx[0] - dx[1];
    c.delK = dx[2] - dx[3];
    c.deljx = dx[4] - dx[5];
    c.deljy = dx[6] - dx[7];
    c.deljz = dx[8] - dx[9];
    c.delT = dx[16] - dx[17];
    c.delvx = dx[10] - dx[11];
    double cv = 0.;
#pragma unroll
    for (int l = 0; l < NS; ++l) cv = cv + hcv[l] * dx[18 + 4 * l + 1] / dx[1];
    c.cvinv = 1.0 / cv;
    c.qmean = cv * dx[17] - 0.5 * (dx[11] * dx[11] + dx[13] * dx[13] + dx[15] * dx[15]);
    c.delG = dx[11] * (dx[4] - dx[5]) + dx[13] * (dx[6] - dx[7]) + dx[15] * (dx[8] - dx[9]);
    return c;
}

// The running averages and derived correlations of one point, entries S(0..ncross-1)
// at stride qs, in the reference's statement order (a later entry reads the earlier
// entries' new values; statsStag.cpp:1007-1104 and :1441-1551 are the same
// statements).  Two reference quirks are kept: the "Y_k" the caller passes, and
// entries 37+nspecies+1 and +2 re-applying the update of entries 37 and
// 37+nspecies-1 that were already updated in the same step.
template <int NS>
FHD_D void cross_update(double* S, int64_t qs, const CrossStar<NS>& x, const CrossHere<NS>& h, double sm1,
                        double sinv) {
    constexpr int H = NS - 1;
    auto at = [&](int q) -> double& { return S[q * qs]; };
    auto upd = [&](int q, double v) { at(q) = (at(q) * sm1 + v) * sinv; };
    upd(0, x.delrho * h.delrho);
    upd(1, x.delK * h.delK);
    upd(2, x.deljx * h.deljx);
    upd(3, x.deljy * h.deljy);
    upd(4, x.deljz * h.deljz);
    upd(5, x.deljx * h.delrho);
    upd(6, x.deljx * h.delrhoYk[0]);
    upd(7, x.deljx * h.delrhoYk[H]);
    upd(8, x.delrho * h.delrhoYk[0]);
    upd(9, x.delrho * h.delrhoYk[H]);
    upd(10, x.delrhoYk[0] * h.delrho);
    upd(11, x.delrhoYk[H] * h.delrho);
    upd(12, x.delG * h.delG);
    upd(13, x.delG * h.delK);
    upd(14, x.delK * h.delG);
    upd(15, x.delrho * h.delK);
    upd(16, x.delK * h.delrho);
    upd(17, x.delrho * h.delG);
    upd(18, x.delG * h.delrho);
    const double meanrhocross = x.meanrho, meanrho = h.meanrho, meanuxcross = x.meanux;
    const double qmeancross = x.qmean, qmean = h.qmean;
    at(19) = (x.cvinv * h.cvinv / (meanrhocross * meanrho)) *
             (at(1) + at(12) - at(13) - at(14) + qmean * qmeancross * at(0) - qmeancross * at(15) - qmean * at(16) +
              qmeancross * at(17) + qmean * at(18));
    at(20) = (x.cvinv / meanrhocross) * (at(16) - at(18) - qmeancross * at(0));
    at(21) = (1.0 / meanrhocross) * (at(5) - meanuxcross * at(0));
    at(22) = (1.0 / meanrhocross) * (at(6) - meanuxcross * at(8));
    at(23) = (1.0 / meanrhocross) * (at(7) - meanuxcross * at(9));
    at(24) = (1.0 / (meanrho * meanrhocross)) *
             (at(6) - meanuxcross * at(8) - h.meanYk[0] * at(5) + meanuxcross * h.meanYk[0] * at(0));
    at(25) = (1.0 / (meanrho * meanrhocross)) *
             (at(7) - meanuxcross * at(9) - h.meanYk[H] * at(5) + meanuxcross * h.meanYk[H] * at(0));
    upd(26, x.delT * h.delT);
    upd(27, x.delT * h.delrho);
    upd(28, x.delT * h.delvx);
    upd(29, x.delvx * h.delrho);
    upd(30, x.delvx * h.delYk[0]);
    upd(31, x.delvx * h.delYk[H]);
    upd(32, x.delvx * h.delrhoYk[0]);
    upd(33, x.delvx * h.delrhoYk[H]);
    upd(34, x.delYk[0] * h.delYk[0]);
    upd(35, x.delYk[H] * h.delYk[H]);
    upd(36, x.delYk[0] * h.delYk[H]);
#pragma unroll
    for (int n = 0; n < NS; ++n) upd(37 + n, x.delrhoYk[n] * h.delrhoYk[n]);
    upd(37 + NS, x.delrhoYk[H] * h.delrhoYk[0]);
    double dd = (at(37) * sm1 + x.delrhoYk[0] * h.delrhoYk[0]) * sinv;
    at(37 + NS + 1) = (1.0 / (meanrho * meanrhocross)) *
                      (dd - x.meanYk[0] * at(8) - h.meanYk[0] * at(10) + x.meanYk[0] * h.meanYk[0] * at(0));
    dd = (at(37 + H) * sm1 + x.delrhoYk[H] * h.delrhoYk[H]) * sinv;
    at(37 + NS + 2) = (1.0 / (meanrho * meanrhocross)) *
                      (dd - x.meanYk[H] * at(9) - h.meanYk[H] * at(11) + x.meanYk[H] * h.meanYk[H] * at(0));
}

template <int NS>
static __global__ void __launch_bounds__(128) k_spatial_cross(CrossArgs a) {
    constexpr int NV = 5 + NS, NP = NS + 4;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nx) return;
    // data_xcross (statsStag.cpp:886-911)
    double dx[18 + 4 * NS];
    {
        const double *cu = a.cu + (int64_t)NV * a.cc, *cm = a.cum + (int64_t)NV * a.cc;
        const double *pr = a.pr + (int64_t)NP * a.cc, *pm = a.pm + (int64_t)NP * a.cc;
        dx[0] = cu[0];  dx[1] = cm[0];  dx[2] = cu[4];  dx[3] = cm[4];
        dx[4] = cu[1];  dx[5] = cm[1];  dx[6] = cu[2];  dx[7] = cm[2];
        dx[8] = cu[3];  dx[9] = cm[3];
        dx[10] = pr[0]; dx[11] = pm[0]; dx[12] = pr[1]; dx[13] = pm[1];
        dx[14] = pr[2]; dx[15] = pm[2]; dx[16] = pr[3]; dx[17] = pm[3];
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            dx[18 + 4 * n + 0] = cu[5 + n];
            dx[18 + 4 * n + 1] = cm[5 + n];
            dx[18 + 4 * n + 2] = pr[4 + n];
            dx[18 + 4 * n + 3] = pm[4 + n];
        }
    }
    if (i == 0)
        for (int q = 0; q < 18 + 4 * NS; ++q) a.xcross[q] = dx[q];
    const CrossStar<NS> x = cross_star<NS>(dx, a.hcv);
    // the x line's quantities (:966-1004); its "Y_k" are the prim line's entries 4+k
    const double *cu = a.cu + (int64_t)NV * i, *cm = a.cum + (int64_t)NV * i;
    const double *pr = a.pr + (int64_t)NP * i, *pm = a.pm + (int64_t)NP * i;
    CrossHere<NS> h;
    h.meanrho = cm[0];
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        h.meanYk[n] = pm[4 + n];
        h.delrhoYk[n] = cu[5 + n] - cm[5 + n];
        h.delYk[n] = pr[4 + n] - pm[4 + n];
    }
    h.delrho = cu[0] - cm[0];
    h.delK = cu[4] - cm[4];
    h.deljx = cu[1] - cm[1];
    h.deljy = cu[2] - cm[2];
    h.deljz = cu[3] - cm[3];
    h.delT = pr[3] - pm[3];
    h.delvx = pr[0] - pm[0];
    double cv = 0.;
#pragma unroll
    for (int l = 0; l < NS; ++l) cv = cv + a.hcv[l] * cm[5 + l] / cm[0];
    h.cvinv = 1.0 / cv;
    h.qmean = cv * pm[3] - 0.5 * (pm[0] * pm[0] + pm[1] * pm[1] + pm[2] * pm[2]);
    h.delG = pm[0] * h.deljx + pm[1] * h.deljy + pm[2] * h.deljz;
    cross_update<NS>(a.S + (int64_t)a.ncross * i, 1, x, h, a.sm1, a.sinv);
}

// ---- quasi-1-D: correlations along each y-z pencil (evaluateStatsStag1D) -------------
// One thread per valid cell; its pencil's cell at x* gives the x* quantities
// (GetPencilCross, statsStag.cpp:830-858: cu 0..4 and 5+k, cuMeans likewise, prim and
// primMeans 1..4 and 6+k) and the cell its own (EvaluateSpatialCorrelations1D,
// :1363-1437: momenta and velocities averaged from the faces, the velocity means
// from velMeans); the updates are the 3-D ones (:1441-1551) on spatialCrossMF
// components star*ncross.. (a cell-centred fab without ghosts).
struct Cross1DArgs {
    Arr4<const double> cu, cum, pr, pm, mom[3], mm[3], velx, vm[3];
    double* S;            // spatialCrossMF component 0 at cell (0, 0, 0)
    int64_t qs;           // component stride (cells of the box)
    int nx, ny, nz, xs, mf;   // x*, first component star*ncross
    double hcv[MAXS];
    double sm1, sinv;
};

template <int NS>
static __global__ void __launch_bounds__(128) k_cross_1d(Cross1DArgs a) {
    const int64_t tot = (int64_t)a.nx * a.ny * a.nz;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % a.nx), j = (int)((q / a.nx) % a.ny), k = (int)(q / ((int64_t)a.nx * a.ny));
        const int xs = a.xs;
        double dx[18 + 4 * NS];
        dx[0] = a.cu(xs, j, k, 0);  dx[1] = a.cum(xs, j, k, 0);
        dx[2] = a.cu(xs, j, k, 4);  dx[3] = a.cum(xs, j, k, 4);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            dx[4 + 2 * d] = a.cu(xs, j, k, 1 + d);
            dx[5 + 2 * d] = a.cum(xs, j, k, 1 + d);
        }
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            dx[10 + 2 * d] = a.pr(xs, j, k, 1 + d);
            dx[11 + 2 * d] = a.pm(xs, j, k, 1 + d);
        }
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            dx[18 + 4 * n + 0] = a.cu(xs, j, k, 5 + n);
            dx[18 + 4 * n + 1] = a.cum(xs, j, k, 5 + n);
            dx[18 + 4 * n + 2] = a.pr(xs, j, k, 6 + n);
            dx[18 + 4 * n + 3] = a.pm(xs, j, k, 6 + n);
        }
        const CrossStar<NS> x = cross_star<NS>(dx, a.hcv);
        CrossHere<NS> h;
        h.meanrho = a.cum(i, j, k, 0);
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            h.meanYk[n] = a.pm(i, j, k, 6 + n);
            h.delrhoYk[n] = a.cu(i, j, k, 5 + n) - a.cum(i, j, k, 5 + n);
            h.delYk[n] = a.pr(i, j, k, 6 + n) - a.pm(i, j, k, 6 + n);
        }
        h.delrho = a.cu(i, j, k, 0) - a.cum(i, j, k, 0);
        h.delK = a.cu(i, j, k, 4) - a.cum(i, j, k, 4);
        h.deljx = 0.5 * (a.mom[0](i, j, k) + a.mom[0](i + 1, j, k)) - 0.5 * (a.mm[0](i, j, k) + a.mm[0](i + 1, j, k));
        h.deljy = 0.5 * (a.mom[1](i, j, k) + a.mom[1](i, j + 1, k)) - 0.5 * (a.mm[1](i, j, k) + a.mm[1](i, j + 1, k));
        h.deljz = 0.5 * (a.mom[2](i, j, k) + a.mom[2](i, j, k + 1)) - 0.5 * (a.mm[2](i, j, k) + a.mm[2](i, j, k + 1));
        h.delT = a.pr(i, j, k, 4) - a.pm(i, j, k, 4);
        h.delvx = 0.5 * (a.velx(i, j, k) + a.velx(i + 1, j, k)) - 0.5 * (a.vm[0](i, j, k) + a.vm[0](i + 1, j, k));
        double cv = 0.;
#pragma unroll
        for (int l = 0; l < NS; ++l) cv = cv + a.hcv[l] * a.cum(i, j, k, 5 + l) / a.cum(i, j, k, 0);
        h.cvinv = 1.0 / cv;
        const double vxmean = 0.5 * (a.vm[0](i, j, k) + a.vm[0](i + 1, j, k));
        const double vymean = 0.5 * (a.vm[1](i, j, k) + a.vm[1](i, j + 1, k));
        const double vzmean = 0.5 * (a.vm[2](i, j, k) + a.vm[2](i, j, k + 1));
        h.qmean = cv * a.pm(i, j, k, 4) - 0.5 * (vxmean * vxmean + vymean * vymean + vzmean * vzmean);
        h.delG = vxmean * h.deljx + vymean * h.deljy + vzmean * h.deljz;
        cross_update<NS>(a.S + (int64_t)a.mf * a.qs + q, a.qs, x, h, a.sm1, a.sinv);
    }
}

template <int NS>
static int cross_launch(const DevParams& P, const fhd_fab& cu, const fhd_fab& prim, const fhd_stats& st,
                        int cross_cell, double sm1, double sinv, double* lines, cudaStream_t s) {
    constexpr int NV = 5 + NS, NP = NS + 4;
    const int nx = P.n[0];
    LineArgs la;
    double* L[4] = {lines, lines + (int64_t)NV * nx, lines + (int64_t)2 * NV * nx,
                    lines + (int64_t)(2 * NV + NP) * nx};
    int q = 0;
    for (int n = 0; n < NV; ++n) la.job[q++] = line_job_dir(cu, n, 0, L[0] + n, NV);
    for (int n = 0; n < NV; ++n) la.job[q++] = line_job_dir(st.cuMeans, n, 0, L[1] + n, NV);
    for (int n = 0; n < NP; ++n) la.job[q++] = line_job_dir(prim, 1 + n, 0, L[2] + n, NP);
    for (int n = 0; n < NP; ++n) la.job[q++] = line_job_dir(st.primMeans, 1 + n, 0, L[3] + n, NP);
    la.njobs = q;
    const int rc = launch_line_sums(la, P.n, 0, s);
    if (rc) return rc;
    CrossArgs ca;
    ca.cu = L[0];
    ca.cum = L[1];
    ca.pr = L[2];
    ca.pm = L[3];
    ca.S = st.spatialCross;
    ca.xcross = st.dataSliceMeans_xcross;
    for (int n = 0; n < MAXS; ++n) ca.hcv[n] = n < NS ? P.hcv[n] : 0.0;
    ca.nx = nx;
    ca.cc = cross_cell;
    ca.ncross = 37 + NS + 3;
    ca.sm1 = sm1;
    ca.sinv = sinv;
    k_spatial_cross<NS><<<(nx + 127) / 128, 128, 0, s>>>(ca);
    return cuda_rc(cudaGetLastError());
}

// quasi-1-D: one launch per x*, in the reference's order (statsStag.cpp:168-193)
template <int NS>
static int cross1d_launch(const DevParams& P, const fhd_fab& cu, const fhd_fab& prim, const fhd_fab vel[3],
                          const fhd_fab mom[3], const fhd_stats& st, const int* stars, int nstars, double sm1,
                          double sinv, cudaStream_t s) {
    Cross1DArgs a;
    a.cu = view<const double>(cu);
    a.cum = view<const double>(st.cuMeans);
    a.pr = view<const double>(prim);
    a.pm = view<const double>(st.primMeans);
    for (int d = 0; d < 3; ++d) {
        a.mom[d] = view<const double>(mom[d]);
        a.mm[d] = view<const double>(st.cumomMeans[d]);
        a.vm[d] = view<const double>(st.velMeans[d]);
    }
    a.velx = view<const double>(vel[0]);
    a.S = st.spatialCross;
    a.nx = P.n[0];
    a.ny = P.n[1];
    a.nz = P.n[2];
    a.qs = (int64_t)a.nx * a.ny * a.nz;
    for (int n = 0; n < MAXS; ++n) a.hcv[n] = n < NS ? P.hcv[n] : 0.0;
    a.sm1 = sm1;
    a.sinv = sinv;
    for (int q = 0; q < nstars; ++q) {
        a.xs = stars[q];
        a.mf = q * (37 + NS + 3);
        k_cross_1d<NS><<<grid_for(a.qs, 128), 128, 0, s>>>(a);
    }
    return cuda_rc(cudaGetLastError());
}

// doubles of the x-line scratch of FHD_STATS_CROSS
int64_t stats_line_doubles(int ns, int nx) { return (int64_t)(2 * (5 + ns) + 2 * (ns + 4)) * nx; }

int exact_stats(const DevParams& P, const fhd_fab& cu, const fhd_fab& prim, const fhd_fab vel[3], const fhd_fab mom[3],
                const fhd_stats& st, int64_t steps, int flags, const int* stars, int nstars, double* lines,
                cudaStream_t s) {
    StatsArgs a;
    a.P = P;
    a.cu = view<const double>(cu);
    a.prim = view<const double>(prim);
    a.cum = view<double>(st.cuMeans);
    a.cuv = view<double>(st.cuVars);
    a.pm = view<double>(st.primMeans);
    a.pv = view<double>(st.primVars);
    a.cov = view<double>(st.coVars);
    a.m3 = view<double>(st.mom3);
    a.m4 = view<double>(st.mom4);
    for (int d = 0; d < 3; ++d) {
        a.mom[d] = view<const double>(mom[d]);
        a.vm[d] = view<double>(st.velMeans[d]);
        a.vv[d] = view<double>(st.velVars[d]);
        a.mm[d] = view<double>(st.cumomMeans[d]);
        a.mv[d] = view<double>(st.cumomVars[d]);
    }
    // statsStag.cpp:211-212 (and :383-384): computed on the host in the same order
    a.sm1 = (double)steps - 1.;
    a.sinv = 1. / (double)steps;
    const bool means = flags & FHD_STATS_MEANS, vars = flags & FHD_STATS_VARS;
    a.mom3 = vars && (flags & FHD_STATS_MOM3);
    a.mom4 = vars && (flags & FHD_STATS_MOM4);
    int rc;
    switch (P.ns) {
        case 1: rc = stats_launch<1>(a, means, vars, st.cuMeans, st.primMeans, st.cuVars, st.primVars, s); break;
        case 2: rc = stats_launch<2>(a, means, vars, st.cuMeans, st.primMeans, st.cuVars, st.primVars, s); break;
        case 3: rc = stats_launch<3>(a, means, vars, st.cuMeans, st.primMeans, st.cuVars, st.primVars, s); break;
        case 4: rc = stats_launch<4>(a, means, vars, st.cuMeans, st.primMeans, st.cuVars, st.primVars, s); break;
        default: return FHD_ERR_UNSUPPORTED;
    }
    // evaluateStatsStag2D has no correlations
    if (rc || !(flags & FHD_STATS_CROSS) || P.dim == 2) return rc;
    if (P.dim == 1) {
        switch (P.ns) {
            case 1: return cross1d_launch<1>(P, cu, prim, vel, mom, st, stars, nstars, a.sm1, a.sinv, s);
            case 2: return cross1d_launch<2>(P, cu, prim, vel, mom, st, stars, nstars, a.sm1, a.sinv, s);
            case 3: return cross1d_launch<3>(P, cu, prim, vel, mom, st, stars, nstars, a.sm1, a.sinv, s);
            default: return cross1d_launch<4>(P, cu, prim, vel, mom, st, stars, nstars, a.sm1, a.sinv, s);
        }
    }
    switch (P.ns) {
        case 1: return cross_launch<1>(P, cu, prim, st, stars[0], a.sm1, a.sinv, lines, s);
        case 2: return cross_launch<2>(P, cu, prim, st, stars[0], a.sm1, a.sinv, lines, s);
        case 3: return cross_launch<3>(P, cu, prim, st, stars[0], a.sm1, a.sinv, lines, s);
        default: return cross_launch<4>(P, cu, prim, st, stars[0], a.sm1, a.sinv, lines, s);
    }
}

}  // namespace fhd
