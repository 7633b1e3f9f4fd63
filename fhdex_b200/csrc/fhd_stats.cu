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
// Every pass reads and writes each operand once per point: it is bound by HBM.
#include "fhd_launch.cuh"

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

int exact_stats(const DevParams& P, const fhd_fab& cu, const fhd_fab& prim, const fhd_fab mom[3],
                const fhd_stats& st, int64_t steps, int flags, cudaStream_t s) {
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
    switch (P.ns) {
        case 1: return stats_launch<1>(a, means, vars, st.cuMeans, st.primMeans, st.cuVars, st.primVars, s);
        case 2: return stats_launch<2>(a, means, vars, st.cuMeans, st.primMeans, st.cuVars, st.primVars, s);
        case 3: return stats_launch<3>(a, means, vars, st.cuMeans, st.primMeans, st.cuVars, st.primVars, s);
        case 4: return stats_launch<4>(a, means, vars, st.cuMeans, st.primMeans, st.cuVars, st.primVars, s);
        default: return FHD_ERR_UNSUPPORTED;
    }
}

}  // namespace fhd
