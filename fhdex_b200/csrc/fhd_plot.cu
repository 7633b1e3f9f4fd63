// fhd_plot.cu — WritePlotFileStag (writePlotFileStag.cpp:7-527): the plotfile
// MultiFab the reference assembles from the state, the transport coefficients and
// the running statistics, and its AMReX plotfile on disk.
//
// Composition: every plotfile component is a copy of one component of one source
// MultiFab (MultiFab::Copy for cell fields, ShiftFaceToCC for face fields, which
// copies face (i,j,k) to cell (i,j,k), ConvertStag.cpp:167-191), in the order and
// under the names of writePlotFileStag.cpp:111-447.  One gather kernel writes all
// of them through a table of per-component source views: block (z-plane,
// component) copies the plane's rows, threads along x, so reads and writes are
// contiguous and the indexing is 32-bit with no divisions.
// plot_deltaY_dir (writePlotFileStag.cpp:282-290) appends Y_k minus its plane
// average (WriteHorizontalAverageToMF, ComputeAverages.cpp:96-190): one thread per
// (plane, species) sums the plane in the reference's loop order (k, j, i) so the
// average is bitwise the reference's, then (-average) + Y_k is written, as
// Ybar.mult(-1) and MultiFab::Add leave it.  Not covered: surface coverage.
//
// On disk (AMReX's single-level plotfile layout, as WriteSingleLevelPlotfile
// writes it for one box): <dir>/Header (text: "HyperCLaw-V1.1", component count
// and names, dimension, time, finest level 0, prob_lo, prob_hi, an empty
// refinement-ratio line, the domain box, the step, the cell sizes, coordinate
// system 0, boundary width 0, then the level's box list in physical coordinates
// and the path "Level_0/Cell"), <dir>/Level_0/Cell_H (the VisMF header of the
// one-box MultiFab with its per-component minima and maxima) and
// <dir>/Level_0/Cell_D_00000 (one FAB: a text descriptor line for little-endian
// IEEE doubles, then the data, components slowest, x fastest).
#include <cstdio>
#include <string>
#include <vector>

#include "fhd_launch.cuh"
#include "fhd_linesum.cuh"
#include "fhd_vismf.h"

namespace fhd {

constexpr int kPlotMax = 224;  // components of the largest composition (4 species, every flag)

struct PlotArgs {
    Arr4<const double> src[kPlotMax];  // per output component, pre-offset to its source component
    Arr4<double> out;
    int n[3];
    int ncomp;
};

// plane averages of Y_k for plot_deltaY_dir (WriteHorizontalAverageToMF,
// ComputeAverages.cpp:96-190): k_sum_to_line (fhd_linesum.cuh), entry r of species n
// the cells with coordinate r along dir summed in the order k, j, i and divided by
// the plane's cell count, into avg[r * ns + n]

// out component c0 + n = (-average) + Y_n, block (z-plane, species) as the pack
struct DeltaYArgs {
    Arr4<const double> y;
    Arr4<double> out;
    const double* avg;
    int n[3], dir, ns, c0;
};
static __global__ void __launch_bounds__(256) k_plot_deltay(DeltaYArgs a) {
    const int c = blockIdx.y;
    for (int k = blockIdx.x; k < a.n[2]; k += gridDim.x)
        for (int j = 0; j < a.n[1]; ++j)
            for (int i = threadIdx.x; i < a.n[0]; i += blockDim.x) {
                const int r = a.dir == 0 ? i : (a.dir == 1 ? j : k);
                a.out(i, j, k, a.c0 + c) = (-a.avg[r * a.ns + c]) + a.y(i, j, k, c);
            }
}

// blockIdx.y: output component; blockIdx.x: z-planes (grid-stride)
static __global__ void __launch_bounds__(256) k_plot_pack(PlotArgs a) {
    const int c = blockIdx.y;
    const Arr4<const double> s = a.src[c];
    for (int k = blockIdx.x; k < a.n[2]; k += gridDim.x)
        for (int j = 0; j < a.n[1]; ++j) {
            const double* __restrict__ sp = &s(0, j, k);
            double* __restrict__ dp = &a.out(0, j, k, c);
            for (int i = threadIdx.x; i < a.n[0]; i += blockDim.x) dp[i] = sp[i];
        }
}

struct PlotComp {
    fhd_fab fab;
    int comp;
    std::string name;
};

static std::string numbered(const char* base, int i) { return std::string(base) + char('0' + i); }

// the composition of writePlotFileStag.cpp:111-311 with the names of :313-447
static bool plot_layout(const fhd_params& prm, int flags, const fhd_fab& cu, const fhd_fab* cumom, const fhd_fab& prim,
                        const fhd_fab* vel, const fhd_fab& eta, const fhd_fab& kappa, const fhd_fab& zeta,
                        const fhd_stats* st, std::vector<PlotComp>& out) {
    const int ns = prm.nspecies, nprim = 6 + 2 * ns;
    const bool visc3 = prm.visc_type == 3 || prm.visc_type == -3;
    const char* xyz[3] = {"x", "y", "z"};
    auto add = [&](const fhd_fab& f, int c, const std::string& nm) { out.push_back(PlotComp{f, c, nm}); };
    const fhd_fab none{};
    auto S = [&](const fhd_fab fhd_stats::*m) -> fhd_fab { return st ? st->*m : none; };
    // instantaneous
    add(cu, 0, "rhoInstant");
    for (int d = 0; d < 3; ++d) add(cu, 1 + d, std::string("j") + xyz[d] + "InstantCC");
    add(cu, 4, "rhoEInstant");
    for (int s = 0; s < ns; ++s) add(cu, 5 + s, numbered("rhoYkInstant_", s));
    for (int d = 0; d < 3; ++d) add(cumom ? cumom[d] : none, 0, std::string("j") + xyz[d] + "InstantFACE");
    for (int d = 0; d < 3; ++d) add(prim, 1 + d, std::string("u") + xyz[d] + "InstantCC");
    add(prim, 4, "tInstant");
    add(prim, 5, "pInstant");
    for (int s = 0; s < ns; ++s) add(prim, 6 + s, numbered("YkInstant_", s));
    for (int s = 0; s < ns; ++s) add(prim, 6 + ns + s, numbered("XkInstant_", s));
    for (int d = 0; d < 3; ++d) add(vel ? vel[d] : none, 0, std::string("u") + xyz[d] + "InstantFACE");
    add(eta, 0, "eta");
    add(kappa, 0, "kappa");
    if (visc3) add(zeta, 0, "zeta");
    if (flags & FHD_PLOT_MEANS) {
        const fhd_fab cm = S(&fhd_stats::cuMeans), pm = S(&fhd_stats::primMeans);
        add(cm, 0, "rhoMean");
        for (int d = 0; d < 3; ++d) add(cm, 1 + d, std::string("j") + xyz[d] + "MeanCC");
        add(cm, 4, "rhoEMean");
        for (int s = 0; s < ns; ++s) add(cm, 5 + s, numbered("rhoYkMean_", s));
        for (int d = 0; d < 3; ++d) add(st ? st->cumomMeans[d] : none, 0, std::string("j") + xyz[d] + "MeanFACE");
        for (int d = 0; d < 3; ++d) add(pm, 1 + d, std::string("u") + xyz[d] + "MeanCC");
        add(pm, 4, "tMean");
        add(pm, 5, "pMean");
        for (int s = 0; s < ns; ++s) add(pm, 6 + s, numbered("YkMean_", s));
        for (int s = 0; s < ns; ++s) add(pm, 6 + ns + s, numbered("XkMean_", s));
        for (int d = 0; d < 3; ++d) add(st ? st->velMeans[d] : none, 0, std::string("u") + xyz[d] + "MeanFACE");
        for (int d = 0; d < 3; ++d) add(pm, nprim + d, std::string("u") + xyz[d] + "MeanCOM");
    }
    if (flags & FHD_PLOT_VARS) {
        const fhd_fab cv = S(&fhd_stats::cuVars), pv = S(&fhd_stats::primVars);
        add(cv, 0, "rhoVar");
        for (int d = 0; d < 3; ++d) add(cv, 1 + d, std::string("j") + xyz[d] + "VarCC");
        add(cv, 4, "rhoEVar");
        for (int s = 0; s < ns; ++s) add(cv, 5 + s, numbered("rhoYkVar_", s));
        for (int d = 0; d < 3; ++d) add(st ? st->cumomVars[d] : none, 0, std::string("j") + xyz[d] + "VarFACE");
        for (int d = 0; d < 3; ++d) add(pv, 1 + d, std::string("u") + xyz[d] + "VarCC");
        add(pv, 4, "TVarDirect");
        for (int s = 0; s < ns; ++s) add(pv, 6 + s, numbered("YkVar_", s));
        const char* extra[5] = {"g-g", "g-energy", "rho-energy", "rho-g", "TVar"};
        for (int e = 0; e < 5; ++e) add(pv, nprim + e, extra[e]);
        for (int d = 0; d < 3; ++d) add(st ? st->velVars[d] : none, 0, std::string("u") + xyz[d] + "VarFACE");
    }
    if (flags & FHD_PLOT_COVARS) {
        const char* cov[26] = {"rho-jx", "rho-jy", "rho-jz", "jx-jy", "jy-jz", "jx-jz", "rho-rhoE", "rhoE-jx",
                               "rhoE-jy", "rhoE-jz", "rhoL-rhoH", "rho-vx", "rho-vy", "rho-vz", "vx-vy", "vy-vz",
                               "vx-vz", "rho-T", "vx-T", "vy-T", "vz-T", "YkL-YkH", "YkL-vx", "YkH-vx",
                               "rhoYkL-vx", "rhoYkH-vx"};
        for (int e = 0; e < 26; ++e) add(S(&fhd_stats::coVars), e, cov[e]);
    }
    for (int q = 0; q < 2; ++q) {
        if (!(flags & (q == 0 ? FHD_PLOT_MOM3 : FHD_PLOT_MOM4))) continue;
        const fhd_fab m = S(q == 0 ? &fhd_stats::mom3 : &fhd_stats::mom4);
        const std::string sfx = q == 0 ? "mom3" : "mom4";
        add(m, 0, "rho" + sfx);
        for (int d = 0; d < 3; ++d) add(m, 1 + d, std::string("vel") + xyz[d] + sfx);
        add(m, 4, "rhoE" + sfx);
        for (int s = 0; s < ns; ++s) add(m, 5 + s, numbered(("Yk" + sfx + "_").c_str(), s));
        add(m, 5 + ns, "T" + sfx);
    }
    // plot_deltaY_dir: computed, not copied (comp -1 marks them)
    if (flags & (FHD_PLOT_DELTAY_X | FHD_PLOT_DELTAY_Y | FHD_PLOT_DELTAY_Z))
        for (int s = 0; s < ns; ++s) out.push_back(PlotComp{prim, -1, numbered("deltaYk_", s)});
    return (int)out.size() <= kPlotMax;
}

// a source fab must exist, cover the domain's valid region and hold the component
static bool plot_src_ok(const fhd_params& prm, const PlotComp& pc) {
    const fhd_fab& f = pc.fab;
    const int need = pc.comp >= 0 ? pc.comp : 6 + prm.nspecies - 1;  // deltaY reads Y_0..Y_{ns-1} of prim
    if (!f.data || f.dtype != FHD_F64 || need >= f.ncomp) return false;
    for (int d = 0; d < 3; ++d)
        if (f.lo[d] > 0 || f.hi[d] < prm.n_cells[d] - 1) return false;
    return true;
}

int plot_pack(const fhd_params& prm, int flags, fhd_fab out, const fhd_fab& cu, const fhd_fab* cumom,
              const fhd_fab& prim, const fhd_fab* vel, const fhd_fab& eta, const fhd_fab& kappa, const fhd_fab& zeta,
              const fhd_stats* st, cudaStream_t s) {
    std::vector<PlotComp> L;
    if (!plot_layout(prm, flags, cu, cumom, prim, vel, eta, kappa, zeta, st, L)) return FHD_ERR_UNSUPPORTED;
    if (!out.data || out.dtype != FHD_F64 || out.ncomp < (int)L.size()) return FHD_ERR_BAD_ARG;
    for (int d = 0; d < 3; ++d)
        if (out.lo[d] > 0 || out.hi[d] < prm.n_cells[d] - 1 || out.nodal[d]) return FHD_ERR_BAD_ARG;
    for (const PlotComp& pc : L)
        if (!plot_src_ok(prm, pc)) return FHD_ERR_BAD_ARG;
    int ncopy = 0;
    while (ncopy < (int)L.size() && L[ncopy].comp >= 0) ++ncopy;  // copies first, deltaY last
    PlotArgs a;
    std::memset(&a, 0, sizeof(a));
    for (int c = 0; c < ncopy; ++c) a.src[c] = view<const double>(L[c].fab, L[c].comp);
    a.out = view<double>(out);
    for (int d = 0; d < 3; ++d) a.n[d] = prm.n_cells[d];
    a.ncomp = ncopy;
    // every block of the (plane, component) grid copies at least a whole plane
    const dim3 grid((unsigned)a.n[2], (unsigned)a.ncomp);
    k_plot_pack<<<grid, 256, 0, s>>>(a);
    int rc = cuda_rc(cudaGetLastError());
    if (rc || ncopy == (int)L.size()) return rc;
    // plot_deltaY_dir
    const int dir = (flags & FHD_PLOT_DELTAY_X) ? 0 : ((flags & FHD_PLOT_DELTAY_Y) ? 1 : 2);
    const int ns = prm.nspecies, npts = prm.n_cells[dir];
    double* avg = nullptr;
    if (cudaMallocAsync(reinterpret_cast<void**>(&avg), sizeof(double) * npts * ns, s) != cudaSuccess) {
        cudaGetLastError();
        return FHD_ERR_OOM;
    }
    LineArgs la;
    for (int c = 0; c < ns; ++c) la.job[c] = line_job_dir(prim, 6 + c, dir, avg + c, ns);
    la.njobs = ns;
    rc = launch_line_sums(la, prm.n_cells, dir, s);
    if (rc) {
        cudaFreeAsync(avg, s);
        return rc;
    }
    DeltaYArgs dy;
    dy.y = view<const double>(prim, 6);
    dy.out = a.out;
    dy.avg = avg;
    for (int d = 0; d < 3; ++d) dy.n[d] = prm.n_cells[d];
    dy.dir = dir;
    dy.ns = ns;
    dy.c0 = ncopy;
    k_plot_deltay<<<dim3((unsigned)dy.n[2], (unsigned)ns), 256, 0, s>>>(dy);
    rc = cuda_rc(cudaGetLastError());
    cudaFreeAsync(avg, s);
    return rc;
}

int plot_names(const fhd_params& prm, int flags, std::vector<std::string>& names) {
    std::vector<PlotComp> L;
    const fhd_fab none{};
    fhd_fab three[3] = {none, none, none};
    fhd_stats st;
    std::memset(&st, 0, sizeof(st));
    if (!plot_layout(prm, flags, none, three, none, three, none, none, none, &st, L)) return FHD_ERR_UNSUPPORTED;
    names.clear();
    for (const PlotComp& pc : L) names.push_back(pc.name);
    return FHD_OK;
}

static std::string box_text(const int n[3]) {
    const int lo[3] = {0, 0, 0}, hi[3] = {n[0] - 1, n[1] - 1, n[2] - 1}, type[3] = {0, 0, 0};
    return vismf_box(lo, hi, type);
}

// Writes the packed host data (ncomp components of the valid box, x fastest,
// components slowest) as a single-level, single-box AMReX plotfile.
int plot_write(const fhd_params& prm, const char* dir, const double* host, const std::vector<std::string>& names,
               double time, int step) {
    const int nc = (int)names.size();
    const int* n = prm.n_cells;
    const std::string root(dir);
    if (!vismf_mkdir(root) || !vismf_mkdir(root + "/Level_0")) return FHD_ERR_IO;
    double dx[3];
    for (int d = 0; d < 3; ++d) dx[d] = (prm.prob_hi[d] - prm.prob_lo[d]) / n[d];
    FILE* h = std::fopen((root + "/Header").c_str(), "w");
    if (!h) return FHD_ERR_IO;
    std::fprintf(h, "HyperCLaw-V1.1\n%d\n", nc);
    for (const std::string& s : names) std::fprintf(h, "%s\n", s.c_str());
    std::fprintf(h, "3\n%.17g\n0\n", time);
    std::fprintf(h, "%.17g %.17g %.17g \n", prm.prob_lo[0], prm.prob_lo[1], prm.prob_lo[2]);
    std::fprintf(h, "%.17g %.17g %.17g \n", prm.prob_hi[0], prm.prob_hi[1], prm.prob_hi[2]);
    std::fprintf(h, "\n%s \n%d \n", box_text(n).c_str(), step);
    std::fprintf(h, "%.17g %.17g %.17g \n", dx[0], dx[1], dx[2]);
    std::fprintf(h, "0\n0\n");
    std::fprintf(h, "0 1 %.17g\n%d\n", time, step);
    for (int d = 0; d < 3; ++d) std::fprintf(h, "%.17g %.17g\n", prm.prob_lo[d], prm.prob_hi[d]);
    std::fprintf(h, "Level_0/Cell\n");
    const bool hok = std::fclose(h) == 0;
    // Level_0/Cell_H and Cell_D_00000: the one-box MultiFab, no ghosts
    const int lo[3] = {0, 0, 0}, hi[3] = {n[0] - 1, n[1] - 1, n[2] - 1}, type[3] = {0, 0, 0};
    const bool cok = vismf_write(root + "/Level_0", "Cell", host, lo, hi, type, nc, 0);
    return (hok && cok) ? FHD_OK : FHD_ERR_IO;
}

}  // namespace fhd
