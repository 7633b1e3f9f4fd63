// fhd_chk.cu — WriteCheckPoint / ReadCheckPoint (Checkpoint.cpp:28-257, 259-575)
// for one periodic box: chk<step, 9 digits>/Header (title line, step, time,
// statsCount, the BoxArray) and Level_0/<name>_H, <name>_D_00000 for every
// MultiFab the reference saves, under its names (cu, cuMeans, cuVars, prim,
// primMeans, primVars, velx..z, velmeanx..z, velvarx..z, cumomx..z,
// cumommeanx..z, cumomvarx..z, coVars, mom3, mom4), whole fabs with their ghost
// cells as VisMF writes them.
//
// With plot_cross (fhd_stats.spatialCross non-NULL) the Header also carries
// spatialCrossVec after the BoxArray, one value per line at 16 significant digits
// (Checkpoint.cpp:112-118, read back at :343-358).  fhd_write_spatial_cross writes
// WriteSpatialCross3D's text file (writePlotFileStag.cpp:528-549).
//
// The reference also saves its C++ random engines' states (rng files); the noise
// here is a function of (seed, step) alone, so the restart step is all the
// generator needs.  Host code: device fabs are copied with cudaMemcpy after a
// device synchronisation, host fabs with memcpy (no GPU needed for those).
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/fhd_capi.h"
#include "fhd_vismf.h"

namespace fhd {

namespace {

bool on_device(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int64_t fab_elems(const fhd_fab& f) {
    int64_t n = f.ncomp;
    for (int d = 0; d < 3; ++d) n *= (int64_t)(f.hi[d] - f.lo[d] + 1);
    return n;
}

bool copy_bytes(void* dst, const void* src, size_t bytes, bool dev) {
    if (!dev) {
        std::memcpy(dst, src, bytes);
        return true;
    }
    if (cudaMemcpy(dst, src, bytes, cudaMemcpyDefault) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

struct Entry {
    std::string name;
    fhd_fab fab;
};

// the MultiFabs of Checkpoint.cpp:172-239 that the caller supplied
std::vector<Entry> entries(fhd_fab cu, const fhd_fab* cumom, fhd_fab prim, const fhd_fab* vel, const fhd_stats* st) {
    const char* xyz = "xyz";
    std::vector<Entry> e;
    auto add = [&](const std::string& n, const fhd_fab& f) {
        if (f.data) e.push_back(Entry{n, f});
    };
    add("cu", cu);
    if (st) {
        add("cuMeans", st->cuMeans);
        add("cuVars", st->cuVars);
    }
    add("prim", prim);
    if (st) {
        add("primMeans", st->primMeans);
        add("primVars", st->primVars);
    }
    for (int d = 0; d < 3; ++d) add(std::string("vel") + xyz[d], vel[d]);
    if (st) {
        for (int d = 0; d < 3; ++d) add(std::string("velmean") + xyz[d], st->velMeans[d]);
        for (int d = 0; d < 3; ++d) add(std::string("velvar") + xyz[d], st->velVars[d]);
    }
    for (int d = 0; d < 3; ++d) add(std::string("cumom") + xyz[d], cumom[d]);
    if (st) {
        for (int d = 0; d < 3; ++d) add(std::string("cumommean") + xyz[d], st->cumomMeans[d]);
        for (int d = 0; d < 3; ++d) add(std::string("cumomvar") + xyz[d], st->cumomVars[d]);
        add("coVars", st->coVars);
        add("mom3", st->mom3);
        add("mom4", st->mom4);
    }
    return e;
}

// a one-box fab of the domain: uniform ghost width, valid box = the domain (+ nodal)
bool geometry(const fhd_params& p, const fhd_fab& f, int vlo[3], int vhi[3], int type[3], int* ng) {
    if (f.dtype != FHD_F64 || f.ncomp < 1) return false;
    *ng = -f.lo[0];
    for (int d = 0; d < 3; ++d) {
        type[d] = f.nodal[d] ? 1 : 0;
        vlo[d] = 0;
        vhi[d] = p.n_cells[d] - 1 + type[d];
        if (f.lo[d] != -*ng || f.hi[d] != vhi[d] + *ng) return false;
    }
    return *ng >= 0;
}

int ncross_of(const fhd_params& p) { return 37 + p.nspecies + 3; }
bool lowdim(const fhd_params& p) { return p.do_1D || p.do_2D; }
// components of a quasi-1-D / 2-D run's spatialCrossMF (main_driver.cpp:717-727)
int crossmf_ncomp(const fhd_params& p) { return (p.do_1D && p.all_correl == 1 ? 5 : 1) * ncross_of(p); }
int64_t cells_of(const fhd_params& p) { return (int64_t)p.n_cells[0] * p.n_cells[1] * p.n_cells[2]; }

// spatialCross (host or device) into a host vector
bool cross_to_host(const fhd_params& p, const double* src, std::vector<double>& out) {
    out.resize((size_t)p.n_cells[0] * ncross_of(p));
    return copy_bytes(out.data(), src, out.size() * sizeof(double), on_device(src));
}

std::string chk_dir(const char* base, int step) {
    char num[32];
    std::snprintf(num, sizeof(num), "%09d", step);
    return std::string(base) + num;
}

}  // namespace
}  // namespace fhd

using namespace fhd;

extern "C" int fhd_write_checkpoint(const fhd_params* params, const char* chk_base, int step, double time,
                                    int stats_count, fhd_fab cu, const fhd_fab cumom[3], fhd_fab prim,
                                    const fhd_fab vel[3], const fhd_stats* stats) {
    if (!params || !chk_base || !cumom || !vel || step < 0 || !cu.data || !prim.data) return FHD_ERR_BAD_ARG;
    const std::vector<Entry> E = entries(cu, cumom, prim, vel, stats);
    bool dev = false;
    for (const Entry& e : E) {
        int vlo[3], vhi[3], type[3], ng;
        if (!geometry(*params, e.fab, vlo, vhi, type, &ng)) return FHD_ERR_BAD_ARG;
        dev = dev || on_device(e.fab.data);
    }
    const bool cross = stats && stats->spatialCross;
    if (cross) dev = dev || on_device(stats->spatialCross);
    if (dev && cudaDeviceSynchronize() != cudaSuccess) {
        cudaGetLastError();
        return FHD_ERR_CUDA;
    }
    // the Header's spatialCrossVec (left at zero by a quasi-1-D / 2-D run, whose
    // correlations are the MultiFab spatialCrossMF: Checkpoint.cpp:251-256)
    std::vector<double> sc, scmf;
    if (cross && !lowdim(*params) && !cross_to_host(*params, stats->spatialCross, sc)) return FHD_ERR_CUDA;
    if (cross && lowdim(*params)) {
        sc.assign((size_t)params->n_cells[0] * ncross_of(*params), 0.0);
        scmf.resize((size_t)cells_of(*params) * crossmf_ncomp(*params));
        if (!copy_bytes(scmf.data(), stats->spatialCross, scmf.size() * sizeof(double), on_device(stats->spatialCross)))
            return FHD_ERR_CUDA;
    }
    const std::string dir = chk_dir(chk_base, step);
    if (!vismf_mkdir(dir) || !vismf_mkdir(dir + "/Level_0")) return FHD_ERR_IO;
    FILE* h = std::fopen((dir + "/Header").c_str(), "w");
    if (!h) return FHD_ERR_IO;
    const int lo[3] = {0, 0, 0}, hi[3] = {params->n_cells[0] - 1, params->n_cells[1] - 1, params->n_cells[2] - 1},
              cc[3] = {0, 0, 0};
    std::fprintf(h, "Checkpoint file for FHDeX/compressStag\n%d\n%.17g\n%d\n(1 0\n%s\n)\n\n", step, time, stats_count,
                 vismf_box(lo, hi, cc).c_str());
    for (double v : sc) std::fprintf(h, "%.16g\n", v);
    if (std::fclose(h) != 0) return FHD_ERR_IO;
    std::vector<double> buf;
    for (const Entry& e : E) {
        int vlo[3], vhi[3], type[3], ng;
        geometry(*params, e.fab, vlo, vhi, type, &ng);
        buf.resize((size_t)fab_elems(e.fab));
        if (!copy_bytes(buf.data(), e.fab.data, buf.size() * sizeof(double), on_device(e.fab.data)))
            return FHD_ERR_CUDA;
        if (!vismf_write(dir + "/Level_0", e.name, buf.data(), vlo, vhi, type, e.fab.ncomp, ng)) return FHD_ERR_IO;
    }
    if (!scmf.empty()) {
        const int vlo[3] = {0, 0, 0}, type[3] = {0, 0, 0};
        if (!vismf_write(dir + "/Level_0", "spatialCrossMF", scmf.data(), vlo, hi, type, crossmf_ncomp(*params), 0))
            return FHD_ERR_IO;
    }
    return FHD_OK;
}

extern "C" int fhd_read_checkpoint(const fhd_params* params, const char* chk_base, int restart, int* step,
                                   double* time, int* stats_count, fhd_fab cu, const fhd_fab cumom[3], fhd_fab prim,
                                   const fhd_fab vel[3], const fhd_stats* stats) {
    if (!params || !chk_base || !cumom || !vel || restart < 0 || !step || !time || !stats_count || !cu.data ||
        !prim.data)
        return FHD_ERR_BAD_ARG;
    const std::string dir = chk_dir(chk_base, restart);
    FILE* h = std::fopen((dir + "/Header").c_str(), "r");
    if (!h) return FHD_ERR_IO;
    char title[256];
    int s = 0, sc = 0;
    double t = 0;
    bool hok = std::fgets(title, sizeof(title), h) && std::fscanf(h, "%d %lf %d", &s, &t, &sc) == 3;
    // spatialCrossVec: the values after the BoxArray's closing ")" line
    std::vector<double> cross;
    if (hok && stats && stats->spatialCross && !lowdim(*params)) {
        char line[512];
        bool end = false;
        while (!end && std::fgets(line, sizeof(line), h)) end = line[0] == ')';
        cross.resize((size_t)params->n_cells[0] * ncross_of(*params));
        for (double& v : cross) hok = hok && end && std::fscanf(h, "%lf", &v) == 1;
    }
    std::fclose(h);
    if (!hok || std::strncmp(title, "Checkpoint file for FHDeX/compressStag", 38) != 0) return FHD_ERR_BAD_ARG;
    const std::vector<Entry> E = entries(cu, cumom, prim, vel, stats);
    std::vector<double> buf;
    bool synced = false;
    for (const Entry& e : E) {
        int vlo[3], vhi[3], type[3], ng;
        if (!geometry(*params, e.fab, vlo, vhi, type, &ng)) return FHD_ERR_BAD_ARG;
        int glo[3], ghi[3];
        for (int d = 0; d < 3; ++d) {
            glo[d] = vlo[d] - ng;
            ghi[d] = vhi[d] + ng;
        }
        const int vr = vismf_read(dir + "/Level_0", e.name, glo, ghi, type, e.fab.ncomp, buf);
        if (vr != kVisOk) return vr == kVisShape ? FHD_ERR_BAD_ARG : FHD_ERR_IO;
        const bool dev = on_device(e.fab.data);
        if (dev && !synced) {
            if (cudaDeviceSynchronize() != cudaSuccess) {
                cudaGetLastError();
                return FHD_ERR_CUDA;
            }
            synced = true;
        }
        if (!copy_bytes(e.fab.data, buf.data(), buf.size() * sizeof(double), dev)) return FHD_ERR_CUDA;
    }
    // a quasi-1-D / 2-D run's correlations: spatialCrossMF (Checkpoint.cpp:529-535)
    if (stats && stats->spatialCross && lowdim(*params)) {
        const int glo[3] = {0, 0, 0}, ghi[3] = {params->n_cells[0] - 1, params->n_cells[1] - 1, params->n_cells[2] - 1};
        const int type[3] = {0, 0, 0};
        const int vr = vismf_read(dir + "/Level_0", "spatialCrossMF", glo, ghi, type, crossmf_ncomp(*params), cross);
        if (vr != kVisOk) return vr == kVisShape ? FHD_ERR_BAD_ARG : FHD_ERR_IO;
    }
    if (!cross.empty()) {
        const bool dev = on_device(stats->spatialCross);
        if (dev && !synced && cudaDeviceSynchronize() != cudaSuccess) {
            cudaGetLastError();
            return FHD_ERR_CUDA;
        }
        if (!copy_bytes(stats->spatialCross, cross.data(), cross.size() * sizeof(double), dev)) return FHD_ERR_CUDA;
    }
    // ReadCheckPoint resumes at the step after the saved one (Checkpoint.cpp:328-329)
    *step = s + 1;
    *time = t;
    *stats_count = sc;
    return FHD_OK;
}

// WriteSpatialCross1D (writePlotFileStag.cpp:551-563): per x*, WriteHorizontalAverage
// (ComputeAverages.cpp:8-94) of its ncross components of spatialCrossMF along x:
// each line the cell centre prob_lo[0] + (i+0.5)*dx[0] and the components' y-z
// averages (each summed from 0.0 with k outer and j inner, divided by
// n_cells[1]*n_cells[2]), every number at the stream's default 6 significant digits
// and followed by a space.
static int write_cross_1d(const fhd_params& p, const char* dir, int step, const double* data) {
    const int nc = ncross_of(p), nstar = crossmf_ncomp(p) / nc;
    const int64_t cells = cells_of(p);
    std::vector<double> mf((size_t)cells * nstar * nc);
    if (!copy_bytes(mf.data(), data, mf.size() * sizeof(double), on_device(data))) return FHD_ERR_CUDA;
    const int nx = p.n_cells[0], ny = p.n_cells[1], nz = p.n_cells[2];
    const double h = (p.prob_hi[0] - p.prob_lo[0]) / nx;
    for (int s = 0; s < nstar; ++s) {
        std::vector<double> avg((size_t)nx * (nc + 1), 0.0);
        for (int n = 0; n < nc; ++n) {
            const double* c = mf.data() + (size_t)(s * nc + n) * cells;
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i) avg[(size_t)i * (nc + 1) + n + 1] += c[((size_t)k * ny + j) * nx + i];
        }
        const int navg = ny * nz;
        for (int r = 0; r < nx; ++r)
            for (int n = 1; n < nc + 1; ++n) avg[(size_t)r * (nc + 1) + n] /= navg;
        for (int r = 0; r < nx; ++r) avg[(size_t)r * (nc + 1)] = p.prob_lo[0] + (r + 0.5) * h;
        const std::string prefix = std::string(dir) + (nstar == 5 ? std::to_string(s) + "_" : std::string()) +
                                   "spatialCross1D_";
        FILE* f = std::fopen(chk_dir(prefix.c_str(), step).c_str(), "w");
        if (!f) return FHD_ERR_IO;
        for (int r = 0; r < nx; ++r) {
            for (int n = 0; n < nc + 1; ++n) std::fprintf(f, "%g ", avg[(size_t)r * (nc + 1) + n]);
            std::fputc('\n', f);
        }
        if (std::fclose(f) != 0) return FHD_ERR_IO;
    }
    return FHD_OK;
}

// WriteSpatialCross3D (writePlotFileStag.cpp:528-549): <dir>spatialCross<step, 9 digits>, one
// line per x cell: the cell centre prob_lo[0] + (i+0.5)*dx[0], then the ncross
// entries, each followed by a space.  The reference sets 16 significant digits
// only before the first entry, so the first line's centre keeps the stream's
// default 6 (every later number has 16).
extern "C" int fhd_write_spatial_cross(const fhd_params* params, const char* dir, int step,
                                       const double* spatial_cross) {
    if (!params || !dir || !spatial_cross || step < 0 || params->nspecies < 1 ||
        params->nspecies > FHD_MAX_SPECIES || params->n_cells[0] < 1)
        return FHD_ERR_BAD_ARG;
    if (params->do_2D) return FHD_OK;   // WriteSpatialCross2D is not enabled in the reference
    std::vector<double> sc;
    if (on_device(spatial_cross) && cudaDeviceSynchronize() != cudaSuccess) {
        cudaGetLastError();
        return FHD_ERR_CUDA;
    }
    if (params->do_1D) return write_cross_1d(*params, dir, step, spatial_cross);
    if (!cross_to_host(*params, spatial_cross, sc)) return FHD_ERR_CUDA;
    FILE* f = std::fopen(chk_dir((std::string(dir) + "spatialCross").c_str(), step).c_str(), "w");
    if (!f) return FHD_ERR_IO;
    const int nc = ncross_of(*params);
    const double h = (params->prob_hi[0] - params->prob_lo[0]) / params->n_cells[0];
    for (int i = 0; i < params->n_cells[0]; ++i) {
        std::fprintf(f, i == 0 ? "%g " : "%.16g ", params->prob_lo[0] + (i + 0.5) * h);
        for (int n = 0; n < nc; ++n) std::fprintf(f, "%.16g ", sc[(size_t)i * nc + n]);
        std::fputc('\n', f);
    }
    return std::fclose(f) == 0 ? FHD_OK : FHD_ERR_IO;
}
