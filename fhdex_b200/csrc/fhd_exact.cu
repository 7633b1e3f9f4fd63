// fhd_exact.cu — dispatch over the species count to the per-NS translation units
// (fhd_kern_ns.cu) and the precision-independent utilities: periodic ghost fill,
// OverrideSync, Philox noise fill, uniform initial state.  Built with -fmad=false.
#include "fhd_launch.cuh"

namespace fhd {

int exact_cellprep_ns1(const StageCall&);
int exact_stage_ns1(const StageCall&, int);
int exact_aux_ns1(const StageCall&);
int mixed_cellprep_ns1(const StageCall&);
int mixed_stage_ns1(const StageCall&, int);
int exact_transport_ns1(const DevParams&, fhd_fab, fhd_fab, fhd_fab, fhd_fab, fhd_fab, fhd_fab, int*, cudaStream_t);
int exact_convert_ns1(const DevParams&, fhd_fab, const fhd_fab*, fhd_fab, const fhd_fab*, int*, cudaStream_t);
int exact_walls_ns1(const StageCall&, int);
int exact_reservoir_ns1(const ResArgs&, cudaStream_t);
int exact_res_reset_ns1(const ResResetArgs&, cudaStream_t);
int exact_bc_prim_ns1(const DevParams&, const WallParams&, fhd_fab, fhd_fab, const fhd_fab*, cudaStream_t);
int exact_bc_seq_ns1(const DevParams&, const WallParams&, fhd_fab, fhd_fab, const fhd_fab*, const fhd_fab*, int,
                     cudaStream_t);
int exact_cellprep_ns2(const StageCall&);
int exact_stage_ns2(const StageCall&, int);
int exact_aux_ns2(const StageCall&);
int mixed_cellprep_ns2(const StageCall&);
int mixed_stage_ns2(const StageCall&, int);
int exact_transport_ns2(const DevParams&, fhd_fab, fhd_fab, fhd_fab, fhd_fab, fhd_fab, fhd_fab, int*, cudaStream_t);
int exact_convert_ns2(const DevParams&, fhd_fab, const fhd_fab*, fhd_fab, const fhd_fab*, int*, cudaStream_t);
int exact_walls_ns2(const StageCall&, int);
int exact_reservoir_ns2(const ResArgs&, cudaStream_t);
int exact_res_reset_ns2(const ResResetArgs&, cudaStream_t);
int exact_bc_prim_ns2(const DevParams&, const WallParams&, fhd_fab, fhd_fab, const fhd_fab*, cudaStream_t);
int exact_bc_seq_ns2(const DevParams&, const WallParams&, fhd_fab, fhd_fab, const fhd_fab*, const fhd_fab*, int,
                     cudaStream_t);
int exact_cellprep_ns3(const StageCall&);
int exact_stage_ns3(const StageCall&, int);
int exact_aux_ns3(const StageCall&);
int mixed_cellprep_ns3(const StageCall&);
int mixed_stage_ns3(const StageCall&, int);
int exact_transport_ns3(const DevParams&, fhd_fab, fhd_fab, fhd_fab, fhd_fab, fhd_fab, fhd_fab, int*, cudaStream_t);
int exact_convert_ns3(const DevParams&, fhd_fab, const fhd_fab*, fhd_fab, const fhd_fab*, int*, cudaStream_t);
int exact_walls_ns3(const StageCall&, int);
int exact_reservoir_ns3(const ResArgs&, cudaStream_t);
int exact_res_reset_ns3(const ResResetArgs&, cudaStream_t);
int exact_bc_prim_ns3(const DevParams&, const WallParams&, fhd_fab, fhd_fab, const fhd_fab*, cudaStream_t);
int exact_bc_seq_ns3(const DevParams&, const WallParams&, fhd_fab, fhd_fab, const fhd_fab*, const fhd_fab*, int,
                     cudaStream_t);
int exact_cellprep_ns4(const StageCall&);
int exact_stage_ns4(const StageCall&, int);
int exact_aux_ns4(const StageCall&);
int mixed_cellprep_ns4(const StageCall&);
int mixed_stage_ns4(const StageCall&, int);
int exact_transport_ns4(const DevParams&, fhd_fab, fhd_fab, fhd_fab, fhd_fab, fhd_fab, fhd_fab, int*, cudaStream_t);
int exact_convert_ns4(const DevParams&, fhd_fab, const fhd_fab*, fhd_fab, const fhd_fab*, int*, cudaStream_t);
int exact_walls_ns4(const StageCall&, int);
int exact_reservoir_ns4(const ResArgs&, cudaStream_t);
int exact_res_reset_ns4(const ResResetArgs&, cudaStream_t);
int exact_bc_prim_ns4(const DevParams&, const WallParams&, fhd_fab, fhd_fab, const fhd_fab*, cudaStream_t);
int exact_bc_seq_ns4(const DevParams&, const WallParams&, fhd_fab, fhd_fab, const fhd_fab*, const fhd_fab*, int,
                     cudaStream_t);

size_t exact_batch_args_size_ns1(int, int);
void exact_batch_pack_ns1(int, int, const StageCall&, void*);
int exact_batch_launch_ns1(int, int, int, const void*, const int*, int, int, cudaStream_t);
size_t mixed_batch_args_size_ns1(int, int);
void mixed_batch_pack_ns1(int, int, const StageCall&, void*);
int mixed_batch_launch_ns1(int, int, int, const void*, const int*, int, int, cudaStream_t);
int exact_batch_persist_ns1(int, int, const PersistArgs&, cudaStream_t);
int mixed_batch_persist_ns1(int, int, const PersistArgs&, cudaStream_t);
size_t exact_batch_args_size_ns2(int, int);
void exact_batch_pack_ns2(int, int, const StageCall&, void*);
int exact_batch_launch_ns2(int, int, int, const void*, const int*, int, int, cudaStream_t);
size_t mixed_batch_args_size_ns2(int, int);
void mixed_batch_pack_ns2(int, int, const StageCall&, void*);
int mixed_batch_launch_ns2(int, int, int, const void*, const int*, int, int, cudaStream_t);
int exact_batch_persist_ns2(int, int, const PersistArgs&, cudaStream_t);
int mixed_batch_persist_ns2(int, int, const PersistArgs&, cudaStream_t);
size_t exact_batch_args_size_ns3(int, int);
void exact_batch_pack_ns3(int, int, const StageCall&, void*);
int exact_batch_launch_ns3(int, int, int, const void*, const int*, int, int, cudaStream_t);
size_t mixed_batch_args_size_ns3(int, int);
void mixed_batch_pack_ns3(int, int, const StageCall&, void*);
int mixed_batch_launch_ns3(int, int, int, const void*, const int*, int, int, cudaStream_t);
int exact_batch_persist_ns3(int, int, const PersistArgs&, cudaStream_t);
int mixed_batch_persist_ns3(int, int, const PersistArgs&, cudaStream_t);
size_t exact_batch_args_size_ns4(int, int);
void exact_batch_pack_ns4(int, int, const StageCall&, void*);
int exact_batch_launch_ns4(int, int, int, const void*, const int*, int, int, cudaStream_t);
size_t mixed_batch_args_size_ns4(int, int);
void mixed_batch_pack_ns4(int, int, const StageCall&, void*);
int mixed_batch_launch_ns4(int, int, int, const void*, const int*, int, int, cudaStream_t);
int exact_batch_persist_ns4(int, int, const PersistArgs&, cudaStream_t);
int mixed_batch_persist_ns4(int, int, const PersistArgs&, cudaStream_t);

#define FHD_DISPATCH(ns, fn, ...)            \
    switch (ns) {                             \
        case 1: return fn##1(__VA_ARGS__);    \
        case 2: return fn##2(__VA_ARGS__);    \
        case 3: return fn##3(__VA_ARGS__);    \
        case 4: return fn##4(__VA_ARGS__);    \
        default: return FHD_ERR_UNSUPPORTED;  \
    }

int exact_cellprep(const StageCall& c) { FHD_DISPATCH(c.P.ns, exact_cellprep_ns, c) }
int exact_stage_part(const StageCall& c, int part) { FHD_DISPATCH(c.P.ns, exact_stage_ns, c, part) }
int exact_aux_fluxes(const StageCall& c) { FHD_DISPATCH(c.P.ns, exact_aux_ns, c) }
int mixed_cellprep(const StageCall& c) { FHD_DISPATCH(c.P.ns, mixed_cellprep_ns, c) }
int mixed_stage_part(const StageCall& c, int part) { FHD_DISPATCH(c.P.ns, mixed_stage_ns, c, part) }
int exact_transport(const DevParams& P, fhd_fab prim, fhd_fab eta, fhd_fab zeta, fhd_fab kappa, fhd_fab chi,
                    fhd_fab D, int* status, cudaStream_t s) {
    FHD_DISPATCH(P.ns, exact_transport_ns, P, prim, eta, zeta, kappa, chi, D, status, s)
}
int exact_convert(const DevParams& P, fhd_fab prim, const fhd_fab vel[3], fhd_fab cons, const fhd_fab mom[3],
                  int* status, cudaStream_t s) {
    FHD_DISPATCH(P.ns, exact_convert_ns, P, prim, vel, cons, mom, status, s)
}

int exact_walls_part(const StageCall& c, int part) { FHD_DISPATCH(c.P.ns, exact_walls_ns, c, part) }
int exact_bc_prim(const DevParams& P, const WallParams& W, fhd_fab prim, fhd_fab cons, const fhd_fab mom[3],
                  cudaStream_t s) {
    FHD_DISPATCH(P.ns, exact_bc_prim_ns, P, W, prim, cons, mom, s)
}

int exact_bc_seq(const DevParams& P, const WallParams& W, fhd_fab prim, fhd_fab cons, const fhd_fab mom[3],
                 const fhd_fab vel[3], bool rre, cudaStream_t s) {
    FHD_DISPATCH(P.ns, exact_bc_seq_ns, P, W, prim, cons, mom, vel, rre ? 1 : 0, s)
}

// the particle reservoir (bc_mass 4) of one stage: its fluxes and momenta into res,
// the resets of the stage's flux scratch / the caller's flux fabs / the momenta
int exact_reservoir(const DevParams& P, const ResBuffers& r, const fhd_fab& cons, const fhd_fab& prim,
                    const fhd_fab vel[3], double dt, int stage, double* rec, int rec_cap, int* status,
                    cudaStream_t s) {
    ResArgs a;
    std::memset(&a, 0, sizeof(a));
    a.P = P;
    a.cons0 = view<const double>(cons);
    a.prim0 = view<const double>(prim);
    for (int d = 0; d < 3; ++d) {
        a.vel[d] = view<const double>(vel[d]);
        a.fres[d] = r.f[d];
        a.mres[d] = r.m[d];
        a.fsy[d] = r.sy[d];
        a.fsz[d] = r.sz[d];
        a.fsn[d] = r.sn[d];
    }
    for (int n = 0; n < MAXS; ++n) a.mass[n] = r.mass[n];
    a.dt = dt;
    a.stage = stage;
    a.nsides = 0;
    a.face_pref[0] = 0;
    for (int side = 0; side < 6; ++side) {
        if (P.bc_mass[side] != 4) continue;
        const int d = side >> 1, e1 = d == 0 ? 1 : 0, e2 = d == 2 ? 1 : 2;
        a.sides[a.nsides] = side;
        a.face_pref[a.nsides + 1] = a.face_pref[a.nsides] + (int64_t)P.n[e1] * P.n[e2];
        ++a.nsides;
    }
    a.rec = rec;
    a.rec_cap = rec_cap;
    a.status = status;
    if (cudaMemsetAsync(r.base, 0, r.bytes, s) != cudaSuccess) return FHD_ERR_CUDA;
    FHD_DISPATCH(P.ns, exact_reservoir_ns, a, s)
}

int exact_res_reset(const DevParams& P, const ResBuffers& r, const fhd_fab* ff, int fc_rho, int fc_rhoE, int fc_Y,
                    const fhd_fab* ef, int ef_comp_base, cudaStream_t s) {
    for (int side = 0; side < 6; ++side) {
        if (P.bc_mass[side] != 4) continue;
        ResResetArgs a;
        std::memset(&a, 0, sizeof(a));
        a.P = P;
        for (int d = 0; d < 3; ++d) {
            a.fres[d] = r.f[d];
            a.fsy[d] = r.sy[d];
            a.fsz[d] = r.sz[d];
            a.fsn[d] = r.sn[d];
            if (ff) a.ff[d] = view<double>(ff[d]);
        }
        a.fc_rho = fc_rho;
        a.fc_rhoE = fc_rhoE;
        a.fc_Y = fc_Y;
        // ef: six one-component fabs, or (ef_comp_base >= 0) one six-component fab
        for (int e = 0; e < 6; ++e) {
            if (!ef) continue;
            a.ef[e] = ef_comp_base >= 0 ? view<double>(ef[0], ef_comp_base + e) : view<double>(ef[e]);
        }
        a.side = side;
        int rc;
        switch (P.ns) {
            case 1: rc = exact_res_reset_ns1(a, s); break;
            case 2: rc = exact_res_reset_ns2(a, s); break;
            case 3: rc = exact_res_reset_ns3(a, s); break;
            case 4: rc = exact_res_reset_ns4(a, s); break;
            default: rc = FHD_ERR_UNSUPPORTED;
        }
        if (rc) return rc;
    }
    return FHD_OK;
}

int exact_res_mom(const DevParams& P, const ResBuffers& r, const fhd_fab mom[3], cudaStream_t s) {
    for (int side = 0; side < 6; ++side) {
        if (P.bc_mass[side] != 4) continue;
        ResMomArgs a;
        std::memset(&a, 0, sizeof(a));
        a.P = P;
        for (int d = 0; d < 3; ++d) {
            a.mres[d] = r.m[d];
            a.fsy[d] = r.sy[d];
            a.fsz[d] = r.sz[d];
            a.mom[d] = view<double>(mom[d]);
        }
        a.side = side;
        const int d = side >> 1, e1 = d == 0 ? 1 : 0, e2 = d == 2 ? 1 : 2;
        k_res_mom<<<grid_for((int64_t)P.n[e1] * P.n[e2], 128), 128, 0, s>>>(a);
        if (cudaGetLastError() != cudaSuccess) return FHD_ERR_CUDA;
    }
    return FHD_OK;
}

int bc_mom(const DevParams& P, const fhd_fab mom[3], const fhd_fab vel[3], cudaStream_t s) {
    BcMomArgs a;
    a.P = P;
    int64_t most = 0;
    for (int d = 0; d < 3; ++d) {
        a.mom[d] = view<double>(mom[d]);
        a.vel[d] = view<double>(vel[d]);
        const int g = -mom[d].lo[0];
        int blo[3], bhi[3], clo[3], chi[3];
        for (int e = 0; e < 3; ++e) {
            const int nod = e == d;
            blo[e] = -g;
            bhi[e] = P.n[e] - 1 + nod + g;
            const bool w = P.walls && !P.periodic[e];
            // the core no condition touches: inside the walls (the wall faces of
            // the nodal direction included in the conditions)
            clo[e] = w ? nod : blo[e];
            chi[e] = w ? P.n[e] - 1 : bhi[e];
        }
        a.sh[d] = make_shell(blo, bhi, clo, chi);
        if (a.sh[d].n > most) most = a.sh[d].n;
    }
    if (most == 0) return FHD_OK;
    k_bc_mom<<<dim3(grid_for(most, 256, 148 * 8), 3), 256, 0, s>>>(a);
    return cuda_rc(cudaGetLastError());
}

size_t batch_args_size(int ns, bool mixed, int kind, int mode) {
    switch (ns) {
        case 1: return mixed ? mixed_batch_args_size_ns1(kind, mode) : exact_batch_args_size_ns1(kind, mode);
        case 2: return mixed ? mixed_batch_args_size_ns2(kind, mode) : exact_batch_args_size_ns2(kind, mode);
        case 3: return mixed ? mixed_batch_args_size_ns3(kind, mode) : exact_batch_args_size_ns3(kind, mode);
        case 4: return mixed ? mixed_batch_args_size_ns4(kind, mode) : exact_batch_args_size_ns4(kind, mode);
        default: return 0;
    }
}
void batch_pack(int ns, bool mixed, int kind, int mode, const StageCall& c, void* dst) {
    switch (ns) {
        case 1: mixed ? mixed_batch_pack_ns1(kind, mode, c, dst) : exact_batch_pack_ns1(kind, mode, c, dst); break;
        case 2: mixed ? mixed_batch_pack_ns2(kind, mode, c, dst) : exact_batch_pack_ns2(kind, mode, c, dst); break;
        case 3: mixed ? mixed_batch_pack_ns3(kind, mode, c, dst) : exact_batch_pack_ns3(kind, mode, c, dst); break;
        case 4: mixed ? mixed_batch_pack_ns4(kind, mode, c, dst) : exact_batch_pack_ns4(kind, mode, c, dst); break;
        default: break;
    }
}
int batch_launch(int ns, bool mixed, int kind, int mode, int tile, const void* dargs, const int* dbpref, int nmem,
                 int nblocks, cudaStream_t s) {
    if (mixed) { FHD_DISPATCH(ns, mixed_batch_launch_ns, kind, mode, tile, dargs, dbpref, nmem, nblocks, s) }
    FHD_DISPATCH(ns, exact_batch_launch_ns, kind, mode, tile, dargs, dbpref, nmem, nblocks, s)
}

int batch_persist(int ns, bool mixed, int mode, int tile, const PersistArgs& a, cudaStream_t s) {
    if (mixed) { FHD_DISPATCH(ns, mixed_batch_persist_ns, mode, tile, a, s) }
    FHD_DISPATCH(ns, exact_batch_persist_ns, mode, tile, a, s)
}

int batch_face_tiles() { return kNumBatchFaceTiles; }
int batch_face_min_blocks(int tile) { return (tile >= 0 && tile < kNumBatchFaceTiles) ? kBatchFaceMinBlocks[tile] : 0; }

int ghost_desc_size() { return (int)sizeof(GhostFab); }

int64_t ghost_pack(const fhd_fab& f, int c0, int nc, const int ncell[3], void* dst) {
    GhostFab g;
    g.p = static_cast<double*>(f.data);
    g.lo = f.lo[0];
    const int gw = -f.lo[0];
    int64_t ext[3];
    for (int d = 0; d < 3; ++d) {
        g.vhi[d] = ncell[d] - 1 + f.nodal[d];
        ext[d] = f.hi[d] - f.lo[d] + 1;
        g.n[d] = ncell[d];
    }
    g.sy = ext[0];
    g.sz = ext[0] * ext[1];
    g.sn = ext[0] * ext[1] * ext[2];
    g.c0 = c0;
    g.nc = nc;
    for (int d = 0; d < 3; ++d) g.per[d] = 1;
    g.mode = 0;
    const int64_t VY = g.vhi[1] + 1, VZ = g.vhi[2] + 1;
    g.npts = gw == 0 ? 0 : 2 * gw * ext[0] * ext[1] + 2 * gw * ext[0] * VZ + 2 * gw * VY * VZ;
    memcpy(dst, &g, sizeof(g));
    return g.npts * g.nc;
}

int ghost_launch_b(const void* dfabs, const int* dbpref, int nfab, int nblocks, cudaStream_t s) {
    if (nblocks <= 0 || nfab <= 0) return FHD_OK;
    k_ghosts_b<<<nblocks, 256, 0, s>>>(static_cast<const GhostFab*>(dfabs), dbpref, nfab);
    return cuda_rc(cudaGetLastError());
}

int steps_set(uint64_t* step, uint64_t v, cudaStream_t s) {
    k_steps_set<<<1, 1, 0, s>>>(step, v);
    return cuda_rc(cudaGetLastError());
}

int steps_inc(uint64_t* steps, int n, cudaStream_t s) {
    if (n <= 0) return FHD_OK;
    k_steps_inc<<<(n + 255) / 256, 256, 0, s>>>(steps, n);
    return cuda_rc(cudaGetLastError());
}

int fill_ghosts(const GhostReq* reqs, int n, const int ncell[3], cudaStream_t s, const int* periodic, int mode) {
    for (int base = 0; base < n; base += 16) {
        GhostArgs a;
        a.nf = 0;
        int64_t maxpts = 0;
        for (int q = base; q < n && q < base + 16; ++q) {
            const fhd_fab& f = reqs[q].f;
            GhostFab& g = a.f[a.nf++];
            g.p = static_cast<double*>(f.data);
            g.lo = f.lo[0];
            const int gw = -f.lo[0];
            int64_t ext[3];
            for (int d = 0; d < 3; ++d) {
                g.vhi[d] = ncell[d] - 1 + f.nodal[d];
                ext[d] = f.hi[d] - f.lo[d] + 1;
            }
            g.sy = ext[0];
            g.sz = ext[0] * ext[1];
            g.sn = ext[0] * ext[1] * ext[2];
            g.c0 = reqs[q].c0;
            g.nc = reqs[q].nc;
            for (int d = 0; d < 3; ++d) {
                g.n[d] = ncell[d];
                g.per[d] = periodic ? periodic[d] : 1;
            }
            g.mode = mode;
            const int64_t VX = g.vhi[0] + 1, VY = g.vhi[1] + 1, VZ = g.vhi[2] + 1;
            g.npts = 2 * gw * ext[0] * ext[1] + 2 * gw * ext[0] * VZ + 2 * gw * VY * VZ;
            (void)VX;
            if (gw == 0) g.npts = 0;
            if (g.npts * g.nc > maxpts) maxpts = g.npts * g.nc;
        }
        for (int d = 0; d < 3; ++d) a.n[d] = ncell[d];
        if (maxpts == 0) continue;
        dim3 grid(grid_for(maxpts, 256, 148 * 8), a.nf);
        k_ghosts<<<grid, 256, 0, s>>>(a);
        if (cudaGetLastError() != cudaSuccess) return FHD_ERR_CUDA;
    }
    return FHD_OK;
}

int override_sync(const fhd_fab& f, const int ncell[3], cudaStream_t s, const int* periodic) {
    SyncArgs a;
    a.p = static_cast<double*>(f.data);
    a.lo = f.lo[0];
    int64_t ext[3];
    for (int d = 0; d < 3; ++d) {
        a.nodal[d] = f.nodal[d] && (!periodic || periodic[d]);
        a.n[d] = ncell[d];
        ext[d] = f.hi[d] - f.lo[d] + 1;
    }
    a.sy = ext[0];
    a.sz = ext[0] * ext[1];
    a.sn = ext[0] * ext[1] * ext[2];
    a.nc = f.ncomp;
    const int64_t tot = (int64_t)(ncell[0] + a.nodal[0]) * (ncell[1] + a.nodal[1]) * (ncell[2] + a.nodal[2]) * f.ncomp;
    if (!a.nodal[0] && !a.nodal[1] && !a.nodal[2]) return FHD_OK;
    k_override_sync<<<grid_for(tot, 256), 256, 0, s>>>(a);
    return cuda_rc(cudaGetLastError());
}

int noise_fill(const DevParams& P, const fhd_fab& f, int c0, int nc, double mean, double sd, uint32_t fid0, int use_b,
               cudaStream_t s, int wall_ghosts) {
    NoiseFillArgs a;
    a.P = P;
    a.f = view<double>(f);
    int ext[3], org[3];
    for (int d = 0; d < 3; ++d) {
        // a wall direction of a field with ghosts: its first ghost layer too
        const bool g = wall_ghosts && P.walls && !P.periodic[d] && -f.lo[d] >= 1;
        ext[d] = P.n[d] + f.nodal[d] + (g ? 2 : 0);
        org[d] = g ? -1 : 0;
    }
    a.vx = ext[0];
    a.vy = ext[1];
    a.vz = ext[2];
    a.ox = org[0];
    a.oy = org[1];
    a.oz = org[2];
    a.c0 = c0;
    a.nc = nc;
    a.mean = mean;
    a.sd = sd;
    a.fid0 = fid0;
    a.use_b = use_b;
    const int64_t tot = (int64_t)a.vx * a.vy * a.vz * nc;
    k_noise_fill<<<grid_for(tot, 256), 256, 0, s>>>(a);
    return cuda_rc(cudaGetLastError());
}

int init_uniform(const fhd_fab& cu, int ns, double rho0, double rhoE, const double* rhoY, cudaStream_t s) {
    InitArgs a;
    a.cu = view<double>(cu);
    a.npts = a.cu.sn;
    a.nvars = cu.ncomp;
    a.ns = ns;
    a.rho0 = rho0;
    a.rhoE = rhoE;
    for (int i = 0; i < MAXS; ++i) a.rhoY[i] = i < ns ? rhoY[i] : 0.0;
    k_init_uniform<<<grid_for(a.npts, 256), 256, 0, s>>>(a);
    return cuda_rc(cudaGetLastError());
}

int num_tiles() { return kNumStageBlocks + kNumZmTiles; }

// 0-4: the split stage (stress, face and update kernels) with the face kernel's
// block size / register cap; 5-8: the fused z-marching stage kernel with its
// block size and z-chunk depth
const char* tile_name(int t) {
    static const char* names[] = {"b128-min4", "b256-min2", "b128-min6", "b128-min10", "b128-min8",
                                  "fused16x8-t128-z32", "fused16x8-t256-z32", "fused16x8-t256-z64",
                                  "fused16x8-t384-z32"};
    return (t >= 0 && t < num_tiles()) ? names[t] : "?";
}

bool tile_fused(int t) { return tile_is_fused(t); }

}  // namespace fhd
