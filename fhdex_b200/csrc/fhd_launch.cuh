// fhd_launch.cuh — templated launchers included by each kernel translation unit.
#pragma once
#include "fhd_host.h"
#include "fhd_kernels.cuh"
#include "fhd_fused.cuh"
#include "fhd_walls.cuh"

namespace fhd {

template <class T>
inline Arr4<T> view(const fhd_fab& f, int comp0 = 0) {
    Arr4<T> a;
    const int64_t nx = f.hi[0] - f.lo[0] + 1, ny = f.hi[1] - f.lo[1] + 1, nz = f.hi[2] - f.lo[2] + 1;
    a.lo0 = f.lo[0];
    a.lo1 = f.lo[1];
    a.lo2 = f.lo[2];
    a.sy = nx;
    a.sz = nx * ny;
    a.sn = nx * ny * nz;
    a.p = f.data ? static_cast<T*>(f.data) + comp0 * a.sn : nullptr;
    return a;
}

// Grid of a grid-stride kernel: as many blocks as the SMs hold at once (the kernel's
// occupancy at this block size, queried once per kernel and block size), so that
// every block runs from the start and all finish together instead of leaving a
// partly filled last wave; fewer when there is less work.
inline int device_sms() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) {
            cudaGetLastError();
            sms = 148;
        }
    }
    return sms;
}

template <auto K>
inline int resident_blocks(int block) {
    static int cache[3] = {0, 0, 0};  // block sizes 128, 256, other
    const int slot = block == 128 ? 0 : (block == 256 ? 1 : 2);
    if (slot == 2 || !cache[slot]) {
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, K, block, 0) != cudaSuccess || nb < 1) {
            cudaGetLastError();
            nb = 1;
        }
        if (slot == 2) return nb * device_sms();
        cache[slot] = nb * device_sms();
    }
    return cache[slot];
}

template <auto K>
inline int resident_grid(int64_t items, int block) {
    int64_t g = (items + block - 1) / block;
    const int cap = resident_blocks<K>(block);
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

inline int grid_for(int64_t items, int block, int cap = 148 * 32) {
    int64_t g = (items + block - 1) / block;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

inline int cuda_rc(cudaError_t e) { return e == cudaSuccess ? FHD_OK : FHD_ERR_CUDA; }

template <int NS, class R>
Fields<NS, R> make_fields(const StageCall& c) {
    Fields<NS, R> F;
    F.cons = view<const double>(c.cons_s);
    for (int d = 0; d < 3; ++d) {
        F.mom[d] = view<const double>(c.mom_s[d]);
        F.vel[d] = view<const double>(c.vel[d]);
    }
    F.pr = view<const double>(c.pr);
    F.pT = c.pT;
    F.eta = view<const R>(c.eta);
    F.zeta = view<const R>(c.zeta);
    F.kappa = view<const R>(c.kappa);
    F.chi = view<const R>(c.chi);
    F.D = view<const R>(c.D);
    return F;
}

template <int MODE>
Noise<MODE> make_noise(const StageCall& c) {
    Noise<MODE> n;
    n.w = c.w;
    for (int d = 0; d < 3; ++d) {
        n.a.fa[d] = view<const double>(c.nz.fa[d]);
        n.a.fb[d] = view<const double>(c.nz.fb[d]);
        n.a.foa[d] = c.nz.fa[d].ncomp - (c.P.ns + 1);
        n.a.fob[d] = c.nz.fb[d].ncomp - (c.P.ns + 1);
        n.a.ea[d] = view<const double>(c.nz.ea[d]);
        n.a.eb[d] = view<const double>(c.nz.eb[d]);
        n.a.ca[d] = view<const double>(c.nz.ca[d]);
        n.a.cb[d] = view<const double>(c.nz.cb[d]);
    }
    return n;
}

template <int NS, class R>
int launch_cellprep(const StageCall& c) {
    PrepArgs<NS, R> a;
    a.P = c.P;
    a.cons = view<const double>(c.cons_s);
    for (int d = 0; d < 3; ++d) {
        a.mom[d] = view<const double>(c.mom_s[d]);
        a.vel[d] = view<double>(c.vel[d]);
    }
    a.pr = view<double>(c.pr, c.pT);
    a.eta = view<R>(c.eta);
    a.zeta = view<R>(c.zeta);
    a.kappa = view<R>(c.kappa);
    a.chi = view<R>(c.chi);
    a.D = view<R>(c.D);
    a.status = c.status;
    const int64_t tot = (int64_t)(c.P.n[0] + 3) * (c.P.n[1] + 3) * (c.P.n[2] + 3);
    // (an occupancy-sized grid was measured slower here: blocks beyond the resident
    // set rebalance this kernel's uneven per-cell cost)
    k_cellprep<NS, R><<<grid_for(tot, 128), 128, 0, c.stream>>>(a);
    return cuda_rc(cudaGetLastError());
}

// launch shapes available to the autotuner: block size of the stage kernels and
// the register cap of the face-flux kernel (minimum resident blocks per SM)
constexpr int kStageBlocks[] = {128, 256, 128, 128, 128};
constexpr int kFaceMinBlocks[] = {4, 2, 6, 10, 8};  // as instantiated in launch_stage_part_t
constexpr int kNumStageBlocks = 5;
// the fused stage kernel (k_stage_zm): tile of 16 x 8 cells; per fused tile the
// block size (128, 256 or 384 threads over the same tile) and the z-chunk depth
constexpr int kZmTX = 16, kZmTY = 8;
constexpr int kZmThreads[] = {128, 256, 256, 384};
constexpr int kZmChunks[] = {32, 32, 64, 32};
constexpr int kNumZmTiles = 4;
inline bool tile_is_fused(int t) { return t >= kNumStageBlocks && t < kNumStageBlocks + kNumZmTiles; }

template <int NS, class R, int NZ>
StageArgs<NS, R, NZ> make_stage_args(const StageCall& c) {
    StageArgs<NS, R, NZ> a;
    a.P = c.P;
    a.F = make_fields<NS, R>(c);
    a.noise = make_noise<NZ>(c);
    a.ct = view<R>(c.ct);
    a.et = view<R>(c.et);
    a.mc = view<double>(c.smc);
    a.me = view<double>(c.sme);
    for (int d = 0; d < 3; ++d) {
        a.ff[d] = view<double>(c.sff[d]);
        a.mom0[d] = view<const double>(c.mom0[d]);
        a.mom_o[d] = view<double>(c.mom_o[d]);
    }
    a.cons0 = view<const double>(c.cons0);
    a.cons_o = view<double>(c.cons_o);
    a.src = view<const double>(c.src);
    a.stage = c.stage;
    return a;
}

inline int stage_block(const StageCall& c) {
    return (c.tile >= 0 && c.tile < kNumStageBlocks) ? kStageBlocks[c.tile] : 128;
}

// part: 0 stresses, 1 face fluxes (all three directions), 2 update
template <int NS, class R, int NZ>
int launch_stage_part_t(const StageCall& c, int part) {
    const StageArgs<NS, R, NZ> a = make_stage_args<NS, R, NZ>(c);
    const int* N = c.P.n;
    const int b = stage_block(c);
    if (part == 0) {
        k_taus<NS, R, NZ><<<grid_for((int64_t)(N[0] + 2) * (N[1] + 2) * (N[2] + 2), b), b, 0, c.stream>>>(a);
    } else if (part == 1) {
        const int t = (c.tile >= 0 && c.tile < kNumStageBlocks) ? c.tile : 0;
#define FHD_FACES(BS, MINB)                                                                                      \
        k_faces<NS, R, NZ, 0, BS, MINB><<<resident_grid<k_faces<NS, R, NZ, 0, BS, MINB>>(                     \
            (int64_t)(N[0] + 1) * N[1] * N[2], BS), BS, 0, c.stream>>>(a);                                     \
        k_faces<NS, R, NZ, 1, BS, MINB><<<resident_grid<k_faces<NS, R, NZ, 1, BS, MINB>>(                     \
            (int64_t)N[0] * (N[1] + 1) * N[2], BS), BS, 0, c.stream>>>(a);                                     \
        k_faces<NS, R, NZ, 2, BS, MINB><<<resident_grid<k_faces<NS, R, NZ, 2, BS, MINB>>(                     \
            (int64_t)N[0] * N[1] * (N[2] + 1), BS), BS, 0, c.stream>>>(a);
        switch (t) {
            case 0: FHD_FACES(128, 4) break;
            case 1: FHD_FACES(256, 2) break;
            case 2: FHD_FACES(128, 6) break;
            case 3: FHD_FACES(128, 10) break;
            default: FHD_FACES(128, 8) break;
        }
#undef FHD_FACES
    } else {
        // 128 threads whatever the tile: the update kernel is capped at 32 registers
        // for full occupancy (16 blocks of 128 per SM)
        k_update<NS, R, NZ><<<resident_grid<k_update<NS, R, NZ>>((int64_t)(N[0] + 1) * (N[1] + 1) * (N[2] + 1), 128),
                               128, 0, c.stream>>>(a);
    }
    return cuda_rc(cudaGetLastError());
}

// resident blocks per SM asked of the register allocator: the shared memory of a
// 16 x 8 tile (56-80 KB) holds 2-4 blocks per SM
template <int NS, class R>
constexpr int zm_min_blocks(int bt) {
    return bt == 128 ? (sizeof(R) == 8 ? (NS <= 2 ? 3 : 2) : (NS <= 2 ? 4 : 3)) : (bt == 256 ? (NS <= 2 ? 3 : 2) : 2);
}

template <int NS, class R, int NZ, int BT>
int launch_stage_zm_bt(const StageCall& c, int zc) {
    constexpr int TX = kZmTX, TY = kZmTY;
    constexpr size_t smem = ZmSmem<NS, R, TX, TY>::bytes;
    auto kern = k_stage_zm<NS, R, NZ, TX, TY, BT, zm_min_blocks<NS, R>(BT)>;
    // the dynamic shared memory above 48 KiB is opted into per device, once
    static bool set[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_CUDA; }
    if (dev < 0 || dev >= 64) return FHD_ERR_UNSUPPORTED;
    if (!set[dev]) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
            cudaGetLastError();
            return FHD_ERR_CUDA;
        }
        set[dev] = true;
    }
    const StageArgs<NS, R, NZ> a = make_stage_args<NS, R, NZ>(c);
    const int* N = c.P.n;
    const dim3 grid((N[0] + TX - 1) / TX, (N[1] + TY - 1) / TY, (N[2] + zc - 1) / zc);
    kern<<<grid, BT, smem, c.stream>>>(a, zc);
    return cuda_rc(cudaGetLastError());
}

template <int NS, class R, int NZ>
int launch_stage_zm_t(const StageCall& c) {
    const int t = tile_is_fused(c.tile) ? c.tile - kNumStageBlocks : 0;
    switch (kZmThreads[t]) {
        case 256: return launch_stage_zm_bt<NS, R, NZ, 256>(c, kZmChunks[t]);
        case 384: return launch_stage_zm_bt<NS, R, NZ, 384>(c, kZmChunks[t]);
        default: return launch_stage_zm_bt<NS, R, NZ, 128>(c, kZmChunks[t]);
    }
}

// the stage parts of a box with physical walls (FP64, one launch shape): the wall
// variants of the stresses and face fluxes, and the common update
template <int NS, int NZ>
int launch_walls_part_t(const StageCall& c, int part) {
    const StageArgs<NS, double, NZ> a = make_stage_args<NS, double, NZ>(c);
    const int* N = c.P.n;
    if (part == 0) {
        k_taus<NS, double, NZ, true><<<grid_for((int64_t)(N[0] + 2) * (N[1] + 2) * (N[2] + 2), 128), 128, 0, c.stream>>>(a);
    } else if (part == 1) {
        // register cap: 64 up to two species (the periodic autotuner's choice at 256^3;
        // 128 was measured twice as slow for the wall variant), 128 above
        constexpr int MB = NS <= 2 ? 8 : 4;
        k_faces<NS, double, NZ, 0, 128, MB, true><<<resident_grid<k_faces<NS, double, NZ, 0, 128, MB, true>>(
            (int64_t)(N[0] + 1) * N[1] * N[2], 128), 128, 0, c.stream>>>(a);
        k_faces<NS, double, NZ, 1, 128, MB, true><<<resident_grid<k_faces<NS, double, NZ, 1, 128, MB, true>>(
            (int64_t)N[0] * (N[1] + 1) * N[2], 128), 128, 0, c.stream>>>(a);
        k_faces<NS, double, NZ, 2, 128, MB, true><<<resident_grid<k_faces<NS, double, NZ, 2, 128, MB, true>>(
            (int64_t)N[0] * N[1] * (N[2] + 1), 128), 128, 0, c.stream>>>(a);
    } else {
        k_update<NS, double, NZ><<<resident_grid<k_update<NS, double, NZ>>(
            (int64_t)(N[0] + 1) * (N[1] + 1) * (N[2] + 1), 128), 128, 0, c.stream>>>(a);
    }
    return cuda_rc(cudaGetLastError());
}

template <int NS>
int launch_walls_part(const StageCall& c, int part) {
    switch (c.mode) {
        case NM_OFF: return launch_walls_part_t<NS, NZ_OFF>(c, part);
        case NM_AB: return launch_walls_part_t<NS, NZ_AB>(c, part);
        case NM_PHILOX: return launch_walls_part_t<NS, NZ_PHILOX>(c, part);
        default: return FHD_ERR_BAD_ARG;
    }
}

// BCMassTempPress + BCRhoRhoE on the ghost cells of the wall directions
template <int NS>
int launch_bc_prim(const DevParams& P, const WallParams& W, const fhd_fab& prim, const fhd_fab& cons,
                   const fhd_fab mom[3], cudaStream_t s) {
    BcPrimArgs<NS> a;
    a.P = P;
    a.W = W;
    a.prim = view<double>(prim);
    a.cons = view<double>(cons);
    for (int d = 0; d < 3; ++d) a.mom[d] = view<const double>(mom[d]);
    const int g = -prim.lo[0];
    int blo[3], bhi[3], clo[3], chi[3];
    for (int d = 0; d < 3; ++d) {
        blo[d] = -g;
        bhi[d] = P.n[d] - 1 + g;
        const bool w = P.walls && !P.periodic[d];
        clo[d] = w ? 0 : blo[d];
        chi[d] = w ? P.n[d] - 1 : bhi[d];
    }
    a.sh = make_shell(blo, bhi, clo, chi);
    if (a.sh.n == 0) return FHD_OK;
    k_bc_prim<NS><<<grid_for(a.sh.n, 128), 128, 0, s>>>(a);
    return cuda_rc(cudaGetLastError());
}

// The reference's boundary passes in its order, one launch each (k_bc_pass):
// for each direction d BCMassTempPress (lo, hi) and BCMomNormal (lo, hi) of
// mom[d] / vel[d] when d has walls, and BCMomTrans of mom[d] / vel[d] across the
// other directions' walls (x lo, x hi, y lo, ...); with rre, BCRhoRhoE of every
// wall side after them (setBCStag); without, the passes RK3stepStag makes before
// the conversion.
template <int NS>
int launch_bc_seq(const DevParams& P, const WallParams& W, const fhd_fab& prim, const fhd_fab& cons,
                  const fhd_fab* mom, const fhd_fab* vel, bool rre, cudaStream_t st) {
    BcPassArgs<NS> a;
    a.P = P;
    a.W = W;
    a.prim = view<double>(prim);
    a.cons = view<double>(cons);
    a.mx = view<const double>(mom[0]);
    a.my = view<const double>(mom[1]);
    a.mz = view<const double>(mom[2]);
    const int g = -prim.lo[0], gm = -mom[0].lo[0];
    auto wall = [&](int d) { return P.walls && !P.periodic[d]; };
    auto launch = [&](int fn, int side, int c) {
        a.fn = fn;
        a.side = side;
        a.c = c;
        const int d = side >> 1, hi = side & 1;
        for (int e = 0; e < 3; ++e) {
            const bool cell = fn == BC_MTP || fn == BC_RRE;
            const int gg = cell ? g : gm;
            const int nod = (!cell && e == c) ? 1 : 0;
            a.blo[e] = -gg;
            a.bhi[e] = P.n[e] - 1 + nod + gg;
            if (e == d) {
                if (fn == BC_MOMN) { a.blo[e] = hi ? P.n[e] : -gg; a.bhi[e] = hi ? P.n[e] + gg : 0; }
                else { a.blo[e] = hi ? P.n[e] : -gg; a.bhi[e] = hi ? P.n[e] + gg - 1 : -1; }
            }
        }
        if (fn == BC_MOMN || fn == BC_MOMT) {
            a.mom = view<double>(mom[c]);
            a.vel = view<double>(vel[c]);
        }
        const int64_t tot = (int64_t)(a.bhi[0] - a.blo[0] + 1) * (a.bhi[1] - a.blo[1] + 1) * (a.bhi[2] - a.blo[2] + 1);
        k_bc_pass<NS><<<grid_for(tot, 128), 128, 0, st>>>(a);
        return cuda_rc(cudaGetLastError());
    };
    int rc = FHD_OK;
    // every direction d: its own sides' passes when it has walls, and BCMomTrans of
    // mom[d] / vel[d] across the other directions' walls in any case
    for (int d = 0; d < 3 && !rc; ++d) {
        for (int h = 0; h < 2 && !rc && wall(d); ++h) rc = launch(BC_MTP, 2 * d + h, d);
        for (int h = 0; h < 2 && !rc && wall(d); ++h) rc = launch(BC_MOMN, 2 * d + h, d);
        for (int e = 0; e < 3 && !rc; ++e) {
            if (e == d || !wall(e)) continue;
            for (int h = 0; h < 2 && !rc; ++h) rc = launch(BC_MOMT, 2 * e + h, d);
        }
    }
    for (int side = 0; side < 6 && rre && !rc; ++side)
        if (wall(side >> 1)) rc = launch(BC_RRE, side, 0);
    return rc;
}

// the particle reservoir's fluxes and momenta (k_reservoir), the flux reset of one
// reservoir side (k_res_reset)
template <int NS>
int launch_reservoir(const ResArgs& a, cudaStream_t s) {
    if (a.face_pref[a.nsides] == 0) return FHD_OK;
    k_reservoir<NS><<<grid_for(a.face_pref[a.nsides], 128), 128, 0, s>>>(a);
    return cuda_rc(cudaGetLastError());
}

template <int NS>
int launch_res_reset(const ResResetArgs& a, cudaStream_t s) {
    const int d = a.side >> 1, e1 = d == 0 ? 1 : 0, e2 = d == 2 ? 1 : 2;
    const int64_t n = (int64_t)a.P.n[e1] * a.P.n[e2] + (int64_t)(a.P.n[e1] + 1) * a.P.n[e2] +
                      (int64_t)a.P.n[e1] * (a.P.n[e2] + 1);
    k_res_reset<NS><<<grid_for(n, 128), 128, 0, s>>>(a);
    return cuda_rc(cudaGetLastError());
}

// part: 0 stresses, 1 face fluxes, 2 update, 3 the fused kernel (all three)
template <int NS, class R>
int launch_stage_part(const StageCall& c, int part) {
    if (part == 3) {
        switch (c.mode) {
            case NM_OFF: return launch_stage_zm_t<NS, R, NZ_OFF>(c);
            case NM_AB: return launch_stage_zm_t<NS, R, NZ_AB>(c);
            case NM_PHILOX: return launch_stage_zm_t<NS, R, NZ_PHILOX>(c);
            default: return FHD_ERR_BAD_ARG;
        }
    }
    switch (c.mode) {
        case NM_OFF: return launch_stage_part_t<NS, R, NZ_OFF>(c, part);
        case NM_AB: return launch_stage_part_t<NS, R, NZ_AB>(c, part);
        case NM_PHILOX: return launch_stage_part_t<NS, R, NZ_PHILOX>(c, part);
        default: return FHD_ERR_BAD_ARG;
    }
}

// ---- batched launches ------------------------------------------------------------
// kinds: 0 cellprep, 1 stresses, 2-4 face fluxes x/y/z, 5 update, 6 conversion.
// For the conversion kind the StageCall carries prim in pr, cu in cons_o, mom in mom_o.
template <int NS>
ConvArgs<NS> make_conv_args(const StageCall& c) {
    ConvArgs<NS> a;
    a.P = c.P;
    a.prim = view<double>(c.pr);
    a.cons = view<double>(c.cons_o);
    for (int d = 0; d < 3; ++d) {
        a.vel[d] = view<double>(c.vel[d]);
        a.mom[d] = view<const double>(c.mom_o[d]);
    }
    a.status = c.status;
    return a;
}

template <int NS, class R>
PrepArgs<NS, R> make_prep_args(const StageCall& c) {
    PrepArgs<NS, R> a;
    a.P = c.P;
    a.cons = view<const double>(c.cons_s);
    for (int d = 0; d < 3; ++d) {
        a.mom[d] = view<const double>(c.mom_s[d]);
        a.vel[d] = view<double>(c.vel[d]);
    }
    a.pr = view<double>(c.pr, c.pT);
    a.eta = view<R>(c.eta);
    a.zeta = view<R>(c.zeta);
    a.kappa = view<R>(c.kappa);
    a.chi = view<R>(c.chi);
    a.D = view<R>(c.D);
    a.status = c.status;
    return a;
}

template <int NS, class R, int NZ>
size_t batch_args_size_t(int kind) {
    if (kind == 0) return sizeof(PrepArgs<NS, R>);
    if (kind == 6) return sizeof(ConvArgs<NS>);
    return sizeof(StageArgs<NS, R, NZ>);
}

template <int NS, class R, int NZ>
void batch_pack_t(int kind, const StageCall& c, void* dst) {
    if (kind == 0) {
        const PrepArgs<NS, R> a = make_prep_args<NS, R>(c);
        memcpy(dst, &a, sizeof(a));
    } else if (kind == 6) {
        const ConvArgs<NS> a = make_conv_args<NS>(c);
        memcpy(dst, &a, sizeof(a));
    } else {
        const StageArgs<NS, R, NZ> a = make_stage_args<NS, R, NZ>(c);
        memcpy(dst, &a, sizeof(a));
    }
}

// register caps of the batched face kernel (resident blocks of 128 per SM), the
// batch autotuner's choices; the default is the first for up to two species and
// the last above
constexpr int kBatchFaceMinBlocks[] = {8, 6, 4};
constexpr int kNumBatchFaceTiles = 3;

template <int NS, class R, int NZ, int MINB>
void batch_faces_t(int kind, const StageArgs<NS, R, NZ>* sa, const int* dbpref, int nmem, int nblocks, cudaStream_t s) {
    if (kind == 2) k_faces_b<NS, R, NZ, 0, MINB><<<nblocks, 128, 0, s>>>(sa, dbpref, nmem);
    else if (kind == 3) k_faces_b<NS, R, NZ, 1, MINB><<<nblocks, 128, 0, s>>>(sa, dbpref, nmem);
    else k_faces_b<NS, R, NZ, 2, MINB><<<nblocks, 128, 0, s>>>(sa, dbpref, nmem);
}

template <int NS, class R, int NZ>
int batch_launch_t(int kind, int tile, const void* dargs, const int* dbpref, int nmem, int nblocks, cudaStream_t s) {
    if (nblocks <= 0 || nmem <= 0) return FHD_OK;
    using SA = StageArgs<NS, R, NZ>;
    const SA* sa = static_cast<const SA*>(dargs);
    switch (kind) {
        case 0: k_cellprep_b<NS, R><<<nblocks, 128, 0, s>>>(static_cast<const PrepArgs<NS, R>*>(dargs), dbpref, nmem); break;
        case 1: k_taus_b<NS, R, NZ><<<nblocks, 128, 0, s>>>(sa, dbpref, nmem); break;
        case 2:
        case 3:
        case 4:
            if (tile < 0 || tile >= kNumBatchFaceTiles) tile = NS <= 2 ? 0 : kNumBatchFaceTiles - 1;
            if (tile == 0) batch_faces_t<NS, R, NZ, kBatchFaceMinBlocks[0]>(kind, sa, dbpref, nmem, nblocks, s);
            else if (tile == 1) batch_faces_t<NS, R, NZ, kBatchFaceMinBlocks[1]>(kind, sa, dbpref, nmem, nblocks, s);
            else batch_faces_t<NS, R, NZ, kBatchFaceMinBlocks[2]>(kind, sa, dbpref, nmem, nblocks, s);
            break;
        case 5: k_update_b<NS, R, NZ><<<nblocks, 128, 0, s>>>(sa, dbpref, nmem); break;
        case 6: k_convert_b<NS><<<nblocks, 128, 0, s>>>(static_cast<const ConvArgs<NS>*>(dargs), dbpref, nmem); break;
        default: return FHD_ERR_BAD_ARG;
    }
    return cuda_rc(cudaGetLastError());
}

// the persistent batched step: grid = the blocks that fit on the GPU at once
template <int NS, class R, int NZ, int MINB>
int batch_persist_minb(const PersistArgs& a, cudaStream_t s) {
    const int grid = resident_blocks<k_batch_persist<NS, R, NZ, MINB>>(128);
    k_batch_persist<NS, R, NZ, MINB><<<grid, 128, 0, s>>>(a);
    return cuda_rc(cudaGetLastError());
}

// tile: the register cap of the batch face tiles (kBatchFaceMinBlocks: 64, 80 or
// 128 registers); -1 the default, 64 registers up to two species (measured on the
// 512-member ensemble: 156 / 170 / 223 ms per step FP64, 112 / 124 / 141 mixed)
// and 128 above
template <int NS, class R, int NZ>
int batch_persist_t(const PersistArgs& a, int tile, cudaStream_t s) {
    if (tile < 0 || tile >= kNumBatchFaceTiles) tile = NS <= 2 ? 0 : 2;
    if (tile == 0) return batch_persist_minb<NS, R, NZ, kBatchFaceMinBlocks[0]>(a, s);
    if (tile == 1) return batch_persist_minb<NS, R, NZ, kBatchFaceMinBlocks[1]>(a, s);
    return batch_persist_minb<NS, R, NZ, kBatchFaceMinBlocks[2]>(a, s);
}

#define FHD_NS_SWITCH(ns, CALL) \
    switch (ns) {                \
        case 1: return CALL(1);  \
        case 2: return CALL(2);  \
        case 3: return CALL(3);  \
        case 4: return CALL(4);  \
        default: return FHD_ERR_UNSUPPORTED; \
    }

}  // namespace fhd
