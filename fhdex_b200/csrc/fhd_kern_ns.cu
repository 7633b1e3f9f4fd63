// fhd_kern_ns.cu — kernel instantiations for one species count, compiled once per
// (FHD_NS, precision) pair so the build runs in parallel:
//   -DFHD_NS=<n>                 exact FP64 (built with -fmad=false)
//   -DFHD_NS=<n> -DFHD_MIXED=1   mixed precision (FP32 compute)
#include "fhd_launch.cuh"

#ifndef FHD_NS
#error "FHD_NS must be defined"
#endif

#define FHD_CAT2(a, b) a##b
#define FHD_CAT(a, b) FHD_CAT2(a, b)

namespace fhd {

#if defined(FHD_MIXED) && FHD_MIXED
#define FHD_R float
#define FHD_PFX mixed
#else
#define FHD_R double
#define FHD_PFX exact
#endif

// batched launches of this (species count, precision); mode is NM_PHILOX or NM_OFF
size_t FHD_CAT(FHD_CAT(FHD_PFX, _batch_args_size_ns), FHD_NS)(int kind, int mode) {
    return mode == NM_OFF ? batch_args_size_t<FHD_NS, FHD_R, NZ_OFF>(kind)
                          : batch_args_size_t<FHD_NS, FHD_R, NZ_PHILOX>(kind);
}
void FHD_CAT(FHD_CAT(FHD_PFX, _batch_pack_ns), FHD_NS)(int kind, int mode, const StageCall& c, void* dst) {
    if (mode == NM_OFF) batch_pack_t<FHD_NS, FHD_R, NZ_OFF>(kind, c, dst);
    else batch_pack_t<FHD_NS, FHD_R, NZ_PHILOX>(kind, c, dst);
}
int FHD_CAT(FHD_CAT(FHD_PFX, _batch_launch_ns), FHD_NS)(int kind, int mode, int tile, const void* dargs,
                                                       const int* dbpref, int nmem, int nblocks, cudaStream_t s) {
    return mode == NM_OFF ? batch_launch_t<FHD_NS, FHD_R, NZ_OFF>(kind, tile, dargs, dbpref, nmem, nblocks, s)
                          : batch_launch_t<FHD_NS, FHD_R, NZ_PHILOX>(kind, tile, dargs, dbpref, nmem, nblocks, s);
}

int FHD_CAT(FHD_CAT(FHD_PFX, _batch_persist_ns), FHD_NS)(int mode, int tile, const PersistArgs& a, cudaStream_t s) {
    return mode == NM_OFF ? batch_persist_t<FHD_NS, FHD_R, NZ_OFF>(a, tile, s)
                          : batch_persist_t<FHD_NS, FHD_R, NZ_PHILOX>(a, tile, s);
}

#if defined(FHD_MIXED) && FHD_MIXED
int FHD_CAT(mixed_cellprep_ns, FHD_NS)(const StageCall& c) { return launch_cellprep<FHD_NS, float>(c); }
int FHD_CAT(mixed_stage_ns, FHD_NS)(const StageCall& c, int part) { return launch_stage_part<FHD_NS, float>(c, part); }
#else
int FHD_CAT(exact_cellprep_ns, FHD_NS)(const StageCall& c) { return launch_cellprep<FHD_NS, double>(c); }
int FHD_CAT(exact_stage_ns, FHD_NS)(const StageCall& c, int part) { return launch_stage_part<FHD_NS, double>(c, part); }

template <int NS, int NZ, bool WL>
int launch_aux_t(const StageCall& c) {
    AuxArgs<NS, double, NZ> a;
    a.P = c.P;
    a.F = make_fields<NS, double>(c);
    a.noise = make_noise<NZ>(c);
    for (int d = 0; d < 3; ++d) {
        a.ff[d] = view<double>(c.ff[d]);
        a.cf[d] = view<double>(c.cf[d]);
    }
    for (int e = 0; e < 6; ++e) a.ef[e] = view<double>(c.ef[e]);
    const int* N = c.P.n;
    const int64_t nf = (int64_t)(N[0] + 1) * N[1] * N[2] + (int64_t)N[0] * (N[1] + 1) * N[2] +
                       (int64_t)N[0] * N[1] * (N[2] + 1);
    const int64_t ne = (int64_t)(N[0] + 1) * (N[1] + 1) * N[2] + (int64_t)(N[0] + 1) * N[1] * (N[2] + 1) +
                       (int64_t)N[0] * (N[1] + 1) * (N[2] + 1) + (int64_t)(N[0] + 2) * (N[1] + 2) * (N[2] + 2);
    if (c.ff[0].data) k_aux_faces<NS, double, NZ, WL><<<grid_for(nf, 128), 128, 0, c.stream>>>(a);
    if (c.ef[0].data) k_aux_edges_cen<NS, double, NZ, WL><<<grid_for(ne, 128), 128, 0, c.stream>>>(a);
    return cuda_rc(cudaGetLastError());
}

template <bool WL>
int aux_mode(const StageCall& c) {
    switch (c.mode) {
        case NM_OFF: return launch_aux_t<FHD_NS, NZ_OFF, WL>(c);
        case NM_W: return launch_aux_t<FHD_NS, NZ_W, WL>(c);
        case NM_AB: return launch_aux_t<FHD_NS, NZ_AB, WL>(c);
        case NM_PHILOX: return launch_aux_t<FHD_NS, NZ_PHILOX, WL>(c);
        default: return FHD_ERR_BAD_ARG;
    }
}

// the wall variants also carry the quasi-1-D / 2-D branches
int FHD_CAT(exact_aux_ns, FHD_NS)(const StageCall& c) {
    return (c.P.walls || c.P.dim < 3) ? aux_mode<true>(c) : aux_mode<false>(c);
}

int FHD_CAT(exact_walls_ns, FHD_NS)(const StageCall& c, int part) { return launch_walls_part<FHD_NS>(c, part); }

int FHD_CAT(exact_bc_prim_ns, FHD_NS)(const DevParams& P, const WallParams& W, fhd_fab prim, fhd_fab cons,
                                      const fhd_fab* mom, cudaStream_t s) {
    return launch_bc_prim<FHD_NS>(P, W, prim, cons, mom, s);
}

int FHD_CAT(exact_reservoir_ns, FHD_NS)(const ResArgs& a, cudaStream_t s) { return launch_reservoir<FHD_NS>(a, s); }
int FHD_CAT(exact_res_reset_ns, FHD_NS)(const ResResetArgs& a, cudaStream_t s) { return launch_res_reset<FHD_NS>(a, s); }

int FHD_CAT(exact_bc_seq_ns, FHD_NS)(const DevParams& P, const WallParams& W, fhd_fab prim, fhd_fab cons,
                                     const fhd_fab* mom, const fhd_fab* vel, int rre, cudaStream_t s) {
    return launch_bc_seq<FHD_NS>(P, W, prim, cons, mom, vel, rre != 0, s);
}

int FHD_CAT(exact_transport_ns, FHD_NS)(const DevParams& P, fhd_fab prim, fhd_fab eta, fhd_fab zeta, fhd_fab kappa,
                                        fhd_fab chi, fhd_fab D, int* status, cudaStream_t s) {
    TransArgs<FHD_NS> a;
    a.P = P;
    a.prim = view<const double>(prim);
    a.eta = view<double>(eta);
    a.zeta = view<double>(zeta);
    a.kappa = view<double>(kappa);
    a.chi = view<double>(chi);
    a.D = view<double>(D);
    // the grown box that every coefficient fab and prim cover
    int g = -prim.lo[0];
    for (const fhd_fab* f : {&eta, &zeta, &kappa, &chi, &D}) g = -f->lo[0] < g ? -f->lo[0] : g;
    // a quasi-1-D run computes them on the box grown by one only (transCoeffs.cpp:18-21)
    if (P.dim == 1 && g > 1) g = 1;
    a.ng = g;
    a.status = status;
    const int64_t tot = (int64_t)(P.n[0] + 2 * a.ng) * (P.n[1] + 2 * a.ng) * (P.n[2] + 2 * a.ng);
    k_transport<FHD_NS><<<grid_for(tot, 128), 128, 0, s>>>(a);
    return cuda_rc(cudaGetLastError());
}

int FHD_CAT(exact_convert_ns, FHD_NS)(const DevParams& P, fhd_fab prim, const fhd_fab vel[3], fhd_fab cons,
                                      const fhd_fab mom[3], int* status, cudaStream_t s) {
    ConvArgs<FHD_NS> a;
    a.P = P;
    a.prim = view<double>(prim);
    a.cons = view<double>(cons);
    for (int d = 0; d < 3; ++d) {
        a.vel[d] = view<double>(vel[d]);
        a.mom[d] = view<const double>(mom[d]);
    }
    a.status = status;
    const int64_t tot = (int64_t)P.n[0] * P.n[1] * P.n[2];
    k_convert<FHD_NS><<<resident_grid<k_convert<FHD_NS>>(tot, 128), 128, 0, s>>>(a);
    return cuda_rc(cudaGetLastError());
}
#endif

}  // namespace fhd
