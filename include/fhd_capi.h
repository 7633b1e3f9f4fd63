/*
 * fhd_capi.h — C ABI of the B200-native compressible staggered-grid FHD step.
 *
 * Drop-in boundary for FHDeX's explicit compressible staggered-grid step.  Every
 * entry point below replaces one C++ free function of the reference; the
 * reference function it stands for is cited beside it (paths are relative to the
 * FHDeX source tree).  The reference passes AMReX MultiFabs and reads physics
 * parameters from global namespaces (common::, compressible::); here a MultiFab
 * of one box is an `fhd_fab` (plain pointer + AMReX Array4 geometry) and the
 * parameters live in an `fhd_params` given once to `fhd_create`.
 *
 * Data layout (identical to AMReX Array4): element (i,j,k,n) of a fab is at
 *   data[(i-lo0) + (j-lo1)*nx + (k-lo2)*nx*ny + n*nx*ny*nz],  nx = hi0-lo0+1, ...
 * i.e. Fortran order with the component slowest.  lo/hi are ghost-inclusive and
 * inclusive.  A fab that is nodal in direction d has valid indices 0..n_cells[d]
 * in d; a cell-centred one 0..n_cells[d]-1.  Ghost width = -lo[d].
 *
 * Memory: fabs handed to the compute entry points are DEVICE pointers on the
 * context's device unless the entry point says otherwise (the *_host variants
 * take host pointers and copy).  All work is ordered on the context's stream;
 * calls return after enqueueing unless stated.  No entry point aborts the
 * process: failures are returned as FHD_ERR_* codes; physics faults detected on
 * the device (non-positive/over-unity mass fraction, non-finite temperature) are
 * latched in a device status word and returned by fhd_status().
 *
 * Threading: one host thread at a time per context.
 */
#ifndef FHD_CAPI_H
#define FHD_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FHD_MAX_SPECIES 8
#define FHD_MAX_REACTIONS 8

/* return / status codes */
enum {
    FHD_OK = 0,
    FHD_ERR_BAD_ARG = 1,     /* shape, dtype or parameter rejected on the host   */
    FHD_ERR_MASSFRAC = 2,    /* Y <= 0 or Y >= 1 seen (transCoeffs.cpp:45-46)     */
    FHD_ERR_NONFINITE = 3,   /* non-finite temperature/pressure produced          */
    FHD_ERR_OOM = 4,         /* device allocation failed                          */
    FHD_ERR_TIMEOUT = 5,     /* a bounded device wait gave up                     */
    FHD_ERR_CUDA = 6,        /* a CUDA runtime call failed                        */
    FHD_ERR_UNSUPPORTED = 7, /* option outside the implemented scope              */
    FHD_ERR_TOO_LARGE = 8,   /* box does not fit fhd_rk3_step_stag_noalloc's scratch */
    FHD_ERR_SINGULAR = 9,    /* a singular Valk/Waldmann system (the reference's Decomp aborts) */
    FHD_ERR_IO = 10          /* a file could not be created, written, read or closed   */
};

/* fab element types */
enum { FHD_F64 = 0, FHD_F32 = 1 };

/* precision modes of the step */
enum {
    FHD_PREC_FP64 = 0,   /* every operation in FP64, reference operation order     */
    FHD_PREC_MIXED = 1   /* FP32 fluxes/coefficients, FP64 state and RK sums       */
};

/* One box of an AMReX MultiFab (Array4 view).  `nodal[d]` = 1 for a
 * face/edge-centred direction (AMReX IndexType). */
typedef struct {
    void* data;
    int lo[3];
    int hi[3];
    int ncomp;
    int nodal[3];
    int dtype;
} fhd_fab;

/* Physics and grid parameters.  Field names follow the reference's inputs-deck
 * keys (common_functions.cpp:293-1010, compressible_functions.cpp:15-88).
 * hcv/hcp < 0 are derived from dof as GetHcGas does
 * (compressible_functions.cpp:91-100). */
typedef struct {
    int nspecies;
    int n_cells[3];
    double prob_lo[3];
    double prob_hi[3];
    double molmass[FHD_MAX_SPECIES];
    double diameter[FHD_MAX_SPECIES];
    double dof[FHD_MAX_SPECIES];
    double e0[FHD_MAX_SPECIES];
    double hcv[FHD_MAX_SPECIES];
    double hcp[FHD_MAX_SPECIES];
    double k_B;
    double Runiv;
    double grav[3];
    double zeta_ratio;
    int algorithm_type;     /* only 2 (multispecies) is accepted, as in every stag deck */
    int visc_type;          /* 1, 2 or 3 (|visc_type| == 3 adds bulk viscosity)         */
    int advection_type;     /* 0, 1 or 2                                               */
    int transport_type;     /* only 1 (Giovangigli) is accepted                         */
    int stoch_stress_form;  /* 0 (no noise) or 1                                       */
    int precision;          /* FHD_PREC_*                                               */
    uint64_t seed;          /* key of the in-kernel Philox noise                        */
    /* Chemistry source of the compressible step
     * (compute_compressible_chemistry_source_CLE, chemistry_functions.cpp:128-193;
     * deck keys chemistry_functions.cpp:45-124, stoich_<m>R / stoich_<m>P per
     * reaction).  nreaction = 0: no chemistry. */
    int nreaction;          /* 0 .. FHD_MAX_REACTIONS                                   */
    int reaction_type;      /* 0 deterministic, 1 chemical Langevin (CLE)               */
    int stoich_R[FHD_MAX_REACTIONS][FHD_MAX_SPECIES];  /* reactant coefficients >= 0   */
    int stoich_P[FHD_MAX_REACTIONS][FHD_MAX_SPECIES];  /* product coefficients >= 0    */
    double rate_const[FHD_MAX_REACTIONS];
    double alpha_param[FHD_MAX_REACTIONS];  /* activation: exp(-alpha/Runiv (1/T - 1/T0)) */
    double beta_param[FHD_MAX_REACTIONS];   /* (T/T0)^beta                                 */
    double T0_chem;         /* > 0 when nreaction > 0                                   */
    double avogadro;        /* <= 0: Runiv / k_B (common_functions.cpp:775)             */
    /* Physical boundaries (boundaryStag.cpp; deck keys bc_vel_lo/hi, bc_mass_lo/hi,
     * bc_therm_lo/hi, t_lo/hi, bc_Yk_<x|y|z>_lo/hi, bc_Xk_<x|y|z>_lo/hi).  walls = 0:
     * fully periodic and the fields below are ignored.  walls = 1: direction d is
     * periodic when bc_vel_lo[d] == bc_vel_hi[d] == -1; otherwise both of its sides
     * are walls with bc_vel 1 (slip) or 2 (no-slip), bc_therm 1 (adiabatic) or 2
     * (isothermal at t_lo[d] / t_hi[d]) and bc_mass 1 (impermeable) or 2 (species
     * held at the wall composition bc_Yk / bc_Xk, of which the one summing to 1
     * defines the other, as SetupCWallStag does; fhd_get_params returns both)
     * or 3 (a reservoir: ghost cells held at the reservoir state t, p_lo / p_hi
     * (<= 0: the initial state's pressure), rho_lo / rho_hi (<= 0: from p, t, Y;
     * else t <= 0 is derived from p and rho) and composition bc_Yk / bc_Xk; flow
     * passes the interface) or 4 (the same reservoir, its interface fluxes and
     * momenta from the particles crossing it: ComputeFluxMomReservoir, with Philox
     * draws under the context's seed).  FP64 only; the state's ghost width is then
     * exactly 2 in fhd_rk3_step_stag(s), and the batched and no-allocation steps
     * return FHD_ERR_UNSUPPORTED. */
    int walls;
    int bc_vel_lo[3], bc_vel_hi[3];
    int bc_mass_lo[3], bc_mass_hi[3];
    int bc_therm_lo[3], bc_therm_hi[3];
    double t_lo[3], t_hi[3];
    double bc_Yk_lo[3][FHD_MAX_SPECIES], bc_Yk_hi[3][FHD_MAX_SPECIES];
    double bc_Xk_lo[3][FHD_MAX_SPECIES], bc_Xk_hi[3][FHD_MAX_SPECIES];
    double p_lo[3], p_hi[3], rho_lo[3], rho_hi[3];
    /* The initial state (InitConsVarStag prob_type 1; deck keys rho0, T_init,
     * rhobar): the reservoirs' default pressure. */
    double rho0, T_init;
    double rhobar[FHD_MAX_SPECIES];
    /* The cell x* of the yz-averaged spatial cross-correlations (deck key cross_cell,
     * 0 <= cross_cell < n_cells[0] when fhd_stats_stag is given FHD_STATS_CROSS,
     * as main_driver.cpp:249-251 requires). */
    int cross_cell;
    /* Quasi-1-D / quasi-2-D runs (deck keys do_1D, do_2D; at most one set): the
     * step's noise and stresses only in x (in x and y) and no transverse diffusive
     * fluxes (timeStepStag.cpp:172-323, fluxStag.cpp:171-295, 504-517, 666-680,
     * 875-1010, 1185-1191, 1324-1330, 1850-1860), transport on one ghost layer in
     * 1-D (transCoeffs.cpp:18-21).  FP64 only, no bulk viscosity (main_driver.cpp:
     * 104-118) and no particle reservoir (bc_mass 4); the state's ghost width is
     * then exactly 2, and the batched and no-allocation steps return
     * FHD_ERR_UNSUPPORTED. */
    int do_1D, do_2D;
    /* With do_1D and FHD_STATS_CROSS: 0 correlates with x* = cross_cell, 1 with the
     * five x* 0, floor(n/4), floor(n/2), floor(3n/4), n-1 (deck key all_correl,
     * statsStag.cpp:168-193). */
    int all_correl;
} fhd_params;

/* Injected Gaussian noise for one RK3 step: the "A" and "B" white-noise fields
 * that RK3stepStag fills once per step (timeStepStag.cpp:99-223) and combines as
 * W = A + w_s B per stage (timeStepStag.cpp:237/568/901).  Index [0] = A,
 * [1] = B.  face[.][d]: nodal in d, 0 ghosts; the energy noise is component
 * ncomp-(nspecies+1) and the species noises follow it (with ncomp = nvars this
 * is the reference's component 4..nvars-1).  edge[.][e]: e = 0 xy, 1 xz, 2 yz
 * edges, 0 ghosts (the reference's stochedge_x[0], stochedge_x[1],
 * stochedge_y[1]; the other three edge fields it fills are never read,
 * fluxStag.cpp:130-132).  cen[.][d]: cell-centred with 1 ghost, variance 2 in
 * 3D.  Values must already be OverrideSync'ed/FillBoundary'ed, as
 * MultiFabFillRandomNormal leaves them.  chem[.]: the reaction noises
 * ranchem_A / ranchem_B (timeStepStag.cpp:148-152, 225-229), cell-centred,
 * nreaction components, 0 ghosts, variance 1; read only when nreaction > 0 and
 * reaction_type is 1 (data == NULL otherwise). */
typedef struct {
    fhd_fab face[2][3];
    fhd_fab edge[2][3];
    fhd_fab cen[2][3];
    fhd_fab chem[2];
} fhd_noise;

typedef struct fhd_ctx fhd_ctx;

/* ---- context ------------------------------------------------------------ */

/* Validates params, derives hcv/hcp, binds `device`, creates a stream. */
int fhd_create(fhd_ctx** ctx, const fhd_params* params, int device);
int fhd_destroy(fhd_ctx* ctx);
const char* fhd_strerror(int code);
/* Enqueue on an external CUDA stream (cudaStream_t as void*; NULL = the legacy
 * default stream).  Until called, the context uses a stream of its own. */
int fhd_set_stream(fhd_ctx* ctx, void* stream);
int fhd_synchronize(fhd_ctx* ctx);
/* Reads and clears the device status word (blocks on the stream). */
int fhd_status(fhd_ctx* ctx);
/* Effective parameters (after GetHcGas and SetupCWallStag). */
int fhd_get_params(const fhd_ctx* ctx, fhd_params* out);
/* Launch shape of the stage kernels (index into fhd_tile_name's list); the
 * autotuner in the host layer times them and sets the fastest.  No reference
 * counterpart (AMReX picks its own launch shapes). */
int fhd_set_tile(fhd_ctx* ctx, int tile);
int fhd_num_tiles(void);
const char* fhd_tile_name(int tile);

/* ---- reference operators -------------------------------------------------- */

/* InitConsVarStag, prob_type 1 (uniform state at rest):
 * compressible_functions_stag.cpp:36-56.  Fills every point incl. ghosts. */
int fhd_init_cons_var_stag(fhd_ctx* ctx, fhd_fab cu, const fhd_fab mom[3],
                           double rho0, double T_init, const double* rhobar);

/* conservedToPrimitiveStag: conservedPrimitiveConversionsStag.cpp:5-144
 * (declared compressible_functions_stag.H:69-70).  Writes vel on valid faces,
 * prim and cu components 1..3 on valid cells; ghosts are left to
 * fhd_fill_boundary, as in the reference. */
int fhd_conserved_to_primitive_stag(fhd_ctx* ctx, fhd_fab prim, const fhd_fab vel[3],
                                    fhd_fab cu, const fhd_fab mom[3]);

/* calculateTransportCoeffs (Giovangigli model): transCoeffs.cpp:7-90
 * (declared compressible_functions.H:37-39).  Fills eta, zeta, kappa, chi, D on
 * the cell box grown by the ghost width of prim. */
int fhd_transport_coeffs(fhd_ctx* ctx, fhd_fab prim, fhd_fab eta, fhd_fab zeta,
                         fhd_fab kappa, fhd_fab chi, fhd_fab D);

/* calculateFluxStag: fluxStag.cpp:5-1868 (declared
 * compressible_functions_stag.H:127-143).  edgeflux[6] = {edgeflux_x[0..1],
 * edgeflux_y[0..1], edgeflux_z[0..1]}; stochedge[3] = {xy, xz, yz} combined
 * noise; stochface[3]/stochcen[3] combined noise W (already weighted). */
int fhd_flux_stag(fhd_ctx* ctx, fhd_fab cu, const fhd_fab mom[3], fhd_fab prim,
                  const fhd_fab vel[3], fhd_fab eta, fhd_fab zeta, fhd_fab kappa,
                  fhd_fab chi, fhd_fab D, const fhd_fab faceflux[3],
                  const fhd_fab edgeflux[6], const fhd_fab cenflux[3],
                  const fhd_fab stochface[3], const fhd_fab stochedge[3],
                  const fhd_fab stochcen[3], double dt);

/* MultiFab::FillBoundary(periodicity) for a single box: ghosts <- periodic
 * images of valid points; valid points untouched.  With walls only the ghosts
 * outside the box in periodic directions alone are filled (AMReX fills no ghost
 * that is outside the domain in a non-periodic direction). */
int fhd_fill_boundary(fhd_ctx* ctx, fhd_fab f);
/* MultiFab::OverrideSync(periodicity): periodic duplicates of nodal points take
 * the value of the low-side owner (point n_cells[d] <- point 0); wall directions
 * have no duplicates. */
int fhd_override_sync(fhd_ctx* ctx, fhd_fab f);

/* setBCStag: boundaryStag.cpp:268-298 (declared compressible_functions_stag.H).
 * BCMassTempPress, BCMomNormal, BCMomTrans of every direction, then BCRhoRhoE:
 * on a box with walls, sets the wall faces' normal momentum and velocity to 0
 * and every ghost of a wall direction of prim (rho, T, p, Y, X), cu (rho, rho E,
 * rho Y), cumom and vel.  prim and cu have one ghost width, cumom and vel all
 * the same one; a fully periodic context does nothing. */
int fhd_set_bc_stag(fhd_ctx* ctx, fhd_fab prim, fhd_fab cu, const fhd_fab cumom[3], const fhd_fab vel[3]);

/* Test hook of the particle reservoir (bc_mass 4): record every random number the
 * reservoir's Poisson processes draw (ComputeFluxMomReservoir), so that a harness can
 * feed the same numbers to the reference.  buf: device memory of
 * 3 x (interface faces of the bc_mass-4 sides, x lo .. z hi) x cap doubles, entry
 * (stage, face, n) the n-th draw of that face in that stage of the next step (draws
 * beyond cap are not recorded); NULL turns recording off. */
int fhd_set_reservoir_record(fhd_ctx* ctx, void* buf, int cap);

/* MultiFabFillRandomNormal: MultiFabFillRandom.cpp:34-50 (declared
 * rng_functions.H:13-22).  Philox-4x32-10 normals; `stream_id` selects an
 * independent stream under the context's seed. */
int fhd_fill_random_normal(fhd_ctx* ctx, fhd_fab mf, int scomp, int ncomp, double mean,
                           double variance, int overridesync, int fillboundary,
                           uint64_t stream_id);

/* MultiFabFillRandomUniform: MultiFabFillRandom.cpp:53-66 (declared
 * rng_functions.H:20-22).  Uniform values in [0, 1) with 53 random bits (one
 * Philox-4x32-10 call per point), then OverrideSync / FillBoundary when asked;
 * `stream_id` selects an independent stream as for the normal fill. */
int fhd_fill_random_uniform(fhd_ctx* ctx, fhd_fab mf, int scomp, int ncomp, int overridesync,
                            int fillboundary, uint64_t stream_id);

/* compute_compressible_chemistry_source_CLE: chemistry_functions.cpp:128-193
 * (declared chemistry_functions.H:20-21).  For every valid cell of `prim`
 * (nprimvars comps, >= 0 ghosts) writes components 5 .. 5+nspecies-1 of
 * `source` (>= 5+nspecies comps, >= 0 ghosts) with the law-of-mass-action
 * rates of the context's reactions and, for reaction_type 1, their Langevin
 * terms driven by `ranchem` (cell-centred, nreaction comps; data == NULL is
 * accepted for reaction_type 0).  dV = dx*dy*dz as the reference's caller
 * passes it (timeStepStag.cpp:360).  FHD_ERR_BAD_ARG when the context has no
 * reactions. */
int fhd_chemistry_source_cle(fhd_ctx* ctx, double dt, double dV, fhd_fab prim, fhd_fab source,
                             fhd_fab ranchem);

/* Fills `noise` with exactly the A/B fields the fused step generates
 * in-kernel for (seed, step): lets a caller replay an in-kernel-noise step
 * through the injected-noise path (chem[.] too when their data is non-NULL). */
int fhd_fill_step_noise(fhd_ctx* ctx, const fhd_noise* noise, int64_t step);

/* RK3stepStag: timeStepStag.cpp:13-1245 (declared
 * compressible_functions_stag.H:113-125).  Advances cu/mom/prim/vel by one
 * SSP-RK3 step in place (ghosts refreshed, as after the reference's final
 * FillBoundary).  prim and vel are recomputed from cu and mom at the start of
 * every stage (the reference reads them as given, which in its driver are
 * always the conversion of cu and mom), so their contents on entry are not read.  source: nvars-component cell fab (the reference's
 * `source`) or data == NULL for zero.  With nreaction > 0, every stage
 * overwrites components 5 .. 5+nspecies-1 of `source` (of a zeroed scratch
 * source when data == NULL) with the chemistry source of the stage's state
 * before the update adds dt * source, as timeStepStag.cpp:354-361 does.
 * eta..D receive the stage-3 transport coefficients and faceflux/edgeflux/
 * cenflux the stage-3 fluxes when their data pointers are non-NULL (pass NULL
 * arrays to skip them; the fused path then never materialises them).
 * injected == NULL -> Philox noise generated in-kernel from (seed, step). */
int fhd_rk3_step_stag(fhd_ctx* ctx, fhd_fab cu, const fhd_fab mom[3], fhd_fab prim,
                      const fhd_fab vel[3], fhd_fab source, fhd_fab eta, fhd_fab zeta,
                      fhd_fab kappa, fhd_fab chi, fhd_fab D, const fhd_fab* faceflux,
                      const fhd_fab* edgeflux, const fhd_fab* cenflux,
                      const fhd_noise* injected, double dt, int64_t step);

/* nsteps RK3stepStag steps (no source, no by-products; in-kernel Philox noise,
 * or none when stoch_stress_form is 0) replayed from a CUDA graph: the first
 * call captures one step and the context keeps it while the fabs, dt and tile
 * stay the same.  For boxes small enough that a step's 23 launches cost more
 * than their work.  Step s of the call draws the noise of step step0 + s, so the
 * result is bitwise that of nsteps fhd_rk3_step_stag calls with steps step0,
 * step0 + 1, ...  On a stream that cannot be captured (the legacy default
 * stream) the steps are launched one by one. */
int fhd_rk3_steps_stag(fhd_ctx* ctx, fhd_fab cu, const fhd_fab mom[3], fhd_fab prim,
                       const fhd_fab vel[3], double dt, int64_t step0, int nsteps);

/* RK3stepStag on HOST fabs (same layouts as above, host pointers; pinned memory
 * gives full copy bandwidth): copies cu and mom to device buffers owned by the
 * context, advances one step there (in-kernel noise, or injected noise given as
 * host fabs), copies cu/mom/prim/vel back and waits for the stream.  prim and vel
 * are outputs only: the step derives them from cu and mom before reading them
 * (as fhd_rk3_step_stag does), so their contents on entry are not read.  For callers whose MultiFabs live in host memory (a CPU AMReX build);
 * no reference counterpart beyond RK3stepStag itself. */
int fhd_rk3_step_stag_host(fhd_ctx* ctx, fhd_fab cu, const fhd_fab mom[3], fhd_fab prim,
                           const fhd_fab vel[3], const fhd_noise* injected, double dt,
                           int64_t step, int64_t* h2d_bytes, int64_t* d2h_bytes);

/* Per-kernel timing of the step with CUDA events on the launching stream
 * (tracing aid in place of the reference's TinyProfiler regions).  Kinds:
 * 0 cellprep (conversion + transport), 1 stresses, 2 face fluxes (the three
 * per-direction launches together), 3 divergence/RK update, 4 ghost fill,
 * 5 final conversion, 6 by-product fluxes, 7 the fused stage kernel (stresses,
 * face fluxes and update in one launch, when the tile selects it).
 * fhd_profile_read synchronizes, sums the elapsed times (ms) and bracketed
 * launches per kind since the last read, and resets. */
#define FHD_PROF_KINDS 8
int fhd_profile(fhd_ctx* ctx, int enable);
int fhd_profile_read(fhd_ctx* ctx, double* ms, int64_t* launches);

/* FMA throughput of `device` in TFLOP/s (2 flops per fma), FP64 (fp64 != 0) or
 * FP32: the best of five timed launches of independent fma chains over a whole
 * number of waves (CUDA events).  The compute denominator of the step's
 * roofline beside the measured HBM bandwidth.  Changes no device setting.  No
 * reference counterpart. */
int fhd_measure_fma_peak(int device, int fp64, double* tflops);

/* ---- ensembles and served runs (no reference counterpart: the reference runs one
 * simulation per process) ------------------------------------------------------
 * A batch advances many independent runs of one species count and precision
 * together: each kernel of the step is launched once for all members, and one
 * step is replayed from a captured CUDA graph.  Members keep their own box size,
 * gas state, dt, seed (Philox key) and step counter, and get exactly the result
 * they would get alone through fhd_rk3_step_stag with in-kernel noise.  The
 * caller owns each member's cu/mom/prim/vel device fabs; the batch owns the
 * members' stage scratch (stream-ordered allocations). */
typedef struct fhd_batch fhd_batch;
int fhd_batch_create(fhd_batch** batch, int nspecies, int precision, int device);
int fhd_batch_destroy(fhd_batch* batch);
int fhd_batch_set_stream(fhd_batch* batch, void* stream);
/* init == NULL: the fabs already hold a converted, ghost-filled state; else
 * init = {rho0, T_init, rhobar[0..nspecies-1]} initialises the uniform rest state
 * (InitConsVarStag prob_type 1 + conversion + FillBoundary). */
int fhd_batch_add(fhd_batch* batch, const fhd_params* params, fhd_fab cu, const fhd_fab mom[3],
                  fhd_fab prim, const fhd_fab vel[3], double dt, int64_t first_step,
                  const double* init, int* member);
int fhd_batch_remove(fhd_batch* batch, int member);
/* Advances every member by nsteps RK3 steps (use_graph: replay a captured graph). */
int fhd_batch_step(fhd_batch* batch, int nsteps, int use_graph);
int fhd_batch_size(const fhd_batch* batch);
/* Run each step of the batch as ONE persistent launch (k_batch_persist) instead of
 * the 23 per-kind launches: blocks take chunks of every member's phases (per stage:
 * cellprep, stresses, faces x/y/z, update, ghost fill; then the conversion, its
 * ghost fill and the step counter) from one device counter in phase-major order
 * and wait, bounded in time, for the member's previous phase.  Results are bitwise
 * those of the per-kind launches.  Replayed from a graph like them.  tile: the
 * kernel's register cap as the batch face tiles (0 .. fhd_batch_num_tiles()-1:
 * 64, 80, 128 registers); -1: 64 up to two species, 128 above. */
int fhd_batch_set_persistent(fhd_batch* batch, int enable, int tile);
/* Time limit of each wait of the persistent step (default 1 s; at most 60 s).  On
 * expiry the member's status becomes FHD_ERR_TIMEOUT and every block stops taking
 * work for that step.  hold_phase >= 0 (0 .. 23) is a failure-injection hook for
 * tests: that phase's completions are never published, so the next phase's wait
 * runs out; -1 turns it off. */
int fhd_batch_set_wait_limit(fhd_batch* batch, double seconds, int hold_phase);
/* Latched device status of one member (waits for the stream). */
int fhd_batch_member_status(fhd_batch* batch, int member);
int fhd_batch_synchronize(fhd_batch* batch);
/* Launch shape of the batched face-flux kernels: tile 0 .. fhd_batch_num_tiles()-1
 * caps them at 64, 80 or 128 registers per thread (8, 6 or 4 resident blocks of
 * 128), -1 restores the default (64 up to two species, 128 above).  Takes effect
 * at the next step. */
int fhd_batch_num_tiles(void);
int fhd_batch_set_tile(fhd_batch* batch, int tile);
/* The batch's autotuner: times the face-flux launches of one RK stage over the
 * current members for every tile (one untimed round, then reps timed rounds,
 * CUDA events on the batch stream) and keeps the fastest.  Those launches write
 * only the stage's face-flux scratch, which every stage recomputes before reading
 * it, so no member's state changes; run it after at least one step so that their
 * inputs are the members' fields.  ms (optional, fhd_batch_num_tiles() entries)
 * receives the mean milliseconds of each tile, *best (optional) the choice. */
int fhd_batch_autotune(fhd_batch* batch, int reps, double* ms, int* best);

/* ---- running statistics ----------------------------------------------------------
 * The per-cell part of evaluateStatsStag3D (statsStag.cpp:10-77), which the
 * reference's time loop calls after every step (main_driver.cpp:1235-1241):
 * EvaluateStatsMeans (statsStag.cpp:200-365) and EvaluateVarsCoVarsMom3
 * (:367-691), each followed by the reference's FillBoundary of the cell-centred
 * means/variances, and with FHD_STATS_CROSS the yz-averaged spatial
 * cross-correlations of plot_cross (:46-76): sumToLine of cu, cuMeans and
 * components 1..nspecies+4 of prim and primMeans, each divided by
 * n_cells[1]*n_cells[2] (every line entry summed over its y-z plane in the order
 * k outer, j inner), and EvaluateSpatialCorrelations3D (:868-1105) at x* =
 * params.cross_cell.  `spatialCross` (device, n_cells[0] * fhd_spatial_cross_ncross
 * doubles, entry i*ncross + n, the reference's spatialCrossVec) is updated in
 * place; `dataSliceMeans_xcross` (device, fhd_spatial_cross_nstats doubles)
 * receives the line averages at x* that the reference appends to its crossMeans
 * file.  In a quasi-1-D run (params.do_1D) FHD_STATS_CROSS is evaluateStatsStag1D's
 * (statsStag.cpp:130-197): per y-z pencil the correlations with the pencil's own
 * cell at x* (GetPencilCross, EvaluateSpatialCorrelations1D :810-866, 1311-1557),
 * into `spatialCross` as the reference's spatialCrossMF: the valid cells of a
 * cell-centred MultiFab without ghosts, fhd_spatial_cross_ncross comps per x* (five
 * x* with params.all_correl), component slowest, x fastest; dataSliceMeans_xcross
 * is unused.  A quasi-2-D run ignores FHD_STATS_CROSS, as evaluateStatsStag2D does.
 * Without surface coverage (nspec_surfcov = 0).  Fabs have the
 * reference's shapes (main_driver.cpp:646-714): cuMeans/cuVars nvars comps,
 * primMeans nprimvars+3 comps, primVars nprimvars+5 comps, coVars 26 comps,
 * mom3/mom4 nvars+1 comps, all cell-centred; velMeans/velVars/cumomMeans/
 * cumomVars nodal in d.  cu and cuMeans need ghost width >= 2 (the density mean
 * is also updated on two ghost layers, as the reference does); the others may
 * have any ghost width (their ghosts are refilled periodically).  The variance
 * fabs and mom3/mom4 may be empty when their flags are off. */
typedef struct {
    fhd_fab cuMeans, cuVars, primMeans, primVars, coVars, mom3, mom4;
    fhd_fab velMeans[3], velVars[3], cumomMeans[3], cumomVars[3];
    double* spatialCross;            /* FHD_STATS_CROSS only; else may be NULL */
    double* dataSliceMeans_xcross;   /* FHD_STATS_CROSS only; else may be NULL */
} fhd_stats;
/* entries per x cell of spatialCross: 37 + nspecies + 3 (main_driver.cpp:283) */
int fhd_spatial_cross_ncross(int nspecies);
/* entries of dataSliceMeans_xcross: 2*nvars + 8 + 2*nspecies (main_driver.cpp:279) */
int fhd_spatial_cross_nstats(int nspecies);

/* ---- plotfiles --------------------------------------------------------------------
 * WritePlotFileStag (writePlotFileStag.cpp:7-527, declared
 * compressible_functions_stag.H): the cell-centred plotfile MultiFab the
 * reference assembles (instantaneous cu, face momenta shifted to cells, prim
 * components 1.., face velocities shifted to cells, eta, kappa, zeta when
 * |visc_type| == 3; then, by flag, the means, variances, covariances and third /
 * fourth moments of fhd_stats), under the reference's variable names, and its
 * single-level AMReX plotfile <plot_base_name><step, 9 digits>/ (Header,
 * Level_0/Cell_H, Level_0/Cell_D_00000).  FHD_PLOT_DELTAY_X/Y/Z (at most one)
 * append plot_deltaY_dir's components, Y_k minus its average over the planes
 * normal to that direction (writePlotFileStag.cpp:282-290; WriteHorizontalAverageToMF,
 * ComputeAverages.cpp:96-190); these take a small stream-ordered device buffer
 * for the averages.  Surface coverage is not covered.  Source fabs must be
 * device-accessible (device, managed or pinned host memory) and cover the valid
 * region. */
enum { FHD_PLOT_MEANS = 1, FHD_PLOT_VARS = 2, FHD_PLOT_COVARS = 4, FHD_PLOT_MOM3 = 8, FHD_PLOT_MOM4 = 16,
       FHD_PLOT_DELTAY_X = 32, FHD_PLOT_DELTAY_Y = 64, FHD_PLOT_DELTAY_Z = 128 };
/* number of plotfile components for `flags` (negative: -error code); no device */
int fhd_plotfile_ncomp(const fhd_params* params, int flags);
/* name of component `comp` into buf (NUL-terminated, at most buflen bytes) */
int fhd_plotfile_varname(const fhd_params* params, int flags, int comp, char* buf, int buflen);
/* writes the plotfile directory `dir` from packed host data (fhd_plotfile_ncomp
 * components of the valid box, x fastest, components slowest); no device */
int fhd_plotfile_write_host(const fhd_params* params, const char* dir, const double* data, int flags,
                            double time, int step);
/* the plotfile MultiFab into `out` (cell-centred, >= fhd_plotfile_ncomp comps) */
int fhd_plotfile_pack(fhd_ctx* ctx, int flags, fhd_fab out, fhd_fab cu, const fhd_fab cumom[3], fhd_fab prim,
                      const fhd_fab vel[3], fhd_fab eta, fhd_fab kappa, fhd_fab zeta, const fhd_stats* stats);
/* ---- checkpoints -----------------------------------------------------------------
 * WriteCheckPoint / ReadCheckPoint (Checkpoint.cpp:28-257, 259-575): the
 * directory <chk_base><step, 9 digits>/ with Header (title, step, time,
 * statsCount, the BoxArray) and Level_0/<name>_H + <name>_D_00000 for cu, prim,
 * vel, cumom and, when `stats` is given, every non-empty statistics fab, under
 * the reference's names, whole fabs with ghost cells.  Fabs may be device or
 * host memory (no device needed for host fabs; with device fabs the call
 * synchronises the device before copying, so pending work on any stream is
 * finished first).  The read fills fabs of the same
 * shapes and returns step = saved step + 1, the time and statsCount, as the
 * reference's restart does; the in-kernel noise needs no saved generator state
 * (it is a function of seed and step).  With plot_cross, stats->spatialCross
 * (host or device, n_cells[0] * fhd_spatial_cross_ncross doubles) is written into
 * the Header after the BoxArray at 16 significant digits, as the reference keeps
 * spatialCrossVec there (Checkpoint.cpp:112-118), and read back from it
 * (:343-358).  For the reference's reset_stats, read with stats = NULL and zero
 * the statistics.  A directory or file that cannot be created, opened, written,
 * read or closed gives FHD_ERR_IO; a checkpoint that holds other shapes or is not
 * a compressible-staggered checkpoint gives FHD_ERR_BAD_ARG.  The file writers
 * below (spatial cross, plotfiles) report file failures as FHD_ERR_IO as well. */
int fhd_write_checkpoint(const fhd_params* params, const char* chk_base, int step, double time, int stats_count,
                         fhd_fab cu, const fhd_fab cumom[3], fhd_fab prim, const fhd_fab vel[3],
                         const fhd_stats* stats);
int fhd_read_checkpoint(const fhd_params* params, const char* chk_base, int restart, int* step, double* time,
                        int* stats_count, fhd_fab cu, const fhd_fab cumom[3], fhd_fab prim, const fhd_fab vel[3],
                        const fhd_stats* stats);

/* WriteSpatialCross3D / WriteSpatialCross1D (writePlotFileStag.cpp:528-563) in the
 * reference's number formatting, from spatialCross in host or device memory, under
 * the reference's file names prefixed by `dir` ("" for the working directory, else
 * e.g. "out/"): 3-D runs <dir>spatialCross<step, 9 digits>, one line per x cell with
 * its centre and the ncross entries; quasi-1-D runs <dir>spatialCross1D_<step> (or,
 * with all_correl, <dir><s>_spatialCross1D_<step> for the five x*), the y-z averages
 * of every component per x cell (WriteHorizontalAverage, ComputeAverages.cpp:8-94).
 * Quasi-2-D runs write nothing (the reference's 2-D writer is not enabled). */
int fhd_write_spatial_cross(const fhd_params* params, const char* dir, int step, const double* spatial_cross);

/* pack, copy to the host and write the plotfile directory (blocks on the stream;
 * allocates and frees a temporary device buffer of the packed size) */
int fhd_write_plotfile_stag(fhd_ctx* ctx, const char* plot_base_name, int step, double time, int flags, fhd_fab cu,
                            const fhd_fab cumom[3], fhd_fab prim, const fhd_fab vel[3], fhd_fab eta, fhd_fab kappa,
                            fhd_fab zeta, const fhd_stats* stats);

/* flags of fhd_stats_stag (the reference's plot_means, plot_vars/plot_covars,
 * plot_mom3, plot_mom4 and plot_cross inputs) */
enum { FHD_STATS_MEANS = 1, FHD_STATS_VARS = 2, FHD_STATS_MOM3 = 4, FHD_STATS_MOM4 = 8, FHD_STATS_CROSS = 16 };

/* One statistics update with sample count `steps` (the reference's statsCount,
 * 1 for the first sample after a reset): stepsminusone = steps - 1 and
 * stepsinv = 1/steps weight every running average.  FHD_STATS_VARS without
 * FHD_STATS_MEANS is rejected (the reference aborts).  cu/prim/vel/mom are the
 * state after the step, with filled ghosts. */
int fhd_stats_stag(fhd_ctx* ctx, fhd_fab cu, fhd_fab prim, const fhd_fab vel[3], const fhd_fab mom[3],
                   const fhd_stats* stats, int64_t steps, int flags);

/* ---- static structure factor -------------------------------------------------------
 * StructFact (src_analysis/StructFact.H, StructFact.cpp) for one periodic box of
 * n_cells cells: covariances of the Fourier transforms of cell-centred
 * variables, accumulated over samples.  Pairs (pairA[c], pairB[c]), c < ncov,
 * index the components of the `variables` fab; pairA == NULL selects all
 * nvar (nvar + 1) / 2 pairs (A = j, B = i for i <= j) as the reference's define
 * without pairs does (StructFact.cpp:45-69).  var_scaling has one entry per pair
 * (the result is divided by it).  The accumulators live in device memory owned
 * by the object (2 x ncov doubles per cell). */
typedef struct fhd_sf fhd_sf;
int fhd_sf_create(fhd_sf** sf, const int n_cells[3], int nvar, int ncov, const int* pairA, const int* pairB,
                  const double* var_scaling, int device);
int fhd_sf_destroy(fhd_sf* sf);
int fhd_sf_set_stream(fhd_sf* sf, void* stream);
int fhd_sf_synchronize(fhd_sf* sf);
int fhd_sf_ncov(const fhd_sf* sf);
int64_t fhd_sf_nsamples(const fhd_sf* sf);
/* StructFact::FortStructure (StructFact.cpp:231-311): one sample from the
 * cell-centred `variables` fab (nvar components, any ghost width, device
 * memory); reset = 1 restarts the accumulation with this sample. */
int fhd_sf_fort_structure(fhd_sf* sf, fhd_fab variables, int reset);
/* StructFact::CallFinalize (StructFact.cpp:598-641): the averaged covariances,
 * zero_avg = 1 zeroes k = 0, shifted so that k = 0 sits at n_cells/2, scaled by
 * 1/var_scaling, into cell-centred fabs of ncov components (real, imaginary,
 * magnitude).  The accumulators are left unchanged. */
int fhd_sf_finalize(fhd_sf* sf, fhd_fab cov_real, fhd_fab cov_imag, fhd_fab cov_mag, int zero_avg);

/* Stacks of structure factors of the quasi-2-D and quasi-1-D runs
 * (main_driver.cpp:923-993, 1503-1557, 1592-1711): one StructFact per z slice
 * (FHD_SF_Z_SLICES, do_2D: members z = 0..n_cells[2]-1 of n_cells[0] x
 * n_cells[1] x 1, ExtractSlice) or per x pencil (FHD_SF_X_PENCILS, do_1D: member
 * i at y = i / n_cells[1], z = i % n_cells[1] of n_cells[0] x 1 x 1,
 * ExtractXPencil; needs n_cells[1] == n_cells[2], since for other shapes that
 * enumeration reads pencils outside the box).  All members transform in one
 * batched cuFFT per variable.  fhd_sf_fort_structure takes the whole box's
 * variables fab and samples every member; fhd_sf_stack_average is the
 * reference's output loop: zeroed mag (ncov comps) and realimag (2 ncov comps:
 * real then imaginary) fabs of the member shape, AddToExternal of every member
 * in order (its Finalize, StructFact.cpp:979-1009), then mult by 1/members.
 * fhd_sf_finalize is refused for a stack. */
enum { FHD_SF_BOX = 0, FHD_SF_Z_SLICES = 1, FHD_SF_X_PENCILS = 2 };
int fhd_sf_create_stack(fhd_sf** sf, const int n_cells[3], int kind, int nvar, int ncov, const int* pairA,
                        const int* pairB, const double* var_scaling, int device);
int fhd_sf_stack_average(fhd_sf* sf, fhd_fab mag, fhd_fab realimag, int zero_avg);

/* RK3stepStag without any device allocation, for callers that cannot allocate:
 * code whose device memory is owned by an arena that a stray cudaMalloc would
 * fail or fragment, framework callbacks that forbid allocation on their hot
 * path, and latency-critical loops that cannot pay the device-wide
 * synchronisation of cudaMalloc/cudaFree.  No reference counterpart (the
 * reference allocates its stage temporaries inside RK3stepStag,
 * timeStepStag.cpp:30-153); this entry point has no context either.
 *
 * Same step as fhd_rk3_step_stag with FP64 precision, in-kernel Philox noise
 * (or none when stoch_stress_form == 0) and no by-product outputs, on the
 * caller's stream (NULL = legacy default stream).  cu, mom, prim and vel must
 * be device memory of the CURRENT device (checked: FHD_ERR_BAD_ARG otherwise),
 * with one ghost width >= 2 per fab, as fhd_rk3_step_stag accepts.  Its stage scratch is a
 * file-scope 16 MiB device array held by every GPU that loads the library until
 * the process exits; boxes whose scratch does not fit (the largest cubes that fit: 29^3
 * cells with 2 species, 26^3 with 4) return FHD_ERR_TOO_LARGE before any GPU work.  The first
 * call on a device looks up the array's device address (cudaGetSymbolAddress,
 * that device current): make it before any stream capture.  Calls share the
 * array and it keeps the last call's contents, so calls whose GPU work overlaps
 * race; serialise them.  status (optional): when non-NULL the call waits for
 * the stream and stores the device status word (0 or FHD_ERR_MASSFRAC /
 * FHD_ERR_NONFINITE). */
int fhd_rk3_step_stag_noalloc(const fhd_params* params, fhd_fab cu, const fhd_fab mom[3],
                              fhd_fab prim, const fhd_fab vel[3], double dt, int64_t step,
                              void* stream, int* status);

#ifdef __cplusplus
}
#endif

#endif /* FHD_CAPI_H */
