/*
 * raven_b200.h -- C ABI of the B200 (sm_100a) DGSEM tendency + LSRK(5,4) library.
 *
 * The library replaces, for one GPU and one rank, the device work behind Raven.jl's
 *   (dg::DGSEM)(dq, q, time; increment)       src/balancelaws/dgsem.jl:84-126
 *   dostep!(q, ::LSRK, after_stage)           src/balancelaws/odesolvers.jl:51-61
 *   weightednorm(dg, q)                       src/balancelaws/measures.jl:6-21
 * The grid data it consumes are exactly the arrays a Raven `Grid` holds
 * (`volumemetrics`, `surfacemetrics`, `facemaps`, `boundarycodes`,
 * `derivatives_1d`, `weights_1d`), in the GridArray parent layouts of
 * src/gridarrays.jl:50-108.  State arrays are Raven's GridArray parent layout
 * (Nq^dim, Ns, E), column-major, FP64, on the device.
 *
 * All functions return an rb200_status and never abort.  Device-pointer arguments
 * are borrowed for the duration of the call; work is enqueued on the caller's stream
 * (a cudaStream_t passed as void*; NULL = legacy default stream).  A handle is not
 * thread-safe.
 */
#ifndef RAVEN_B200_H
#define RAVEN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RB200_ABI_VERSION 1

typedef enum rb200_status {
    RB200_OK = 0,
    RB200_ERR_BAD_ARG = 1,     /* null pointer, out-of-range enum or size */
    RB200_ERR_SHAPE = 2,       /* array sizes inconsistent (DimensionMismatch in Raven) */
    RB200_ERR_OOM = 3,         /* device allocation failed */
    RB200_ERR_CUDA = 4,        /* a CUDA runtime call failed */
    RB200_ERR_TIMEOUT = 5,     /* a bounded wait expired */
    RB200_ERR_UNSUPPORTED = 6  /* valid input this build does not implement */
} rb200_status;

/* Balance laws: AdvectionLaw{FT,D}(u) (balancelaws/advection.jl:8-16),
 * EulerLaw{FT,D}(; gamma) (balancelaws/euler.jl:9-19). */
enum { RB200_LAW_ADVECTION = 0, RB200_LAW_EULER = 1 };
/* Volume forms: WeakForm(), FluxDifferencingForm(flux) (dgsem.jl:5-17). */
enum { RB200_FORM_WEAK = 0, RB200_FORM_FLUXDIFF = 1 };
/* Numerical fluxes (numericalfluxes.jl:39-55, euler.jl:93-300).  Surface fluxes:
 * Rusanov and Central for every law and precision; Kennedy-Gruber, entropy conservative
 * (their two-point flux contracted with the normal), Roe and matrix dissipation for the
 * Euler law in FP64. */
enum {
    RB200_FLUX_CENTRAL = 0,
    RB200_FLUX_KENNEDY_GRUBER = 1,
    RB200_FLUX_ENTROPY_CONSERVATIVE = 2,
    RB200_FLUX_RUSANOV = 3,
    RB200_FLUX_ROE = 4,
    RB200_FLUX_MATRIX = 5
};
/* Arithmetic of the volume/surface bulk.  FP32_BULK keeps the state q, the
 * geometry and all reductions in FP64 and the LSRK register dq in FP32. */
enum { RB200_PRECISION_FP64 = 0, RB200_PRECISION_FP32_BULK = 1 };

typedef struct rb200_desc {
    int32_t abi_version;      /* RB200_ABI_VERSION */
    int32_t dim;              /* 1, 2 or 3 */
    int32_t nq;               /* nodes per direction, 2..8 (N = nq-1) */
    int32_t law;              /* RB200_LAW_* */
    int64_t num_elements;     /* E (local elements; no ghosts on one rank) */
    int32_t volume_form;      /* RB200_FORM_* */
    int32_t volume_flux;      /* two-point flux of FluxDifferencingForm */
    int32_t surface_flux;     /* RB200_FLUX_*; see the flux enum for what each law takes */
    int32_t precision;        /* RB200_PRECISION_* */
    double gamma;             /* Euler ratio of specific heats (Raven default 7//5) */
    double advection_velocity[3];
    /* Host arrays, read during rb200_create only: */
    const double* D;               /* (nq, nq) col-major, derivatives_1d(cell)[1] (lobattocells.jl:263) */
    const double* w;               /* (nq), weights_1d */
    const double* volume_metrics;  /* (nq^dim, dim*dim+2, E): dRdX (col-major), J, wJ
                                      = parent(first(volumemetrics(grid))) */
    const double* surface_metrics; /* (dim+2, 2*dim*nq^(dim-1), E): n, sJ, wsJ
                                      = parent(first(surfacemetrics(grid))) */
    const int64_t* vmapM;          /* (2*dim*nq^(dim-1), E), 1-based (facemaps(grid).vmapM) */
    const int64_t* vmapP;          /* same shape (facemaps(grid).vmapP) */
    const int64_t* boundary_codes; /* (2*dim, E) boundarycodes(grid); NULL = all 0 */
    int32_t device;                /* CUDA device ordinal */
} rb200_desc;

typedef struct rb200_handle rb200_handle;

/* DGSEM(; law, grid, surface_numericalflux, volume_form)  (dgsem.jl:46-81).
 * Uploads the grid once; compresses vmapM/vmapP into a per-face neighbour table
 * after checking, node by node, that it reproduces them.  A grid of an unstructured
 * coarse grid, whose faces may meet rotated or on another face of the neighbour
 * (lobattocells.jl:2177-2206), keeps vmapP as a table read by the kernels; its faces
 * must each map onto one face of one element (RB200_ERR_SHAPE otherwise). */
rb200_status rb200_create(const rb200_desc* desc, rb200_handle** out);
rb200_status rb200_destroy(rb200_handle* h);

/* (dg::DGSEM)(dq, q, time; increment)  (dgsem.jl:84-126).
 * dq = (increment ? dq : 0) + RHS(q).  dq, q: device, (nq^dim, Ns, E) FP64. */
rb200_status rb200_tendency(rb200_handle* h, double* dq, const double* q, double time, int32_t increment,
                            void* stream);

/* nsteps of dostep!(q, LSRK54(dg, q, dt))  (odesolvers.jl:51-66): for each of the 5
 * stages  dq = rka*dq + RHS(q);  q = q + rkb*dt*dq,  fused into one kernel per stage.
 * q, dq: device FP64 (dq is the LSRK register, ignored in FP32_BULK mode where the
 * handle keeps an FP32 register).  `time` is the time at the start of the first step. */
rb200_status rb200_lsrk54_step(rb200_handle* h, double* q, double* dq, double time, double dt, int32_t nsteps,
                               void* stream);

/* nsteps of dostep!(q, LSRK144(dg, q, dt))  (odesolvers.jl:51-61, 68-71, 191-239): the
 * same fused stages with the 14-stage, fourth-order low-storage coefficients of
 * coefficients_lsrk144.  Arguments as for rb200_lsrk54_step. */
rb200_status rb200_lsrk144_step(rb200_handle* h, double* q, double* dq, double time, double dt, int32_t nsteps,
                                void* stream);

/* nsteps of dostep!(q, LSRK(rhs!, rka, rkb, rkc, q, dt, t0))  (odesolvers.jl:32-61): any
 * low-storage table of 1..32 stages (host arrays rka[nstages], rkb[nstages], copied;
 * rka[i] == 0 skips reading the register in stage i).  The fused steps of
 * rb200_lsrk54_step with the caller's coefficients; the captured step graph is reused
 * while the table's values stay the same.  Arguments otherwise as for rb200_lsrk54_step. */
rb200_status rb200_lsrk_step(rb200_handle* h, double* q, double* dq, const double* rka, const double* rkb,
                             int32_t nstages, double time, double dt, int32_t nsteps, void* stream);

/* Same as rb200_lsrk54_step for a state held in HOST memory: copies q in, runs the
 * steps, copies q back, synchronously.  The LSRK register lives on the device. */
rb200_status rb200_lsrk54_step_host(rb200_handle* h, double* q_host, double time, double dt, int32_t nsteps,
                                    void* stream);

/* One stage (0..4) of LSRK(5,4) (odesolvers.jl:163-189) from q_in to q_out:
 * dq = rka[stage]*dq + RHS(q_in);  q_out = q_in + rkb[stage]*dt*dq, for the active
 * elements.  q_in and q_out must be different device buffers.  A distributed step calls
 * it five times, refreshing the ghost elements of q_in (start!/finish! around the
 * right-hand side, dgsem.jl:95-100) before each; see rb200_set_active_elements. */
rb200_status rb200_lsrk54_stage(rb200_handle* h, const double* q_in, double* q_out, double* dq, int32_t stage,
                                double time, double dt, void* stream);

/* The same stage on the active elements e_begin..e_end-1 only (0 <= e_begin <= e_end <=
 * the active count).  A rank numbers its interior elements (no ghost neighbour) first:
 * it runs them while its ghost exchange is in flight, then the rest once the ghosts
 * have arrived (Raven's start!, volume term, finish!, dgsem.jl:95-100). */
rb200_status rb200_lsrk54_stage_range(rb200_handle* h, const double* q_in, double* q_out, double* dq,
                                      int32_t stage, int64_t e_begin, int64_t e_end, double time, double dt,
                                      void* stream);

/* One stage of any low-storage scheme (odesolvers.jl:51-60): dq = rka*dq + RHS(q_in);
 * q_out = q_in + rkb*dt*dq on the active elements (rka == 0: the register is not read).
 * The stage-by-stage form of rb200_lsrk_step, for stage callbacks. */
rb200_status rb200_lsrk_stage(rb200_handle* h, const double* q_in, double* q_out, double* dq, double rka,
                              double rkb, double time, double dt, void* stream);

/* rb200_lsrk_stage on the active elements e_begin..e_end-1 only (the partitioned path's
 * interior / partition-boundary split, as rb200_lsrk54_stage_range). */
rb200_status rb200_lsrk_stage_range(rb200_handle* h, const double* q_in, double* q_out, double* dq, double rka,
                                    double rkb, int64_t e_begin, int64_t e_end, double time, double dt,
                                    void* stream);

/* Ghost elements: only elements 0..num_active-1 are computed and summed by the
 * reductions; elements num_active..E-1 hold other ranks' data (Raven's GridArray ghost
 * cells, gridarrays.jl:26-40).  Their face maps point to themselves; the faces of active
 * elements may point into them.  Default: all E elements.  Not available with mortars. */
rb200_status rb200_set_active_elements(rb200_handle* h, int64_t num_active);

/* Buffer fills of the ghost exchange (setbuffer!/getbuffer!, communication.jl:267-293),
 * 0-based indices, device arrays, asynchronous on `stream`:
 *   pack:    buffer[i] = src[indices[i]],   i < n;
 *   unpack:  dest[indices[i]] = buffer[i],  i < n.
 * An index outside [0, src_len) or [0, dest_len) is skipped. */
rb200_status rb200_pack_values(const double* src, int64_t src_len, const int64_t* indices, int64_t n,
                               double* buffer, void* stream);
rb200_status rb200_unpack_values(const double* buffer, const int64_t* indices, int64_t n, double* dest,
                                 int64_t dest_len, void* stream);

/* weightednorm(dg, q, 2; componentwise=true)  (measures.jl:6-21): out[s] =
 * sqrt(sum(MJ .* q_s.^2)) for s < Ns, out[Ns] = 2-norm of those.  FP64, synchronous,
 * deterministic (fixed reduction order).  out: host, Ns+1 doubles. */
rb200_status rb200_weightednorm(rb200_handle* h, const double* q, double* out, void* stream);

/* weightednorm(dg, q, p; componentwise=true) for any p > 0 (measures.jl:6-14) and for
 * p = Inf (measures.jl:16-21; pass INFINITY): out[s] = (sum(MJ .* abs.(q_s).^p))^(1/p),
 * or maximum(abs.(q_s)) for p = Inf (unweighted, as in the reference); out[Ns] =
 * norm(out[0..Ns-1], p).  p = 2 gives rb200_weightednorm's result.  FP64, synchronous,
 * deterministic (fixed reduction order; NaN propagates through the maximum).  p <= 0 or
 * NaN: BAD_ARG.  out: host, Ns+1 doubles. */
rb200_status rb200_weightednorm_p(rb200_handle* h, const double* q, double p, double* out, void* stream);

/* Conservation integrals out[s] = sum(MJ .* q_s)  (FP64, synchronous).  out: host, Ns. */
rb200_status rb200_integrals(rb200_handle* h, const double* q, double* out, void* stream);

/* entropyintegral(dg, q) = sum(MJ .* entropy.(q)) (measures.jl:23-27) into *out (host;
 * FP64, deterministic, synchronous).  Replaces Raven.BalanceLaws.entropyintegral. */
rb200_status rb200_entropy_integral(rb200_handle* h, const double* q, double* out, void* stream);

/* entropyproduct(dg, p, q) = sum(MJ .* dot.(entropyvariables.(p), q)) (measures.jl:28-33)
 * into *out (host; synchronous). */
rb200_status rb200_entropy_product(rb200_handle* h, const double* p, const double* q, double* out, void* stream);

/* `nsteps` steps of RLSRK54(dg, q, dt) (odesolvers.jl:73-161, 153-156): LSRK(5,4) stages
 * with the entropy production of each stage, then the relaxation q = q0 + gamma (q - q0)
 * with gamma solving eta(q) = eta0 + gamma deta.  dq: FP64 LSRK register (zero before the
 * first step); *gamma: the relaxation parameter carried between steps (1 at the start),
 * updated in place.  FP64 handles only.  Synchronous: the scalar solve reads two device
 * sums per iterate on the host. */
rb200_status rb200_rlsrk54_step(rb200_handle* h, double* q, double* dq, double* gamma, double time, double dt,
                                int32_t nsteps, void* stream);

/* `nsteps` steps of RLSRK144(dg, q, dt) (odesolvers.jl:158-161): the relaxation step of
 * rb200_rlsrk54_step over the 14 LSRK(14,4) stages.  Arguments as for rb200_rlsrk54_step. */
rb200_status rb200_rlsrk144_step(rb200_handle* h, double* q, double* dq, double* gamma, double time, double dt,
                                 int32_t nsteps, void* stream);

/* `nsteps` steps of RLSRK(rhs!, rka, rkb, rkc, q, dt, t0)  (odesolvers.jl:73-151) with
 * any low-storage table of 1..32 stages (host arrays, copied).  Arguments otherwise as
 * for rb200_rlsrk54_step. */
rb200_status rb200_rlsrk_step(rb200_handle* h, double* q, double* dq, double* gamma, const double* rka,
                              const double* rkb, int32_t nstages, double time, double dt, int32_t nsteps,
                              void* stream);

/* Snapshot / resume of the time-stepper state.  The reference keeps (q, dq, time, dt)
 * in its LSRK struct (odesolvers.jl:32-49; RLSRK adds gamma, :73-84) and has no
 * checkpoint; these copy that state to a host buffer and back.  The buffer holds a
 * 128-byte header (magic "RB200SNP", version, sizes, time, dt, gamma, a fingerprint of the
 * discretization, checksums of the header and of the payload), then q (FP64) and dq (FP64,
 * or FP32 for FP32_BULK handles, whose LSRK register is the handle's own and the dq
 * argument is ignored).  rb200_restore checks the header, the fingerprint
 * (RB200_ERR_SHAPE: another discretization) and the checksums (RB200_ERR_BAD_ARG:
 * corrupted) before it copies anything.  Both are synchronous on `stream`. */
rb200_status rb200_snapshot_bytes(const rb200_handle* h, size_t* bytes);
rb200_status rb200_snapshot(rb200_handle* h, const double* q, const void* dq, double time, double dt, double gamma,
                            void* host, size_t bytes, void* stream);
rb200_status rb200_restore(rb200_handle* h, const void* host, size_t bytes, double* q, void* dq, double* time,
                           double* dt, double* gamma, void* stream);

/* Rebuilds vmapP (1-based, (2*dim*nq^(dim-1), E) int64) on the device from the
 * neighbour table the kernels use (or from the vmapP table they read, on a grid with
 * rotated faces), for bit-exact comparison with facemaps(grid).vmapP. */
rb200_status rb200_face_vmapP(rb200_handle* h, int64_t* vmapP_out, void* stream);

/* Mortars of an adapted (non-conforming) grid, after rb200_create.  The reference's
 * surfaceterm! leaves hanging faces uncoupled (vmapP = vmapM there,
 * lobattocells.jl:2073-2074); with mortars each hanging face is coupled to its small
 * neighbours instead, conservatively:
 *   - the large face's trace is interpolated to each small face (tohalves operators,
 *     lobattocells.jl:16-17);
 *   - the surface flux is taken there;
 *   - the large face gets the lumped L2 projection of the small faces' fluxes.
 * mortars: host (2 + 2^(dim-1), M) int64 0-based columns: large element, its face
 * (0..2*dim-1: x-, x+, y-, y+, z-, z+), the small elements by position on the face (first
 * in-face direction fastest).  The large face and the small elements' opposite faces must
 * be unconnected in the face maps.  IL, IU: (nq, nq) row-major interpolation from the
 * LGL nodes to those of the lower / upper half, I[i*nq + j] = l_j((r_i -+ 1)/2).  PL, PU:
 * the projections back, P[j*nq + i] = I[i*nq + j] w_i / (2 w_j).  Unwarped elements
 * only; the generic stage kernel runs with one mortar launch before each stage. */
rb200_status rb200_set_mortars(rb200_handle* h, const int64_t* mortars, int64_t num_mortars, const double* IL,
                               const double* IU, const double* PL, const double* PU);

/* Kernel selection: 0 = automatic, 1 = generic stage kernel only.  Automatic runs a
 * persistent bulk-copy-pipelined kernel where one exists and the state pointers are
 * 16-byte aligned: 3-D unwarped bricks with nq = 4, 6, 8 (Euler Kennedy-Gruber or
 * entropy-conservative flux differencing with Rusanov or central surface flux; weak-form
 * advection), and 3-D nq = 8 curved grids in FP32_BULK (Euler Kennedy-Gruber).  Every
 * other configuration runs the generic stage kernel. */
rb200_status rb200_set_kernel_path(rb200_handle* h, int32_t path);

/* DGSEM(; directions)  (dgsem.jl:46-81): the volume term (dgsem.jl:257-348, 514-608) and
 * the surface term (dgsem.jl:756-782) are computed for the directions in `mask` only (bit
 * d = direction d + 1, e.g. 3 = directions (1, 2) of a 3-D grid, 4 = direction 3).  The
 * default is every direction; a proper subset runs the generic stage kernel.  mask must
 * be a non-empty subset of 1:dim (BAD_ARG otherwise).  Applies to every later tendency
 * and step of the handle. */
rb200_status rb200_set_directions(rb200_handle* h, int32_t mask);

/* boundarystate(law, problem, n, q-, aux-, tag)  (balancelaw.jl:22; the reference's
 * examples overload it per problem, e.g. examples/balancelaws/euler/sod.jl:15-21 and
 * euler_gravity/gravitywave.jl:16-21).  Sets the exterior state of the boundary faces
 * whose code (boundarycodes(grid)) is `tag` (1..8):
 *   kind 0: q+ = q- (the reference's default);
 *   kind 1: q+ = state (Ns host doubles, copied), a prescribed exterior state;
 *   kind 2: a reflecting wall, q+ = q- with rho u+ = rho u- - 2 (n . rho u-) n (Euler only).
 * Faces of other tags keep their condition.  A handle with a non-default condition runs
 * the generic stage kernel. */
#define RB200_BC_DEFAULT 0
#define RB200_BC_PRESCRIBED 1
#define RB200_BC_WALL 2
rb200_status rb200_set_boundary_condition(rb200_handle* h, int32_t tag, int32_t kind, const double* state);

/* Synchronizes `stream` and returns RB200_ERR_TIMEOUT if a kernel of this handle gave
 * up a bounded wait since the handle was created, RB200_OK otherwise. */
rb200_status rb200_sync_status(rb200_handle* h, void* stream);

/* Diagnostics of the bounded waits: launches one CTA that polls an mbarrier nothing
 * completes, with the stage kernels' try_wait loop limited to `polls` polls
 * (1..2^30).  Returns RB200_ERR_TIMEOUT when the kernel gave up and recorded it (the
 * expected outcome; the context stays usable), RB200_OK if the wait ended otherwise.
 * Synchronous on `stream`; allocates and frees 4 bytes of device memory. */
rb200_status rb200_probe_bounded_wait(int64_t polls, void* stream);

/* Measures the device's FP64 fma throughput: a grid of 8 CTAs per SM x 256 threads,
 * each thread running 8 independent chains of `iters` fmas (4..2^26, a multiple of 4),
 * timed with CUDA events on `stream` (best of 3 after a warm-up launch).  Writes
 * TFLOP/s (2 flops per fma) to *tflops_out.  Synchronous. */
rb200_status rb200_probe_fp64_rate(int64_t iters, double* tflops_out, void* stream);

/* Handle properties: info[0]=dim, [1]=nq, [2]=Ns, [3]=E, [4]=geometry kind
 * (0 affine brick, 1 curved), [5]=precision, [6]=kernel launches per LSRK step,
 * [7]=algorithmic HBM bytes per node per stage, [8]=CTAs of the pipelined kernel of the
 * handle's geometry (brick, or the FP32-bulk curved one; 0 when the configuration does
 * not use one), [9]=CTAs of the cluster step kernel (small weak-form advection grids on
 * unwarped bricks: one launch of one thread-block cluster runs all stages of all steps
 * of an rb200_lsrk54_step / rb200_lsrk144_step / rb200_lsrk_step call, and [6] does not
 * apply to those calls; 0 when the steps run as stage launches).  n <= 10 values are
 * written. */
rb200_status rb200_get_info(const rb200_handle* h, int64_t* info, int32_t n);

/* Weighted sums without any device allocation (no counterpart in the reference).
 *
 * For callers that cannot call cudaMalloc: code whose device memory is owned by a
 * pooling allocator (CUDA.jl and PyTorch keep most of the device reserved in their
 * caching pools, so a raw cudaMalloc from inside a library can fail or fragment the
 * pool), and code that runs where allocating is not allowed, such as a monitoring hook
 * called between the steps of a solve.  The handle API allocates in rb200_create;
 * this entry point needs no handle and allocates nothing.
 *
 * sums_out[s] = sum(MJ .* q_s.^2) and sums_out[ns + s] = sum(MJ .* q_s), s < ns, in
 * FP64 with a fixed reduction order: the squares give weightednorm (take square
 * roots), the plain sums the conservation integrals.  q: device (np, ns, E) FP64, MJ:
 * device (np, E) FP64 nodal weights (DGSEM's MJ), sums_out: device, 2*ns doubles.
 *
 * Scratch: a file-scope device array of 256 * 2 * 5 doubles (20 KB) that every device
 * loading the library holds until exit; hence ns <= 5 (larger ns returns
 * RB200_ERR_UNSUPPORTED), np <= 512.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress, with that device current); make that first call
 * before any stream capture.  The address is kept per device and CUDA context: after a
 * device reset (or any new context on the device) the next call looks it up again, so
 * that call too should come before any stream capture.  q, MJ and sums_out must be device
 * (or managed) memory usable on the current device; otherwise RB200_ERR_BAD_ARG.  All
 * calls share the array: calls that overlap on the GPU (for instance on two streams)
 * race and must be ordered by the caller. */
rb200_status rb200_weighted_sums_noalloc(const double* q, const double* MJ, int32_t np, int32_t ns,
                                         int64_t num_elements, double* sums_out, void* stream);

/* ------------------------------------------------------------------------------------
 * Serving loop: many independent brick solves on one GPU (no counterpart in the
 * reference, whose drivers run one solve!(q, timeend, LSRK54(dg, q, dt)) per process,
 * odesolvers.jl:9-30).
 *
 * A server owns one device arena, allocated in rb200_server_create.  It admits submitted
 * solves in FIFO order as their footprint fits, and a request that does not fit yet lets
 * later ones pass.  A solve's footprint is 2 state buffers + the LSRK register + 32 B of
 * geometry and 8*dim B of connectivity per element.  Admitted solves advance one
 * LSRK(5,4) step per tick, batched with every running solve of the same class:
 *   class = (dim, nq, law, volume form and flux, surface flux, precision, gamma,
 *            advection velocity, D, w).
 * A finished solve's state is copied to q_out.  A solve's result does not depend on the
 * solves it shares launches with: it equals the same solve run alone, bit for bit.
 *
 * Served configurations are unwarped bricks (affine elements): dim 2 or 3, nq 4, 6 or 8.
 *   - Advection: weak form.
 *   - Euler: flux differencing with Kennedy-Gruber.  3-D nq = 8 Euler classes run the
 *     persistent TMA-pipelined kernel of the DGSEM handle over their chunks.
 * The surface flux is Rusanov or central, and the precision is FP64 or FP32_BULK.
 * ------------------------------------------------------------------------------------ */
typedef struct rb200_request {
    int32_t abi_version;       /* RB200_ABI_VERSION */
    int32_t dim;               /* 2 or 3 */
    int32_t nq;                /* 4, 6 or 8 */
    int32_t law;               /* RB200_LAW_* */
    int64_t num_elements;      /* E */
    int32_t volume_form;       /* RB200_FORM_* */
    int32_t volume_flux;       /* RB200_FLUX_KENNEDY_GRUBER for Euler */
    int32_t surface_flux;      /* RB200_FLUX_RUSANOV or RB200_FLUX_CENTRAL */
    int32_t precision;         /* RB200_PRECISION_* */
    double gamma;
    double advection_velocity[3];
    const double* D;           /* (nq, nq) col-major derivative matrix */
    const double* w;           /* (nq) LGL weights */
    const double* r;           /* (nq) LGL points; needed when q0 is NULL */
    const double* elem_geo;    /* (4, E): dr/dx, ds/dy, dt/dz (0 in 2-D), J of each element */
    const int32_t* neighbors;  /* (2*dim, E): element across faces -x,+x,-y,+y(,-z,+z),
                                  0-based; -1 = boundary face (exterior state = interior) */
    const double* q0;          /* host (nq^dim, Ns, E) initial state, copied during submit;
                                  NULL = initial data evaluated on the device (init_kind) */
    int32_t init_kind;         /* with q0 NULL: 1 = Euler isentropic vortex (init_params:
                                  strength, u0, centre x, centre y); 2 = advection
                                  sin(2 pi x)sin(2 pi y)[sin(2 pi z)] + Gaussian (width,
                                  centre xyz) */
    double init_params[8];
    const double* corners;     /* (2, dim, E): lower corner and width of each element along
                                  each direction (node x = fma(width, (r+1)/2, corner)) */
    double dt;
    int32_t nsteps;            /* LSRK54 steps */
    double* q_out;             /* host (nq^dim, Ns, E) final state; NULL = discard.  Must
                                  stay valid until rb200_server_wait returns */
} rb200_request;

typedef struct rb200_server rb200_server;

/* Allocates the arena (arena_bytes of device memory on `device`) and starts the loop. */
rb200_status rb200_server_create(int32_t device, uint64_t arena_bytes, rb200_server** out);

/* Queues one solve; the request's host arrays are copied before return.  ticket: id for
 * rb200_server_wait.  RB200_ERR_OOM: the footprint exceeds the whole arena.  Thread-safe. */
rb200_status rb200_server_submit(rb200_server* s, const rb200_request* req, uint64_t* ticket);

/* Blocks until the solve finishes (q_out written) or timeout_s passes (RB200_ERR_TIMEOUT;
 * the ticket stays valid).  latency_s: submit-to-finish wall time.  Thread-safe. */
rb200_status rb200_server_wait(rb200_server* s, uint64_t ticket, double timeout_s, double* latency_s);

/* out[0..8]: completed, submitted, running, queued, DOF updates (nodes * Ns * 5 stages *
 * steps of completed solves), arena bytes in use, peak arena bytes, class ticks, seconds
 * from the first submit to the last completion.  Returns the server's error status. */
rb200_status rb200_server_stats(rb200_server* s, double* out, int32_t n);

/* Per class, 4 values: dim, nq, internal kernel combination, elements per CTA that the
 * autotuner chose (0 while it is still timing).  Unused entries are 0. */
rb200_status rb200_server_class_tiles(rb200_server* s, int32_t* out, int32_t n);

/* Per class, 6 values: dim, nq, internal kernel combination, completed ticks, device
 * milliseconds of those ticks (from events around each tick on the class's stream;
 * classes run concurrently, so the times of different classes overlap), DOF updates of
 * those ticks (elements x Np x Ns x 5 stages).  Unused entries are 0. */
rb200_status rb200_server_class_stats(rb200_server* s, double* out, int32_t n);

/* Message of the error that stopped the server (empty if none).  Valid until destroy. */
const char* rb200_server_last_error(rb200_server* s);

/* Stops the loop (unfinished solves are abandoned) and frees everything.  No call on
 * the server may run concurrently with or after this one. */
rb200_status rb200_server_destroy(rb200_server* s);

/* ------------------------------------------------------------------------------------
 * Utilities Raven exports beside the DGSEM path: Kron (kron.jl), gather!/scatter!
 * (gatherscatter.jl) and decode (facecode.jl).  Device arrays, asynchronous on
 * `stream`.  Results are bit-identical to the reference's arithmetic.
 * ------------------------------------------------------------------------------------ */

/* Kron(args) * f  (kron.jl:15-387).  args = (X_n, ..., X_1) as in Julia, X_1 acting on
 * the fastest index.  mats[d] = X_{d+1}: a HOST column-major rows[d] x cols[d] matrix
 * of `dtype` (0 = double, 1 = float), or NULL for Eye(rows[d]) (cols[d] = rows[d]);
 * rows, cols <= 16.  The node index of f runs over prod(cols) entries, that of the
 * result over prod(rows); element (node, comp, col) of f is at
 * in[node*in_strides[0] + comp*in_strides[1] + col*in_strides[2]], likewise for out.
 * A GridArray parent (Np, Ns, E) has strides (1, Np, Np*Ns) and ncomp = Ns; an array of
 * SVector{C} columns has strides (C, 1, C*Np) and ncomp = C.  The arithmetic is that
 * of the method Julia dispatches to:
 *   - all factors Eye: a copy;
 *   - one dense factor: one fma chain;
 *   - otherwise: the generic nested sum, with Eye entries used as 0/1 values. */
rb200_status rb200_kron_apply(int32_t nfactors, const void* const* mats, const int32_t* rows, const int32_t* cols,
                              int32_t dtype, const void* in, const int64_t* in_strides, void* out,
                              const int64_t* out_strides, int64_t ncols, int32_t ncomp, void* stream);

/* Where element i, component c of an array lives:
 *   (i % block) * node_stride + (i / block) * block_stride + c * comp_stride.
 * A discontinuous GridArray (Np, Ns, E) is {Np, 1, Np*Ns, Np}.  A continuous one
 * (Ns, Nc) is {Nc, Ns, 0, 1}. */
typedef struct rb200_layout {
    int64_t block, node_stride, block_stride, comp_stride;
} rb200_layout;

/* scatter!(dest, src, dtoc)  (gatherscatter.jl:17-34): dest[i] = src[dtoc[i]] for
 * i < n, for every component.  dtoc: device int64, 1-based (discontinuoustocontinuous).
 * dtype: 0 double, 1 float, 2 int64, 3 int32. */
rb200_status rb200_scatter(void* dest, const rb200_layout* dest_layout, const void* src,
                           const rb200_layout* src_layout, const int64_t* dtoc, int64_t n, int32_t ncomp,
                           int32_t dtype, void* stream);

/* gather!(dest, src, ctod; op, init)  (gatherscatter.jl:36-103): for each column j of
 * the CSC matrix ctod (continuoustodiscontinuous; colptr: ncols+1, rowval: nnz, device
 * int64, 1-based), dest[j] = op(...op(init, src[r_1])..., src[r_k]) over the column's
 * rows in stored order.  op: 0 = +, 1 = min, 2 = max (Julia semantics: NaN propagates,
 * -0.0 < 0.0).  init is converted to dtype. */
rb200_status rb200_gather(void* dest, const rb200_layout* dest_layout, const void* src,
                          const rb200_layout* src_layout, const int64_t* colptr, const int64_t* rowval, int64_t ncols,
                          int32_t ncomp, int32_t dtype, int32_t op, double init, void* stream);

/* decode(facecode)  (facecode.jl:1-140) for n device codes.  bits = 8 (2-D quadrant
 * codes, uint8): out (4, n) hanging-face values.  bits = 16 (3-D octant codes,
 * uint16): out (18, n) = 6 hanging-face then 12 hanging-edge values. */
rb200_status rb200_decode_facecodes(const void* codes, int32_t bits, int64_t n, uint8_t* out, void* stream);

/* Last error message of a handle (empty if none); static text for NULL. */
const char* rb200_last_error(const rb200_handle* h);
const char* rb200_status_string(rb200_status s);

#ifdef __cplusplus
}
#endif

#endif /* RAVEN_B200_H */
