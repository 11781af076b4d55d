// Internal declarations shared by the host runtime (api.cu) and the kernel
// instantiation units (stage_*.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>

namespace rb200 {

// Raises a kernel's dynamic shared-memory limit once per device: the attribute belongs
// to the kernel's instance in the current device's context.  `done` holds one bit per
// device ordinal (devices beyond 63 set the attribute on every call).
template <typename Kernel>
cudaError_t ensure_smem_limit(Kernel kern, int bytes, std::atomic<uint64_t>& done) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = (dev >= 0 && dev < 64) ? (uint64_t{1} << dev) : 0;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// Physics + volume-form combination (template parameter of the stage kernel).
enum Combo : int {
    ADV_WEAK = 0,  // AdvectionLaw, WeakForm
    ADV_FDC = 1,   // AdvectionLaw, FluxDifferencingForm(CentralFlux())
    EUL_WEAK = 2,  // EulerLaw, WeakForm
    EUL_FDC = 3,   // EulerLaw, FluxDifferencingForm(CentralFlux())
    EUL_KG = 4,    // EulerLaw, FluxDifferencingForm(KennedyGruberFlux())
    EUL_EC = 5,    // EulerLaw, FluxDifferencingForm(EntropyConservativeFlux())
    NUM_COMBOS = 6
};

enum Geom : int { GEOM_AFFINE = 0, GEOM_CURVED = 1 };

// What a launch of the stage kernel does with dq and q.
enum Mode : int {
    MODE_TENDENCY_SET = 0,  // dq = RHS(q)
    MODE_TENDENCY_INC = 1,  // dq = dq + RHS(q)
    MODE_STAGE = 2,         // dq = rka*dq + RHS(q); q_out = q_in + rkb_dt*dq
    MODE_STAGE_FIRST = 3    // rka == 0: dq = RHS(q) without reading dq; q_out = q_in + rkb_dt*dq
};

constexpr int kMaxNq = 8;
constexpr int32_t kStatusTimeout = 5;  // RB200_ERR_TIMEOUT
// Numerical flux codes (RB200_FLUX_* of raven_b200.h)
constexpr int kFluxCentral = 0, kFluxKG = 1, kFluxEC = 2, kFluxRusanov = 3, kFluxRoe = 4, kFluxMatrix = 5;

struct StageArgs {
    const double* q_in;   // (Np, Ns, E)
    double* q_out;        // stage modes only (may alias nothing that q_in aliases)
    void* dq;             // double* (FP64) or float* (FP32 bulk), read-modify-write in place
    const double* elem_geo;  // affine: (4, E): drdx, dsdy, dtdz, J
    const double* vgeo;      // curved: (Np, dim*dim+2, E): wJ*dRdX[dir,d] (dir-major), MJI, MJ
    const double* sgeo;      // curved: (dim+1, 2*dim*Nfp, E): n, wsJ
    const int32_t* nbr;      // (2*dim, E): neighbour element across each face, -1 = boundary,
                             // -2 = a mortar face (its flux is in ncflux)
    const double* ncflux;    // mortar face fluxes ((2*dim, E) faces x (Ns, Nfp)), or null
    const int32_t* vmapP;    // general connectivity (rotated faces, any neighbour face): per face
                             // node (2*dim*Nfp, E) the 0-based global node e'*Np + n' across the
                             // face; null on grids whose faces meet aligned (implied indexing)
    int64_t E;                // elements e_begin..E-1 are computed
    int64_t e_begin;
    int32_t mode;
    int32_t surface_rusanov;  // 1 Rusanov, 0 central (with surface_flux Rusanov or central)
    int32_t surface_flux;     // kFlux*: the entropy family (EC, KG, Roe, matrix) runs its own kernels
    int32_t dir_mask;         // DGSEM(; directions): bit d set = direction d's volume and face terms
                              // are computed (dgsem.jl:46-81, 257-348, 733-784); 0 reads as all
    // boundarystate (balancelaw.jl:22) per boundary tag 1..kMaxBcTags: a face whose
    // neighbour entry is -(kBcBase + tag) takes bc_kind[tag] (BC_PRESCRIBED: q+ = bc_state[tag],
    // BC_WALL: q+ = q- with the normal momentum reversed); other boundary faces keep q+ = q-
    int32_t bc_kind[9];
    double bc_state[9][5];
    double rka;
    double rkb_dt;
    double gamma;
    double adv[3];
    double D[kMaxNq * kMaxNq];  // D[i + nq*j] = l_j'(r_i)
    double w[kMaxNq];
};

// Programmatic dependent launch between the kernels of a step: a kernel launched with it
// may start while the previous kernel of the stream drains; it touches no global memory
// that kernel writes or reads before grid_dependency_wait() (griddepcontrol.wait: the
// previous grid has completed and its writes are visible; a no-op in a kernel launched
// without it).  RB200_PDL=0 launches the kernels in plain stream order.
#ifndef RB200_PDL
#define RB200_PDL 1
#endif
#ifdef __CUDACC__
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
#endif
// Launches kern<<<grid, block, smem, s>>>(args...) with programmatic stream serialization.
template <typename Kern, typename... Args>
cudaError_t launch_pdl(Kern kern, int grid, int block, size_t smem, cudaStream_t s, const Args&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3((unsigned)block, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = RB200_PDL;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, kern, args...);
    return e != cudaSuccess ? e : cudaGetLastError();
}

constexpr int kMaxBcTags = 8;
constexpr int kBcBase = 16;
enum { BC_DEFAULT = 0, BC_PRESCRIBED = 1, BC_WALL = 2 };

// Small grids: all stages of `nsteps` LSRK steps in one launch of one thread-block
// cluster (weak-form advection on unwarped bricks, stage_kernel.cuh).  The state q is
// read at the start and written at the end; stage s of a step has rka[s] and rkb_dt[s];
// the LSRK register is a.dq.
// CTAs of the cluster at most: 16, the largest size B200 runs (above the portable 8, with
// the kernel's opt-in), and nodes (threads) of a CTA at most.  On the 16^2, N=4 grid 13
// CTAs of 500 threads take 5.3 us a step against 7.7 us for 7 CTAs of 1000 threads.
#ifndef RB200_CLUSTER_CTAS
#define RB200_CLUSTER_CTAS 16
#endif
#ifndef RB200_CLUSTER_NODES
#define RB200_CLUSTER_NODES 512
#endif
constexpr int kClusterCtas = RB200_CLUSTER_CTAS;
constexpr int kClusterNodes = RB200_CLUSTER_NODES;
constexpr int kClusterStages = 32;   // stages of a step at most
struct ClusterStepsArgs {
    StageArgs a;                     // q_in, q_out, mode, rka and rkb_dt unused
    double* q;
    int32_t nsteps;
    int32_t nstages;
    double rka[kClusterStages];
    double rkb_dt[kClusterStages];
};
// Elements per CTA of the cluster kernel: up to kClusterNodes nodes a CTA.
inline int64_t cluster_elements_per_cta(int64_t np) { return np >= kClusterNodes ? 1 : kClusterNodes / np; }
cudaError_t launch_cluster_steps(int dim, int nq, int fp32, const ClusterStepsArgs& c, int ctas, cudaStream_t s);

// Mortars of an adapted grid (mortar.cu).
struct MortarArgs {
    const double* q;          // q_in (Np, Ns, E)
    double* ncflux;           // (2*dim, E) faces x (Ns, Nfp)
    const int64_t* mortars;   // (2 + 2^(dim-1), M): large element, its face, small elements
    int64_t M;
    int32_t surface_rusanov;
    int32_t surface_flux;     // kFlux*: the Euler entropy family uses surface_fluxes.cuh
    double gamma;
    double adv[3];
    double IL[kMaxNq * kMaxNq], IU[kMaxNq * kMaxNq];  // to the halves, [i*nq + j]
    double PL[kMaxNq * kMaxNq], PU[kMaxNq * kMaxNq];  // projections back, [j*nq + i]
    // curved (warped) grids: the per-face-node (n, wsJ) rows of the stage kernel
    // ((dim+1, 2*dim*Nfp, E)), null on affine grids; and the LGL weights
    const double* sgeo;
    double w[kMaxNq];
};
cudaError_t launch_mortars(int dim, int nq, int euler, int fp32, const MortarArgs& a, cudaStream_t s);

// Serving loop: one running solve of a class, and one chunk of its elements.
struct SolveDesc {
    double* q[2];             // ping-pong state buffers
    void* dq;                 // LSRK register (FP64 or FP32)
    const double* elem_geo;   // (4, E) unwarped brick geometry
    const int32_t* nbr;       // (2*dim, E) neighbour table
    int64_t E;
    double dt;
    int64_t start_tick;       // class tick at which the solve's state sat in q[0]
};

struct Chunk {
    int32_t solve;  // index into the descriptor table, or -1
    int32_t count;  // elements in this chunk (0: empty slot)
    int64_t first;  // first element of the chunk within the solve
};

// Launches one stage kernel; returns cudaSuccess or the launch error.
cudaError_t launch_stage(int dim, int nq, int combo, int geom, int fp32, const StageArgs& a, cudaStream_t s);
// Dynamic shared memory the kernel needs (bytes) and threads per block; 0 if not built.
size_t stage_smem_bytes(int dim, int nq, int combo, int geom, int fp32);

struct PipeArgs;  // pipelined_kernel.cuh
// Persistent TMA-pipelined kernel for 3-D Nq = 8 affine flux differencing (KG, EC).
cudaError_t launch_pipelined(int nq, int combo, int fp32, const PipeArgs& a, int grid, cudaStream_t s);
int pipelined_blocks_per_sm(int nq, int combo, int fp32);
struct PipeBatch;  // pipelined_kernel.cuh
// The same kernel over the chunks of a serving class (Euler KG only).
cudaError_t launch_pipelined_batch(int nq, int combo, int fp32, const PipeArgs& a, const PipeBatch& b, int grid,
                                   cudaStream_t s);
int pipelined_batch_blocks_per_sm(int nq, int combo, int fp32);
struct PipeCurvedArgs;  // pipelined_curved.cuh
// Persistent pipelined kernel for 3-D Nq = 8 curved grids (FP32 bulk, Kennedy-Gruber, stage modes).
cudaError_t launch_pipelined_curved(const PipeCurvedArgs& a, int grid, cudaStream_t s);
int pipelined_curved_blocks_per_sm();
// The same in FP64 (Kennedy-Gruber, stage modes).
cudaError_t launch_pipelined_curved64(const PipeCurvedArgs& a, int grid, cudaStream_t s);
int pipelined_curved64_blocks_per_sm();

// Reductions and face-map expansion (reduce.cu).
cudaError_t launch_weighted_sums(const double* q, const double* elem_geo, const double* vgeo, const double* w,
                                 int dim, int nq, int ns, int64_t E, int geom, double* partial, int nblocks,
                                 double* out_dev, cudaStream_t s);
// weightednorm for p != 2: out_dev[s] = sum MJ |q_s|^p, or max |q_s| for p = Inf.
cudaError_t launch_weighted_pnorm(const double* q, const double* elem_geo, const double* vgeo, const double* w,
                                  int dim, int nq, int ns, int64_t E, int geom, double p, double* partial,
                                  int nblocks, double* out_dev, cudaStream_t s);
cudaError_t launch_face_vmapP(const int32_t* nbr, int dim, int nq, int64_t E, int64_t* out, cudaStream_t s);
// out[k] = vmapP0[k] + 1: the 1-based vmapP of a grid kept with general connectivity
cudaError_t launch_copy_vmapP(const int32_t* vmapP0, int64_t n, int64_t* out, cudaStream_t s);

// Entropy measures and the RLSRK(5,4) step (relaxation.cu).  Sums land in out[0..1]
// (device): (sum MJ eta, sum MJ v.k); the stage kernel writes only out[1].
struct RelaxGeo {
    const double* elem_geo;  // affine: (4, E)
    const double* vgeo;      // curved: (Np, dim*dim+2, E), MJ at dim*dim+1
    int dim, nq, np, geom, euler;
    int64_t E;
    double gamma;
    double w[kMaxNq];
};
cudaError_t launch_entropy_sums(const RelaxGeo& G, const double* base, const double* dir, double c, const double* k,
                                double* partial, int nblocks, double* out, cudaStream_t s);
cudaError_t launch_rlsrk_stage(const RelaxGeo& G, double* q, double* dq, const double* k, double rka, double rkb_dt,
                               double* partial, int nblocks, double* out, cudaStream_t s);
cudaError_t launch_state_diff(const double* q, const double* q0, double* k, int64_t n, cudaStream_t s);
cudaError_t launch_relax(double* q, const double* q0, const double* k, double gamma, int64_t n, cudaStream_t s);

}  // namespace rb200
