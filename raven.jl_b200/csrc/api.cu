// Host runtime behind the C ABI (include/raven_b200.h).
//
// rb200_create turns the arrays of a Raven `Grid` into the compact device form the
// kernels read:
//  * geometry: an unwarped brick (what Raven's `isunwarpedbrick` path produces,
//    gridmanager.jl:1166) is detected node by node and stored as 4 doubles per
//    element (dRdX diagonal, J); anything else keeps per-node metric rows
//    wJ*dRdX[dir,:] plus MJI and MJ, and per-face-node (n, wsJ);
//  * connectivity: vmapM/vmapP (lobattocells.jl:2278-2291) become one int32
//    neighbour per element face.  Every node of every face is checked against the
//    given vmapP before the table is accepted, so the kernels' implied indexing is
//    the reference's indexing bit for bit (rb200_face_vmapP rebuilds it on the GPU).
//    A grid whose faces do not all meet aligned, face x- against face x+ and so on
//    (rotated faces of an unstructured coarse grid, lobattocells.jl:2177-2206), keeps
//    vmapP itself as an int32 table; the generic stage kernel then reads qP = q[vmapP]
//    node by node, and the handle takes the per-node (curved) geometry path.
#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/raven_b200.h"
#include "pipelined_curved.cuh"
#include "pipelined_kernel.cuh"
#include "rb200_internal.h"

using namespace rb200;

struct rb200_handle {
    int dim = 0, nq = 0, np = 0, nfp = 0, nf = 0, ns = 0;
    int64_t E = 0;
    int64_t E_active = 0;  // elements the kernels and reductions process; E_active..E-1 are ghosts
    int law = 0, form = 0, vflux = 0, sflux = 0, prec = 0, combo = 0, geom = 0;
    double gamma = 1.4, adv[3] = {0, 0, 0};
    double D[kMaxNq * kMaxNq] = {0}, w[kMaxNq] = {0};
    int device = 0;
    double* d_elem_geo = nullptr;
    double* d_vgeo = nullptr;
    double* d_sgeo = nullptr;
    double* d_w = nullptr;
    int32_t* d_nbr = nullptr;
    int32_t* d_vmapP = nullptr;  // general connectivity only: vmapP - 1 per face node
    double* d_qtmp = nullptr;
    float* d_dq32 = nullptr;
    double* d_hq = nullptr;   // device copy of a host state (rb200_lsrk54_step_host)
    double* d_hdq = nullptr;  // its LSRK register
    double* d_partial = nullptr;
    double* d_sums = nullptr;
    int32_t* d_status = nullptr;  // bounded-wait error word written by the kernels
    int red_blocks = 0;
    int kernel_path = 0;          // 0 automatic, 1 generic stage kernel only
    int dir_mask = 0;             // DGSEM(; directions) as a bit mask; 0 = all directions
    // boundarystate per boundary tag (rb200_set_boundary_condition); the face codes kept
    std::vector<int8_t> bcode;    // (nf, E) boundary codes of the grid
    int32_t bc_kind[kMaxBcTags + 1] = {0};
    double bc_state[kMaxBcTags + 1][5] = {{0}};
    bool has_bc = false;
    // CUDA graph of two LSRK steps (10 stage launches) for one (q, dq, dt), replayed by
    // rb200_lsrk54_step; captured on a stream of the handle, launched on the caller's
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    const double* graph_q = nullptr;
    const void* graph_dq = nullptr;
    double graph_dt = 0.0;
    // the captured graph's scheme, by value (a caller's table may change between calls)
    int graph_nst = 0;
    double graph_rka[32] = {0}, graph_rkb[32] = {0};
    // a caller's coefficient table (rb200_lsrk_step, rb200_rlsrk_step), copied per call
    double user_rka[32] = {0}, user_rkb[32] = {0};
    int use_graphs = 1;
    int pipe_grid = 0;            // CTAs of the pipelined kernel (0: not eligible)
    int pipe_curved_grid = 0;     // CTAs of the curved-grid pipelined kernel, FP32 bulk or FP64 (0: not eligible)
    double pipe_S[64] = {0};      // D[a,id] w[a] / w[id] - D[id,a] (advection: D[a,id] w[a] / w[id])
    // mortars of an adapted grid (rb200_set_mortars)
    int64_t nmortars = 0;
    int64_t* d_mortars = nullptr;
    double* d_ncflux = nullptr;
    MortarArgs mortar{};
    // RLSRK workspace (rb200_rlsrk54_step, rb200_rlsrk144_step): q0, the stage tendency k, and device sums
    double* d_rq0 = nullptr;
    double* d_rk = nullptr;
    double* d_rsums = nullptr;  // (eta, prod) pairs: [0] eta0, [1..stages] the stages
    std::string err;
};

namespace {

// LSRK(5,4) coefficients (odesolvers.jl:163-189): exact rationals, each rounded once.
const double RKA[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                       -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double RKB[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                       1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                       2277821191437.0 / 14882151754819.0};

// LSRK(14,4) coefficients (odesolvers.jl:191-239, coefficients_lsrk144): the reference's
// Float64 literals.
const double RKA144[14] = {0.0,
                           -0.7188012108672410,
                           -0.7785331173421570,
                           -0.0053282796654044,
                           -0.8552979934029281,
                           -3.9564138245774565,
                           -1.5780575380587385,
                           -2.0837094552574054,
                           -0.7483334182761610,
                           -0.7032861106563359,
                           0.0013917096117681,
                           -0.0932075369637460,
                           -0.9514200470875948,
                           -7.1151571693922548};
const double RKB144[14] = {0.0367762454319673, 0.3136296607553959, 0.1531848691869027, 0.0030097086818182,
                           0.3326293790646110, 0.2440251405350864, 0.3718879239592277, 0.6204126221582444,
                           0.1524043173028741, 0.0760894927419266, 0.0077604214040978, 0.0024647284755382,
                           0.0780348340049386, 5.5059777270269628};

// A low-storage Runge-Kutta scheme: its stage count and its a and b coefficients.
struct Scheme {
    int stages;
    const double* rka;
    const double* rkb;
};
constexpr int kMaxStages = 32;
const Scheme kLSRK54{5, RKA, RKB};
const Scheme kLSRK144{14, RKA144, RKB144};

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

rb200_status fail(rb200_handle* h, rb200_status st, const std::string& msg) {
    if (h) h->err = msg;
    return st;
}

rb200_status cuda_fail(rb200_handle* h, cudaError_t e, const char* where) {
    return fail(h, RB200_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// 0-based volume node of face f at in-face index j (cellfaceindices, lobattocells.jl:2012-2053)
int face_node(int dim, int nq, int f, int j) {
    const int dir = f / 2, c = (f % 2) ? nq - 1 : 0;
    if (dim == 1) return c;
    if (dim == 2) return dir == 0 ? c + nq * j : j + nq * c;
    const int j1 = j % nq, j2 = j / nq;
    if (dir == 0) return c + nq * (j1 + nq * j2);
    if (dir == 1) return j1 + nq * (c + nq * j2);
    return j1 + nq * (j2 + nq * c);
}

template <typename T>
rb200_status dev_alloc(rb200_handle* h, T** p, size_t count) {
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(h, RB200_ERR_OOM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
    }
    return RB200_OK;
}

void free_graph(rb200_handle* h) {
    if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    h->graph_exec = nullptr;
    h->graph_q = nullptr;
    h->graph_dq = nullptr;
}

void free_all(rb200_handle* h) {
    free_graph(h);
    if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
    h->cap_stream = nullptr;
    void* ptrs[] = {h->d_elem_geo, h->d_vgeo, h->d_sgeo,    h->d_w,    h->d_nbr,   h->d_qtmp,
                    h->d_dq32,     h->d_hq,   h->d_hdq,     h->d_partial, h->d_sums, h->d_status,
                    h->d_vmapP};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (h->d_mortars) cudaFree(h->d_mortars);
    if (h->d_ncflux) cudaFree(h->d_ncflux);
    h->d_mortars = nullptr;
    h->d_ncflux = nullptr;
    for (double** p : {&h->d_rq0, &h->d_rk, &h->d_rsums}) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    h->d_elem_geo = h->d_vgeo = h->d_sgeo = h->d_w = h->d_qtmp = h->d_hq = h->d_hdq = h->d_partial = h->d_sums =
        nullptr;
    h->d_nbr = nullptr;
    h->d_vmapP = nullptr;
    h->d_dq32 = nullptr;
    h->d_status = nullptr;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// One stage (or tendency) launch: the pipelined kernel when the configuration and the
// pointers allow it, the generic stage kernel otherwise.
cudaError_t launch_any(rb200_handle* h, const StageArgs& a, cudaStream_t st) {
    if (h->nmortars > 0) {  // adapted grid: the mortar fluxes of this q, then the stage
        MortarArgs m = h->mortar;
        m.q = a.q_in;
        cudaError_t e = launch_mortars(h->dim, h->nq, h->law == RB200_LAW_EULER, h->prec, m, st);
        if (e != cudaSuccess) return e;
    }
    const bool stage_mode = a.mode >= MODE_STAGE;
    // the pipelined kernels compute every direction; a direction subset runs the generic one
    const bool all_dirs = h->dir_mask == 0 && !h->has_bc;
    if (all_dirs && h->pipe_curved_grid > 0 && h->kernel_path == 0 && stage_mode && aligned16(a.q_in) && aligned16(a.q_out) &&
        aligned16(a.dq)) {
        PipeCurvedArgs c;
        std::memset(&c, 0, sizeof(c));
        c.q_in = a.q_in;
        c.q_out = a.q_out;
        if (h->prec == RB200_PRECISION_FP64) c.dq64 = static_cast<double*>(a.dq);
        else c.dq = static_cast<float*>(a.dq);
        c.vgeo = h->d_vgeo;
        c.sgeo = h->d_sgeo;
        c.nbr = h->d_nbr;
        c.status = h->d_status;
        c.E = a.E;
        c.e_begin = a.e_begin;
        c.mode = a.mode;
        c.surface_rusanov = a.surface_rusanov;
        c.rka = a.rka;
        c.rkb_dt = a.rkb_dt;
        c.gamma = a.gamma;
        std::memcpy(c.D, h->D, sizeof(c.D));
        const int grid = (int)std::min<int64_t>(h->pipe_curved_grid, a.E - a.e_begin);
        return h->prec == RB200_PRECISION_FP64 ? launch_pipelined_curved64(c, grid, st)
                                               : launch_pipelined_curved(c, grid, st);
    }
    const bool eligible = all_dirs && h->kernel_path == 0 && h->pipe_grid > 0 && aligned16(a.q_in) && aligned16(a.dq) &&
                          (!stage_mode || aligned16(a.q_out)) &&
                          (h->prec == RB200_PRECISION_FP64 || stage_mode);
    if (!eligible) return launch_stage(h->dim, h->nq, h->combo, h->geom, h->prec, a, st);
    PipeArgs p;
    std::memset(&p, 0, sizeof(p));
    p.q_in = a.q_in;
    p.q_out = a.q_out;
    p.dq = a.dq;
    p.elem_geo = a.elem_geo;
    p.nbr = a.nbr;
    p.ncflux = h->d_ncflux;
    p.status = h->d_status;
    p.E = a.E;
    p.e_begin = a.e_begin;
    p.mode = a.mode;
    p.surface_rusanov = a.surface_rusanov;
    p.rka = a.rka;
    p.rkb_dt = a.rkb_dt;
    p.gamma = a.gamma;
    std::memcpy(p.S, h->pipe_S, sizeof(p.S));
    for (int i = 0; i < 64; ++i) p.Sf[i] = (float)h->pipe_S[i];
    std::memcpy(p.w, h->w, sizeof(p.w));
    std::memcpy(p.adv, a.adv, sizeof(p.adv));
    const int grid = (int)std::min<int64_t>(h->pipe_grid, a.E - a.e_begin);
    return launch_pipelined(h->nq, h->combo, h->prec, p, grid, st);
}

StageArgs base_args(const rb200_handle* h) {
    StageArgs a;
    std::memset(&a, 0, sizeof(a));
    a.elem_geo = h->d_elem_geo;
    a.vgeo = h->d_vgeo;
    a.sgeo = h->d_sgeo;
    a.nbr = h->d_nbr;
    a.ncflux = h->d_ncflux;
    a.vmapP = h->d_vmapP;
    a.dir_mask = h->dir_mask;
    std::memcpy(a.bc_kind, h->bc_kind, sizeof(a.bc_kind));
    std::memcpy(a.bc_state, h->bc_state, sizeof(a.bc_state));
    a.E = h->E_active;
    a.surface_rusanov = h->sflux == RB200_FLUX_RUSANOV ? 1 : 0;
    a.surface_flux = h->sflux;
    a.gamma = h->gamma;
    for (int d = 0; d < 3; ++d) a.adv[d] = h->adv[d];
    std::memcpy(a.D, h->D, sizeof(a.D));
    std::memcpy(a.w, h->w, sizeof(a.w));
    return a;
}

// Enqueues `nsteps` steps of the scheme with q_in/q_out alternating between q and the
// handle's second state buffer; returns the buffer holding the result.
rb200_status enqueue_steps(rb200_handle* h, const Scheme& sc, double* q, void* dq, double dt, int32_t nsteps,
                           cudaStream_t st, double** result) {
    StageArgs a = base_args(h);
    a.dq = dq;
    double* cur = q;
    double* oth = h->d_qtmp;
    for (int32_t step = 0; step < nsteps; ++step) {
        for (int stg = 0; stg < sc.stages; ++stg) {
            a.q_in = cur;
            a.q_out = oth;
            a.mode = sc.rka[stg] == 0.0 ? MODE_STAGE_FIRST : MODE_STAGE;
            a.rka = sc.rka[stg];
            a.rkb_dt = sc.rkb[stg] * dt;
            cudaError_t e = launch_any(h, a, st);
            if (e != cudaSuccess) return cuda_fail(h, e, "stage kernel launch");
            double* t = cur;
            cur = oth;
            oth = t;
        }
    }
    *result = cur;
    return RB200_OK;
}

// CTAs of the cluster step kernel for this handle, or 0 where the steps run as stage
// launches: weak-form advection on an unwarped brick without mortars whose stages would
// run the generic stage kernel (no pipelined kernel for its Nq), the automatic kernel
// choice, and a grid whose elements kClusterCtas CTAs of kClusterNodes nodes hold.  The
// cluster kernel then computes what the stage launches compute, bit for bit.
int cluster_ctas(const rb200_handle* h) {
    // (every neighbour an element of the cluster: no ghost elements beyond E_active)
    if (h->kernel_path != 0 || h->combo != ADV_WEAK || h->geom != GEOM_AFFINE || h->nmortars > 0 ||
        h->pipe_grid > 0 || h->E_active != h->E)
        return 0;
    const int64_t epb = cluster_elements_per_cta(h->np);
    const int64_t groups = (h->E_active + epb - 1) / epb;
    if (groups < 1 || groups > kClusterCtas) return 0;
    return (int)groups;
}

rb200_status run_steps(rb200_handle* h, const Scheme& sc, double* q, void* dq, double dt, int32_t nsteps,
                       cudaStream_t st) {
    const size_t nstate = (size_t)h->np * h->ns * h->E;
    if (!h->d_qtmp) {
        rb200_status s = dev_alloc(h, &h->d_qtmp, nstate);
        if (s != RB200_OK) return s;
    }
    if (h->prec == RB200_PRECISION_FP32_BULK) dq = h->d_dq32;
    double* cur = q;
    rb200_status rs;
    int32_t done = 0;
    const int cctas = cluster_ctas(h);
    if (cctas > 0 && nsteps > 0 && sc.stages <= kClusterStages) {
        // a small grid: all stages of all steps in one launch of one cluster
        ClusterStepsArgs c;
        std::memset(&c, 0, sizeof(c));
        c.a = base_args(h);
        c.a.dq = dq;
        c.q = q;
        c.nsteps = nsteps;
        c.nstages = sc.stages;
        for (int s = 0; s < sc.stages; ++s) {
            c.rka[s] = sc.rka[s];
            c.rkb_dt[s] = sc.rkb[s] * dt;
        }
        cudaError_t e = launch_cluster_steps(h->dim, h->nq, h->prec == RB200_PRECISION_FP32_BULK ? 1 : 0, c, cctas, st);
        if (e == cudaSuccess) {
            done = nsteps;  // the result is in q
        } else if (e != cudaErrorNotSupported) {  // not supported: stage launches below
            return cuda_fail(h, e, "cluster step kernel launch");
        }
    }
    if (done < nsteps && h->use_graphs && nsteps >= 4) {
        // two steps (an even number of stages, so the state is back in q) run eagerly:
        // kernel attributes get configured outside the capture
        if ((rs = enqueue_steps(h, sc, q, dq, dt, 2, st, &cur)) != RB200_OK) return rs;
        done = 2;
        const bool same_scheme = h->graph_nst == sc.stages &&
                                 std::memcmp(h->graph_rka, sc.rka, sizeof(double) * sc.stages) == 0 &&
                                 std::memcmp(h->graph_rkb, sc.rkb, sizeof(double) * sc.stages) == 0;
        if (!h->graph_exec || h->graph_q != q || h->graph_dq != dq || h->graph_dt != dt || !same_scheme) {
            free_graph(h);
            cudaError_t e = cudaSuccess;
            if (!h->cap_stream) e = cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking);
            if (e != cudaSuccess) return cuda_fail(h, e, "graph stream");
            cudaGraph_t graph = nullptr;
            e = cudaStreamBeginCapture(h->cap_stream, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return cuda_fail(h, e, "graph capture");
            double* gres = nullptr;
            rs = enqueue_steps(h, sc, q, dq, dt, 2, h->cap_stream, &gres);
            e = cudaStreamEndCapture(h->cap_stream, &graph);
            if (rs != RB200_OK) {
                if (graph) cudaGraphDestroy(graph);
                return rs;
            }
            if (e == cudaSuccess) e = cudaGraphInstantiate(&h->graph_exec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (e != cudaSuccess) {
                h->graph_exec = nullptr;
                return cuda_fail(h, e, "graph instantiate");
            }
            h->graph_q = q;
            h->graph_dq = dq;
            h->graph_dt = dt;
            h->graph_nst = sc.stages;
            std::memcpy(h->graph_rka, sc.rka, sizeof(double) * sc.stages);
            std::memcpy(h->graph_rkb, sc.rkb, sizeof(double) * sc.stages);
        }
        for (; done + 2 <= nsteps; done += 2) {
            cudaError_t e = cudaGraphLaunch(h->graph_exec, st);
            if (e != cudaSuccess) return cuda_fail(h, e, "graph launch");
        }
    }
    if (done < nsteps) {
        if ((rs = enqueue_steps(h, sc, q, dq, dt, nsteps - done, st, &cur)) != RB200_OK) return rs;
    }
    if (cur != q) {
        cudaError_t e = cudaMemcpyAsync(q, cur, nstate * sizeof(double), cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return cuda_fail(h, e, "state copy-back");
    }
    return RB200_OK;
}

RelaxGeo relax_geo(const rb200_handle* h) {
    RelaxGeo G;
    std::memset(&G, 0, sizeof(G));
    G.elem_geo = h->d_elem_geo;
    G.vgeo = h->d_vgeo;
    G.dim = h->dim;
    G.nq = h->nq;
    G.np = h->np;
    G.geom = h->geom;
    G.euler = h->law == RB200_LAW_EULER ? 1 : 0;
    G.E = h->E_active;
    G.gamma = h->gamma;
    std::memcpy(G.w, h->w, sizeof(G.w));
    return G;
}

// (sum MJ eta(base + c dir), sum MJ v(base + c dir).k) into host out[0..1]
rb200_status entropy_sums_host(rb200_handle* h, const double* base, const double* dir, double c, const double* k,
                               double* out, cudaStream_t s) {
    cudaError_t e = launch_entropy_sums(relax_geo(h), base, dir, c, k, h->d_partial, h->red_blocks, h->d_sums, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, h->d_sums, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(h, e, "entropy reduction");
    return RB200_OK;
}

// rkb_full: the b coefficients of the standard Butcher form (odesolvers.jl:91-97)
void rkb_full(const Scheme& sc, double* bf) {
    const int n = sc.stages;
    bf[n - 1] = sc.rkb[n - 1];
    for (int i = n - 2; i >= 0; --i) bf[i] = sc.rka[i + 1] * bf[i + 1] + sc.rkb[i];
}

// One RLSRK step of the scheme (odesolvers.jl:118-151).  The relaxation solve r(gamma) = 0 with
// r(gamma) = eta(q0 + gamma k) - eta0 - gamma deta and r'(gamma) = v(q0 + gamma k).k - deta
// takes Newton steps from the previous gamma, as the reference's NLsolve trust-region
// method does for a scalar problem whose steps stay inside the region: a step is kept
// when it reduces r^2 by more than 1e-4 of the predicted reduction; the solve ends at
// |r| <= 10 eps (the reference's ftol) or at the first step that is not kept (the
// residual is then at round-off), after at most 1000 iterations.
rb200_status rlsrk_step(rb200_handle* h, const Scheme& sc, double* q, double* dq, double* gamma, double dt,
                        cudaStream_t s) {
    const int64_t n = (int64_t)h->np * h->ns * h->E;
    const RelaxGeo G = relax_geo(h);
    cudaError_t e = cudaMemcpyAsync(h->d_rq0, q, n * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
        e = launch_entropy_sums(G, h->d_rq0, nullptr, 0.0, nullptr, h->d_partial, h->red_blocks, h->d_rsums, s);
    if (e != cudaSuccess) return cuda_fail(h, e, "relaxation set-up");
    StageArgs a = base_args(h);
    a.mode = MODE_TENDENCY_SET;
    a.dq = h->d_rk;
    for (int st = 0; st < sc.stages; ++st) {
        a.q_in = q;
        e = launch_any(h, a, s);  // k = RHS(q)
        if (e == cudaSuccess)
            e = launch_rlsrk_stage(G, q, dq, h->d_rk, sc.rka[st], sc.rkb[st] * dt, h->d_partial, h->red_blocks,
                                   h->d_rsums + 2 * (1 + st), s);
        if (e != cudaSuccess) return cuda_fail(h, e, "relaxation stage");
    }
    e = launch_state_diff(q, h->d_rq0, h->d_rk, n, s);  // k = q - q0
    double sums[2 * (1 + kMaxStages)];
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(sums, h->d_rsums, 2 * (1 + sc.stages) * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(h, e, "relaxation stages");
    double bf[kMaxStages];
    rkb_full(sc, bf);
    const double eta0 = sums[0];
    double deta = -0.0;
    for (int st = 0; st < sc.stages; ++st) deta = deta + bf[st] * dt * sums[2 * (1 + st) + 1];
    const double ftol = 10 * 2.220446049250313e-16;
    auto eval = [&](double g, double* F, double* J) -> rb200_status {
        double s2[2];
        rb200_status rs = entropy_sums_host(h, h->d_rq0, h->d_rk, g, h->d_rk, s2, s);
        *F = s2[0] - eta0 - g * deta;
        *J = s2[1] - deta;
        return rs;
    };
    double g = *gamma, F, J;
    rb200_status rs = eval(g, &F, &J);
    if (rs != RB200_OK) return rs;
    if (!(std::fabs(F) <= ftol)) {
        for (int it = 0; it < 1000; ++it) {
            if (!(J != 0)) break;
            const double step = -F / J;
            const double gn = g + step;
            double Fn, Jn;
            if ((rs = eval(gn, &Fn, &Jn)) != RB200_OK) return rs;
            if (!(Fn * Fn < F * F * (1 - 1e-4))) break;
            g = gn;
            F = Fn;
            J = Jn;
            if (std::fabs(F) <= ftol || step == 0) break;
        }
    }
    if (!std::isfinite(g)) return fail(h, RB200_ERR_BAD_ARG, "relaxation parameter is not finite");
    *gamma = g;
    e = launch_relax(q, h->d_rq0, h->d_rk, g, n, s);
    if (e != cudaSuccess) return cuda_fail(h, e, "relaxation update");
    return RB200_OK;
}

}  // namespace

extern "C" {

const char* rb200_status_string(rb200_status s) {
    switch (s) {
        case RB200_OK: return "ok";
        case RB200_ERR_BAD_ARG: return "bad argument";
        case RB200_ERR_SHAPE: return "shape mismatch";
        case RB200_ERR_OOM: return "out of device memory";
        case RB200_ERR_CUDA: return "CUDA error";
        case RB200_ERR_TIMEOUT: return "timeout";
        case RB200_ERR_UNSUPPORTED: return "unsupported";
    }
    return "unknown status";
}

const char* rb200_last_error(const rb200_handle* h) {
    if (!h) return "null handle";
    return h->err.c_str();
}

rb200_status rb200_create(const rb200_desc* d, rb200_handle** out) {
    if (!out) return RB200_ERR_BAD_ARG;
    *out = nullptr;
    if (!d) return RB200_ERR_BAD_ARG;
    if (d->abi_version != RB200_ABI_VERSION) return RB200_ERR_BAD_ARG;
    rb200_handle* h = new (std::nothrow) rb200_handle();
    if (!h) return RB200_ERR_OOM;
    auto bail = [&](rb200_status s) {
        // the handle is returned even on failure so that rb200_last_error can explain;
        // the caller must still rb200_destroy it
        *out = h;
        return s;
    };
    if (d->dim < 1 || d->dim > 3) return bail(fail(h, RB200_ERR_UNSUPPORTED, "dim must be 1, 2 or 3"));
    if (d->nq < 2 || d->nq > kMaxNq) return bail(fail(h, RB200_ERR_UNSUPPORTED, "nq must be in 2..8"));
    if (d->num_elements < 0 || d->num_elements > (int64_t)INT32_MAX)
        return bail(fail(h, RB200_ERR_BAD_ARG, "num_elements out of range"));
    if (!d->D || !d->w || !d->volume_metrics || !d->surface_metrics || !d->vmapM || !d->vmapP)
        return bail(fail(h, RB200_ERR_BAD_ARG, "null host array in descriptor"));
    h->dim = d->dim;
    h->nq = d->nq;
    h->np = d->dim == 1 ? d->nq : d->dim == 2 ? d->nq * d->nq : d->nq * d->nq * d->nq;
    h->nfp = h->np / d->nq;
    h->nf = 2 * d->dim;
    h->E = d->num_elements;
    h->E_active = d->num_elements;
    h->law = d->law;
    h->form = d->volume_form;
    h->vflux = d->volume_flux;
    h->sflux = d->surface_flux;
    h->prec = d->precision;
    h->gamma = d->gamma;
    h->device = d->device;
    for (int i = 0; i < 3; ++i) h->adv[i] = d->advection_velocity[i];
    if (h->prec != RB200_PRECISION_FP64 && h->prec != RB200_PRECISION_FP32_BULK)
        return bail(fail(h, RB200_ERR_BAD_ARG, "unknown precision"));
    const bool entropy_flux = h->sflux == RB200_FLUX_KENNEDY_GRUBER || h->sflux == RB200_FLUX_ENTROPY_CONSERVATIVE ||
                              h->sflux == RB200_FLUX_ROE || h->sflux == RB200_FLUX_MATRIX;
    if (h->sflux != RB200_FLUX_RUSANOV && h->sflux != RB200_FLUX_CENTRAL && !entropy_flux)
        return bail(fail(h, RB200_ERR_BAD_ARG, "unknown surface flux"));
    if (entropy_flux && (h->law != RB200_LAW_EULER || h->prec != RB200_PRECISION_FP64))
        return bail(fail(h, RB200_ERR_UNSUPPORTED,
                         "the KG, EC, Roe and matrix surface fluxes are implemented for Euler in FP64"));
    if (h->law == RB200_LAW_ADVECTION) {
        h->ns = 1;
        if (h->form == RB200_FORM_WEAK) h->combo = ADV_WEAK;
        else if (h->form == RB200_FORM_FLUXDIFF && h->vflux == RB200_FLUX_CENTRAL) h->combo = ADV_FDC;
        else return bail(fail(h, RB200_ERR_UNSUPPORTED, "advection supports WeakForm and FluxDifferencing(Central)"));
    } else if (h->law == RB200_LAW_EULER) {
        h->ns = h->dim + 2;
        if (!(h->gamma > 1.0)) return bail(fail(h, RB200_ERR_BAD_ARG, "gamma must be > 1"));
        if (h->form == RB200_FORM_WEAK) h->combo = EUL_WEAK;
        else if (h->form == RB200_FORM_FLUXDIFF) {
            if (h->vflux == RB200_FLUX_CENTRAL) h->combo = EUL_FDC;
            else if (h->vflux == RB200_FLUX_KENNEDY_GRUBER) h->combo = EUL_KG;
            else if (h->vflux == RB200_FLUX_ENTROPY_CONSERVATIVE) h->combo = EUL_EC;
            else return bail(fail(h, RB200_ERR_UNSUPPORTED, "unknown volume flux"));
        } else return bail(fail(h, RB200_ERR_BAD_ARG, "unknown volume form"));
    } else {
        return bail(fail(h, RB200_ERR_BAD_ARG, "unknown law"));
    }
    const int dim = h->dim, nq = h->nq, np = h->np, nfp = h->nfp, nf = h->nf;
    const int64_t E = h->E;
    for (int i = 0; i < nq * nq; ++i) h->D[i] = d->D[i];
    for (int i = 0; i < nq; ++i) h->w[i] = d->w[i];

    // ---------------------------------------------------------------- geometry
    const int nvm = dim * dim + 2;  // dRdX, J, wJ
    const int nsm = dim + 2;        // n, sJ, wsJ
    const double* vm = d->volume_metrics;
    const double* sm = d->surface_metrics;
    bool affine = true;
    std::vector<double> eg(4 * (size_t)E, 0.0);
    for (int64_t e = 0; e < E && affine; ++e) {
        const double* m = vm + (size_t)np * nvm * e;
        double diag[3], J = m[(size_t)np * (dim * dim)];
        for (int a = 0; a < dim; ++a) diag[a] = m[(size_t)np * (a + dim * a)];
        for (int n = 0; n < np && affine; ++n) {
            for (int a = 0; a < dim; ++a)
                for (int b = 0; b < dim; ++b) {
                    const double v = m[n + (size_t)np * (a + dim * b)];
                    if (a == b ? v != diag[a] : v != 0.0) affine = false;
                }
            if (m[n + (size_t)np * (dim * dim)] != J) affine = false;
            const int idx[3] = {n % nq, (n / nq) % nq, n / (nq * nq)};
            double wJ = h->w[idx[0]];
            for (int k = 1; k < dim; ++k) wJ = wJ * h->w[idx[k]];
            wJ = wJ * J;
            if (m[n + (size_t)np * (dim * dim + 1)] != wJ) affine = false;
        }
        for (int f = 0; f < nf && affine; ++f) {
            const int dir = f / 2;
            const double sJ = std::fabs(J * diag[dir]);
            for (int j = 0; j < nfp && affine; ++j) {
                const double* s = sm + (size_t)nsm * ((size_t)nf * nfp * e + (size_t)f * nfp + j);
                for (int k = 0; k < dim; ++k) {
                    const double want = k == dir ? (f % 2 ? 1.0 : -1.0) : 0.0;
                    if (s[k] != want) affine = false;
                }
                double wsJ;
                if (dim == 1) wsJ = sJ;  // one node a face: weight 1 (lobattocells.jl:2656)
                else if (dim == 2) wsJ = sJ * h->w[j];
                else wsJ = (sJ * h->w[j % nq]) * h->w[j / nq];
                if (s[dim + 1] != wsJ) affine = false;
            }
        }
        for (int a = 0; a < dim; ++a) eg[4 * e + a] = diag[a];
        eg[4 * e + 3] = J;
    }
    h->geom = affine ? GEOM_AFFINE : GEOM_CURVED;

    // ------------------------------------------------------------- connectivity
    std::vector<int32_t> nbr((size_t)nf * E, -1);
    h->bcode.assign((size_t)nf * E, 0);
    bool general = false;  // some face meets its neighbour rotated or on another face
    for (int64_t e = 0; e < E; ++e)
        for (int f = 0; f < nf; ++f) {
            const size_t base = (size_t)nf * nfp * e + (size_t)f * nfp;
            const int64_t bcode = d->boundary_codes ? d->boundary_codes[(size_t)nf * e + f] : 0;
            for (int j = 0; j < nfp; ++j)
                if (d->vmapM[base + j] != (int64_t)np * e + face_node(dim, nq, f, j) + 1)
                    return bail(fail(h, RB200_ERR_SHAPE, "vmapM is not Raven's face-node numbering"));
            if (bcode != 0) {
                h->bcode[(size_t)nf * e + f] = (int8_t)(bcode >= 1 && bcode <= kMaxBcTags ? bcode : 0);
                nbr[(size_t)nf * e + f] = -1;
                continue;
            }
            const int64_t p0 = d->vmapP[base] - 1;
            const int64_t ne = p0 / np;
            bool ok = ne >= 0 && ne < E;
            for (int j = 0; j < nfp && ok; ++j)
                ok = d->vmapP[base + j] == ne * np + face_node(dim, nq, f ^ 1, j) + 1;
            if (!ok) {
                bool self = true;  // non-conforming / unconnected faces keep vmapP = vmapM
                for (int j = 0; j < nfp && self; ++j) self = d->vmapP[base + j] == d->vmapM[base + j];
                if (self) {
                    nbr[(size_t)nf * e + f] = -1;
                    continue;
                }
                // a conforming neighbour in another orientation or on another face: every
                // node must name a node of one other element, on one of its faces
                const int64_t tot = (int64_t)np * E;
                const int64_t e2 = ne;
                ok = ne >= 0 && ne < E;
                for (int j = 0; j < nfp && ok; ++j) {
                    const int64_t g = d->vmapP[base + j] - 1;
                    ok = g >= 0 && g < tot && g / np == e2;
                    if (ok) {
                        const int n2 = (int)(g % np);
                        const int i0 = n2 % nq, i1 = (n2 / nq) % nq, i2 = dim == 3 ? n2 / (nq * nq) : 0;
                        ok = i0 == 0 || i0 == nq - 1 || i1 == 0 || i1 == nq - 1 ||
                             (dim == 3 && (i2 == 0 || i2 == nq - 1));
                    }
                }
                if (!ok)
                    return bail(fail(h, RB200_ERR_SHAPE,
                                     "vmapP: a face's nodes do not all lie on one face of one other element"));
                general = true;
            }
            nbr[(size_t)nf * e + f] = (int32_t)ne;
        }
    std::vector<int32_t> vmapP32;
    if (general) {
        if ((int64_t)np * E > (int64_t)INT32_MAX)
            return bail(fail(h, RB200_ERR_UNSUPPORTED, "general face connectivity needs Np*E < 2^31"));
        vmapP32.resize((size_t)nf * nfp * E);
        for (size_t k = 0; k < vmapP32.size(); ++k) vmapP32[k] = (int32_t)(d->vmapP[k] - 1);
        // the kernels with implied face indexing (bricks) do not apply: per-node geometry
        affine = false;
        h->geom = GEOM_CURVED;
    }

    // ----------------------------------------------------------------- upload
    DeviceGuard guard(h->device);
    rb200_status st;
    if ((st = dev_alloc(h, &h->d_nbr, nbr.size())) != RB200_OK) return bail(st);
    if ((st = dev_alloc(h, &h->d_w, (size_t)nq)) != RB200_OK) return bail(st);
    cudaError_t ce = cudaMemcpy(h->d_nbr, nbr.data(), nbr.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemcpy(h->d_w, h->w, nq * sizeof(double), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) return bail(cuda_fail(h, ce, "upload"));
    if (general) {
        if ((st = dev_alloc(h, &h->d_vmapP, vmapP32.size())) != RB200_OK) return bail(st);
        ce = cudaMemcpy(h->d_vmapP, vmapP32.data(), vmapP32.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
        if (ce != cudaSuccess) return bail(cuda_fail(h, ce, "upload"));
    }
    if (affine) {
        if ((st = dev_alloc(h, &h->d_elem_geo, eg.size())) != RB200_OK) return bail(st);
        ce = cudaMemcpy(h->d_elem_geo, eg.data(), eg.size() * sizeof(double), cudaMemcpyHostToDevice);
        if (ce != cudaSuccess) return bail(cuda_fail(h, ce, "upload"));
    } else {
        const int nvg = dim * dim + 2;  // wJ*dRdX[dir,d] (dir-major), MJI, MJ
        std::vector<double> vg((size_t)np * nvg * E);
        for (int64_t e = 0; e < E; ++e) {
            const double* m = vm + (size_t)np * nvm * e;
            double* g = vg.data() + (size_t)np * nvg * e;
            for (int n = 0; n < np; ++n) {
                const double wJ = m[n + (size_t)np * (dim * dim + 1)];
                for (int dir = 0; dir < dim; ++dir)
                    for (int k = 0; k < dim; ++k)
                        g[n + (size_t)np * (dir * dim + k)] = wJ * m[n + (size_t)np * (dir + dim * k)];
                g[n + (size_t)np * (dim * dim)] = 1.0 / wJ;
                g[n + (size_t)np * (dim * dim + 1)] = wJ;
            }
        }
        std::vector<double> sg((size_t)(dim + 1) * nf * nfp * E);
        for (size_t k = 0; k < (size_t)nf * nfp * E; ++k) {
            for (int c = 0; c < dim; ++c) sg[(dim + 1) * k + c] = sm[nsm * k + c];
            sg[(dim + 1) * k + dim] = sm[nsm * k + dim + 1];
        }
        if ((st = dev_alloc(h, &h->d_vgeo, vg.size())) != RB200_OK) return bail(st);
        if ((st = dev_alloc(h, &h->d_sgeo, sg.size())) != RB200_OK) return bail(st);
        ce = cudaMemcpy(h->d_vgeo, vg.data(), vg.size() * sizeof(double), cudaMemcpyHostToDevice);
        if (ce == cudaSuccess) ce = cudaMemcpy(h->d_sgeo, sg.data(), sg.size() * sizeof(double), cudaMemcpyHostToDevice);
        if (ce != cudaSuccess) return bail(cuda_fail(h, ce, "upload"));
    }
    if (h->prec == RB200_PRECISION_FP32_BULK) {
        const size_t n = (size_t)np * h->ns * E;
        if ((st = dev_alloc(h, &h->d_dq32, n)) != RB200_OK) return bail(st);
        ce = cudaMemset(h->d_dq32, 0, n * sizeof(float));
        if (ce != cudaSuccess) return bail(cuda_fail(h, ce, "memset"));
    }
    if ((st = dev_alloc(h, &h->d_status, 1)) != RB200_OK) return bail(st);
    ce = cudaMemset(h->d_status, 0, sizeof(int32_t));
    if (ce != cudaSuccess) return bail(cuda_fail(h, ce, "memset"));
    if (dim == 3 && (nq == 4 || nq == 6 || nq == 8) && affine &&
        (h->combo == EUL_KG || h->combo == EUL_EC || h->combo == ADV_WEAK) && !entropy_flux) {
        // flux differencing: S[a, id] = D[a,id] w[a] / w[id] - D[id,a]; weak-form
        // advection: W[a, id] = D[a,id] w[a] / w[id]
        for (int a = 0; a < nq; ++a)
            for (int id = 0; id < nq; ++id)
                h->pipe_S[a * nq + id] = h->combo == ADV_WEAK
                                             ? h->D[a + nq * id] * (h->w[a] / h->w[id])
                                             : h->D[a + nq * id] * (h->w[a] / h->w[id]) - h->D[id + nq * a];
        int dev = 0, nsm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        const int per_sm = pipelined_blocks_per_sm(nq, h->combo, h->prec);
        h->pipe_grid = per_sm > 0 ? per_sm * nsm : 0;
        cudaGetLastError();
    }
    if (dim == 3 && nq == 8 && !affine && !general && h->combo == EUL_KG && !entropy_flux && h->d_vgeo && h->d_sgeo &&
        aligned16(h->d_vgeo) && aligned16(h->d_sgeo)) {
        // curved 3-D Nq = 8 Kennedy-Gruber: the curved pipelined kernel of the handle's precision
        int dev = 0, nsm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        const int per_sm = h->prec == RB200_PRECISION_FP64 ? pipelined_curved64_blocks_per_sm()
                                                           : pipelined_curved_blocks_per_sm();
        h->pipe_curved_grid = per_sm > 0 ? per_sm * nsm : 0;
        cudaGetLastError();
    }
    h->red_blocks = 296;
    if ((st = dev_alloc(h, &h->d_partial, (size_t)h->red_blocks * 2 * h->ns)) != RB200_OK) return bail(st);
    if ((st = dev_alloc(h, &h->d_sums, (size_t)2 * h->ns)) != RB200_OK) return bail(st);
    if (stage_smem_bytes(dim, nq, h->combo, h->geom, h->prec) == 0)
        return bail(fail(h, RB200_ERR_UNSUPPORTED, "no kernel instantiation for this configuration"));
    *out = h;
    return RB200_OK;
}

rb200_status rb200_destroy(rb200_handle* h) {
    if (!h) return RB200_ERR_BAD_ARG;
    {
        DeviceGuard guard(h->device);
        free_all(h);
    }
    delete h;
    return RB200_OK;
}

rb200_status rb200_tendency(rb200_handle* h, double* dq, const double* q, double time, int32_t increment,
                            void* stream) {
    (void)time;  // the advection and Euler laws have no time-dependent sources
    if (!h) return RB200_ERR_BAD_ARG;
    if (!dq || !q) return fail(h, RB200_ERR_BAD_ARG, "null state pointer");
    if (h->E_active == 0) return RB200_OK;
    DeviceGuard guard(h->device);
    StageArgs a = base_args(h);
    a.q_in = q;
    a.dq = dq;
    a.mode = increment ? MODE_TENDENCY_INC : MODE_TENDENCY_SET;
    cudaError_t e = launch_any(h, a, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "tendency kernel launch");
    return RB200_OK;
}

static rb200_status lsrk_steps(rb200_handle* h, const Scheme& sc, double* q, double* dq, double dt, int32_t nsteps,
                               void* stream) {
    if (!h) return RB200_ERR_BAD_ARG;
    if (!q || (!dq && h->prec == RB200_PRECISION_FP64)) return fail(h, RB200_ERR_BAD_ARG, "null state pointer");
    if (nsteps < 0 || !std::isfinite(dt)) return fail(h, RB200_ERR_BAD_ARG, "bad nsteps or dt");
    if (h->E_active == 0 || nsteps == 0) return RB200_OK;
    DeviceGuard guard(h->device);
    return run_steps(h, sc, q, dq, dt, nsteps, (cudaStream_t)stream);
}

rb200_status rb200_lsrk54_step(rb200_handle* h, double* q, double* dq, double time, double dt, int32_t nsteps,
                               void* stream) {
    (void)time;
    return lsrk_steps(h, kLSRK54, q, dq, dt, nsteps, stream);
}

rb200_status rb200_lsrk144_step(rb200_handle* h, double* q, double* dq, double time, double dt, int32_t nsteps,
                                void* stream) {
    (void)time;
    return lsrk_steps(h, kLSRK144, q, dq, dt, nsteps, stream);
}

// A caller's low-storage table: finite, at most kMaxStages stages, copied into the handle.
static rb200_status user_scheme(rb200_handle* h, const double* rka, const double* rkb, int32_t nstages, Scheme* sc) {
    if (!rka || !rkb) return fail(h, RB200_ERR_BAD_ARG, "null coefficient table");
    if (nstages < 1 || nstages > kMaxStages) return fail(h, RB200_ERR_BAD_ARG, "nstages must be in 1..32");
    for (int i = 0; i < nstages; ++i)
        if (!std::isfinite(rka[i]) || !std::isfinite(rkb[i])) return fail(h, RB200_ERR_BAD_ARG, "coefficients not finite");
    std::memcpy(h->user_rka, rka, sizeof(double) * nstages);
    std::memcpy(h->user_rkb, rkb, sizeof(double) * nstages);
    *sc = Scheme{nstages, h->user_rka, h->user_rkb};
    return RB200_OK;
}

rb200_status rb200_lsrk_step(rb200_handle* h, double* q, double* dq, const double* rka, const double* rkb,
                             int32_t nstages, double time, double dt, int32_t nsteps, void* stream) {
    (void)time;
    if (!h) return RB200_ERR_BAD_ARG;
    Scheme sc;
    rb200_status st = user_scheme(h, rka, rkb, nstages, &sc);
    if (st != RB200_OK) return st;
    return lsrk_steps(h, sc, q, dq, dt, nsteps, stream);
}

// One stage of LSRK(5,4) (odesolvers.jl:163-189) from q_in to q_out on elements
// e_begin..e_end-1: the building block of a step whose ghost elements are refreshed
// between stages (the start!/finish! exchange of dgsem.jl:95-100 around every
// right-hand side), with the interior elements computed while the exchange runs.
static rb200_status stage_range(rb200_handle* h, const double* q_in, double* q_out, double* dq, double rka,
                                double rkb, int64_t e_begin, int64_t e_end, double dt, cudaStream_t s) {
    if (!q_in || !q_out || (!dq && h->prec == RB200_PRECISION_FP64))
        return fail(h, RB200_ERR_BAD_ARG, "null state pointer");
    if (q_in == q_out) return fail(h, RB200_ERR_BAD_ARG, "q_in and q_out must be different buffers");
    if (!std::isfinite(rka) || !std::isfinite(rkb) || !std::isfinite(dt))
        return fail(h, RB200_ERR_BAD_ARG, "bad coefficients or dt");
    if (e_begin < 0 || e_begin > e_end || e_end > h->E_active)
        return fail(h, RB200_ERR_BAD_ARG, "element range outside the active elements");
    if (e_begin == e_end) return RB200_OK;
    DeviceGuard guard(h->device);
    StageArgs a = base_args(h);
    a.e_begin = e_begin;
    a.E = e_end;
    a.q_in = q_in;
    a.q_out = q_out;
    a.dq = h->prec == RB200_PRECISION_FP32_BULK ? static_cast<void*>(h->d_dq32) : static_cast<void*>(dq);
    a.mode = rka == 0.0 ? MODE_STAGE_FIRST : MODE_STAGE;
    a.rka = rka;
    a.rkb_dt = rkb * dt;
    cudaError_t e = launch_any(h, a, s);
    if (e != cudaSuccess) return cuda_fail(h, e, "stage kernel launch");
    return RB200_OK;
}

rb200_status rb200_lsrk54_stage(rb200_handle* h, const double* q_in, double* q_out, double* dq, int32_t stage,
                                double time, double dt, void* stream) {
    (void)time;
    if (!h) return RB200_ERR_BAD_ARG;
    if (stage < 0 || stage > 4) return fail(h, RB200_ERR_BAD_ARG, "bad stage or dt");
    return stage_range(h, q_in, q_out, dq, RKA[stage], RKB[stage], 0, h->E_active, dt, (cudaStream_t)stream);
}

rb200_status rb200_lsrk54_stage_range(rb200_handle* h, const double* q_in, double* q_out, double* dq,
                                      int32_t stage, int64_t e_begin, int64_t e_end, double time, double dt,
                                      void* stream) {
    (void)time;
    if (!h) return RB200_ERR_BAD_ARG;
    if (stage < 0 || stage > 4) return fail(h, RB200_ERR_BAD_ARG, "bad stage or dt");
    return stage_range(h, q_in, q_out, dq, RKA[stage], RKB[stage], e_begin, e_end, dt, (cudaStream_t)stream);
}

rb200_status rb200_lsrk_stage(rb200_handle* h, const double* q_in, double* q_out, double* dq, double rka,
                              double rkb, double time, double dt, void* stream) {
    (void)time;
    if (!h) return RB200_ERR_BAD_ARG;
    return stage_range(h, q_in, q_out, dq, rka, rkb, 0, h->E_active, dt, (cudaStream_t)stream);
}

rb200_status rb200_lsrk_stage_range(rb200_handle* h, const double* q_in, double* q_out, double* dq, double rka,
                                    double rkb, int64_t e_begin, int64_t e_end, double time, double dt,
                                    void* stream) {
    (void)time;
    if (!h) return RB200_ERR_BAD_ARG;
    return stage_range(h, q_in, q_out, dq, rka, rkb, e_begin, e_end, dt, (cudaStream_t)stream);
}

rb200_status rb200_set_active_elements(rb200_handle* h, int64_t num_active) {
    if (!h) return RB200_ERR_BAD_ARG;
    if (num_active < 0 || num_active > h->E) return fail(h, RB200_ERR_BAD_ARG, "active elements out of range");
    if (h->nmortars > 0 && num_active != h->E)
        return fail(h, RB200_ERR_UNSUPPORTED, "ghost elements on an adapted grid");
    DeviceGuard guard(h->device);
    free_graph(h);  // a captured step holds the old element count
    h->E_active = num_active;
    return RB200_OK;
}

rb200_status rb200_lsrk54_step_host(rb200_handle* h, double* q_host, double time, double dt, int32_t nsteps,
                                    void* stream) {
    (void)time;
    if (!h) return RB200_ERR_BAD_ARG;
    if (!q_host) return fail(h, RB200_ERR_BAD_ARG, "null state pointer");
    if (nsteps < 0 || !std::isfinite(dt)) return fail(h, RB200_ERR_BAD_ARG, "bad nsteps or dt");
    if (h->E == 0) return RB200_OK;
    DeviceGuard guard(h->device);
    const size_t n = (size_t)h->np * h->ns * h->E;
    rb200_status st;
    if (!h->d_hq && (st = dev_alloc(h, &h->d_hq, n)) != RB200_OK) return st;
    if (!h->d_hdq && (st = dev_alloc(h, &h->d_hdq, n)) != RB200_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(h->d_hq, q_host, n * sizeof(double), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(h, e, "host-to-device copy");
    if ((st = run_steps(h, kLSRK54, h->d_hq, h->d_hdq, dt, nsteps, s)) != RB200_OK) return st;
    e = cudaMemcpyAsync(q_host, h->d_hq, n * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(h, e, "device-to-host copy");
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(h, e, "stream synchronize");
    return RB200_OK;
}

static rb200_status sums(rb200_handle* h, const double* q, double* host, cudaStream_t s) {
    if (!h) return RB200_ERR_BAD_ARG;
    if (!q || !host) return fail(h, RB200_ERR_BAD_ARG, "null pointer");
    DeviceGuard guard(h->device);
    cudaError_t e = launch_weighted_sums(q, h->d_elem_geo, h->d_vgeo, h->d_w, h->dim, h->nq, h->ns, h->E_active, h->geom,
                                         h->d_partial, h->red_blocks, h->d_sums, s);
    if (e != cudaSuccess) return cuda_fail(h, e, "reduction launch");
    e = cudaMemcpyAsync(host, h->d_sums, 2 * h->ns * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(h, e, "reduction readback");
    return RB200_OK;
}

rb200_status rb200_weightednorm(rb200_handle* h, const double* q, double* out, void* stream) {
    double buf[2 * 5];
    rb200_status st = sums(h, q, buf, (cudaStream_t)stream);
    if (st != RB200_OK) return st;
    double tot = 0.0;
    for (int s = 0; s < h->ns; ++s) {
        out[s] = std::sqrt(buf[s]);
        tot += out[s] * out[s];
    }
    out[h->ns] = std::sqrt(tot);
    return RB200_OK;
}

rb200_status rb200_weightednorm_p(rb200_handle* h, const double* q, double p, double* out, void* stream) {
    if (!h) return RB200_ERR_BAD_ARG;
    if (!q || !out) return fail(h, RB200_ERR_BAD_ARG, "null pointer");
    if (std::isnan(p) || p <= 0.0) return fail(h, RB200_ERR_BAD_ARG, "weightednorm: p must be > 0 or Inf");
    if (p == 2.0) return rb200_weightednorm(h, q, out, stream);
    DeviceGuard guard(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = launch_weighted_pnorm(q, h->d_elem_geo, h->d_vgeo, h->d_w, h->dim, h->nq, h->ns, h->E_active,
                                          h->geom, p, h->d_partial, h->red_blocks, h->d_sums, s);
    if (e != cudaSuccess) return cuda_fail(h, e, "reduction launch");
    double buf[5];
    e = cudaMemcpyAsync(buf, h->d_sums, h->ns * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(h, e, "reduction readback");
    // per field: the sum to the power 1/p (measures.jl:11), or the maximum (:18); then
    // norm(n, p) over the fields: maximum, sum, or (sum n^p)^(1/p)
    const bool inf = std::isinf(p);
    double tot = 0.0, mx = 0.0;
    for (int f = 0; f < h->ns; ++f) {
        const double c = inf ? buf[f] : (p == 1.0 ? buf[f] : std::pow(buf[f], 1.0 / p));
        out[f] = c;
        if (std::isnan(c) || c > mx) mx = c;
        tot += p == 1.0 ? c : std::pow(c, p);
    }
    out[h->ns] = inf ? mx : (p == 1.0 ? tot : std::pow(tot, 1.0 / p));
    return RB200_OK;
}

rb200_status rb200_integrals(rb200_handle* h, const double* q, double* out, void* stream) {
    double buf[2 * 5];
    rb200_status st = sums(h, q, buf, (cudaStream_t)stream);
    if (st != RB200_OK) return st;
    for (int s = 0; s < h->ns; ++s) out[s] = buf[h->ns + s];
    return RB200_OK;
}

rb200_status rb200_entropy_integral(rb200_handle* h, const double* q, double* out, void* stream) {
    if (!h) return RB200_ERR_BAD_ARG;
    if (!q || !out) return fail(h, RB200_ERR_BAD_ARG, "null pointer");
    DeviceGuard guard(h->device);
    double s2[2];
    rb200_status st = entropy_sums_host(h, q, nullptr, 0.0, nullptr, s2, (cudaStream_t)stream);
    if (st == RB200_OK) *out = s2[0];
    return st;
}

rb200_status rb200_entropy_product(rb200_handle* h, const double* p, const double* q, double* out, void* stream) {
    if (!h) return RB200_ERR_BAD_ARG;
    if (!p || !q || !out) return fail(h, RB200_ERR_BAD_ARG, "null pointer");
    DeviceGuard guard(h->device);
    double s2[2];
    rb200_status st = entropy_sums_host(h, p, nullptr, 0.0, q, s2, (cudaStream_t)stream);
    if (st == RB200_OK) *out = s2[1];
    return st;
}

static rb200_status rlsrk_steps(rb200_handle* h, const Scheme& sc, double* q, double* dq, double* gamma, double dt,
                                int32_t nsteps, void* stream) {
    if (!h) return RB200_ERR_BAD_ARG;
    if (!q || !dq || !gamma) return fail(h, RB200_ERR_BAD_ARG, "null pointer");
    if (nsteps < 0 || !std::isfinite(dt) || !std::isfinite(*gamma)) return fail(h, RB200_ERR_BAD_ARG, "bad nsteps, dt or gamma");
    if (h->prec != RB200_PRECISION_FP64)
        return fail(h, RB200_ERR_UNSUPPORTED, "RLSRK keeps its LSRK register in FP64: create the handle in FP64");
    if (h->E == 0 || nsteps == 0) return RB200_OK;
    DeviceGuard guard(h->device);
    const size_t n = (size_t)h->np * h->ns * h->E;
    rb200_status st;
    if (!h->d_rq0 && (st = dev_alloc(h, &h->d_rq0, n)) != RB200_OK) return st;
    if (!h->d_rk && (st = dev_alloc(h, &h->d_rk, n)) != RB200_OK) return st;
    if (!h->d_rsums && (st = dev_alloc(h, &h->d_rsums, 2 * (1 + kMaxStages))) != RB200_OK) return st;
    for (int32_t i = 0; i < nsteps; ++i)
        if ((st = rlsrk_step(h, sc, q, dq, gamma, dt, (cudaStream_t)stream)) != RB200_OK) return st;
    return RB200_OK;
}

rb200_status rb200_rlsrk54_step(rb200_handle* h, double* q, double* dq, double* gamma, double time, double dt,
                                int32_t nsteps, void* stream) {
    (void)time;
    return rlsrk_steps(h, kLSRK54, q, dq, gamma, dt, nsteps, stream);
}

rb200_status rb200_rlsrk144_step(rb200_handle* h, double* q, double* dq, double* gamma, double time, double dt,
                                 int32_t nsteps, void* stream) {
    (void)time;
    return rlsrk_steps(h, kLSRK144, q, dq, gamma, dt, nsteps, stream);
}

rb200_status rb200_rlsrk_step(rb200_handle* h, double* q, double* dq, double* gamma, const double* rka,
                              const double* rkb, int32_t nstages, double time, double dt, int32_t nsteps,
                              void* stream) {
    (void)time;
    if (!h) return RB200_ERR_BAD_ARG;
    Scheme sc;
    rb200_status st = user_scheme(h, rka, rkb, nstages, &sc);
    if (st != RB200_OK) return st;
    return rlsrk_steps(h, sc, q, dq, gamma, dt, nsteps, stream);
}

// ---------------------------------------------------------------------------------
// Snapshot / resume of the time-stepper state (q, dq, time, dt, gamma)
// ---------------------------------------------------------------------------------

// 64-bit multiply-xor hash over little-endian 64-bit words (FNV-1a's prime and offset,
// applied per word rather than per byte), then per byte for a ragged tail.
static uint64_t snap_hash(const void* data, size_t bytes, uint64_t h = 0xcbf29ce484222325ull) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    const uint64_t prime = 0x100000001b3ull;
    size_t i = 0;
    for (; i + 8 <= bytes; i += 8) {
        uint64_t w;
        std::memcpy(&w, p + i, 8);
        h = (h ^ w) * prime;
    }
    for (; i < bytes; ++i) h = (h ^ p[i]) * prime;
    return h;
}

struct SnapHeader {
    char magic[8];  // "RB200SNP"
    uint32_t version;
    uint32_t header_bytes;
    int32_t dim, nq, ns, law, precision, combo;
    int64_t E;
    uint64_t q_bytes, dq_bytes;
    double time, dt, gamma;
    uint64_t fingerprint;  // the discretization: sizes, law, scheme, D, w, gamma, velocity,
                           // directions and boundary conditions when set
    uint64_t payload_sum;  // hash of the q bytes, then the dq bytes
    uint64_t reserved[2];
    uint64_t header_sum;   // hash of every byte before this field
};
static_assert(sizeof(SnapHeader) == 128, "snapshot header layout");

static uint64_t snap_fingerprint(const rb200_handle* h) {
    const int32_t ints[9] = {h->dim, h->nq, h->ns, h->law, h->form, h->vflux, h->sflux, h->prec, h->combo};
    uint64_t f = snap_hash(ints, sizeof(ints));
    f = snap_hash(&h->E, sizeof(h->E), f);
    f = snap_hash(h->D, sizeof(double) * h->nq * h->nq, f);
    f = snap_hash(h->w, sizeof(double) * h->nq, f);
    f = snap_hash(&h->gamma, sizeof(double), f);
    f = snap_hash(h->adv, sizeof(h->adv), f);
    // a direction subset or boundary conditions change the operator too (hashed only when
    // set, so a default handle's fingerprint does not depend on them)
    if (h->dir_mask) f = snap_hash(&h->dir_mask, sizeof(h->dir_mask), f);
    if (h->has_bc) {
        f = snap_hash(h->bc_kind, sizeof(h->bc_kind), f);
        f = snap_hash(h->bc_state, sizeof(h->bc_state), f);
    }
    return f;
}

static size_t snap_dq_bytes(const rb200_handle* h) {
    return (size_t)h->np * h->ns * h->E * (h->prec == RB200_PRECISION_FP32_BULK ? sizeof(float) : sizeof(double));
}

rb200_status rb200_snapshot_bytes(const rb200_handle* h, size_t* bytes) {
    if (!h || !bytes) return RB200_ERR_BAD_ARG;
    *bytes = sizeof(SnapHeader) + (size_t)h->np * h->ns * h->E * sizeof(double) + snap_dq_bytes(h);
    return RB200_OK;
}

rb200_status rb200_snapshot(rb200_handle* h, const double* q, const void* dq, double time, double dt, double gamma,
                            void* host, size_t bytes, void* stream) {
    if (!h) return RB200_ERR_BAD_ARG;
    size_t need = 0;
    rb200_snapshot_bytes(h, &need);
    const bool fp32 = h->prec == RB200_PRECISION_FP32_BULK;
    if (!q || !host || (!dq && !fp32)) return fail(h, RB200_ERR_BAD_ARG, "null pointer");
    if (bytes < need) return fail(h, RB200_ERR_SHAPE, "snapshot buffer is smaller than rb200_snapshot_bytes");
    DeviceGuard guard(h->device);
    const size_t qb = (size_t)h->np * h->ns * h->E * sizeof(double), db = snap_dq_bytes(h);
    unsigned char* out = static_cast<unsigned char*>(host);
    cudaStream_t s = (cudaStream_t)stream;
    // the FP32-bulk LSRK register is the handle's own (rb200_lsrk54_step ignores dq there)
    const void* dq_src = fp32 ? (const void*)h->d_dq32 : dq;
    cudaError_t e = cudaSuccess;
    if (qb) e = cudaMemcpyAsync(out + sizeof(SnapHeader), q, qb, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && db) e = cudaMemcpyAsync(out + sizeof(SnapHeader) + qb, dq_src, db, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(h, e, "snapshot copy");
    SnapHeader hd;
    std::memset(&hd, 0, sizeof(hd));
    std::memcpy(hd.magic, "RB200SNP", 8);
    hd.version = 1;
    hd.header_bytes = sizeof(SnapHeader);
    hd.dim = h->dim;
    hd.nq = h->nq;
    hd.ns = h->ns;
    hd.law = h->law;
    hd.precision = h->prec;
    hd.combo = h->combo;
    hd.E = h->E;
    hd.q_bytes = qb;
    hd.dq_bytes = db;
    hd.time = time;
    hd.dt = dt;
    hd.gamma = gamma;
    hd.fingerprint = snap_fingerprint(h);
    hd.payload_sum = snap_hash(out + sizeof(SnapHeader), qb + db);
    hd.header_sum = snap_hash(&hd, offsetof(SnapHeader, header_sum));
    std::memcpy(out, &hd, sizeof(hd));
    return RB200_OK;
}

rb200_status rb200_restore(rb200_handle* h, const void* host, size_t bytes, double* q, void* dq, double* time,
                           double* dt, double* gamma, void* stream) {
    if (!h) return RB200_ERR_BAD_ARG;
    const bool fp32 = h->prec == RB200_PRECISION_FP32_BULK;
    if (!host || !q || (!dq && !fp32)) return fail(h, RB200_ERR_BAD_ARG, "null pointer");
    if (bytes < sizeof(SnapHeader)) return fail(h, RB200_ERR_SHAPE, "snapshot is shorter than its header");
    SnapHeader hd;
    std::memcpy(&hd, host, sizeof(hd));
    if (std::memcmp(hd.magic, "RB200SNP", 8) != 0 || hd.version != 1 || hd.header_bytes != sizeof(SnapHeader))
        return fail(h, RB200_ERR_BAD_ARG, "not a snapshot of this format");
    if (hd.header_sum != snap_hash(&hd, offsetof(SnapHeader, header_sum)))
        return fail(h, RB200_ERR_BAD_ARG, "snapshot header checksum mismatch");
    const size_t qb = (size_t)h->np * h->ns * h->E * sizeof(double), db = snap_dq_bytes(h);
    if (hd.fingerprint != snap_fingerprint(h) || hd.q_bytes != qb || hd.dq_bytes != db)
        return fail(h, RB200_ERR_SHAPE, "snapshot was taken with another discretization or precision");
    if (bytes < sizeof(SnapHeader) + qb + db) return fail(h, RB200_ERR_SHAPE, "snapshot is truncated");
    const unsigned char* in = static_cast<const unsigned char*>(host);
    if (hd.payload_sum != snap_hash(in + sizeof(SnapHeader), qb + db))
        return fail(h, RB200_ERR_BAD_ARG, "snapshot payload checksum mismatch");
    DeviceGuard guard(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    void* dq_dst = fp32 ? (void*)h->d_dq32 : dq;
    cudaError_t e = cudaSuccess;
    if (qb) e = cudaMemcpyAsync(q, in + sizeof(SnapHeader), qb, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && db) e = cudaMemcpyAsync(dq_dst, in + sizeof(SnapHeader) + qb, db, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(h, e, "restore copy");
    if (time) *time = hd.time;
    if (dt) *dt = hd.dt;
    if (gamma) *gamma = hd.gamma;
    return RB200_OK;
}

rb200_status rb200_face_vmapP(rb200_handle* h, int64_t* vmapP_out, void* stream) {
    if (!h) return RB200_ERR_BAD_ARG;
    if (!vmapP_out) return fail(h, RB200_ERR_BAD_ARG, "null pointer");
    DeviceGuard guard(h->device);
    cudaError_t e = h->d_vmapP ? launch_copy_vmapP(h->d_vmapP, (int64_t)h->nf * h->nfp * h->E, vmapP_out,
                                                   (cudaStream_t)stream)
                               : launch_face_vmapP(h->d_nbr, h->dim, h->nq, h->E, vmapP_out, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "vmapP kernel launch");
    return RB200_OK;
}

rb200_status rb200_set_mortars(rb200_handle* h, const int64_t* mortars, int64_t num_mortars, const double* IL,
                               const double* IU, const double* PL, const double* PU) {
    if (!h) return RB200_ERR_BAD_ARG;
    if (num_mortars < 0 || (num_mortars > 0 && (!mortars || !IL || !IU || !PL || !PU))) return RB200_ERR_BAD_ARG;
    if (h->nmortars > 0) return fail(h, RB200_ERR_BAD_ARG, "mortars are already set");
    if (num_mortars == 0) return RB200_OK;
    if (h->E_active != h->E) return fail(h, RB200_ERR_UNSUPPORTED, "mortars on a grid with ghost elements");
    if (h->d_vmapP)
        return fail(h, RB200_ERR_UNSUPPORTED, "mortars on a grid with general (rotated) face connectivity");
    const int nf = h->nf, mcols = 2 + (h->dim == 3 ? 4 : 2);
    DeviceGuard guard(h->device);
    std::vector<int32_t> nbr((size_t)nf * h->E);
    cudaError_t ce = cudaMemcpy(nbr.data(), h->d_nbr, nbr.size() * sizeof(int32_t), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return cuda_fail(h, ce, "mortar set-up");
    for (int64_t m = 0; m < num_mortars; ++m) {
        const int64_t* col = mortars + (size_t)mcols * m;
        if (col[0] < 0 || col[0] >= h->E || col[1] < 0 || col[1] >= nf)
            return fail(h, RB200_ERR_BAD_ARG, "mortar: large element or face out of range");
        // a hanging face is unconnected in the face maps (vmapP = vmapM)
        if (nbr[(size_t)nf * col[0] + col[1]] != -1) return fail(h, RB200_ERR_SHAPE, "mortar: the large face is connected");
        nbr[(size_t)nf * col[0] + col[1]] = -2;
        for (int k = 2; k < mcols; ++k) {
            if (col[k] < 0 || col[k] >= h->E) return fail(h, RB200_ERR_BAD_ARG, "mortar: small element out of range");
            int32_t& v = nbr[(size_t)nf * col[k] + (col[1] ^ 1)];
            if (v != -1) return fail(h, RB200_ERR_SHAPE, "mortar: a small face is connected or in two mortars");
            v = -2;
        }
    }
    const size_t nflux = (size_t)nf * h->E * h->ns * h->nfp;
    rb200_status st;
    if ((st = dev_alloc(h, &h->d_mortars, (size_t)mcols * num_mortars)) != RB200_OK) return st;
    if ((st = dev_alloc(h, &h->d_ncflux, nflux)) != RB200_OK) return st;
    ce = cudaMemcpy(h->d_mortars, mortars, (size_t)mcols * num_mortars * sizeof(int64_t), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemset(h->d_ncflux, 0, nflux * sizeof(double));
    if (ce == cudaSuccess) ce = cudaMemcpy(h->d_nbr, nbr.data(), nbr.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) return cuda_fail(h, ce, "mortar upload");
    MortarArgs& a = h->mortar;
    std::memset(&a, 0, sizeof(a));
    a.ncflux = h->d_ncflux;
    a.mortars = h->d_mortars;
    a.M = num_mortars;
    a.surface_rusanov = h->sflux == RB200_FLUX_RUSANOV ? 1 : 0;
    a.surface_flux = h->sflux;
    a.gamma = h->gamma;
    for (int d = 0; d < 3; ++d) a.adv[d] = h->adv[d];
    a.sgeo = h->geom == GEOM_CURVED ? h->d_sgeo : nullptr;
    std::memcpy(a.w, h->w, sizeof(a.w));
    const int q2 = h->nq * h->nq;
    std::memcpy(a.IL, IL, q2 * sizeof(double));
    std::memcpy(a.IU, IU, q2 * sizeof(double));
    std::memcpy(a.PL, PL, q2 * sizeof(double));
    std::memcpy(a.PU, PU, q2 * sizeof(double));
    h->nmortars = num_mortars;
    h->pipe_curved_grid = 0;  // the curved pipelined kernel has no mortar faces
    free_graph(h);
    return RB200_OK;
}

rb200_status rb200_set_kernel_path(rb200_handle* h, int32_t path) {
    if (!h || path < 0 || path > 1) return RB200_ERR_BAD_ARG;
    if (path != h->kernel_path) {
        DeviceGuard guard(h->device);
        free_graph(h);  // a captured step holds the other kernel
    }
    h->kernel_path = path;
    return RB200_OK;
}

rb200_status rb200_set_boundary_condition(rb200_handle* h, int32_t tag, int32_t kind, const double* state) {
    if (!h) return RB200_ERR_BAD_ARG;
    if (tag < 1 || tag > kMaxBcTags) return fail(h, RB200_ERR_BAD_ARG, "boundary tag must be in 1..8");
    if (kind != BC_DEFAULT && kind != BC_PRESCRIBED && kind != BC_WALL)
        return fail(h, RB200_ERR_BAD_ARG, "unknown boundary condition kind");
    if (kind == BC_WALL && h->law != RB200_LAW_EULER)
        return fail(h, RB200_ERR_UNSUPPORTED, "a reflecting wall needs the Euler law");
    if (kind == BC_PRESCRIBED) {
        if (!state) return fail(h, RB200_ERR_BAD_ARG, "null boundary state");
        for (int s = 0; s < h->ns; ++s)
            if (!std::isfinite(state[s])) return fail(h, RB200_ERR_BAD_ARG, "boundary state is not finite");
    }
    DeviceGuard guard(h->device);
    std::vector<int32_t> nbr((size_t)h->nf * h->E);
    cudaError_t ce = cudaMemcpy(nbr.data(), h->d_nbr, nbr.size() * sizeof(int32_t), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return cuda_fail(h, ce, "boundary condition set-up");
    for (size_t k = 0; k < nbr.size(); ++k)
        if (h->bcode[k] == tag) nbr[k] = kind == BC_DEFAULT ? -1 : -(kBcBase + tag);
    ce = cudaMemcpy(h->d_nbr, nbr.data(), nbr.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) return cuda_fail(h, ce, "boundary condition upload");
    h->bc_kind[tag] = kind;
    for (int s = 0; s < 5; ++s) h->bc_state[tag][s] = (kind == BC_PRESCRIBED && s < h->ns) ? state[s] : 0.0;
    h->has_bc = false;
    for (int t = 1; t <= kMaxBcTags; ++t) h->has_bc = h->has_bc || h->bc_kind[t] != BC_DEFAULT;
    free_graph(h);  // a captured step holds the old arguments
    return RB200_OK;
}

rb200_status rb200_set_directions(rb200_handle* h, int32_t mask) {
    if (!h) return RB200_ERR_BAD_ARG;
    const int32_t all = (1 << h->dim) - 1;
    if (mask < 1 || mask > all) return fail(h, RB200_ERR_BAD_ARG, "directions: a non-empty subset of 1:dim");
    const int32_t m = mask == all ? 0 : mask;
    if (m != h->dir_mask) {
        DeviceGuard guard(h->device);
        free_graph(h);  // a captured step holds the old directions
    }
    h->dir_mask = m;
    return RB200_OK;
}

rb200_status rb200_sync_status(rb200_handle* h, void* stream) {
    if (!h) return RB200_ERR_BAD_ARG;
    DeviceGuard guard(h->device);
    int32_t v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, h->d_status, sizeof(v), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "status readback");
    if (v != 0) return fail(h, (rb200_status)v, "a kernel wait exceeded its iteration limit");
    return RB200_OK;
}

rb200_status rb200_get_info(const rb200_handle* h, int64_t* info, int32_t n) {
    if (!h || !info) return RB200_ERR_BAD_ARG;
    const int64_t bytes_q = 8, bytes_dq = h->prec == RB200_PRECISION_FP32_BULK ? 4 : 8;
    int64_t per_node = h->ns * (2 * bytes_q + 2 * bytes_dq);
    if (h->geom == GEOM_CURVED)
        per_node += (h->dim * h->dim + 1) * 8 + (int64_t)h->nf * h->nfp * (h->dim + 1) * 8 / h->np;
    const int64_t v[10] = {h->dim, h->nq, h->ns, h->E, h->geom, h->prec, h->nmortars > 0 ? 10 : 5, per_node,
                           h->dir_mask || h->has_bc ? 0 : (h->geom == GEOM_CURVED ? h->pipe_curved_grid : h->pipe_grid),
                           cluster_ctas(h)};
    for (int i = 0; i < n && i < 10; ++i) info[i] = v[i];
    return RB200_OK;
}

}  // extern "C"
