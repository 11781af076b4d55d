// Serving runtime: continuous batching of independent brick solves.
//
// A server owns one device arena, allocated once.  Submitted solves wait in a FIFO
// queue and are admitted, between ticks, as soon as their HBM footprint fits in the
// arena; a request that does not fit yet lets later ones pass.  Admitted solves keep
// their state, geometry and connectivity resident until they finish.
//
// Solves are grouped into classes of equal (dim, Nq, law, form, precision, physical
// constants).  Each class advances all of its solves one LSRK(5,4) step per tick:
// * the tick is a CUDA graph of five batched stage launches plus a tick counter update,
//   captured once per class and per tile;
// * the launches read a chunk table (solve, first element, count) and the solve
//   descriptors from device memory, so admissions and completions only rewrite those
//   tables;
// * each class has its own stream and advances as soon as its previous tick is done,
//   so the ticks of different classes overlap on the device.
//
// The autotuner times the candidate element-per-CTA tiles of a class over its first
// ticks and keeps the fastest.
//
// A host thread runs the loop, and nothing on the device waits on the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/raven_b200.h"
#include "pipelined_kernel.cuh"
#include "serve_kernel.cuh"

namespace rb200 {
cudaError_t launch_batched_d2(int nq, int combo, int fp32, int tile, const BatchArgs& b, int grid, cudaStream_t s,
                              int* blocks_per_sm);
cudaError_t launch_batched_d3(int nq, int combo, int fp32, int tile, const BatchArgs& b, int grid, cudaStream_t s,
                              int* blocks_per_sm);
int batched_tiles_d2(int nq, int* epb);
int batched_tiles_d3(int nq, int* epb);

__global__ void brick_init_kernel(const __grid_constant__ InitArgs A) {
    const int np = A.dim == 2 ? A.nq * A.nq : A.nq * A.nq * A.nq;
    const int64_t total = A.E * np;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t / np;
        const int n = (int)(t % np);
        const int idx[3] = {n % A.nq, (n / A.nq) % A.nq, n / (A.nq * A.nq)};
        double x[3] = {0, 0, 0};
        for (int d = 0; d < A.dim; ++d) {
            const double c1 = A.corners[(e * A.dim + d) * 2], dx = A.corners[(e * A.dim + d) * 2 + 1];
            x[d] = fma(dx, fma(0.5, A.r[idx[d]] + 1.0, 0.0), c1);
        }
        double* qe = A.q + (size_t)e * A.ns * np + n;
        if (A.kind == 1) {
            const double g = A.gamma, pi = 3.141592653589793;
            const double r0 = x[0] - A.p[2], r1 = x[1] - A.p[3];
            const double f = A.p[0] * exp(1 - (r0 * r0 + r1 * r1));
            const double rho = pow(1 - ((g - 1) * (f * f)) / ((16 * g) * (pi * pi)), 1 / (g - 1));
            const double c = f / (2 * pi);
            const double u[3] = {A.p[1] + c * (-r1), 0.0 + c * r0, 0.0};
            const double pr = pow(rho, g);
            double ke = 0;
            qe[0] = rho;
            for (int d = 0; d < A.dim; ++d) {
                qe[(size_t)(1 + d) * np] = rho * u[d];
                ke += (rho * u[d]) * (rho * u[d]);
            }
            qe[(size_t)(A.dim + 1) * np] = pr / (g - 1) + ke / (2 * rho);
        } else {
            const double pi = 3.141592653589793;
            double sv = 1.0, r2 = 0.0;
            for (int d = 0; d < A.dim; ++d) {
                sv *= sin(2 * pi * x[d]);
                r2 += (x[d] - A.p[1 + d]) * (x[d] - A.p[1 + d]);
            }
            qe[0] = sv + exp(-r2 / (2 * A.p[0] * A.p[0]));
        }
    }
}

__global__ void advance_tick_kernel(int64_t* tick) { *tick += 1; }

}  // namespace rb200

using namespace rb200;

namespace {

// LSRK(5,4) coefficients (coefficients_lsrk54, odesolvers.jl:163-189), the same values
// the DGSEM handle uses.
const double kRKA[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                        -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double kRKB[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                        1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                        2277821191437.0 / 14882151754819.0};

constexpr int kMaxSolvesPerClass = 1024;
constexpr int kMaxChunksPerClass = 1 << 16;
constexpr size_t kAlign = 256;

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

cudaError_t launch_batched(int dim, int nq, int combo, int fp32, int tile, const BatchArgs& b, int grid,
                           cudaStream_t s, int* bps) {
    return dim == 2 ? launch_batched_d2(nq, combo, fp32, tile, b, grid, s, bps)
                    : launch_batched_d3(nq, combo, fp32, tile, b, grid, s, bps);
}

// First-fit allocator over byte offsets of the arena.
class Arena {
   public:
    explicit Arena(size_t size) : size_(size) { free_[0] = size; }
    bool alloc(size_t bytes, size_t* off) {
        bytes = align_up(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                *off = it->first;
                const size_t rest = it->second - bytes;
                const size_t start = it->first + bytes;
                free_.erase(it);
                if (rest) free_[start] = rest;
                used_ += bytes;
                peak_ = std::max(peak_, used_);
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        bytes = align_up(bytes);
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t size() const { return size_; }
    size_t used() const { return used_; }
    size_t peak() const { return peak_; }

   private:
    size_t size_, used_ = 0, peak_ = 0;
    std::map<size_t, size_t> free_;
};

struct Req {
    uint64_t ticket = 0;
    // class fields: the first seven ints and the four doubles form the class key
    int dim = 0, nq = 0, law = 0, form = 0, vflux = 0, sflux = 0, prec = 0;
    int combo = 0, ns = 0, np = 0;
    double gamma = 1.4, adv[3] = {0, 0, 0};
    double D[64] = {0}, w[8] = {0}, r[8] = {0};
    int64_t E = 0;
    std::vector<double> geo, corners;
    std::vector<int32_t> nbr;
    std::vector<double> q0;  // host copy of the initial state (empty: device initial data)
    int init_kind = 0;
    double initp[8] = {0};
    double dt = 0;
    int nsteps = 0;
    double* q_out = nullptr;
    double t_submit = 0, t_admit = 0, t_done = 0;
    int state = 0;  // 0 queued, 1 running, 2 done, 3 failed
    size_t bytes = 0;
    std::string key;
};

struct Solve {
    std::shared_ptr<Req> req;
    size_t off = 0;
    int slot = -1;
    int64_t steps_done = 0;
    SolveDesc desc{};
    const double* final_state = nullptr;  // set when the last step's tick has completed
};

struct Class {
    std::string key;
    int dim = 0, nq = 0, combo = 0, prec = 0, ns = 0, np = 0;
    cudaStream_t stream = nullptr;
    StageArgs base{};
    SolveDesc* d_solves = nullptr;
    Chunk* d_chunks = nullptr;
    int32_t* d_nchunks = nullptr;
    int64_t* d_tick = nullptr;
    std::vector<SolveDesc> h_solves;
    std::vector<Chunk> h_chunks;
    std::vector<Solve*> slots;
    int chunk_elems = 1;
    int nchunks = 0;
    int64_t tick = 0;
    bool dirty = true;
    int ntiles = 0;
    int epb[3] = {1, 1, 1};
    cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
    int tile = 1;
    int tune_done = 0;
    double tune_ms[3] = {0, 0, 0};
    int tune_n[3] = {0, 0, 0};
    int last_tile = 1;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // tick start and end
    // totals of the completed ticks: device time between the tick's events (classes run
    // concurrently, so these overlap across classes) and DOF updates
    int64_t ticks_done = 0;
    double busy_ms = 0.0, dof_updates = 0.0;
    bool pipelined = false;                      // 3-D Nq=4, 6, 8 Euler KG or advection: the pipelined kernel
    int32_t* d_status = nullptr;                 // its bounded waits report here
    int active = 0;
    bool launched = false;
};

}  // namespace

struct rb200_server {
    int device = 0;
    char* arena_base = nullptr;
    std::unique_ptr<Arena> arena;
    cudaStream_t upload = nullptr;
    cudaEvent_t uploaded = nullptr;  // recorded after each admission's uploads
    cudaStream_t download = nullptr;  // copies of finished states to the host
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_drain;
    std::deque<std::shared_ptr<Req>> queue;
    std::unordered_map<uint64_t, std::shared_ptr<Req>> reqs;
    std::map<std::string, std::unique_ptr<Class>> classes;
    std::vector<std::unique_ptr<Solve>> running;
    // finished solves whose state is being copied to the host: they have left their
    // class (no tick reads or writes them) and keep their arena space until the copy ends
    std::deque<std::unique_ptr<Solve>> draining;
    std::thread loop, completer;
    bool stop = false;
    uint64_t next_ticket = 1;
    std::string err;
    rb200_status err_status = RB200_OK;
    // statistics
    double completed = 0, submitted = 0, dof_updates = 0, ticks = 0, first_submit = 0, last_done = 0;
};

namespace {

std::string class_key(const Req& r) {
    std::string k(reinterpret_cast<const char*>(&r.dim), sizeof(int) * 7);
    k.append(reinterpret_cast<const char*>(&r.gamma), sizeof(double) * 4);
    k.append(reinterpret_cast<const char*>(r.D), sizeof(double) * r.nq * r.nq);
    k.append(reinterpret_cast<const char*>(r.w), sizeof(double) * r.nq);
    return k;
}

// Two state buffers, the LSRK register, elem_geo and the neighbour table.
size_t footprint(const Req& r) {
    const size_t nstate = (size_t)r.np * r.ns * r.E;
    const size_t dqb = r.prec == RB200_PRECISION_FP32_BULK ? 4 : 8;
    return 2 * align_up(nstate * 8) + align_up(nstate * dqb) + align_up((size_t)r.E * 4 * 8) +
           align_up((size_t)r.E * 2 * r.dim * 4);
}

// Caller holds s->mu.
rb200_status fail_server(rb200_server* s, rb200_status st, const std::string& msg) {
    s->err = msg;
    s->err_status = st;
    for (auto& kv : s->reqs)
        if (kv.second->state < 2) kv.second->state = 3;
    s->cv_done.notify_all();
    return st;
}

cudaError_t make_class(rb200_server* s, Class& c, const Req& r) {
    c.dim = r.dim;
    c.nq = r.nq;
    c.combo = r.combo;
    c.prec = r.prec;
    c.ns = r.ns;
    c.np = r.np;
    std::memset(&c.base, 0, sizeof(c.base));
    c.base.surface_rusanov = r.sflux == RB200_FLUX_RUSANOV ? 1 : 0;
    c.base.gamma = r.gamma;
    for (int d = 0; d < 3; ++d) c.base.adv[d] = r.adv[d];
    std::memcpy(c.base.D, r.D, sizeof(c.base.D));
    std::memcpy(c.base.w, r.w, sizeof(c.base.w));
    c.h_solves.assign(kMaxSolvesPerClass, SolveDesc{});
    c.h_chunks.assign(kMaxChunksPerClass, Chunk{-1, 0, 0});
    c.slots.assign(kMaxSolvesPerClass, nullptr);
    cudaError_t e = cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&c.d_solves, sizeof(SolveDesc) * kMaxSolvesPerClass);
    if (e == cudaSuccess) e = cudaMalloc(&c.d_chunks, sizeof(Chunk) * kMaxChunksPerClass);
    if (e == cudaSuccess) e = cudaMalloc(&c.d_nchunks, sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&c.d_tick, sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMemsetAsync(c.d_nchunks, 0, sizeof(int32_t), c.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c.d_tick, 0, sizeof(int64_t), c.stream);
    if (e == cudaSuccess) e = cudaMalloc(&c.d_status, sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemsetAsync(c.d_status, 0, sizeof(int32_t), c.stream);
    if (e == cudaSuccess) e = cudaEventCreate(&c.ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&c.ev1);
    if (e != cudaSuccess) return e;
    c.ntiles = c.dim == 2 ? batched_tiles_d2(c.nq, c.epb) : batched_tiles_d3(c.nq, c.epb);
    if (c.ntiles <= 0) return cudaErrorInvalidValue;
    // a chunk is 8 default tiles: a multiple of every candidate tile
    c.chunk_elems = 8 * c.epb[1];
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, s->device);
    c.pipelined = c.dim == 3 && (c.nq == 4 || c.nq == 6 || c.nq == 8) && (c.combo == EUL_KG || c.combo == ADV_WEAK);
    if (c.pipelined) {
        // one configuration (the persistent TMA-pipelined kernel): nothing to tune
        c.ntiles = 1;
        c.tile = 0;
        const int bps = pipelined_batch_blocks_per_sm(c.nq, c.combo, c.prec);
        if (bps <= 0) return cudaErrorInvalidConfiguration;
        PipeArgs pa{};
        pa.status = c.d_status;
        pa.surface_rusanov = c.base.surface_rusanov;
        pa.gamma = c.base.gamma;
        const int q = c.nq;
        for (int a = 0; a < q; ++a)
            for (int id = 0; id < q; ++id)
                pa.S[a * q + id] = c.combo == ADV_WEAK
                                       ? c.base.D[a + q * id] * (c.base.w[a] / c.base.w[id])
                                       : c.base.D[a + q * id] * (c.base.w[a] / c.base.w[id]) - c.base.D[id + q * a];
        for (int i = 0; i < q; ++i) pa.w[i] = c.base.w[i];
        for (int d = 0; d < 3; ++d) pa.adv[d] = c.base.adv[d];
        for (int i = 0; i < 64; ++i) pa.Sf[i] = (float)pa.S[i];
        cudaGraph_t g = nullptr;
        e = cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        for (int st = 0; st < 5 && e == cudaSuccess; ++st) {
            pa.mode = kRKA[st] == 0.0 ? MODE_STAGE_FIRST : MODE_STAGE;
            pa.rka = kRKA[st];
            const PipeBatch b{c.d_solves, c.d_chunks, c.d_nchunks, c.d_tick, st, kRKB[st]};
            e = launch_pipelined_batch(c.nq, c.combo, c.prec, pa, b, bps * nsm, c.stream);
        }
        if (e == cudaSuccess) {
            advance_tick_kernel<<<1, 1, 0, c.stream>>>(c.d_tick);
            e = cudaGetLastError();
        }
        cudaError_t e2 = cudaStreamEndCapture(c.stream, &g);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&c.graph[0], g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) return e;
        return cudaStreamSynchronize(c.stream);
    }
    for (int t = 0; t < c.ntiles; ++t) {
        int bps = 0;
        BatchArgs probe{};
        e = launch_batched(c.dim, c.nq, c.combo, c.prec, t, probe, 0, c.stream, &bps);
        if (e != cudaSuccess) return e;
        const int grid = std::max(1, bps) * nsm;  // fixed persistent grid
        cudaGraph_t g = nullptr;
        e = cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        for (int st = 0; st < 5 && e == cudaSuccess; ++st) {
            BatchArgs b{};
            b.base = c.base;
            b.base.mode = kRKA[st] == 0.0 ? MODE_STAGE_FIRST : MODE_STAGE;
            b.base.rka = kRKA[st];
            b.solves = c.d_solves;
            b.chunks = c.d_chunks;
            b.nchunks = c.d_nchunks;
            b.tick = c.d_tick;
            b.stage = st;
            b.rkb = kRKB[st];
            e = launch_batched(c.dim, c.nq, c.combo, c.prec, t, b, grid, c.stream, nullptr);
        }
        if (e == cudaSuccess) {
            advance_tick_kernel<<<1, 1, 0, c.stream>>>(c.d_tick);
            e = cudaGetLastError();
        }
        cudaError_t e2 = cudaStreamEndCapture(c.stream, &g);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&c.graph[t], g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) return e;
    }
    return cudaStreamSynchronize(c.stream);
}

void destroy_class(Class& c) {
    for (auto& g : c.graph)
        if (g) cudaGraphExecDestroy(g);
    if (c.d_solves) cudaFree(c.d_solves);
    if (c.d_chunks) cudaFree(c.d_chunks);
    if (c.d_nchunks) cudaFree(c.d_nchunks);
    if (c.d_tick) cudaFree(c.d_tick);
    if (c.d_status) cudaFree(c.d_status);
    if (c.ev0) cudaEventDestroy(c.ev0);
    if (c.ev1) cudaEventDestroy(c.ev1);
    if (c.stream) cudaStreamDestroy(c.stream);
}

int chunks_needed(const Class& c, int64_t E) { return (int)((E + c.chunk_elems - 1) / c.chunk_elems); }

// Admits queued requests that fit; caller holds s->mu.
cudaError_t admit(rb200_server* s) {
    for (auto it = s->queue.begin(); it != s->queue.end();) {
        auto r = *it;
        auto cit = s->classes.find(r->key);
        if (cit == s->classes.end()) {
            auto c = std::make_unique<Class>();
            c->key = r->key;
            cudaError_t e = make_class(s, *c, *r);
            if (e != cudaSuccess) {
                destroy_class(*c);
                return e;
            }
            cit = s->classes.emplace(r->key, std::move(c)).first;
        }
        Class& c = *cit->second;
        int slot = -1;
        for (int i = 0; i < kMaxSolvesPerClass; ++i)
            if (!c.slots[i]) {
                slot = i;
                break;
            }
        size_t off = 0;
        if (slot < 0 || c.nchunks + chunks_needed(c, r->E) > kMaxChunksPerClass || !s->arena->alloc(r->bytes, &off)) {
            ++it;  // does not fit now; later requests may
            continue;
        }
        auto sv = std::make_unique<Solve>();
        sv->req = r;
        sv->off = off;
        sv->slot = slot;
        const size_t nstate = (size_t)r->np * r->ns * r->E;
        const size_t dqb = r->prec == RB200_PRECISION_FP32_BULK ? 4 : 8;
        char* base = s->arena_base + off;
        SolveDesc& d = sv->desc;
        d.q[0] = reinterpret_cast<double*>(base);
        d.q[1] = reinterpret_cast<double*>(base + align_up(nstate * 8));
        d.dq = base + 2 * align_up(nstate * 8);
        char* g = base + 2 * align_up(nstate * 8) + align_up(nstate * dqb);
        d.elem_geo = reinterpret_cast<const double*>(g);
        d.nbr = reinterpret_cast<const int32_t*>(g + align_up((size_t)r->E * 4 * 8));
        d.E = r->E;
        d.dt = r->dt;
        d.start_tick = c.tick + (c.launched ? 1 : 0);  // joins at the class's next tick
        cudaError_t e = cudaMemcpyAsync(const_cast<double*>(d.elem_geo), r->geo.data(), r->geo.size() * 8,
                                        cudaMemcpyHostToDevice, s->upload);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(const_cast<int32_t*>(d.nbr), r->nbr.data(), r->nbr.size() * 4, cudaMemcpyHostToDevice,
                                s->upload);
        if (e == cudaSuccess && !r->q0.empty()) {
            e = cudaMemcpyAsync(d.q[0], r->q0.data(), nstate * 8, cudaMemcpyHostToDevice, s->upload);
        } else if (e == cudaSuccess) {
            double* dcorn = d.q[1];  // scratch: q[1] is first written by stage 1
            e = cudaMemcpyAsync(dcorn, r->corners.data(), r->corners.size() * 8, cudaMemcpyHostToDevice, s->upload);
            if (e == cudaSuccess) {
                InitArgs ia{};
                ia.q = d.q[0];
                ia.corners = dcorn;
                ia.E = r->E;
                ia.dim = r->dim;
                ia.nq = r->nq;
                ia.ns = r->ns;
                ia.kind = r->init_kind;
                ia.gamma = r->gamma;
                std::memcpy(ia.r, r->r, sizeof(ia.r));
                std::memcpy(ia.p, r->initp, sizeof(ia.p));
                const int64_t total = r->E * r->np;
                const int blocks = (int)std::min<int64_t>((total + 255) / 256, 4096);
                brick_init_kernel<<<blocks, 256, 0, s->upload>>>(ia);
                e = cudaGetLastError();
            }
        }
        // the class's next tick waits for the uploads on the device; the host does not
        // (pageable sources are staged by the time cudaMemcpyAsync returns)
        if (e == cudaSuccess) e = cudaEventRecord(s->uploaded, s->upload);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c.stream, s->uploaded, 0);
        if (e != cudaSuccess) return e;
        r->geo = std::vector<double>();
        r->nbr = std::vector<int32_t>();
        r->corners = std::vector<double>();
        r->q0 = std::vector<double>();
        r->state = 1;
        r->t_admit = now_s();
        c.slots[slot] = sv.get();
        c.h_solves[slot] = d;
        c.nchunks += chunks_needed(c, r->E);
        c.active += 1;
        c.dirty = true;
        s->running.push_back(std::move(sv));
        it = s->queue.erase(it);
    }
    return cudaSuccess;
}

cudaError_t launch_tick(Class& c) {
    cudaError_t e = cudaSuccess;
    if (c.dirty) {
        int n = 0;
        for (int i = 0; i < kMaxSolvesPerClass; ++i) {
            if (!c.slots[i]) continue;
            const int64_t E = c.h_solves[i].E;
            for (int64_t f = 0; f < E; f += c.chunk_elems)
                c.h_chunks[n++] = Chunk{i, (int32_t)std::min<int64_t>(c.chunk_elems, E - f), f};
        }
        c.nchunks = n;
        e = cudaMemcpyAsync(c.d_solves, c.h_solves.data(), sizeof(SolveDesc) * kMaxSolvesPerClass,
                            cudaMemcpyHostToDevice, c.stream);
        if (e == cudaSuccess && n)
            e = cudaMemcpyAsync(c.d_chunks, c.h_chunks.data(), sizeof(Chunk) * n, cudaMemcpyHostToDevice, c.stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(c.d_nchunks, &c.nchunks, sizeof(int32_t), cudaMemcpyHostToDevice, c.stream);
        if (e != cudaSuccess) return e;
        c.dirty = false;
    }
    // autotuner: the first 2*ntiles ticks cycle through the tiles, then the fastest stays
    const bool tuning = c.tune_done < 2 * c.ntiles;
    c.last_tile = tuning ? c.tune_done % c.ntiles : c.tile;
    e = cudaEventRecord(c.ev0, c.stream);
    if (e == cudaSuccess) e = cudaGraphLaunch(c.graph[c.last_tile], c.stream);
    if (e == cudaSuccess) e = cudaEventRecord(c.ev1, c.stream);  // completion of the tick
    c.launched = e == cudaSuccess;
    return e;
}

// After the class's tick completed on the device: bookkeeping; caller holds s->mu.
cudaError_t finish_tick(rb200_server* s, Class& c) {
    c.launched = false;
    const int64_t done_tick = c.tick;
    float ms = 0;
    cudaEventElapsedTime(&ms, c.ev0, c.ev1);
    int64_t elems = 0;  // elements of the solves the tick advanced
    for (auto* sv : c.slots)
        if (sv && sv->desc.start_tick <= done_tick) elems += sv->desc.E;
    c.ticks_done += 1;
    c.busy_ms += ms;
    c.dof_updates += (double)elems * c.np * c.ns * 5.0;
    if (c.tune_done < 2 * c.ntiles) {
        // normalise by the elements of the tick so that ticks of different batches compare
        c.tune_ms[c.last_tile] += elems > 0 ? ms / (double)elems : ms;
        c.tune_n[c.last_tile] += 1;
        if (++c.tune_done == 2 * c.ntiles) {
            int best = 0;
            for (int t = 1; t < c.ntiles; ++t)
                if (c.tune_ms[t] / c.tune_n[t] < c.tune_ms[best] / c.tune_n[best]) best = t;
            c.tile = best;
        }
    }
    c.tick += 1;
    s->ticks += 1;
    bool status_read = false;
    for (int i = 0; i < kMaxSolvesPerClass; ++i) {
        Solve* sv = c.slots[i];
        if (!sv || sv->desc.start_tick > done_tick) continue;  // admitted while the tick ran
        sv->steps_done += 1;
        Req& r = *sv->req;
        if (sv->steps_done < r.nsteps) continue;
        if (c.pipelined && !status_read) {  // a bounded wait of the pipelined kernel gave up: the result is void
            int32_t status = 0;
            cudaError_t e = cudaMemcpyAsync(&status, c.d_status, sizeof(status), cudaMemcpyDeviceToHost, c.stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);  // the tick has completed: idle stream
            if (e != cudaSuccess) return e;
            if (status != 0) return cudaErrorTimeout;
            status_read = true;
        }
        // the solve leaves its class now (the next tick's chunk table no longer names it)
        // and its final state goes to the completion thread, which copies it to the host
        // while the class's next ticks run
        sv->final_state = sv->desc.q[sv->steps_done & 1];
        c.slots[i] = nullptr;
        c.h_solves[i] = SolveDesc{};
        c.nchunks -= chunks_needed(c, r.E);
        c.active -= 1;
        c.dirty = true;
        auto pos = std::find_if(s->running.begin(), s->running.end(), [&](auto& p) { return p.get() == sv; });
        if (pos != s->running.end()) {
            s->draining.push_back(std::move(*pos));
            s->running.erase(pos);
        }
    }
    s->cv_drain.notify_all();
    return cudaSuccess;
}

// Completion thread: copies each finished solve's state to its host buffer on the
// download stream, outside the server lock, then marks the request done and releases its
// arena space.  Pending copies are finished before the thread exits.
void completion_loop(rb200_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        if (s->draining.empty()) {
            if (s->stop) break;
            s->cv_drain.wait(lk);
            continue;
        }
        std::unique_ptr<Solve> sv = std::move(s->draining.front());
        s->draining.pop_front();
        Req& r = *sv->req;
        const size_t nstate = (size_t)r.np * r.ns * r.E;
        lk.unlock();
        cudaError_t e = cudaSuccess;
        if (r.q_out && r.state < 2) {
            e = cudaMemcpyAsync(r.q_out, sv->final_state, nstate * 8, cudaMemcpyDeviceToHost, s->download);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->download);
        }
        const double t = now_s();
        lk.lock();
        if (e != cudaSuccess) {
            fail_server(s, RB200_ERR_CUDA, std::string("result copy: ") + cudaGetErrorString(e));
        } else if (r.state < 2) {
            r.state = 2;
            r.t_done = t;
            s->completed += 1;
            s->last_done = t;
            s->dof_updates += (double)nstate * 5.0 * r.nsteps;  // one update per RHS evaluation
        }
        s->arena->release(sv->off, r.bytes);
        s->cv_done.notify_all();
        s->cv_work.notify_all();  // arena space for queued requests
    }
}

// Each class advances independently: as soon as a class's tick has completed, its
// bookkeeping runs and its next tick is launched, so small classes are not held back by
// the step time of large ones.
void server_loop(rb200_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        if (s->err_status != RB200_OK) break;
        cudaError_t e = admit(s);
        if (e != cudaSuccess) {
            fail_server(s, RB200_ERR_CUDA, std::string("admission: ") + cudaGetErrorString(e));
            break;
        }
        int in_flight = 0;
        for (auto& kv : s->classes) {
            Class& c = *kv.second;
            if (c.launched) {
                const cudaError_t qe = cudaEventQuery(c.ev1);
                if (qe == cudaErrorNotReady) {
                    ++in_flight;
                    continue;
                }
                if (qe != cudaSuccess) {
                    e = qe;
                    break;
                }
                e = finish_tick(s, c);
                if (e != cudaSuccess) break;
            }
            if (c.active > 0) {
                e = launch_tick(c);
                if (e != cudaSuccess) break;
                ++in_flight;
            }
        }
        if (e == cudaErrorTimeout) {
            fail_server(s, RB200_ERR_TIMEOUT, "a bounded wait of the pipelined stage kernel expired");
            break;
        }
        if (e != cudaSuccess) {
            fail_server(s, RB200_ERR_CUDA, std::string("tick: ") + cudaGetErrorString(e));
            break;
        }
        if (in_flight == 0) {
            if (s->stop && s->queue.empty()) break;
            s->cv_work.wait_for(lk, std::chrono::milliseconds(2));
        } else {
            // the device runs without the lock: submitters and waiters proceed meanwhile
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(20));
            lk.lock();
        }
    }
    // drain: no graph of this server may still run when its memory is freed
    for (auto& kv : s->classes)
        if (kv.second->stream) cudaStreamSynchronize(kv.second->stream);
    if (s->upload) cudaStreamSynchronize(s->upload);
}

}  // namespace

extern "C" {

rb200_status rb200_server_create(int32_t device, uint64_t arena_bytes, rb200_server** out) {
    if (!out || arena_bytes < (1u << 20)) return RB200_ERR_BAD_ARG;
    *out = nullptr;
    auto* s = new (std::nothrow) rb200_server();
    if (!s) return RB200_ERR_OOM;
    s->device = device;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaMalloc(&s->arena_base, arena_bytes);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->upload, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->download, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->uploaded, cudaEventDisableTiming);
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (s->arena_base) cudaFree(s->arena_base);
        delete s;
        return e == cudaErrorMemoryAllocation ? RB200_ERR_OOM : RB200_ERR_CUDA;
    }
    s->arena = std::make_unique<Arena>(arena_bytes);
    s->loop = std::thread(server_loop, s);
    s->completer = std::thread(completion_loop, s);
    *out = s;
    return RB200_OK;
}

rb200_status rb200_server_submit(rb200_server* s, const rb200_request* q, uint64_t* ticket) {
    if (!s || !q || !ticket) return RB200_ERR_BAD_ARG;
    if (q->abi_version != RB200_ABI_VERSION) return RB200_ERR_BAD_ARG;
    auto r = std::make_shared<Req>();
    r->dim = q->dim;
    r->nq = q->nq;
    r->law = q->law;
    r->form = q->volume_form;
    r->vflux = q->volume_flux;
    r->sflux = q->surface_flux;
    r->prec = q->precision;
    r->gamma = q->gamma;
    for (int d = 0; d < 3; ++d) r->adv[d] = q->advection_velocity[d];
    if ((r->dim != 2 && r->dim != 3) || (r->nq != 4 && r->nq != 6 && r->nq != 8)) return RB200_ERR_UNSUPPORTED;
    if (r->prec != RB200_PRECISION_FP64 && r->prec != RB200_PRECISION_FP32_BULK) return RB200_ERR_BAD_ARG;
    if (r->sflux != RB200_FLUX_RUSANOV && r->sflux != RB200_FLUX_CENTRAL) return RB200_ERR_UNSUPPORTED;
    if (r->law == RB200_LAW_ADVECTION && r->form == RB200_FORM_WEAK) {
        r->combo = ADV_WEAK;
        r->ns = 1;
    } else if (r->law == RB200_LAW_EULER && r->form == RB200_FORM_FLUXDIFF &&
               r->vflux == RB200_FLUX_KENNEDY_GRUBER) {
        r->combo = EUL_KG;
        r->ns = r->dim + 2;
        if (!(r->gamma > 1.0)) return RB200_ERR_BAD_ARG;
    } else {
        return RB200_ERR_UNSUPPORTED;  // served classes: advection weak form, Euler KG
    }
    r->np = r->dim == 2 ? r->nq * r->nq : r->nq * r->nq * r->nq;
    r->E = q->num_elements;
    if (r->E <= 0 || r->E > (int64_t)1 << 31 || !q->D || !q->w || !q->elem_geo || !q->neighbors)
        return RB200_ERR_BAD_ARG;
    if (q->nsteps < 1 || !(q->dt > 0)) return RB200_ERR_BAD_ARG;
    if (!q->q0) {
        if (!q->corners || !q->r) return RB200_ERR_BAD_ARG;
        if (q->init_kind == 1 && r->combo != EUL_KG) return RB200_ERR_BAD_ARG;
        if (q->init_kind == 2 && r->combo != ADV_WEAK) return RB200_ERR_BAD_ARG;
        if (q->init_kind != 1 && q->init_kind != 2) return RB200_ERR_BAD_ARG;
    }
    for (int i = 0; i < r->nq * r->nq; ++i) r->D[i] = q->D[i];
    for (int i = 0; i < r->nq; ++i) {
        r->w[i] = q->w[i];
        if (q->r) r->r[i] = q->r[i];
    }
    r->geo.assign(q->elem_geo, q->elem_geo + 4 * r->E);
    r->nbr.assign(q->neighbors, q->neighbors + 2 * r->dim * r->E);
    for (int32_t v : r->nbr)
        if (v < -1 || v >= r->E) return RB200_ERR_BAD_ARG;
    if (q->q0) {
        r->q0.assign(q->q0, q->q0 + (size_t)r->np * r->ns * r->E);
    } else {
        r->corners.assign(q->corners, q->corners + 2 * r->dim * r->E);
    }
    r->init_kind = q->init_kind;
    for (int i = 0; i < 8; ++i) r->initp[i] = q->init_params[i];
    r->dt = q->dt;
    r->nsteps = q->nsteps;
    r->q_out = q->q_out;
    r->bytes = footprint(*r);
    r->key = class_key(*r);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->err_status != RB200_OK) return s->err_status;
    if (r->bytes > s->arena->size()) return RB200_ERR_OOM;  // could never be admitted
    r->ticket = s->next_ticket++;
    r->t_submit = now_s();
    if (s->submitted == 0) s->first_submit = r->t_submit;
    s->submitted += 1;
    s->reqs[r->ticket] = r;
    s->queue.push_back(r);
    *ticket = r->ticket;
    s->cv_work.notify_all();
    return RB200_OK;
}

rb200_status rb200_server_wait(rb200_server* s, uint64_t ticket, double timeout_s, double* latency_s) {
    if (!s) return RB200_ERR_BAD_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return RB200_ERR_BAD_ARG;
    auto r = it->second;
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(std::max(0.0, timeout_s));
    while (r->state < 2) {
        if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && r->state < 2) return RB200_ERR_TIMEOUT;
    }
    if (r->state == 3) return s->err_status != RB200_OK ? s->err_status : RB200_ERR_CUDA;
    if (latency_s) *latency_s = r->t_done - r->t_submit;
    s->reqs.erase(it);
    return RB200_OK;
}

rb200_status rb200_server_stats(rb200_server* s, double* out, int32_t n) {
    if (!s || !out) return RB200_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    double active = 0;
    for (auto& kv : s->classes) active += kv.second->active;
    const double v[9] = {s->completed,
                         s->submitted,
                         active,
                         (double)s->queue.size(),
                         s->dof_updates,
                         (double)s->arena->used(),
                         (double)s->arena->peak(),
                         s->ticks,
                         s->last_done > s->first_submit ? s->last_done - s->first_submit : 0.0};
    for (int i = 0; i < n && i < 9; ++i) out[i] = v[i];
    return s->err_status;
}

rb200_status rb200_server_class_tiles(rb200_server* s, int32_t* out, int32_t n) {
    if (!s || !out) return RB200_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    for (int i = 0; i < n; ++i) out[i] = 0;
    int i = 0;
    for (auto& kv : s->classes) {
        if (i + 4 > n) break;
        const Class& c = *kv.second;
        out[i++] = c.dim;
        out[i++] = c.nq;
        out[i++] = c.combo;
        out[i++] = c.tune_done >= 2 * c.ntiles ? c.epb[c.tile] : 0;
    }
    return RB200_OK;
}

rb200_status rb200_server_class_stats(rb200_server* s, double* out, int32_t n) {
    if (!s || !out) return RB200_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    for (int i = 0; i < n; ++i) out[i] = 0.0;
    int i = 0;
    for (auto& kv : s->classes) {
        if (i + 6 > n) break;
        const Class& c = *kv.second;
        out[i++] = c.dim;
        out[i++] = c.nq;
        out[i++] = c.combo;
        out[i++] = (double)c.ticks_done;
        out[i++] = c.busy_ms;
        out[i++] = c.dof_updates;
    }
    return RB200_OK;
}

const char* rb200_server_last_error(rb200_server* s) {
    if (!s) return "null server";
    std::lock_guard<std::mutex> lk(s->mu);
    return s->err.c_str();
}

rb200_status rb200_server_destroy(rb200_server* s) {
    if (!s) return RB200_ERR_BAD_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        // unfinished work is abandoned
        s->queue.clear();
        for (auto& kv : s->classes) {
            for (auto*& sv : kv.second->slots) sv = nullptr;
            kv.second->active = 0;
        }
        for (auto& kv : s->reqs)
            if (kv.second->state < 2) kv.second->state = 3;
        s->cv_work.notify_all();
        s->cv_done.notify_all();
    }
    if (s->loop.joinable()) s->loop.join();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->cv_drain.notify_all();
    }
    if (s->completer.joinable()) s->completer.join();  // finishes the copies in flight
    cudaSetDevice(s->device);
    for (auto& kv : s->classes) destroy_class(*kv.second);
    if (s->uploaded) cudaEventDestroy(s->uploaded);
    if (s->download) cudaStreamDestroy(s->download);
    if (s->upload) cudaStreamDestroy(s->upload);
    if (s->arena_base) cudaFree(s->arena_base);
    delete s;
    return RB200_OK;
}

}  // extern "C"
