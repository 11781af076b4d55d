// Persistent, TMA-pipelined stage kernel for 3-D hexahedra on unwarped bricks (Nq = 4, 6
// or 8), flux-differencing volume forms (Kennedy-Gruber, entropy conservative).
//
// Each CTA owns a strided set of elements (e = blockIdx.x + k*gridDim.x); three CTAs
// share an SM (Nq = 8).
// * The element's state q arrives by one 1-D bulk copy (cp.async.bulk, completion on an
//   mbarrier) into shared memory.  It is only needed to build the per-node partner
//   values, so right after the first barrier the copy of the CTA's next element is
//   issued into the same buffer and lands while the current element's flux arithmetic
//   runs.
// * The next element's geometry and neighbour ids, the neighbour face traces and (FP32
//   bulk) the element's LSRK register are fetched with cp.async during the volume term.
// * The element's own old q (and the FP64 register) are read with coalesced loads at
//   the end, so that they hold no registers across the flux arithmetic.
//
// A thread owns two nodes of one z line (their eight z-partners are loaded once for
// both), or in FP64 at Nq = 8 four nodes on a 2 x 2 block of y and z lines (each y- and
// z-partner is loaded once for two of them; a quarter of the partner loads saved).  The metric of an unwarped brick is folded into
// a per-element table S_dir[a][id] = drdx_dir * (D[a,id] w_a / w_id - D[id,a]), which
// equals MJI_id * (D[a,id] l_g[a] - D[id,a] l_g[id]) of esvolumeterm_dir!
// (src/balancelaws/dgsem.jl:576-600); S_dir[id][id] = 0, so the z pair of a node with
// itself is skipped.  Face fluxes are applied in the order x-, x+, y-, y+, z-, z+ of
// surfaceterm! (dgsem.jl:756-782) by the owner of each face node.
//
// Every wait on an mbarrier is bounded: after kWaitLimit polls the CTA records
// RB200 status TIMEOUT in *A.status and returns.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rb200_internal.h"
#include "stage_kernel.cuh"  // logavg, Mode

namespace rb200 {

struct PipeArgs {
    const double* q_in;
    double* q_out;
    void* dq;
    const double* elem_geo;  // (4, E)
    const int32_t* nbr;      // (6, E); -2 marks a mortar face of an adapted grid
    const double* ncflux;    // mortar face fluxes ((6, E) faces x (Ns, Nfp)), or null
    int32_t* status;         // device status word (0 = ok)
    int64_t E;        // elements e_begin..E-1 are computed (one state)
    int64_t e_begin;
    int32_t mode;
    int32_t surface_rusanov;
    double rka, rkb_dt, gamma;
    double S[64];  // S[a*Nq + id] = D[a,id] * w[a] / w[id] - D[id,a] (advection: D[a,id] * w[a] / w[id])
    double w[8];
    double adv[3];  // advection velocity (advection law only)
    float Sf[64];   // (float)S, for FP32 arithmetic on table entries at fixed indices
};

// Serving loop: the elements of a launch are the chunks of a class's running solves
// instead of the strided elements of one state (SolveDesc, Chunk: rb200_internal.h).
struct PipeBatch {
    const SolveDesc* solves;
    const Chunk* chunks;
    const int32_t* nchunks;  // chunk slots in use (device)
    const int64_t* tick;     // class tick counter (device)
    int32_t stage;           // 0..4: selects the ping-pong buffer with the tick
    double rkb;              // LSRK b coefficient of the stage (times each solve's dt)
};

// One element as the kernel sees it: its state's buffers and its index there.
struct ElemRef {
    const double* q;     // q_in of the element's state (neighbours are in the same state)
    double* q_out;
    void* dq;
    const double* geo;   // elem_geo of the state
    const int32_t* nbr;  // neighbour table of the state
    int64_t e;           // element index in its state; -1: none (end of the CTA's work)
    double rkb_dt;
};

namespace pipe {

constexpr int NQ = 8, NP = 512, NS = 5, NAUX = 6, NSLOT = 384;  // the Nq = 8 element
constexpr int PAD(int n) { return n + (n >> 3); }  // one vector slot of padding every 8 nodes
constexpr int NPP = PAD(NP);                       // padded plane length

// Sizes of an element with Q nodes per direction (Q even: an element's state is then a
// whole number of 16-byte units, as the bulk copies need).
template <int Q>
struct Geo {
    static_assert(Q % 2 == 0 && Q >= 4 && Q <= 8, "Nq = 4, 6 or 8");
    static constexpr int NQ = Q, NP = Q * Q * Q, NFP = Q * Q, NSLOT = 6 * Q * Q, NPP = PAD(Q * Q * Q);
};
constexpr long kWaitLimit = 1L << 26;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Per-node partner values (6 per node), read as vectors: three 16-byte loads in FP64, one
// 16-byte and one 8-byte load in FP32.
template <typename T, int NPP_ = NPP>
struct AuxBuf;
template <int NPP_>
struct AuxBuf<double, NPP_> {
    double2 v[NAUX / 2][NPP_];
    __device__ __forceinline__ void put(int i, const double (&o)[NAUX]) {
#pragma unroll
        for (int c = 0; c < NAUX / 2; ++c) v[c][i] = make_double2(o[2 * c], o[2 * c + 1]);
    }
    __device__ __forceinline__ void get(int i, double (&o)[NAUX]) const {
#pragma unroll
        for (int c = 0; c < NAUX / 2; ++c) {
            const double2 x = v[c][i];
            o[2 * c] = x.x;
            o[2 * c + 1] = x.y;
        }
    }
};
template <int NPP_>
struct AuxBuf<float, NPP_> {
    float4 a[NPP_];
    float2 b[NPP_];
    __device__ __forceinline__ void put(int i, const float (&o)[NAUX]) {
        a[i] = make_float4(o[0], o[1], o[2], o[3]);
        b[i] = make_float2(o[4], o[5]);
    }
    __device__ __forceinline__ void get(int i, float (&o)[NAUX]) const {
        const float4 x = a[i];
        const float2 y = b[i];
        o[0] = x.x;
        o[1] = x.y;
        o[2] = x.z;
        o[3] = x.w;
        o[4] = y.x;
        o[5] = y.y;
    }
};

template <typename T, int Q = 8>
struct Smem {
    using G = Geo<Q>;
    double q[NS][G::NP];                        // state of the element (TMA destination)
    AuxBuf<T, G::NPP> aux;                      // per-node partner values
    double slot[NS][G::NSLOT];                  // neighbour trace, then (wsJ * nf) * MJI, per face slot
    T S[3][Q][Q];                               // S_dir[a][id] * drdx_dir of the current element
    // FP32 LSRK register of the element, staged during the volume term.  FP64 reads its
    // register at the end instead: staging the state or the register in shared memory (by
    // cp.async or bulk copies, with bulk stores of the results) measured slower, because the
    // stage is bound by shared-memory bandwidth (the partner loads of the volume term)
    __align__(16) T dqs[sizeof(T) == 4 ? NS : 1][sizeof(T) == 4 ? G::NP : 1];
    T rs[3][Q];                                 // sum_a S[dir][a][id]
    double geo[2][4];                           // elem_geo of the current / next element
    int32_t nb[2][8];                           // neighbours of the current / next element
    ElemRef ref[2];                             // the current / next element
    uint64_t bar;
};

__device__ __forceinline__ bool bounded_wait(uint64_t* bar, uint32_t parity) {
    long it = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++it > kWaitLimit) return false;
    }
    return true;
}

// 0-based volume node of face slot `slot` (faces x-, x+, y-, y+, z-, z+; Q*Q slots each)
// and the node of the opposite face with the same in-face index.
template <int Q = 8>
__device__ __forceinline__ void slot_nodes(int slot, int& vn, int& opp) {
    const int f = slot / (Q * Q), jf = slot % (Q * Q);
    const int dir = f >> 1, side = f & 1;
    const int j1 = jf % Q, j2 = jf / Q, c = side ? Q - 1 : 0;
    if (dir == 0) {
        vn = c + Q * (j1 + Q * j2);
        opp = (Q - 1 - c) + Q * (j1 + Q * j2);
    } else if (dir == 1) {
        vn = j1 + Q * (c + Q * j2);
        opp = j1 + Q * ((Q - 1 - c) + Q * j2);
    } else {
        vn = j1 + Q * (j2 + Q * c);
        opp = j1 + Q * (j2 + Q * (Q - 1 - c));
    }
}

// The CTA's sequence of elements, advanced by thread 0 one element ahead of the work.
// One state: elements blockIdx.x + k*gridDim.x.  Serving batch: the elements of chunks
// blockIdx.x + k*gridDim.x, in order.
template <bool BATCH>
struct Cursor {
    int64_t e = 0;  // one state: element; batch: index within the chunk
    int ci = 0;     // batch: chunk slot
    int nch = 0;    // batch: chunk slots in use

    __device__ bool start(const PipeArgs& A, const PipeBatch& B) {
        if constexpr (!BATCH) {
            e = A.e_begin + blockIdx.x;
            return e < A.E;
        } else {
            nch = *B.nchunks;
            ci = blockIdx.x;
            e = 0;
            return skip_empty(B);
        }
    }
    __device__ bool advance(const PipeArgs& A, const PipeBatch& B) {
        if constexpr (!BATCH) {
            e += gridDim.x;
            return e < A.E;
        } else {
            if (++e < B.chunks[ci].count) return true;
            ci += gridDim.x;
            e = 0;
            return skip_empty(B);
        }
    }
    __device__ bool skip_empty(const PipeBatch& B) {
        while (ci < nch && (B.chunks[ci].solve < 0 || B.chunks[ci].count <= 0)) ci += gridDim.x;
        return ci < nch;
    }
    __device__ void resolve(const PipeArgs& A, const PipeBatch& B, ElemRef& r) const {
        if constexpr (!BATCH) {
            r = ElemRef{A.q_in, A.q_out, A.dq, A.elem_geo, A.nbr, e, A.rkb_dt};
        } else {
            const Chunk c = B.chunks[ci];
            const SolveDesc& sd = B.solves[c.solve];
            const int par = (int)((*B.tick - sd.start_tick + B.stage) & 1);
            r = ElemRef{sd.q[par], sd.q[par ^ 1], sd.dq, sd.elem_geo, sd.nbr, c.first + e, B.rkb * sd.dt};
        }
    }
};

// Threads 0..9: one value each of the geometry (4) and neighbour ids (6) of element r
// into a shared slot (cp.async).
__device__ __forceinline__ void fetch_part(const ElemRef& r, int t, double (&geo)[4], int32_t (&nb)[8]) {
    if (t < 4) cp_async8(&geo[t], r.geo + 4 * r.e + t);
    else cp_async4(&nb[t - 4], r.nbr + 6 * r.e + (t - 4));
}

}  // namespace pipe

// CTAs per SM the register allocation is sized for.  Nq = 8: 3 for FP64 (128 threads of
// 168 registers), 3 for FP32 bulk (256 threads of 80).  Smaller elements have fewer
// threads a CTA, so more CTAs share an SM at about the same registers a thread.
#ifndef RB200_PIPE_MIN6
#define RB200_PIPE_MIN6 4, 6
#endif
#ifndef RB200_PIPE_MIN4
#define RB200_PIPE_MIN4 14, 20
#endif
#ifndef RB200_PIPE_MIN8_FP64
#define RB200_PIPE_MIN8_FP64 3
#endif
#ifndef RB200_PIPE_MIN8_FP32
#define RB200_PIPE_MIN8_FP32 3
#endif
// unroll factor of the pair loop over partners (8: fully unrolled)
#ifndef RB200_PIPE_UNROLL_A
#define RB200_PIPE_UNROLL_A 8
#endif
template <typename T, int Q = 8>
constexpr int pipe_min_ctas() {
    constexpr int m8[2] = {RB200_PIPE_MIN8_FP64, RB200_PIPE_MIN8_FP32}, m6[2] = {RB200_PIPE_MIN6}, m4[2] = {RB200_PIPE_MIN4};
    return Q == 8 ? m8[sizeof(T) == 4] : Q == 6 ? m6[sizeof(T) == 4] : m4[sizeof(T) == 4];
}

// Nodes per thread of the kernel: 4 (the 2 x 2 (y, z) block) in FP64 at Nq = 8, else 2.
template <typename T, int Q>
constexpr int pipe_npt() {
    return (sizeof(T) == 8 && Q == 8) ? 4 : 2;
}

// NPT nodes per thread, with i = t mod Nq:
// * NPT = 2: (i, j, k0) and (i, j, k0 + Nq/2), j = (t / Nq) mod Nq, k0 = t / Nq^2 — one z
//   line, so their z-partners are loaded once;
// * NPT = 4: (i, j0 + Nq/2 hj, k0 + Nq/2 hk), hj, hk in {0, 1}, j0 = (t / Nq) mod Nq/2,
//   k0 = t / (Nq^2/2) — two y lines and two z lines, so each y- and z-partner serves two
//   nodes.  A quarter-warp still spans an x line (x partners: one address a quarter), and
//   k0 is the same across a warp (the z pair of a node with itself is skipped uniformly).
template <int COMBO, typename T, int NPT, bool BATCH, int Q = 8>
__global__ void __launch_bounds__(Q * Q * Q / NPT, (pipe_min_ctas<T, Q>()))
    pipelined_stage_kernel(const __grid_constant__ PipeArgs A, const __grid_constant__ PipeBatch B) {
    using namespace pipe;
    using G = Geo<Q>;
    constexpr int NQ = Q, NP = G::NP, NFP = G::NFP, NSLOT = G::NSLOT;
    static_assert(NPT == 2 || NPT == 4, "a z pair or a 2 x 2 (y, z) block");
    constexpr bool YZ = NPT == 4;
    constexpr int NT = NP / NPT, H = Q / 2;
    extern __shared__ __align__(128) unsigned char pipe_smem_raw[];
    Smem<T, Q>& sm = *reinterpret_cast<Smem<T, Q>*>(pipe_smem_raw);
    const int t = threadIdx.x;
    const int ii = t % Q;
    const int jj = YZ ? (t / Q) % H : (t / Q) % Q;
    const int k0 = YZ ? t / (Q * H) : t / (Q * Q);
    // coordinates and index of the thread's node h
    auto jj_of = [&](int h) { return YZ ? jj + H * (h & 1) : jj; };
    auto kk_of = [&](int h) { return YZ ? k0 + H * (h >> 1) : k0 + H * h; };
    auto node_of = [&](int h) { return YZ ? ii + Q * (jj_of(h) + Q * kk_of(h)) : t + NT * h; };
    const bool stage = A.mode >= MODE_STAGE;
    const bool dq_is_f32 = stage && sizeof(T) == 4;
    constexpr bool kStageDq = sizeof(T) == 4;
    const uint32_t qbytes = NS * NP * sizeof(double);
    const T gm1 = (T)(A.gamma - 1.0), gam = (T)A.gamma;

    Cursor<BATCH> cur;  // meaningful in threads 0..9
    if (t == 0) {
        mbar_init(&sm.bar, 1);
        fence_mbar_init();
    }
    if (t < 10) {
        ElemRef r{};
        r.e = -1;
        if (cur.start(A, B)) cur.resolve(A, B, r);
        if (t == 0) sm.ref[0] = r;
        if (r.e >= 0) fetch_part(r, t, sm.geo[0], sm.nb[0]);  // geometry: written by no kernel
    }
    // the previous kernel of the stream (the last stage, or this stage's mortar fluxes)
    // has completed before any state, register or mortar flux is read or written
    grid_dependency_wait();
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();

    if (t == 0 && sm.ref[0].e >= 0) {
        mbar_expect_tx(&sm.bar, qbytes);
        bulk_g2s(&sm.q[0][0], sm.ref[0].q + (size_t)sm.ref[0].e * NS * NP, qbytes, &sm.bar);
    }
    uint32_t phase = 0;
    int64_t es = A.e_begin + blockIdx.x;  // one state: the current element, kept in registers
    for (int buf = 0;; buf ^= 1, es += gridDim.x) {
        const int64_t e = BATCH ? sm.ref[buf].e : (es < A.E ? es : -1);
        if (e < 0) break;
        const double drdx[3] = {sm.geo[buf][0], sm.geo[buf][1], sm.geo[buf][2]};
        for (int q = t; q < 3 * Q * Q; q += NT) {
            const int dir = q / (Q * Q), a = (q / Q) % Q, id = q % Q;
            const double dd = dir == 0 ? drdx[0] : (dir == 1 ? drdx[1] : drdx[2]);
            sm.S[dir][a][id] = (T)(A.S[a * Q + id] * dd);
        }
        if constexpr (COMBO == EUL_KG) {
            for (int q = t; q < 3 * Q; q += NT) {
                const int dir = q / Q, id = q % Q;
                const double dd = dir == 0 ? drdx[0] : (dir == 1 ? drdx[1] : drdx[2]);
                T r = T(0);
#pragma unroll
                for (int a = 0; a < NQ; ++a) r += (T)(A.S[a * Q + id] * dd);
                sm.rs[dir][id] = r;
            }
        }
        // ---- this element's state
        if (__syncthreads_or(!bounded_wait(&sm.bar, phase))) {
            if (t == 0) atomicExch(A.status, kStatusTimeout);
            return;
        }
        phase ^= 1;
        // ---- per-node partner values
        T own[NPT][NAUX];
#pragma unroll
        for (int h = 0; h < NPT; ++h) {
            const int n = node_of(h);
            const T rho = (T)sm.q[0][n];
            const T rinv = T(1) / rho;
            const T m0 = (T)sm.q[1][n], m1 = (T)sm.q[2][n], m2 = (T)sm.q[3][n];
            const T u0 = m0 * rinv, u1 = m1 * rinv, u2 = m2 * rinv;
            const T rhoe = (T)sm.q[4][n];
            const T p = gm1 * (rhoe - (m0 * m0 + m1 * m1 + m2 * m2) * (T(0.5) * rinv));
            if constexpr (COMBO == EUL_KG) {
                own[h][0] = rho * T(0.5);
                own[h][1] = u0 * T(0.5);
                own[h][2] = u1 * T(0.5);
                own[h][3] = u2 * T(0.5);
                own[h][4] = rhoe * rinv * T(0.5);
                own[h][5] = p * T(0.5);
            } else {  // EUL_EC: rho, u, b = rho/(2p), |u|^2
                own[h][0] = rho;
                own[h][1] = u0;
                own[h][2] = u1;
                own[h][3] = u2;
                own[h][4] = rho / (T(2) * p);
                own[h][5] = u0 * u0 + u1 * u1 + u2 * u2;
            }
            sm.aux.put(PAD(n), own[h]);
        }
        __syncthreads();  // #1: aux and S ready; q and the slot buffer are free
        if (t < 10) {  // the next element: its state by TMA, its geometry and neighbours with the traces
            ElemRef rn{};
            rn.e = -1;
            if (cur.advance(A, B)) cur.resolve(A, B, rn);
            if (t == 0) {
                sm.ref[buf ^ 1] = rn;
                if (rn.e >= 0) {
                    fence_proxy_async();
                    mbar_expect_tx(&sm.bar, qbytes);
                    bulk_g2s(&sm.q[0][0], rn.q + (size_t)rn.e * NS * NP, qbytes, &sm.bar);
                }
            }
            if (rn.e >= 0) fetch_part(rn, t, sm.geo[buf ^ 1], sm.nb[buf ^ 1]);
        }
        // the element's state buffers (one state: the kernel parameters)
        const double* const qin_e = BATCH ? sm.ref[buf].q : A.q_in;
        void* const dq_e = BATCH ? sm.ref[buf].dq : A.dq;
        // neighbour traces of this thread's face slots t + NT * sl
#pragma unroll
        for (int sl = 0; sl < (NSLOT + NT - 1) / NT; ++sl) {
            const int slot = t + NT * sl;
            if (slot >= NSLOT) continue;
            int vn, opp;
            slot_nodes<Q>(slot, vn, opp);
            const int ne = sm.nb[buf][slot / NFP];
            if (ne >= 0) {
                const double* qn = qin_e + (size_t)ne * NS * NP + opp;
#pragma unroll
                for (int s = 0; s < NS; ++s) cp_async8(&sm.slot[s][slot], qn + s * NP);
            }
        }
        if (kStageDq && A.mode == MODE_STAGE) {  // the element's FP32 register, for the end of the stage
            const char* src = reinterpret_cast<const char*>(dq_e) + (size_t)e * NS * NP * sizeof(T);
            char* dst = reinterpret_cast<char*>(&sm.dqs[0][0]);
            for (int c = t; c < NS * NP * (int)sizeof(T) / 16; c += NT) cp_async16(dst + 16 * c, src + 16 * c);
        }
        cp_async_commit();

        // ---- volume term (ordered pairs along x, y, z)
        T acc[NPT][NS], accu[NPT];
#pragma unroll
        for (int h = 0; h < NPT; ++h) {
            accu[h] = T(0);
#pragma unroll
            for (int s = 0; s < NS; ++s) acc[h][s] = T(0);
        }

        // KG with the own-node parts of the averages factored out of the sums:
        //   sum F (o_k + p_k) = o_k sum F + sum F p_k, F = rho_avg * u_avg,dir * S,
        //   sum S (o_5 + p_5) = o_5 rs_dir + sum S p_5,
        //   sum U (rho_avg (o_4 + p_4) + o_5 + p_5) = o_4 sum F + o_5 sum U + sum (F p_4 + U p_5)
        // (o, p: halves of the own and partner rho, u, e, p); the own parts are added after
        // the pair loop.
        auto pair = [&](T (&ac)[NS], T& au, const T (&o)[NAUX], const T (&pv)[NAUX], const T sc, const int dir) {
            if constexpr (COMBO == EUL_KG) {
                const T rb = o[0] + pv[0];
                const T un = (dir == 0 ? o[1] + pv[1] : dir == 1 ? o[2] + pv[2] : o[3] + pv[3]) * sc;
                const T f1 = rb * un;
                ac[0] += f1;
                au += un;
                ac[1] = fma(f1, pv[1], ac[1]);
                ac[2] = fma(f1, pv[2], ac[2]);
                ac[3] = fma(f1, pv[3], ac[3]);
                ac[1 + dir] = fma(pv[5], sc, ac[1 + dir]);
                ac[4] = fma(f1, pv[4], ac[4]);
                ac[4] = fma(un, pv[5], ac[4]);
            } else {
                const T ua0 = (o[1] + pv[1]) * T(0.5), ua1 = (o[2] + pv[2]) * T(0.5), ua2 = (o[3] + pv[3]) * T(0.5);
                const T ra = (o[0] + pv[0]) * T(0.5);
                const T ba = (o[4] + pv[4]) * T(0.5);
                const T u2a = (o[5] + pv[5]) * T(0.5);
                const T rlog = logavg(o[0], pv[0]);
                const T blog = logavg(o[4], pv[4]);
                const T pt = ra / (T(2) * ba);
                const T cc = T(1) / ((T(2) * gm1) * blog) - u2a * T(0.5);
                const T un = (dir == 0 ? ua0 : dir == 1 ? ua1 : ua2) * sc;
                const T uaa = ua0 * ua0 + ua1 * ua1 + ua2 * ua2;
                const T f0 = rlog * un;
                ac[0] += f0;
                ac[1] = fma(f0, ua0, ac[1]);
                ac[2] = fma(f0, ua1, ac[2]);
                ac[3] = fma(f0, ua2, ac[3]);
                ac[1 + dir] = fma(pt, sc, ac[1 + dir]);
                ac[4] = fma(un, cc * rlog + rlog * uaa + pt, ac[4]);
            }
        };
        auto load_aux = [&](T (&pv)[NAUX], const int n) { sm.aux.get(PAD(n), pv); };
        constexpr int kUnrA = RB200_PIPE_UNROLL_A < NQ ? RB200_PIPE_UNROLL_A : NQ;
#pragma unroll kUnrA
        for (int a = 0; a < NQ; ++a) {
            const T sx = sm.S[0][a][ii];
            if constexpr (YZ) {
#pragma unroll
                for (int h = 0; h < NPT; ++h) {
                    T pv[NAUX];
                    load_aux(pv, a + Q * (jj_of(h) + Q * kk_of(h)));
                    pair(acc[h], accu[h], own[h], pv, sx, 0);
                }
#pragma unroll
                for (int hk = 0; hk < 2; ++hk) {  // y-partner (ii, a, kk): nodes 2hk, 2hk+1
                    T pv[NAUX];
                    load_aux(pv, ii + Q * (a + Q * kk_of(2 * hk)));
#pragma unroll
                    for (int hj = 0; hj < 2; ++hj) {
                        const int h = 2 * hk + hj;
                        pair(acc[h], accu[h], own[h], pv, sm.S[1][a][jj_of(h)], 1);
                    }
                }
#pragma unroll
                for (int hj = 0; hj < 2; ++hj) {  // z-partner (ii, jj, a): nodes hj, hj+2
                    T pv[NAUX];
                    load_aux(pv, ii + Q * (jj_of(hj) + Q * a));
#pragma unroll
                    for (int hk = 0; hk < 2; ++hk) {
                        const int h = 2 * hk + hj;
                        if (a != kk_of(h)) pair(acc[h], accu[h], own[h], pv, sm.S[2][a][kk_of(h)], 2);  // S_aa = 0
                    }
                }
            } else {
                const T sy = sm.S[1][a][jj];
#pragma unroll
                for (int h = 0; h < NPT; ++h) {
                    const int kk = kk_of(h);
                    T pv[NAUX];
                    load_aux(pv, a + Q * (jj + Q * kk));
                    pair(acc[h], accu[h], own[h], pv, sx, 0);
                    load_aux(pv, ii + Q * (a + Q * kk));
                    pair(acc[h], accu[h], own[h], pv, sy, 1);
                }
                T pv[NAUX];
                load_aux(pv, ii + Q * (jj + Q * a));
#pragma unroll
                for (int h = 0; h < NPT; ++h)
                    if (a != kk_of(h)) pair(acc[h], accu[h], own[h], pv, sm.S[2][a][kk_of(h)], 2);  // S_aa = 0
            }
        }

        if constexpr (COMBO == EUL_KG) {
#pragma unroll
            for (int h = 0; h < NPT; ++h) {
                const int kk = kk_of(h), jh = jj_of(h);
                if constexpr (sizeof(T) == 4) {
                    // FP32: e/2 and p/2 of the own node again from shared memory: they are not
                    // used in the pair loop and would hold registers across it (80 a thread)
                    T ov[NAUX];
                    load_aux(ov, node_of(h));
                    own[h][4] = ov[4];
                    own[h][5] = ov[5];
                }
                const T o5 = own[h][5];
                acc[h][1] = fma(own[h][1], acc[h][0], acc[h][1]);
                acc[h][2] = fma(own[h][2], acc[h][0], acc[h][2]);
                acc[h][3] = fma(own[h][3], acc[h][0], acc[h][3]);
                acc[h][1] = fma(o5, sm.rs[0][ii], acc[h][1]);
                acc[h][2] = fma(o5, sm.rs[1][jh], acc[h][2]);
                acc[h][3] = fma(o5, sm.rs[2][kk], acc[h][3]);
                acc[h][4] = fma(own[h][4], acc[h][0], fma(o5, accu[h], acc[h][4]));
            }
        }
        // ---- face-slot contributions (wsJ * nf) * MJI, written over the slot's trace
        cp_async_wait_all();
#pragma unroll
        for (int sl = 0; sl < (NSLOT + NT - 1) / NT; ++sl) {
            const int slot = t + NT * sl;
            if (slot >= NSLOT) continue;
            const int f = slot / NFP, dir = f >> 1, side = f & 1;
            int vn, opp;
            slot_nodes<Q>(slot, vn, opp);
            const int nbf = sm.nb[buf][f];
            const bool open_face = nbf >= 0;
            if (nbf == -2) {  // mortar face: its flux comes from the mortar kernel
                const T fsc = (T)(fabs(dir == 0 ? drdx[0] : (dir == 1 ? drdx[1] : drdx[2])) / A.w[0]);
                const double* nfp = A.ncflux + (((size_t)e * 6 + f) * NS) * NFP + (slot - f * NFP);
#pragma unroll
                for (int s = 0; s < NS; ++s) sm.slot[s][slot] = (double)((T)nfp[s * NFP] * fsc);
                continue;
            }
            if constexpr (sizeof(T) == 4) {
                // FP32: fluxes field by field from the two sides' primitives, so that no flux
                // arrays stay live beside the accumulators (80 registers, no spills)
            // q- and its primitives from the staged partner values of the element
            T rm, um0, um1, um2, pm, Em;
            {
                T v[NAUX];
                sm.aux.get(PAD(vn), v);
                if constexpr (COMBO == EUL_KG) {
                    rm = T(2) * v[0];
                    um0 = T(2) * v[1];
                    um1 = T(2) * v[2];
                    um2 = T(2) * v[3];
                    pm = T(2) * v[5];
                    Em = rm * (T(2) * v[4]);
                } else {
                    rm = v[0];
                    um0 = v[1];
                    um1 = v[2];
                    um2 = v[3];
                    pm = rm / (T(2) * v[4]);
                    Em = pm / gm1 + T(0.5) * rm * v[5];
                }
            }
            const T sn = side ? T(1) : T(-1);
            const T udm = dir == 0 ? um0 : dir == 1 ? um1 : um2;
            // wave speeds |u.n| + sqrt(gamma p / rho) of both sides (euler.jl:62-68)
            const T wsm = fabs(udm * sn) + sqrt(gam * pm * (T(1) / rm));
            // q+: the neighbour's trace, or q- itself on a boundary face (balancelaw.jl:77)
            T rp = rm, mp0 = rm * um0, mp1 = rm * um1, mp2 = rm * um2, Ep = Em;
            T up0 = um0, up1 = um1, up2 = um2, pp = pm, wsp = wsm;
            if (open_face) {
                rp = (T)sm.slot[0][slot];
                mp0 = (T)sm.slot[1][slot];
                mp1 = (T)sm.slot[2][slot];
                mp2 = (T)sm.slot[3][slot];
                Ep = (T)sm.slot[4][slot];
                const T rinv = T(1) / rp;
                up0 = mp0 * rinv;
                up1 = mp1 * rinv;
                up2 = mp2 * rinv;
                pp = gm1 * (Ep - (mp0 * mp0 + mp1 * mp1 + mp2 * mp2) * (T(0.5) * rinv));
                wsp = fabs((dir == 0 ? up0 : dir == 1 ? up1 : up2) * sn) + sqrt(gam * pp * rinv);
            }
            const T mx = fmax(wsm, wsp);
            // (wsJ * MJI) of a face node of an unwarped brick: wsJ = |J drdx| w_a w_b and
            // MJI = 1 / (w_i w_j w_k J) leave |drdx_dir| / w_end (w_end = w_0 = w_N)
            const T fsc = (T)(fabs(dir == 0 ? drdx[0] : (dir == 1 ? drdx[1] : drdx[2])) / A.w[0]);
            // normal fluxes of both sides (euler.jl:50-60 with n = sn e_dir), field by field,
            // so that no flux arrays stay live next to the volume accumulators
            const T mnm = (rm * udm) * sn, mnp = (dir == 0 ? mp0 : dir == 1 ? mp1 : mp2) * sn;
            const T unm = udm * sn, unp = (dir == 0 ? up0 : dir == 1 ? up1 : up2) * sn;
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                T fm, fp, qms, qps;
                if (s == 0) {
                    fm = mnm;
                    fp = mnp;
                    qms = rm;
                    qps = rp;
                } else if (s == 4) {
                    fm = unm * (Em + pm);
                    fp = unp * (Ep + pp);
                    qms = Em;
                    qps = Ep;
                } else {
                    const T am = s == 1 ? um0 : s == 2 ? um1 : um2, ap = s == 1 ? up0 : s == 2 ? up1 : up2;
                    fm = mnm * am + (dir == s - 1 ? pm * sn : T(0));
                    fp = mnp * ap + (dir == s - 1 ? pp * sn : T(0));
                    qms = rm * am;
                    qps = s == 1 ? mp0 : s == 2 ? mp1 : mp2;
                }
                const T fc = (fm + fp) * T(0.5);
                const T nf = A.surface_rusanov ? fc - (mx * (qps - qms)) * T(0.5) : fc;
                sm.slot[s][slot] = (double)(nf * fsc);
            }
            } else {
            // q- and its primitives from the staged partner values of the element
            T qm[NS], u0, u1, u2, p, rinv;
            {
                T v[NAUX];
                sm.aux.get(PAD(vn), v);
                if constexpr (COMBO == EUL_KG) {
                    const T rho = T(2) * v[0];
                    u0 = T(2) * v[1];
                    u1 = T(2) * v[2];
                    u2 = T(2) * v[3];
                    p = T(2) * v[5];
                    rinv = T(1) / rho;
                    qm[0] = rho;
                    qm[4] = rho * (T(2) * v[4]);
                } else {
                    const T rho = v[0];
                    u0 = v[1];
                    u1 = v[2];
                    u2 = v[3];
                    p = rho / (T(2) * v[4]);
                    rinv = T(1) / rho;
                    qm[0] = rho;
                    qm[4] = p / gm1 + T(0.5) * rho * v[5];
                }
                qm[1] = qm[0] * u0;
                qm[2] = qm[0] * u1;
                qm[3] = qm[0] * u2;
            }
            const T sn = side ? T(1) : T(-1);
            T Fn[2][NS], ws[2];
            // normal flux and wave speed of one side (euler.jl:50-68 with n = sn e_dir)
            auto side_flux = [&](const T (&qq)[NS], const T a0, const T a1, const T a2, const T pp, const T ri,
                                 T (&F)[NS], T& w) {
                const T ud = dir == 0 ? a0 : dir == 1 ? a1 : a2;
                const T un = ud * sn;
                const T mn = (dir == 0 ? qq[1] : dir == 1 ? qq[2] : qq[3]) * sn;
                F[0] = mn;
                F[1] = mn * a0 + (dir == 0 ? pp * sn : T(0));
                F[2] = mn * a1 + (dir == 1 ? pp * sn : T(0));
                F[3] = mn * a2 + (dir == 2 ? pp * sn : T(0));
                F[4] = un * (qq[4] + pp);
                w = fabs(un) + sqrt(gam * pp * ri);
            };
            side_flux(qm, u0, u1, u2, p, rinv, Fn[0], ws[0]);
            T qp[NS];
            if (open_face) {
#pragma unroll
                for (int s = 0; s < NS; ++s) qp[s] = (T)sm.slot[s][slot];
                rinv = T(1) / qp[0];
                u0 = qp[1] * rinv;
                u1 = qp[2] * rinv;
                u2 = qp[3] * rinv;
                p = gm1 * (qp[4] - (qp[1] * qp[1] + qp[2] * qp[2] + qp[3] * qp[3]) * (T(0.5) * rinv));
                side_flux(qp, u0, u1, u2, p, rinv, Fn[1], ws[1]);
            } else {  // boundary face: q+ = q- (balancelaw.jl:77)
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    qp[s] = qm[s];
                    Fn[1][s] = Fn[0][s];
                }
                ws[1] = ws[0];
            }
            const T mx = fmax(ws[0], ws[1]);
            // (wsJ * MJI) of a face node of an unwarped brick: wsJ = |J drdx| w_a w_b and
            // MJI = 1 / (w_i w_j w_k J) leave |drdx_dir| / w_end (w_end = w_0 = w_N)
            const T fsc = (T)(fabs(dir == 0 ? drdx[0] : (dir == 1 ? drdx[1] : drdx[2])) / A.w[0]);
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const T fc = (Fn[0][s] + Fn[1][s]) * T(0.5);
                const T nf = A.surface_rusanov ? fc - (mx * (qp[s] - qm[s])) * T(0.5) : fc;
                sm.slot[s][slot] = (double)(nf * fsc);
            }
            }
        }
        __syncthreads();  // #2: face-slot contributions ready
        // ---- own old state and register, read now so that the loads overlap the faces
        const size_t g0 = (size_t)e * NS * NP;
        double* const qout_e = BATCH ? sm.ref[buf].q_out : A.q_out;
        const double rkb_dt = BATCH ? sm.ref[buf].rkb_dt : A.rkb_dt;
        double qold[NPT][NS];
        T dqold[NPT][NS];
#pragma unroll
        for (int h = 0; h < NPT; ++h)
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const size_t g = g0 + node_of(h) + s * NP;
                qold[h][s] = stage ? __ldg(qin_e + g) : 0.0;
                if (kStageDq && A.mode == MODE_STAGE)
                    dqold[h][s] = sm.dqs[kStageDq ? s : 0][kStageDq ? node_of(h) : 0];
                else if (A.mode == MODE_STAGE || A.mode == MODE_TENDENCY_INC)
                    dqold[h][s] = dq_is_f32 ? (T)__ldg(reinterpret_cast<const float*>(dq_e) + g)
                                            : (T)__ldg(reinterpret_cast<const double*>(dq_e) + g);
                else
                    dqold[h][s] = T(0);
            }

        // ---- own nodes: dq = rka*dq + volume - faces (x, y, z order); q_out = q + rkb*dt*dq
#pragma unroll
        for (int h = 0; h < NPT; ++h) {
            const int kk = kk_of(h), jn = jj_of(h);
            int slots[3] = {-1, -1, -1};
            if (ii == 0) slots[0] = jn + Q * kk;
            else if (ii == NQ - 1) slots[0] = NFP + jn + Q * kk;
            if (jn == 0) slots[1] = 2 * NFP + ii + Q * kk;
            else if (jn == NQ - 1) slots[1] = 3 * NFP + ii + Q * kk;
            if (kk == 0) slots[2] = 4 * NFP + ii + Q * jn;
            else if (kk == NQ - 1) slots[2] = 5 * NFP + ii + Q * jn;
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                T v = acc[h][s];
                if (A.mode == MODE_STAGE) v = (T)A.rka * dqold[h][s] + v;
                else if (A.mode == MODE_TENDENCY_INC) v = (T)((double)dqold[h][s] + (double)v);
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    if (slots[d] >= 0) v = v - (T)sm.slot[s][slots[d]];
                const size_t g = g0 + node_of(h) + s * NP;
                if (stage) {
                    if (dq_is_f32) reinterpret_cast<float*>(dq_e)[g] = (float)v;
                    else reinterpret_cast<double*>(dq_e)[g] = (double)v;
                    qout_e[g] = qold[h][s] + rkb_dt * (double)v;
                } else {
                    reinterpret_cast<double*>(dq_e)[g] = (double)v;
                }
            }
        }
    }
}

}  // namespace rb200
