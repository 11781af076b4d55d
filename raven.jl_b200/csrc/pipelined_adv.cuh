// Persistent, bulk-copy-pipelined LSRK stage kernel for the weak-form advection law on
// unwarped 3-D bricks with Nq = 4, 6 or 8 (one field).
//
// The stage is the one of the generic kernel's brick advection path, with the same
// operations in the same order:
//     dq_i += sum_dir (drdx_dir a_dir) sum_a W[a][i] q_a,    W[a][i] = D[a,i] w_a / w_i,
// (volumeterm!, src/balancelaws/dgsem.jl:299-343, with MJI_i wJ_a = w_a / w_i along a
// line of a brick) and the upwind (Rusanov) or central face flux times
// wsJ MJI = |drdx_dir| / w_0 (surfaceterm!, dgsem.jl:733-784).
//
// One field carries little arithmetic per byte, so the kernel is built to keep many
// bytes in flight.  Each CTA walks elements blockIdx.x + k*gridDim.x (or the chunks of a
// serving class) through a ring of NST shared-memory stages.  A stage holds one
// element's state and LSRK register (two 1-D bulk copies) and its geometry and neighbour
// ids (cp.async by threads 0..9), all completing on the stage's mbarrier; the copies of
// element k + NST - 1 are issued while element k runs.  The neighbour traces of element
// k + 1 are fetched (cp.async) during element k.
//
// A thread owns NPT nodes of one z-line (same i, j), whose z partners are loaded once.
// At Nq = 8 it owns the whole line: its x and y weights W[.][i], W[.][j] stay in
// registers, and the z weights are kernel parameters at fixed indices.  Every mbarrier
// wait is bounded: after kWaitLimit polls the CTA records RB200 status TIMEOUT and returns.
#pragma once

#include "pipelined_kernel.cuh"

namespace rb200 {

namespace pipea {

// nodes a thread owns, and ring stages (NST - 1 elements in flight ahead)
template <int Q>
constexpr int npt() { return Q == 8 ? 8 : 2; }
template <int Q>
constexpr int nst() { return Q == 8 ? 3 : 4; }

template <typename T, int Q>
struct Smem {
    using G = pipe::Geo<Q>;
    static constexpr int NST = nst<Q>();
    static_assert(NST >= 3, "the stage refilled at element k must differ from those of k and k + 1");
    __align__(16) double q[NST][G::NP];  // element state (bulk copy)
    __align__(16) T dq[NST][G::NP];      // element LSRK register (bulk copy)
    T qa[G::NPP];                        // the state in T, padded, for the partners
    double tr[2][G::NSLOT];              // neighbour traces, then (wsJ nf) MJI, per face slot
    T W[Q][Q];                           // W[a][i] = D[a,i] w_a / w_i
    T fc[2][6];                          // per element: |drdx_dir| / w_0 and drdx_dir a_dir
    double geo[NST][4];
    int32_t nb[NST][8];
    ElemRef ref[NST];
    uint64_t bar[NST];
};

// Arrivals a stage's mbarrier expects: thread 0's expect_tx arrive plus one cp.async
// completion arrive from each of threads 0..9.
constexpr uint32_t kArrivals = 11;

__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t* bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(pipe::smem_addr(bar)) : "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Entry i of the weight table as a kernel parameter in type T.
template <typename T>
__device__ __forceinline__ T wpar(const PipeArgs& A, int i) {
    if constexpr (sizeof(T) == 8) return A.S[i];
    else return A.Sf[i];
}

}  // namespace pipea

// CTAs per SM the registers are sized for (one field: few registers a thread)
template <typename T, int Q>
constexpr int pipe_adv_min_ctas() {
    return Q == 8 ? (sizeof(T) == 4 ? 8 : 6) : (Q == 6 ? 7 : 32);
}

template <typename T, bool BATCH, int Q>
__global__ void __launch_bounds__(Q * Q * Q / pipea::npt<Q>(), (pipe_adv_min_ctas<T, Q>()))
    pipelined_adv_kernel(const __grid_constant__ PipeArgs A, const __grid_constant__ PipeBatch B) {
    using namespace pipe;
    using G = Geo<Q>;
    constexpr int NPT = pipea::npt<Q>(), NST = pipea::nst<Q>();
    constexpr int NP = G::NP, NFP = G::NFP, NSLOT = G::NSLOT, NT = NP / NPT, KS = Q / NPT;
    constexpr int NSL = (NSLOT + NT - 1) / NT;  // face slots a thread owns
    constexpr bool LINE = NPT == Q;             // the thread owns its whole z-line
    extern __shared__ __align__(128) unsigned char pipe_smem_raw[];
    pipea::Smem<T, Q>& sm = *reinterpret_cast<pipea::Smem<T, Q>*>(pipe_smem_raw);
    const int t = threadIdx.x;
    const int ii = t % Q, jj = (t / Q) % Q, k0 = LINE ? 0 : t / (Q * Q);
    const bool stage = A.mode >= MODE_STAGE;
    const bool dq_is_f32 = stage && sizeof(T) == 4;
    // the register arrives by bulk copy whenever the stage reads it in type T
    const bool bulk_dq = A.mode == MODE_STAGE || (A.mode == MODE_TENDENCY_INC && sizeof(T) == 8);
    const uint32_t qbytes = NP * sizeof(double), dqbytes = bulk_dq ? NP * sizeof(T) : 0;

    // Threads 0..9 put element `r` into ring stage `s`: thread 0 the bulk copies of its
    // state and register, each thread one value of its geometry or neighbour ids.
    auto issue = [&](const ElemRef& r, int s) {
        if (t == 0) {
            sm.ref[s] = r;
            if (r.e >= 0) {
                fence_proxy_async();
                mbar_expect_tx(&sm.bar[s], qbytes + dqbytes);
                bulk_g2s(&sm.q[s][0], r.q + (size_t)r.e * NP, qbytes, &sm.bar[s]);
                if (bulk_dq)
                    bulk_g2s(&sm.dq[s][0], static_cast<const char*>(r.dq) + (size_t)r.e * dqbytes, dqbytes,
                             &sm.bar[s]);
            }
        }
        if (r.e >= 0) {
            fetch_part(r, t, sm.geo[s], sm.nb[s]);
            pipea::cp_async_arrive_noinc(&sm.bar[s]);
        }
    };
    // The face slots t + NT*sl this thread owns, packed once: face (bits 0-2), padded
    // own node (bits 3-12), node of the neighbour across the face (bits 13-22); -1: none.
    int pk[NSL];
#pragma unroll
    for (int sl = 0; sl < NSL; ++sl) {
        const int slot = t + NT * sl;
        int vn = 0, opp = 0;
        if (slot < NSLOT) slot_nodes<Q>(slot, vn, opp);
        pk[sl] = slot < NSLOT ? (slot / NFP) | (PAD(vn) << 3) | (opp << 13) : -1;
    }
    // Neighbour traces of the element in ring stage `s` into trace buffer `b`; slot
    // t + NT*sl is fetched and later used by thread t alone.
    auto traces = [&](int s, int b) {
        const double* qin = BATCH ? sm.ref[s].q : A.q_in;
#pragma unroll
        for (int sl = 0; sl < NSL; ++sl) {
            if (pk[sl] < 0) continue;
            const int ne = sm.nb[s][pk[sl] & 7];
            if (ne >= 0) cp_async8(&sm.tr[b][t + NT * sl], qin + (size_t)ne * NP + (pk[sl] >> 13));
        }
    };

    for (int c = t; c < Q * Q; c += NT) sm.W[c / Q][c % Q] = (T)A.S[c];  // S carries W[a*Q + i]
    if (t == 0) {
        for (int s = 0; s < NST; ++s) mbar_init(&sm.bar[s], pipea::kArrivals);
        fence_mbar_init();
    }
    __syncthreads();
    Cursor<BATCH> cur;  // meaningful in threads 0..9
    bool more = false;
    if (t < 10) {
        more = cur.start(A, B);
        for (int s = 0; s < NST - 1; ++s) {
            ElemRef r{};
            r.e = -1;
            if (more) {
                cur.resolve(A, B, r);
                more = cur.advance(A, B);
            }
            issue(r, s);
        }
    }
    cp_async_commit();
    __syncthreads();  // the stage references and the weight table are visible
    T wx[LINE ? Q : 1], wy[LINE ? Q : 1];
    if constexpr (LINE) {
#pragma unroll
        for (int a = 0; a < Q; ++a) {
            wx[a] = sm.W[a][ii];
            wy[a] = sm.W[a][jj];
        }
    }
    if (sm.ref[0].e >= 0) {
        if (__syncthreads_or(!bounded_wait(&sm.bar[0], 0))) {
            if (t == 0) atomicExch(A.status, kStatusTimeout);
            return;
        }
        traces(0, 0);
    }
    cp_async_commit();

    int64_t es = A.e_begin + blockIdx.x;
    for (int k = 0;; ++k, es += gridDim.x) {
        const int r = k % NST, r1 = (k + 1) % NST, b = k & 1;
        const int64_t e = BATCH ? sm.ref[r].e : (es < A.E ? es : -1);
        if (e < 0) break;
        if (t < 3) {  // the element's face factors and advection coefficients
            const double dd = sm.geo[r][t];
            sm.fc[b][t] = (T)(fabs(dd) / A.w[0]);
            sm.fc[b][3 + t] = (T)dd * (T)A.adv[t];
        }
#pragma unroll
        for (int h = 0; h < NPT; ++h) {
            const int n = t + NT * h;
            sm.qa[PAD(n)] = (T)sm.q[r][n];
        }
        // the next element's stage (issued NST - 2 elements ago): wait, then fetch its traces
        const bool next = sm.ref[r1].e >= 0;
        const bool late = next && !bounded_wait(&sm.bar[r1], (uint32_t)(((k + 1) / NST) & 1));
        if (__syncthreads_or(late)) {  // #1: partner values ready; stage k - 1 is free
            if (t == 0) atomicExch(A.status, kStatusTimeout);
            return;
        }
        if (t < 10) {
            ElemRef rn{};
            rn.e = -1;
            if (more) {
                cur.resolve(A, B, rn);
                more = cur.advance(A, B);
            }
            issue(rn, (k + NST - 1) % NST);
        }
        cp_async_commit();
        if (next) traces(r1, b ^ 1);
        cp_async_commit();

        // ---- volume term: the derivative sums along x, y, z
        const T cx = sm.fc[b][3], cy = sm.fc[b][4], cz = sm.fc[b][5];
        T acc[NPT];
        if constexpr (LINE) {
            T qz[Q];
#pragma unroll
            for (int a = 0; a < Q; ++a) qz[a] = sm.qa[PAD(ii + Q * (jj + Q * a))];
#pragma unroll
            for (int h = 0; h < Q; ++h) {
                T sx = T(0), sy = T(0), sz = T(0);
#pragma unroll
                for (int a = 0; a < Q; ++a) {
                    sx += wx[a] * sm.qa[PAD(a + Q * (jj + Q * h))];
                    sy += wy[a] * sm.qa[PAD(ii + Q * (a + Q * h))];
                    sz += pipea::wpar<T>(A, a * Q + h) * qz[a];
                }
                acc[h] = T(0);
                acc[h] += cx * sx;
                acc[h] += cy * sy;
                acc[h] += cz * sz;
            }
        } else {
            T sx[NPT], sy[NPT], sz[NPT];
#pragma unroll
            for (int h = 0; h < NPT; ++h) sx[h] = sy[h] = sz[h] = T(0);
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                const T wxa = sm.W[a][ii], wya = sm.W[a][jj];
#pragma unroll
                for (int h = 0; h < NPT; ++h) {
                    const int kk = k0 + KS * h;
                    sx[h] += wxa * sm.qa[PAD(a + Q * (jj + Q * kk))];
                    sy[h] += wya * sm.qa[PAD(ii + Q * (a + Q * kk))];
                }
                const T qz = sm.qa[PAD(ii + Q * (jj + Q * a))];
#pragma unroll
                for (int h = 0; h < NPT; ++h) sz[h] += sm.W[a][k0 + KS * h] * qz;
            }
#pragma unroll
            for (int h = 0; h < NPT; ++h) {
                acc[h] = T(0);
                acc[h] += cx * sx[h];
                acc[h] += cy * sy[h];
                acc[h] += cz * sz[h];
            }
        }

        // ---- face-slot contributions (wsJ nf) MJI over the slot's trace (this thread's
        // own copies; the two groups committed since belong to later elements)
        pipea::cp_async_wait_group<2>();
#pragma unroll
        for (int sl = 0; sl < NSL; ++sl) {
            if (pk[sl] < 0) continue;
            const int slot = t + NT * sl;
            const int f = pk[sl] & 7, dir = f >> 1, side = f & 1;
            const int nbf = sm.nb[r][f];
            T nf;
            if (nbf == -2) {  // mortar face: the flux comes from the mortar kernel
                nf = (T)A.ncflux[((size_t)e * 6 + f) * NFP + (slot - f * NFP)];
            } else {
                const T qm = sm.qa[(pk[sl] >> 3) & 1023];
                const T qp = nbf >= 0 ? (T)sm.tr[b][slot] : qm;  // default boundarystate (balancelaw.jl:77)
                const T an = (T)A.adv[dir] * (side ? T(1) : T(-1));
                const T fcen = (an * qm + an * qp) * T(0.5);
                nf = A.surface_rusanov ? fcen - (fabs(an) * (qp - qm)) * T(0.5) : fcen;
            }
            sm.tr[b][slot] = (double)(nf * sm.fc[b][dir]);
        }
        __syncthreads();  // #2: face-slot contributions ready

        // ---- own nodes: dq = rka dq + volume - faces (x, y, z order); q_out = q + rkb dt dq
        void* const dq_e = BATCH ? sm.ref[r].dq : A.dq;
        double* const qout_e = BATCH ? sm.ref[r].q_out : A.q_out;
        const double rkb_dt = BATCH ? sm.ref[r].rkb_dt : A.rkb_dt;
        const double* fl = sm.tr[b];
#pragma unroll
        for (int h = 0; h < NPT; ++h) {
            const int kk = k0 + KS * h;
            const int n = t + NT * h;
            const size_t g = (size_t)e * NP + n;
            T v = acc[h];
            if (A.mode == MODE_STAGE) {
                v = (T)A.rka * sm.dq[r][n] + v;
            } else if (A.mode == MODE_TENDENCY_INC) {
                const double old = bulk_dq ? (double)sm.dq[r][n] : __ldg(reinterpret_cast<const double*>(dq_e) + g);
                v = (T)(old + (double)v);
            }
            if (ii == 0) v = v - (T)fl[jj + Q * kk];
            else if (ii == Q - 1) v = v - (T)fl[NFP + jj + Q * kk];
            if (jj == 0) v = v - (T)fl[2 * NFP + ii + Q * kk];
            else if (jj == Q - 1) v = v - (T)fl[3 * NFP + ii + Q * kk];
            if (kk == 0) v = v - (T)fl[4 * NFP + ii + Q * jj];
            else if (kk == Q - 1) v = v - (T)fl[5 * NFP + ii + Q * jj];
            if (stage) {
                if (dq_is_f32) reinterpret_cast<float*>(dq_e)[g] = (float)v;
                else reinterpret_cast<double*>(dq_e)[g] = (double)v;
                qout_e[g] = sm.q[r][n] + rkb_dt * (double)v;  // stage r is refilled at element k + 1
            } else {
                reinterpret_cast<double*>(dq_e)[g] = (double)v;
            }
        }
    }
    cp_async_wait_all();
}

}  // namespace rb200
