// Persistent, TMA-pipelined stage kernel for 3-D hexahedra with Nq = 8 on unwarped
// bricks, flux-differencing volume forms (Kennedy-Gruber, entropy conservative).
//
// Each CTA owns a strided set of elements (e = blockIdx.x + k*gridDim.x).  While it
// computes element e, one thread has already issued 1-D bulk copies (cp.async.bulk,
// completion on an mbarrier) of the next element's state q and LSRK register dq into
// the other half of a double buffer, so the HBM stream overlaps the flux arithmetic.
// Two CTAs share an SM.
//
// Thread t owns the two nodes t and t+256 of the element (same i, j; k and k+4), so
// the eight z-partners of its line are loaded once for both nodes.  The metric of an
// unwarped brick is folded into a per-element table S_dir[a][id] =
// drdx_dir * (D[a,id] w_a / w_id - D[id,a]), which equals MJI_id * (D[a,id] l_g[a] -
// D[id,a] l_g[id]) of esvolumeterm_dir! (src/balancelaws/dgsem.jl:576-600).
// Neighbour traces are prefetched into registers before the volume loop; the face
// fluxes are then applied in the order x-, x+, y-, y+, z-, z+ of surfaceterm!
// (dgsem.jl:756-782).
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
    const int32_t* nbr;      // (6, E)
    int32_t* status;         // device status word (0 = ok)
    int64_t E;
    int32_t mode;
    int32_t surface_rusanov;
    double rka, rkb_dt, gamma;
    double S[64];  // S[a*8 + id] = D[a,id] * w[a] / w[id] - D[id,a]
    double w[8];
};

namespace pipe {

constexpr int NQ = 8, NP = 512, NS = 5, NT = 256, NAUX = 6;
constexpr int PAD(int n) { return n + (n >> 3); }  // one vector slot of padding every 8 nodes
constexpr int NPP = PAD(NP);                       // padded plane length
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

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

template <typename T>
struct Vec2;
template <>
struct Vec2<double> {
    using type = double2;
};
template <>
struct Vec2<float> {
    using type = float2;
};

template <typename T>
struct Smem {
    double q[2][NS][NP];      // state: element being computed / element prefetched
    T dq[NS][NP];             // LSRK register of the element being computed
    typename Vec2<T>::type aux[NAUX / 2][NPP];  // per-node partner values, two per vector load
    T sflux[NS][384];         // face-slot contributions (wsJ * nf) * MJI
    T S[3][NQ][NQ];           // S_dir[a][id] * drdx_dir of the current element
    uint64_t bar[3];          // q buffers 0/1, dq buffer
};

__device__ __forceinline__ bool bounded_wait(uint64_t* bar, uint32_t parity) {
    long it = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++it > kWaitLimit) return false;
    }
    return true;
}

}  // namespace pipe

template <int COMBO, typename T>
__global__ void __launch_bounds__(pipe::NT, 2) pipelined_stage_kernel(const __grid_constant__ PipeArgs A) {
    using namespace pipe;
    extern __shared__ __align__(128) unsigned char pipe_smem_raw[];
    Smem<T>& sm = *reinterpret_cast<Smem<T>*>(pipe_smem_raw);
    const int t = threadIdx.x;
    const int ii = t & 7, jj = (t >> 3) & 7, k0 = t >> 6;  // nodes (ii, jj, k0) and (ii, jj, k0 + 4)
    const int n0 = t, n1 = t + 256;
    const bool stage = A.mode >= MODE_STAGE;
    const bool read_dq = A.mode == MODE_STAGE || A.mode == MODE_TENDENCY_INC;
    const bool dq_is_f32 = stage && sizeof(T) == 4;
    const uint32_t qbytes = NS * NP * sizeof(double);
    const uint32_t dqbytes = NS * NP * (dq_is_f32 ? 4 : 8);
    const T gm1 = (T)(A.gamma - 1.0), gam = (T)A.gamma;

    if (t == 0) {
        mbar_init(&sm.bar[0], 1);
        mbar_init(&sm.bar[1], 1);
        mbar_init(&sm.bar[2], 1);
        fence_mbar_init();
    }
    __syncthreads();

    int64_t e = blockIdx.x;
    if (t == 0 && e < A.E) {
        mbar_expect_tx(&sm.bar[0], qbytes);
        bulk_g2s(&sm.q[0][0][0], A.q_in + (size_t)e * NS * NP, qbytes, &sm.bar[0]);
    }
    uint32_t qphase[2] = {0, 0}, dqphase = 0;
    int b = 0;
    for (; e < A.E; e += gridDim.x, b ^= 1) {
        const int64_t enext = e + gridDim.x;
        // ---- element geometry, scaled S table, neighbour traces (global/L2) issued early
        const double* eg = A.elem_geo + 4 * e;
        const double drdx[3] = {__ldg(eg), __ldg(eg + 1), __ldg(eg + 2)};
        const double J = __ldg(eg + 3);
        if (t < 192) {
            const int dir = t >> 6, a = (t >> 3) & 7, id = t & 7;
            const double dd = dir == 0 ? drdx[0] : (dir == 1 ? drdx[1] : drdx[2]);
            sm.S[dir][a][id] = (T)(A.S[a * 8 + id] * dd);
        }
        // face slots: s0 = t (faces x-, x+, y-, y+), s1 = 256 + t for t < 128 (z-, z+)
        T qp[2][NS];
        int vnode[2] = {0, 0};
        bool open_face[2] = {false, false};  // false: boundary face, q+ = q- (balancelaw.jl:77)
#pragma unroll
        for (int sl = 0; sl < 2; ++sl) {
            const int slot = sl == 0 ? t : 256 + t;
            if (slot >= 384) continue;
            const int f = slot >> 6, jf = slot & 63;
            const int dir = f >> 1, side = f & 1;
            const int j1 = jf & 7, j2 = jf >> 3, c = side ? NQ - 1 : 0;
            int vn, opp;
            if (dir == 0) { vn = c + 8 * (j1 + 8 * j2); opp = (NQ - 1 - c) + 8 * (j1 + 8 * j2); }
            else if (dir == 1) { vn = j1 + 8 * (c + 8 * j2); opp = j1 + 8 * ((NQ - 1 - c) + 8 * j2); }
            else { vn = j1 + 8 * (j2 + 8 * c); opp = j1 + 8 * (j2 + 8 * (NQ - 1 - c)); }
            vnode[sl] = vn;
            const int ne = __ldg(A.nbr + 6 * e + f);
            open_face[sl] = ne >= 0;
            if (ne >= 0) {
                const double* qn = A.q_in + (size_t)ne * NS * NP + opp;
#pragma unroll
                for (int s = 0; s < NS; ++s) qp[sl][s] = (T)__ldg(qn + s * NP);
            }
        }
        // ---- this element's state
        if (__syncthreads_or(!bounded_wait(&sm.bar[b], qphase[b]))) {
            if (t == 0) atomicExch(A.status, kStatusTimeout);
            return;
        }
        qphase[b] ^= 1;
        // ---- per-node partner values
        T own[2][NAUX];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int n = h ? n1 : n0;
            const T rho = (T)sm.q[b][0][n];
            const T rinv = T(1) / rho;
            const T m0 = (T)sm.q[b][1][n], m1 = (T)sm.q[b][2][n], m2 = (T)sm.q[b][3][n];
            const T u0 = m0 * rinv, u1 = m1 * rinv, u2 = m2 * rinv;
            const T rhoe = (T)sm.q[b][4][n];
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
#pragma unroll
            for (int c = 0; c < NAUX / 2; ++c) {
                sm.aux[c][PAD(n)].x = own[h][2 * c];
                sm.aux[c][PAD(n)].y = own[h][2 * c + 1];
            }
        }
        __syncthreads();  // #1: aux and S ready; every thread is past the previous element
        if (t == 0) {
            // the other q buffer and the dq buffer were last read before barrier #1
            fence_proxy_async();
            if (enext < A.E) {
                mbar_expect_tx(&sm.bar[b ^ 1], qbytes);
                bulk_g2s(&sm.q[b ^ 1][0][0], A.q_in + (size_t)enext * NS * NP, qbytes, &sm.bar[b ^ 1]);
            }
            if (read_dq) {
                mbar_expect_tx(&sm.bar[2], dqbytes);
                bulk_g2s(&sm.dq[0][0], reinterpret_cast<const char*>(A.dq) + (size_t)e * dqbytes, dqbytes,
                         &sm.bar[2]);
            }
        }

        // ---- volume term (ordered pairs along x, y, z)
        T acc[2][NS];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int s = 0; s < NS; ++s) acc[h][s] = T(0);

        auto pair = [&](T (&ac)[NS], const T (&o)[NAUX], const T (&pv)[NAUX], const T sc, const int dir) {
            if constexpr (COMBO == EUL_KG) {
                const T rb = o[0] + pv[0];
                const T ub0 = o[1] + pv[1], ub1 = o[2] + pv[2], ub2 = o[3] + pv[3];
                const T eb = o[4] + pv[4], pb = o[5] + pv[5];
                const T un = (dir == 0 ? ub0 : dir == 1 ? ub1 : ub2) * sc;
                const T f1 = rb * un;
                ac[0] += f1;
                ac[1] = fma(f1, ub0, ac[1]);
                ac[2] = fma(f1, ub1, ac[2]);
                ac[3] = fma(f1, ub2, ac[3]);
                ac[1 + dir] = fma(pb, sc, ac[1 + dir]);
                ac[4] = fma(un, fma(rb, eb, pb), ac[4]);
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

        auto load_aux = [&](T (&pv)[NAUX], const int n) {
#pragma unroll
            for (int c = 0; c < NAUX / 2; ++c) {
                const auto v = sm.aux[c][PAD(n)];
                pv[2 * c] = v.x;
                pv[2 * c + 1] = v.y;
            }
        };
#pragma unroll
        for (int a = 0; a < NQ; ++a) {
            const T sx = sm.S[0][a][ii], sy = sm.S[1][a][jj];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int kk = k0 + 4 * h;
                T pv[NAUX];
                const int nx = a + 8 * (jj + 8 * kk);
                load_aux(pv, nx);
                pair(acc[h], own[h], pv, sx, 0);
                const int ny = ii + 8 * (a + 8 * kk);
                load_aux(pv, ny);
                pair(acc[h], own[h], pv, sy, 1);
            }
            {
                T pv[NAUX];
                const int nz = ii + 8 * (jj + 8 * a);
                load_aux(pv, nz);
                pair(acc[0], own[0], pv, sm.S[2][a][k0], 2);
                pair(acc[1], own[1], pv, sm.S[2][a][k0 + 4], 2);
            }
        }

        // ---- face-slot contributions (wsJ * nf) * MJI into shared memory
#pragma unroll
        for (int sl = 0; sl < 2; ++sl) {
            const int slot = sl == 0 ? t : 256 + t;
            if (slot >= 384) continue;
            const int f = slot >> 6, dir = f >> 1, side = f & 1;
            const int vn = vnode[sl];
            T qm[NS];
#pragma unroll
            for (int s = 0; s < NS; ++s) qm[s] = (T)sm.q[b][s][vn];
            if (!open_face[sl]) {
#pragma unroll
                for (int s = 0; s < NS; ++s) qp[sl][s] = qm[s];
            }
            const T sn = side ? T(1) : T(-1);
            T Fn[2][NS], ws[2];
            // normal flux and wave speed of one side (euler.jl:50-68 with n = sn e_dir),
            // from the conserved state and its primitives u, p
            auto side_flux = [&](const T (&qq)[NS], const T u0, const T u1, const T u2, const T p, const T rinv,
                                 T (&F)[NS], T& w) {
                const T ud = dir == 0 ? u0 : dir == 1 ? u1 : u2;
                const T un = ud * sn;
                const T mn = (dir == 0 ? qq[1] : dir == 1 ? qq[2] : qq[3]) * sn;
                F[0] = mn;
                F[1] = mn * u0 + (dir == 0 ? p * sn : T(0));
                F[2] = mn * u1 + (dir == 1 ? p * sn : T(0));
                F[3] = mn * u2 + (dir == 2 ? p * sn : T(0));
                F[4] = un * (qq[4] + p);
                w = fabs(un) + sqrt(gam * p * rinv);
            };
            auto prim = [&](const T (&qq)[NS], T& u0, T& u1, T& u2, T& p, T& rinv) {
                rinv = T(1) / qq[0];
                u0 = qq[1] * rinv;
                u1 = qq[2] * rinv;
                u2 = qq[3] * rinv;
                p = gm1 * (qq[4] - (qq[1] * qq[1] + qq[2] * qq[2] + qq[3] * qq[3]) * (T(0.5) * rinv));
            };
            {
                T u0, u1, u2, p, rinv;
                if constexpr (COMBO == EUL_KG) {
                    // the element's own primitives are already staged (halves)
                    const auto v0 = sm.aux[0][PAD(vn)], v1 = sm.aux[1][PAD(vn)], v2 = sm.aux[2][PAD(vn)];
                    u0 = T(2) * v0.y;
                    u1 = T(2) * v1.x;
                    u2 = T(2) * v1.y;
                    p = T(2) * v2.y;
                    rinv = T(0.5) / v0.x;
                } else {
                    prim(qm, u0, u1, u2, p, rinv);
                }
                side_flux(qm, u0, u1, u2, p, rinv, Fn[0], ws[0]);
                if (open_face[sl]) {
                    prim(qp[sl], u0, u1, u2, p, rinv);
                    side_flux(qp[sl], u0, u1, u2, p, rinv, Fn[1], ws[1]);
                } else {
#pragma unroll
                    for (int s = 0; s < NS; ++s) Fn[1][s] = Fn[0][s];
                    ws[1] = ws[0];
                }
            }
            const T mx = fmax(ws[0], ws[1]);
            // (wsJ * MJI) of a face node of an unwarped brick: wsJ = |J drdx| w_a w_b and
            // MJI = 1 / (w_i w_j w_k J) leave |drdx_dir| / w_end (w_end = w_0 = w_N)
            const T fsc = (T)(fabs(dir == 0 ? drdx[0] : (dir == 1 ? drdx[1] : drdx[2])) / A.w[0]);
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const T fc = (Fn[0][s] + Fn[1][s]) * T(0.5);
                const T nf = A.surface_rusanov ? fc - (mx * (qp[sl][s] - qm[s])) * T(0.5) : fc;
                sm.sflux[s][slot] = nf * fsc;
            }
        }
        __syncthreads();  // #2: face-slot contributions ready
        if (read_dq) {
            if (__syncthreads_or(!bounded_wait(&sm.bar[2], dqphase))) {
                if (t == 0) atomicExch(A.status, kStatusTimeout);
                return;
            }
            dqphase ^= 1;
        }
        // ---- own nodes: dq = rka*dq + volume - faces (x, y, z order); q_out = q + rkb*dt*dq
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int n = h ? n1 : n0;
            const int kk = k0 + 4 * h;
            int slots[3] = {-1, -1, -1};
            if (ii == 0) slots[0] = jj + 8 * kk;
            else if (ii == NQ - 1) slots[0] = 64 + jj + 8 * kk;
            if (jj == 0) slots[1] = 128 + ii + 8 * kk;
            else if (jj == NQ - 1) slots[1] = 192 + ii + 8 * kk;
            if (kk == 0) slots[2] = 256 + ii + 8 * jj;
            else if (kk == NQ - 1) slots[2] = 320 + ii + 8 * jj;
            const size_t g = (size_t)e * NS * NP + n;
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                T v = acc[h][s];
                if (A.mode == MODE_STAGE) v = (T)A.rka * sm.dq[s][n] + v;
                else if (A.mode == MODE_TENDENCY_INC) v = (T)((double)sm.dq[s][n] + (double)v);
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    if (slots[d] >= 0) v = v - sm.sflux[s][slots[d]];
                if (stage) {
                    if (dq_is_f32) reinterpret_cast<float*>(A.dq)[g + s * NP] = (float)v;
                    else reinterpret_cast<double*>(A.dq)[g + s * NP] = (double)v;
                    A.q_out[g + s * NP] = sm.q[b][s][n] + A.rkb_dt * (double)v;
                } else {
                    reinterpret_cast<double*>(A.dq)[g + s * NP] = (double)v;
                }
            }
        }
    }
}

}  // namespace rb200
