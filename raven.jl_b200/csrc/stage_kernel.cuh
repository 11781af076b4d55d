// Fused DGSEM stage kernel: volume term + surface term + LSRK(5,4) stage update.
//
// One thread owns one volume node; EPB elements share a CTA (EPB*Np threads).  The
// thread keeps its own state, accumulators and metric in registers; the per-node
// quantities its line partners need (primitive half-values, fluxes, metric rows) are
// staged once in shared memory.  The surface term is evaluated by the thread that
// owns the face node, face by face in Raven's order (x-, x+, y-, y+, z-, z+), so no
// atomics or extra barriers are needed and corner nodes accumulate in the same order
// as surfaceterm! (src/balancelaws/dgsem.jl:756-782).  The neighbour's trace is read
// straight from the previous stage's state (ping-pong buffers: q_in is never written).
//
// Reference kernels restated: volumeterm! (dgsem.jl:257-348), esvolumeterm_dir!
// (dgsem.jl:514-608), surfaceterm! (dgsem.jl:733-784), the LSRK stage broadcasts
// (odesolvers.jl:55-57); fluxes from balancelaws/euler.jl:34-68,150-216,
// balancelaws/advection.jl:18-19 and numericalfluxes.jl:9-50.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rb200_internal.h"
#include "surface_fluxes.cuh"

namespace rb200 {

template <int N, int D>
struct IPow {
    static constexpr int v = N * IPow<N, D - 1>::v;
};
template <int N>
struct IPow<N, 0> {
    static constexpr int v = 1;
};

// EPBX > 0 overrides the default number of elements per CTA (the serving loop's tiles).
template <int DIM, int NQ, int EPBX = 0>
struct Shape {
    static constexpr int NP = IPow<NQ, DIM>::v;
    static constexpr int NFP = IPow<NQ, DIM - 1>::v;
    static constexpr int NF = 2 * DIM;
    static constexpr int EPB = EPBX > 0 ? EPBX : (NP >= 256 ? 1 : 256 / NP);  // elements per CTA
    static constexpr int THREADS = EPB * NP;
};

template <int COMBO, int DIM>
struct CSize {
    static constexpr bool ADV = (COMBO == ADV_WEAK || COMBO == ADV_FDC);
    static constexpr int NS = ADV ? 1 : DIM + 2;
    // per-node values staged in shared memory for the line partners
    static constexpr int NAUX = COMBO == ADV_WEAK   ? DIM              // l_F[dir]
                                : COMBO == ADV_FDC  ? 1                // q/2
                                : COMBO == EUL_WEAK ? DIM * (DIM + 2)  // l_F[dir][s]
                                : COMBO == EUL_FDC  ? DIM * (DIM + 2)  // F[d][s]/2
                                : COMBO == EUL_KG   ? DIM + 3          // rho/2, u/2, e/2, p/2
                                                    : DIM + 3;         // EC: rho, u, b, |u|^2
};

template <int DIM, int NQ, int COMBO, int GEOM, typename T, int EPBX = 0>
struct KernelCfg {
    using S = Shape<DIM, NQ, EPBX>;
    using C = CSize<COMBO, DIM>;
    static constexpr int NLG = GEOM == GEOM_AFFINE ? DIM : DIM * DIM;
    // partner values and metric rows of the CTA's elements, then the derivative matrix D
    // (read per pair with thread-dependent indices: from shared memory rather than the
    // kernel parameters, whose constant cache serialises distinct addresses in a warp)
    static constexpr size_t off_D = (size_t)S::EPB * (C::NAUX + NLG) * S::NP * sizeof(T);
    static constexpr size_t smem = off_D + (size_t)NQ * NQ * sizeof(T);
};

// Products and differences that must not be contracted into an FMA (they make the
// diagonal pair term cancel exactly).
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
// cp.async of one value into shared memory (the persistent kernels' prefetch)
__device__ __forceinline__ void cpa8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cpa4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// A thread's own state and LSRK register, already copied into shared memory by the
// thread itself (field s at q[s * stride]); null pointers: read them from global memory.
// tables_ready: the element-independent shared tables (D, or W of the brick advection
// stage) already hold this CTA's values from an earlier group.
struct Prefetched {
    const double* q = nullptr;
    const void* dq = nullptr;
    int stride = 0;
    bool tables_ready = false;
};

__device__ __forceinline__ double dev_log(double x) { return log(x); }
__device__ __forceinline__ float dev_log(float x) { return logf(x); }
__device__ __forceinline__ double dev_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float dev_sqrt(float x) { return sqrtf(x); }

// logavg (numericalfluxes.jl:9-22)
template <typename T>
__device__ __forceinline__ T logavg(T a, T b) {
    const T zeta = a / b;
    const T f = (zeta - T(1)) / (zeta + T(1));
    const T u = f * f;
    const T eps = sizeof(T) == 8 ? T(2.220446049250313e-16) : T(1.1920929e-07f);
    T F;
    if (u < eps) {
        F = fma(u, fma(u, fma(u, fma(u, T(1) / T(9), T(1) / T(7)), T(1) / T(5)), T(1) / T(3)), T(1));
    } else {
        F = dev_log(zeta) / (T(2) * f);
    }
    return (a + b) / (T(2) * F);
}

// Buffers of the element being updated: the DGSEM handle takes them from StageArgs,
// the serving loop from each solve's descriptor.
struct ElemPtrs {
    const double* q_in;
    double* q_out;
    void* dq;
    const double* elem_geo;
    const double* vgeo;
    const double* sgeo;
    const int32_t* nbr;
    double rkb_dt;
    const double* ncflux;
    const int32_t* vmapP;  // general connectivity, or null (StageArgs::vmapP)
};

__device__ __forceinline__ ElemPtrs elem_ptrs(const StageArgs& A) {
    return ElemPtrs{A.q_in, A.q_out, A.dq, A.elem_geo, A.vgeo, A.sgeo, A.nbr, A.rkb_dt, A.ncflux, A.vmapP};
}

// Weak-form advection on an unwarped element (the stage of stage_element, refactored for
// bricks).  Along a line in direction dir the metric and mass factors of volumeterm!
// (dgsem.jl:299-308, 326-343) reduce to MJI_i wJ_a drdx = (w_a / w_i) drdx, so
//     dq_i += sum_dir drdx_dir a_dir sum_a W[a][i] q_a,    W[a][i] = D[a,i] w_a / w_i,
// and on a face (wsJ MJI) = |drdx_dir| / w_0 (lobattocells.jl:3285-3291; LGL weights are
// symmetric).  One field: the partner values are the state itself.
template <int DIM, int NQ, typename T, int EPBX>
__device__ __forceinline__ void stage_element_adv_brick(const StageArgs& A, const ElemPtrs& P, const int64_t e,
                                                        const bool active, unsigned char* smem_raw,
                                                        const Prefetched pf) {
    using S = Shape<DIM, NQ, EPBX>;
    constexpr int NP = S::NP, NFP = S::NFP, NF = S::NF, EPB = S::EPB;
    T* sq = reinterpret_cast<T*>(smem_raw);  // q of the CTA's elements
    T* sW = sq + EPB * NP;                   // W[a + NQ i]
    const int tid = threadIdx.x;
    const int el = tid / NP;
    const int n = tid - el * NP;
    int id[3];
    id[0] = n % NQ;
    id[1] = DIM > 1 ? (n / NQ) % NQ : 0;
    id[2] = DIM > 2 ? n / (NQ * NQ) : 0;
    double qd = 0.0, drdx[3] = {0.0, 0.0, 0.0};
    T q0 = T(0);
    if (active) {
        qd = pf.q ? pf.q[0] : __ldg(P.q_in + (size_t)e * NP + n);
        q0 = (T)qd;
        const double* eg = P.elem_geo + 4 * e;
#pragma unroll
        for (int d = 0; d < DIM; ++d) drdx[d] = __ldg(eg + d);
        sq[el * NP + n] = q0;
    }
    if (!pf.tables_ready)
        for (int i = tid; i < NQ * NQ; i += S::THREADS) {
            const int a = i % NQ, ii = i / NQ;
            sW[i] = (T)(A.D[a + NQ * ii] * (A.w[a] / A.w[ii]));
        }
    __syncthreads();
    if (!active) return;

    // ---- volume term
    const T* qe = sq + el * NP;
    const int dmask = A.dir_mask ? A.dir_mask : 7;
    T acc = T(0);
#pragma unroll
    for (int dir = 0; dir < DIM; ++dir) {
        if (!((dmask >> dir) & 1)) continue;
        const int stride = dir == 0 ? 1 : (dir == 1 ? NQ : NQ * NQ);
        const int idd = id[dir];
        const int base = n - idd * stride;
        T sum = T(0);
#pragma unroll
        for (int a = 0; a < NQ; ++a) sum += sW[a + NQ * idd] * qe[base + a * stride];
        acc += ((T)drdx[dir] * (T)A.adv[dir]) * sum;
    }

    // ---- combine with dq
    const bool stage = A.mode >= MODE_STAGE;
    const size_t node0 = (size_t)e * NP + n;
    T v = acc;
    if (A.mode == MODE_STAGE) {
        T old;
        if (pf.dq) old = static_cast<const T*>(pf.dq)[0];
        else if (sizeof(T) == 4) old = (T) reinterpret_cast<const float*>(P.dq)[node0];
        else old = (T) reinterpret_cast<const double*>(P.dq)[node0];
        v = (T)A.rka * old + v;
    } else if (A.mode == MODE_TENDENCY_INC) {
        v = (T)(reinterpret_cast<const double*>(P.dq)[node0] + (double)v);
    }

    // ---- surface term, faces in the order x-, x+, y-, y+, z-, z+ (dgsem.jl:756-782)
#pragma unroll
    for (int dir = 0; dir < DIM; ++dir) {
        const int idd = id[dir];
        if (idd != 0 && idd != NQ - 1) continue;
        if (!((dmask >> dir) & 1)) continue;
        const int side = idd == 0 ? 0 : 1;
        const int f = 2 * dir + side;
        const int stride = dir == 0 ? 1 : (dir == 1 ? NQ : NQ * NQ);
        const int ne = __ldg(P.nbr + (size_t)NF * e + f);
        T nf;
        if (ne == -2) {  // mortar face: the flux comes from the mortar kernel
            int j;
            if (DIM == 1) j = 0;
            else if (DIM == 2) j = (dir == 0) ? id[1] : id[0];
            else j = (dir == 0) ? id[1] + NQ * id[2] : (dir == 1 ? id[0] + NQ * id[2] : id[0] + NQ * id[1]);
            nf = (T)__ldg(P.ncflux + ((size_t)e * NF + f) * NFP + j);
        } else {
            T qp = q0;  // default boundarystate (balancelaw.jl:77)
            if (ne >= 0) {
                const int nn = n + (side == 0 ? (NQ - 1) * stride : -(NQ - 1) * stride);
                qp = (T)__ldg(P.q_in + (size_t)ne * NP + nn);
            } else if (ne <= -kBcBase && A.bc_kind[-ne - kBcBase] == BC_PRESCRIBED) {
                qp = (T)A.bc_state[-ne - kBcBase][0];
            }
            const T an = (T)A.adv[dir] * (side == 0 ? T(-1) : T(1));
            const T fc = (an * q0 + an * qp) * T(0.5);
            nf = A.surface_rusanov ? fc - (fabs(an) * (qp - q0)) * T(0.5) : fc;
        }
        v = v - nf * (T)(fabs(drdx[dir]) / A.w[0]);
    }

    // ---- write back
    if (stage) {
        if (sizeof(T) == 4) reinterpret_cast<float*>(P.dq)[node0] = (float)v;
        else reinterpret_cast<double*>(P.dq)[node0] = (double)v;
        P.q_out[node0] = qd + P.rkb_dt * (double)v;
    } else {
        reinterpret_cast<double*>(P.dq)[node0] = (double)v;
    }
}

// One element per group of Np threads: the whole fused stage for element e.  All
// threads of the CTA must call it (it contains a barrier); inactive groups pass
// active = false.  SF = 1: the Euler surface flux is one of the entropy family
// (entropy conservative, Kennedy-Gruber, Roe, matrix dissipation; A.surface_flux).
template <int DIM, int NQ, int COMBO, int GEOM, typename T, int EPBX, int SF = 0>
__device__ __forceinline__ void stage_element(const StageArgs& A, const ElemPtrs& P, const int64_t e,
                                              const bool active, unsigned char* smem_raw,
                                              const Prefetched pf = Prefetched{}) {
    using S = Shape<DIM, NQ, EPBX>;
    using C = CSize<COMBO, DIM>;
    using K = KernelCfg<DIM, NQ, COMBO, GEOM, T, EPBX>;
    constexpr int NP = S::NP, NFP = S::NFP, NF = S::NF, EPB = S::EPB;
    constexpr int NS = C::NS, NAUX = C::NAUX, NLG = K::NLG;
    constexpr bool AFF = GEOM == GEOM_AFFINE;
    if constexpr (COMBO == ADV_WEAK && AFF) {
        stage_element_adv_brick<DIM, NQ, T, EPBX>(A, P, e, active, smem_raw, pf);
        return;
    }

    T* s_aux = reinterpret_cast<T*>(smem_raw);
    T* s_lg = s_aux + EPB * NAUX * NP;
    T* sD = reinterpret_cast<T*>(smem_raw + K::off_D);  // D[i + NQ j] = l_j'(r_i)

    const int tid = threadIdx.x;
    const int el = tid / NP;
    const int n = tid - el * NP;
    int id[3];
    id[0] = n % NQ;
    id[1] = DIM > 1 ? (n / NQ) % NQ : 0;
    id[2] = DIM > 2 ? n / (NQ * NQ) : 0;
    T* aux = s_aux + el * NAUX * NP;
    T* lgs = s_lg + el * NLG * NP;

    double qd[NS];
    T q[NS];
    T lg[NLG];
    T own[NAUX > 0 ? NAUX : 1];
    double mji = 0.0, J = 0.0, wJ = 0.0;
    double drdx[3] = {0.0, 0.0, 0.0};

    if (active) {
        const double* qe = P.q_in + (size_t)e * NS * NP;
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            qd[s] = pf.q ? pf.q[s * pf.stride] : __ldg(qe + s * NP + n);
            q[s] = (T)qd[s];
        }
        if constexpr (AFF) {
            const double* eg = P.elem_geo + 4 * e;
#pragma unroll
            for (int d = 0; d < DIM; ++d) drdx[d] = __ldg(eg + d);
            J = __ldg(eg + 3);
            // wJ = wr[i]*ws[j]*wt[k]*J (lobattocells.jl:3231), MJI = 1 ./ MJ (dgsem.jl:56)
            wJ = A.w[id[0]];
#pragma unroll
            for (int d = 1; d < DIM; ++d) wJ = wJ * A.w[id[d]];
            wJ = wJ * J;
            mji = 1.0 / wJ;
#pragma unroll
            for (int d = 0; d < DIM; ++d) lg[d] = (T)(wJ * drdx[d]);
        } else {
            const double* vg = P.vgeo + (size_t)e * (DIM * DIM + 2) * NP;  // fields: wJ*dRdX rows, MJI, MJ
#pragma unroll
            for (int c = 0; c < DIM * DIM; ++c) lg[c] = (T)__ldg(vg + c * NP + n);
            mji = __ldg(vg + DIM * DIM * NP + n);
        }
#pragma unroll
        for (int c = 0; c < NLG; ++c) lgs[c * NP + n] = lg[c];

        // ---- per-node values for the partners ----
        if constexpr (COMBO == ADV_WEAK) {
#pragma unroll
            for (int dir = 0; dir < DIM; ++dir) {
                T v;
                if constexpr (AFF) {
                    // l_F = (dRdX[dir,dir] * f[dir]) * MJ  (dgsem.jl:299-308)
                    v = ((T)drdx[dir] * ((T)A.adv[dir] * q[0])) * (T)wJ;
                } else {
                    T acc = T(0);
#pragma unroll
                    for (int dd = 0; dd < DIM; ++dd) acc += lg[dir * DIM + dd] * ((T)A.adv[dd] * q[0]);
                    v = acc;
                }
                own[dir] = v;
            }
        } else if constexpr (COMBO == ADV_FDC) {
            own[0] = q[0] * T(0.5);
        } else {
            const T rho = q[0];
            const T rhoe = q[DIM + 1];
            T u[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) u[d] = q[1 + d] / rho;
            T rr = q[1] * q[1];
#pragma unroll
            for (int d = 1; d < DIM; ++d) rr = rr + q[1 + d] * q[1 + d];
            const T gm1 = (T)(A.gamma - 1.0);
            const T p = gm1 * (rhoe - rr / (T(2) * rho));
            if constexpr (COMBO == EUL_KG) {
                own[0] = rho * T(0.5);
#pragma unroll
                for (int d = 0; d < DIM; ++d) own[1 + d] = u[d] * T(0.5);
                own[DIM + 1] = (rhoe / rho) * T(0.5);
                own[DIM + 2] = p * T(0.5);
            } else if constexpr (COMBO == EUL_EC) {
                own[0] = rho;
#pragma unroll
                for (int d = 0; d < DIM; ++d) own[1 + d] = u[d];
                own[DIM + 1] = rho / (T(2) * p);
                T uu = u[0] * u[0];
#pragma unroll
                for (int d = 1; d < DIM; ++d) uu = uu + u[d] * u[d];
                own[DIM + 2] = uu;
            } else {
                // physical flux F[d][s] (euler.jl:50-61)
                T F[DIM][NS];
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    F[d][0] = q[1 + d];
#pragma unroll
                    for (int b = 0; b < DIM; ++b) F[d][1 + b] = (d == b) ? q[1 + d] * u[b] + p : q[1 + d] * u[b];
                    F[d][DIM + 1] = u[d] * (rhoe + p);
                }
                if constexpr (COMBO == EUL_FDC) {
#pragma unroll
                    for (int d = 0; d < DIM; ++d)
#pragma unroll
                        for (int s = 0; s < NS; ++s) own[d * NS + s] = F[d][s] * T(0.5);
                } else {  // EUL_WEAK: l_F[dir][s] = MJ * sum_dd dRdX[dir,dd] F[dd,s]
#pragma unroll
                    for (int dir = 0; dir < DIM; ++dir)
#pragma unroll
                        for (int s = 0; s < NS; ++s) {
                            if constexpr (AFF) {
                                own[dir * NS + s] = ((T)drdx[dir] * F[dir][s]) * (T)wJ;
                            } else {
                                T acc = T(0);
#pragma unroll
                                for (int dd = 0; dd < DIM; ++dd) acc += lg[dir * DIM + dd] * F[dd][s];
                                own[dir * NS + s] = acc;
                            }
                        }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < NAUX; ++k) aux[k * NP + n] = own[k];
    }
    if (!pf.tables_ready)
        for (int i = tid; i < NQ * NQ; i += S::THREADS) sD[i] = (T)A.D[i];
    __syncthreads();
    if (!active) return;

    // ------------------------------------------------------------------ volume term
    T acc[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) acc[s] = T(0);
    const int dmask = A.dir_mask ? A.dir_mask : 7;  // DGSEM(; directions)

#pragma unroll
    for (int dir = 0; dir < DIM; ++dir) {
        if (!((dmask >> dir) & 1)) continue;
        const int stride = dir == 0 ? 1 : (dir == 1 ? NQ : NQ * NQ);
        const int idd = id[dir];
        const int base = n - idd * stride;
#pragma unroll
        for (int a = 0; a < NQ; ++a) {
            const int na = base + a * stride;
            // D[a, id]: FP32 from shared memory (measured faster), FP64 from the parameters
            const T Dai = sizeof(T) == 4 ? sD[a + NQ * idd] : (T)A.D[a + NQ * idd];
            if constexpr (COMBO == ADV_WEAK) {
                acc[0] += Dai * aux[dir * NP + na];
            } else if constexpr (COMBO == EUL_WEAK) {
#pragma unroll
                for (int s = 0; s < NS; ++s) acc[s] += Dai * aux[(dir * NS + s) * NP + na];
            } else {
                const T Dia = sizeof(T) == 4 ? sD[idd + NQ * a] : (T)A.D[idd + NQ * a];  // D[id, a]
                // metric combination G_d = D[a,id] l_g[a][d] - D[id,a] l_g[i][d]
                T G[DIM];
                if constexpr (AFF) {
#pragma unroll
                    for (int d = 0; d < DIM; ++d) G[d] = T(0);
                    G[dir] = sub_rn(mul_rn(Dai, lgs[dir * NP + na]), mul_rn(Dia, lg[dir]));
                } else {
#pragma unroll
                    for (int d = 0; d < DIM; ++d)
                        G[d] = sub_rn(mul_rn(Dai, lgs[(dir * DIM + d) * NP + na]), mul_rn(Dia, lg[dir * DIM + d]));
                }
                if constexpr (COMBO == ADV_FDC) {
                    T aG = (T)A.adv[0] * G[0];
#pragma unroll
                    for (int d = 1; d < DIM; ++d) aG += (T)A.adv[d] * G[d];
                    acc[0] += (own[0] + aux[na]) * aG;
                } else if constexpr (COMBO == EUL_FDC) {
#pragma unroll
                    for (int s = 0; s < NS; ++s) {
                        T v = T(0);
#pragma unroll
                        for (int d = 0; d < DIM; ++d) v += (own[d * NS + s] + aux[(d * NS + s) * NP + na]) * G[d];
                        acc[s] += v;
                    }
                } else if constexpr (COMBO == EUL_KG) {
                    const T rb = own[0] + aux[na];
                    T ub[DIM];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) ub[d] = own[1 + d] + aux[(1 + d) * NP + na];
                    const T eb = own[DIM + 1] + aux[(DIM + 1) * NP + na];
                    const T pb = own[DIM + 2] + aux[(DIM + 2) * NP + na];
                    T un;
                    if constexpr (AFF) {
                        un = ub[dir] * G[dir];
                    } else {
                        un = ub[0] * G[0];
#pragma unroll
                        for (int d = 1; d < DIM; ++d) un += ub[d] * G[d];
                    }
                    const T f1 = rb * un;
                    acc[0] += f1;
#pragma unroll
                    for (int b = 0; b < DIM; ++b) {
                        if (AFF && b != dir) acc[1 + b] += f1 * ub[b];
                        else acc[1 + b] += f1 * ub[b] + pb * G[b];
                    }
                    acc[DIM + 1] += un * (rb * eb + pb);
                } else {  // EUL_EC
                    const T r2 = aux[na];
                    T u2[DIM], ua[DIM];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        u2[d] = aux[(1 + d) * NP + na];
                        ua[d] = (own[1 + d] + u2[d]) * T(0.5);
                    }
                    const T b2 = aux[(DIM + 1) * NP + na];
                    const T uu2 = aux[(DIM + 2) * NP + na];
                    const T ra = (own[0] + r2) * T(0.5);
                    const T ba = (own[DIM + 1] + b2) * T(0.5);
                    const T u2a = (own[DIM + 2] + uu2) * T(0.5);
                    const T rlog = logavg(own[0], r2);
                    const T blog = logavg(own[DIM + 1], b2);
                    const T pt = ra / (T(2) * ba);
                    const T c = T(1) / ((T(2) * (T)(A.gamma - 1.0)) * blog) - u2a * T(0.5);
                    T un = ua[0] * G[0], uaa = ua[0] * ua[0];
#pragma unroll
                    for (int d = 1; d < DIM; ++d) {
                        un += ua[d] * G[d];
                        uaa += ua[d] * ua[d];
                    }
                    const T f0 = rlog * un;
                    acc[0] += f0;
#pragma unroll
                    for (int b = 0; b < DIM; ++b) acc[1 + b] += f0 * ua[b] + pt * G[b];
                    acc[DIM + 1] += un * (c * rlog + rlog * uaa + pt);
                }
            }
        }
    }

    // ------------------------------------------------------------- combine with dq
    const T mjiT = (T)mji;
    const bool stage = A.mode >= MODE_STAGE;
    const size_t node0 = (size_t)e * NS * NP + n;
    T t[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        T v = acc[s] * mjiT;
        if (A.mode == MODE_STAGE) {
            T old;
            if (pf.dq) old = static_cast<const T*>(pf.dq)[s * pf.stride];
            else if (sizeof(T) == 4) old = (T) reinterpret_cast<const float*>(P.dq)[node0 + s * NP];
            else old = (T) reinterpret_cast<const double*>(P.dq)[node0 + s * NP];
            v = (T)A.rka * old + v;
        } else if (A.mode == MODE_TENDENCY_INC) {
            v = (T)(reinterpret_cast<const double*>(P.dq)[node0 + s * NP] + (double)v);
        }
        t[s] = v;
    }

    // ---------------------------------------------------------------- surface term
#pragma unroll
    for (int dir = 0; dir < DIM; ++dir) {
        const int idd = id[dir];
        if (idd != 0 && idd != NQ - 1) continue;
        if (!((dmask >> dir) & 1)) continue;
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            if ((side == 0 && idd != 0) || (side == 1 && idd != NQ - 1)) continue;
            const int f = 2 * dir + side;
            const int stride = dir == 0 ? 1 : (dir == 1 ? NQ : NQ * NQ);
            const int ne = __ldg(P.nbr + (size_t)NF * e + f);
            // in-face index of this node (column-major over the face dims)
            int j;
            if (DIM == 1) j = 0;
            else if (DIM == 2) j = (dir == 0) ? id[1] : id[0];
            else j = (dir == 0) ? id[1] + NQ * id[2] : (dir == 1 ? id[0] + NQ * id[2] : id[0] + NQ * id[1]);
            T qp[NS];
            if (ne >= 0) {
                const double* qn;
                if (!AFF && P.vmapP) {
                    // qP = q[vmapP] (dgsem.jl:756-770): the neighbour's node may sit on any of
                    // its faces, in any orientation
                    const int32_t gn = __ldg(P.vmapP + ((size_t)e * NF + f) * NFP + j);
                    const int32_t en = gn / NP;
                    qn = P.q_in + (size_t)en * NS * NP + (gn - en * NP);
                } else {
                    const int nn = n + (side == 0 ? (NQ - 1) * stride : -(NQ - 1) * stride);
                    qn = P.q_in + (size_t)ne * NS * NP + nn;
                }
#pragma unroll
                for (int s = 0; s < NS; ++s) qp[s] = (T)__ldg(qn + s * NP);
            } else {
#pragma unroll
                for (int s = 0; s < NS; ++s) qp[s] = q[s];  // default boundarystate (balancelaw.jl:77)
            }
            T nv[DIM];
            double wsJ;
            if constexpr (AFF) {
                // hexsurfacemetrics! on an unwarped brick (lobattocells.jl:3278-3291)
                const double sJ = fabs(J * drdx[dir]);
#pragma unroll
                for (int d = 0; d < DIM; ++d) nv[d] = T(0);
                nv[dir] = side == 0 ? T(-1) : T(1);
                if (DIM == 1) wsJ = sJ;  // one node a face: weight 1 (lobattocells.jl:2656)
                else if (DIM == 2) wsJ = sJ * A.w[dir == 0 ? id[1] : id[0]];
                else {
                    const int i1 = dir == 0 ? id[1] : id[0];
                    const int i2 = dir == 2 ? id[1] : id[2];
                    wsJ = (sJ * A.w[i1]) * A.w[i2];
                }
            } else {
                const double* sg = P.sgeo + ((size_t)e * NF * NFP + (size_t)f * NFP + j) * (DIM + 1);
#pragma unroll
                for (int d = 0; d < DIM; ++d) nv[d] = (T)__ldg(sg + d);
                wsJ = __ldg(sg + DIM);
            }
            if (ne <= -kBcBase) {  // a boundary tag with its own boundarystate
                const int tag = -ne - kBcBase;
                if (A.bc_kind[tag] == BC_PRESCRIBED) {
#pragma unroll
                    for (int s = 0; s < NS; ++s) qp[s] = (T)A.bc_state[tag][s];
                } else if constexpr (!C::ADV) {
                    if (A.bc_kind[tag] == BC_WALL) {
                        // reflecting wall: rho u+ = rho u- - 2 (n . rho u-) n
                        T mn = nv[0] * q[1];
#pragma unroll
                        for (int d = 1; d < DIM; ++d) mn += nv[d] * q[1 + d];
#pragma unroll
                        for (int d = 0; d < DIM; ++d) qp[1 + d] = q[1 + d] - (T(2) * mn) * nv[d];
                    }
                }
            }
            T nf[NS];
            if (ne == -2) {  // mortar face of an adapted grid: the flux comes from the mortar kernel
#pragma unroll
                for (int s = 0; s < NS; ++s) nf[s] = (T)__ldg(P.ncflux + (((size_t)e * NF + f) * NS + s) * NFP + j);
            } else if constexpr (SF == 1 && !C::ADV) {
                euler_entropy_surface_flux<DIM, T>(A.surface_flux, nv, q, qp, (T)A.gamma, nf);
            } else if constexpr (C::ADV) {
                T an;
                if constexpr (AFF) an = (T)A.adv[dir] * nv[dir];
                else {
                    an = (T)A.adv[0] * nv[0];
#pragma unroll
                    for (int d = 1; d < DIM; ++d) an += (T)A.adv[d] * nv[d];
                }
                const T fc = (an * q[0] + an * qp[0]) * T(0.5);
                nf[0] = A.surface_rusanov ? fc - (fabs(an) * (qp[0] - q[0])) * T(0.5) : fc;
            } else {
                // Rusanov: central flux of the physical fluxes, minus the max wave speed jump
                // (numericalfluxes.jl:44-50, euler.jl:50-68)
                const T gm1 = (T)(A.gamma - 1.0);
                T Fn[2][NS], ws[2];
#pragma unroll
                for (int side2 = 0; side2 < 2; ++side2) {
                    const T* qq = side2 == 0 ? q : qp;
                    const T rho = qq[0], rhoe = qq[DIM + 1];
                    T u[DIM];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) u[d] = qq[1 + d] / rho;
                    T rr = qq[1] * qq[1];
#pragma unroll
                    for (int d = 1; d < DIM; ++d) rr = rr + qq[1 + d] * qq[1 + d];
                    const T p = gm1 * (rhoe - rr / (T(2) * rho));
                    T un, mn;
                    if constexpr (AFF) {
                        un = u[dir] * nv[dir];
                        mn = qq[1 + dir] * nv[dir];
                    } else {
                        un = u[0] * nv[0];
                        mn = qq[1] * nv[0];
#pragma unroll
                        for (int d = 1; d < DIM; ++d) {
                            un += u[d] * nv[d];
                            mn += qq[1 + d] * nv[d];
                        }
                    }
                    Fn[side2][0] = mn;
#pragma unroll
                    for (int b = 0; b < DIM; ++b) Fn[side2][1 + b] = mn * u[b] + p * nv[b];
                    Fn[side2][DIM + 1] = un * (rhoe + p);
                    ws[side2] = fabs(un) + dev_sqrt((T)A.gamma * p / rho);
                }
                const T mx = fmax(ws[0], ws[1]);
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    const T fc = (Fn[0][s] + Fn[1][s]) * T(0.5);
                    nf[s] = A.surface_rusanov ? fc - (mx * (qp[s] - q[s])) * T(0.5) : fc;
                }
            }
            const T wsJT = (T)wsJ;
#pragma unroll
            for (int s = 0; s < NS; ++s) t[s] = t[s] - (wsJT * nf[s]) * mjiT;
        }
    }

    // ----------------------------------------------------------------- write back
    if (stage) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            if (sizeof(T) == 4) reinterpret_cast<float*>(P.dq)[node0 + s * NP] = (float)t[s];
            else reinterpret_cast<double*>(P.dq)[node0 + s * NP] = (double)t[s];
            P.q_out[node0 + s * NP] = qd[s] + P.rkb_dt * (double)t[s];
        }
    } else {
#pragma unroll
        for (int s = 0; s < NS; ++s) reinterpret_cast<double*>(P.dq)[node0 + s * NP] = (double)t[s];
    }
}

// Shared memory of the generic kernels: stage_element's arrays and, where the state and
// register are prefetched (PF), two buffers of per-thread slots (FP64 state, T register).
// Prefetching pays on 3-D elements in FP32 bulk (measured: 1.2-1.4x at Nq = 4 and 6);
// 2-D elements and FP64 keep one group per CTA with direct loads, which measured faster.
template <int DIM, int NQ, int COMBO, int GEOM, typename T, int EPBX = 0>
struct PersistentCfg {
    using S = Shape<DIM, NQ, EPBX>;
    using K = KernelCfg<DIM, NQ, COMBO, GEOM, T, EPBX>;
    static constexpr bool PF = DIM == 3 && sizeof(T) == 4;
    static constexpr int NS = CSize<COMBO, DIM>::NS;
    static constexpr size_t off_q = (K::smem + 15) / 16 * 16;
    static constexpr size_t off_dq = off_q + (size_t)2 * NS * S::THREADS * sizeof(double);
    static constexpr size_t smem = PF ? off_dq + (size_t)2 * NS * S::THREADS * sizeof(T) : K::smem;
    // CTAs per SM the registers are sized for: about 768 resident threads per SM when the
    // kernel loops over groups with prefetches (the loop otherwise lets the compiler keep
    // more values live than one group needs, at the cost of residency)
#ifndef RB200_ADV_TARGET
#define RB200_ADV_TARGET 2048
#endif
    static constexpr int TARGET = NS == 1 ? RB200_ADV_TARGET : 768;
    static constexpr int MIN_CTAS = PF && S::THREADS < TARGET ? TARGET / S::THREADS : 1;
};

// Generic stage kernel.  Without prefetch (PC::PF false) one CTA runs one group of EPB
// elements.  With it, each CTA walks element groups blockIdx.x + k*gridDim.x; while a
// group runs, every thread copies the state (and, in stage mode, the LSRK register) of
// its node in the CTA's next group into its own shared-memory slots with cp.async, so
// those loads overlap the current group's arithmetic.  A thread reads only slots it
// filled itself, so the copies need no barrier.
template <int DIM, int NQ, int COMBO, int GEOM, typename T, int SF>
__global__ void __launch_bounds__(Shape<DIM, NQ>::THREADS, (PersistentCfg<DIM, NQ, COMBO, GEOM, T>::MIN_CTAS))
    stage_kernel(const __grid_constant__ StageArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using S = Shape<DIM, NQ>;
    using PC = PersistentCfg<DIM, NQ, COMBO, GEOM, T>;
    if constexpr (!PC::PF) {
        const int64_t e = A.e_begin + (int64_t)blockIdx.x * S::EPB + threadIdx.x / S::NP;
        stage_element<DIM, NQ, COMBO, GEOM, T, 0, SF>(A, elem_ptrs(A), e, e < A.E, smem_raw);
        return;
    }
    constexpr int NS = PC::NS, TH = S::THREADS, NP = S::NP;
    double* qs = reinterpret_cast<double*>(smem_raw + PC::off_q);  // [2][NS][TH]
    T* dqs = reinterpret_cast<T*>(smem_raw + PC::off_dq);           // [2][NS][TH]
    const int tid = threadIdx.x, el = tid / NP, n = tid - el * NP;
    const bool pf_dq = A.mode == MODE_STAGE;
    const int64_t ngroups = (A.E - A.e_begin + S::EPB - 1) / S::EPB;
    const ElemPtrs P = elem_ptrs(A);
    auto prefetch = [&](int64_t g, int b) {
        const int64_t e = A.e_begin + g * S::EPB + el;
        if (g < ngroups && e < A.E) {
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const size_t gi = ((size_t)e * NS + s) * NP + n;
                cpa8(qs + (b * NS + s) * TH + tid, A.q_in + gi);
                if (pf_dq) {
                    if constexpr (sizeof(T) == 4) cpa4(dqs + (b * NS + s) * TH + tid, static_cast<const float*>(A.dq) + gi);
                    else cpa8(dqs + (b * NS + s) * TH + tid, static_cast<const double*>(A.dq) + gi);
                }
            }
        }
        cpa_commit();
    };
    prefetch(blockIdx.x, 0);
    int b = 0;
    for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x, b ^= 1) {
        cpa_wait_all();                  // this group's values (issued one iteration ago)
        prefetch(g + gridDim.x, b ^ 1);  // the next group's, into the other buffer
        const int64_t e = A.e_begin + g * S::EPB + el;
        Prefetched pf;
        pf.q = qs + b * NS * TH + tid;
        pf.dq = pf_dq ? static_cast<const void*>(dqs + b * NS * TH + tid) : nullptr;
        pf.stride = TH;
        pf.tables_ready = g != blockIdx.x;
        stage_element<DIM, NQ, COMBO, GEOM, T, 0, SF>(A, P, e, e < A.E, smem_raw, pf);
        __syncthreads();  // the shared partner values are reused by the next group
    }
    cpa_wait_all();
}

template <int DIM, int NQ, int COMBO, int GEOM, typename T, int SF = 0>
cudaError_t launch_one(const StageArgs& a, cudaStream_t st) {
    using S = Shape<DIM, NQ>;
    using PC = PersistentCfg<DIM, NQ, COMBO, GEOM, T>;
    auto kern = stage_kernel<DIM, NQ, COMBO, GEOM, T, SF>;
    static std::atomic<uint64_t> configured{0};
    cudaError_t err = ensure_smem_limit(kern, (int)PC::smem, configured);
    if (err != cudaSuccess) return err;
    const int64_t groups = (a.E - a.e_begin + S::EPB - 1) / S::EPB;
    if (groups <= 0) return cudaSuccess;
    if constexpr (!PC::PF) {
        kern<<<(unsigned)groups, S::THREADS, PC::smem, st>>>(a);
        return cudaGetLastError();
    }
    // persistent grid: the resident CTAs of every SM, cached per device
    static std::atomic<int> grid_of_device[64];
    int dev = 0;
    if ((err = cudaGetDevice(&dev)) != cudaSuccess) return err;
    int grid = (dev >= 0 && dev < 64) ? grid_of_device[dev].load(std::memory_order_relaxed) : 0;
    if (grid <= 0) {
        int per_sm = 0, nsm = 0;
        if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, S::THREADS, PC::smem)) != cudaSuccess)
            return err;
        if ((err = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return err;
        grid = per_sm > 0 ? per_sm * nsm : 1;
        if (dev >= 0 && dev < 64) grid_of_device[dev].store(grid, std::memory_order_relaxed);
    }
    kern<<<(unsigned)std::min<int64_t>(grid, groups), S::THREADS, PC::smem, st>>>(a);
    return cudaGetLastError();
}

// Small grids: every stage of every step of an LSRK call in one launch of one
// thread-block cluster (weak-form advection on unwarped bricks).  On a grid that one pass
// of a few CTAs covers (a 16^2, N=4 grid has 6400 nodes) a stage launch is mostly launch
// latency and dependent trips to L2.  Here CTA r of the cluster owns elements
// e_begin + r*EPB .. +EPB-1 (one node a thread, up to kClusterNodes a CTA) for the whole
// call: a thread keeps its node's state and LSRK register in registers, the CTA keeps its
// elements' state of the current stage in shared memory (two buffers by stage parity),
// the volume term reads the element's own nodes there, and the surface term reads the
// neighbour's trace from the shared memory of the CTA that owns it (distributed shared
// memory).  One hardware cluster barrier a stage (arrive.release / wait.acquire) orders
// a stage's shared-memory writes before the next stage's reads.  Global memory is read
// at the start and written at the end only.  The arithmetic per node is that of
// stage_element_adv_brick, expression for expression, so the results are bit for bit
// those of the stage launches.
template <int DIM, int NQ>
struct ClusterShape {
    static constexpr int NP = IPow<NQ, DIM>::v;
    static constexpr int EPB = NP >= kClusterNodes ? 1 : kClusterNodes / NP;
    using S = Shape<DIM, NQ, EPB>;
    static constexpr size_t smem = (size_t)(2 * EPB * NP + NQ * NQ) * sizeof(double);
};

__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// The address of `p` (this CTA's shared memory) in the shared memory of cluster CTA `rank`.
template <typename T>
__device__ __forceinline__ const T* cluster_peer(const T* p, unsigned rank) {
    uint64_t out;
    asm("mapa.u64 %0, %1, %2;" : "=l"(out) : "l"(reinterpret_cast<uint64_t>(p)), "r"(rank));
    return reinterpret_cast<const T*>(out);
}

template <int DIM, int NQ, typename T>
__global__ void __launch_bounds__(ClusterShape<DIM, NQ>::S::THREADS, 1)
    cluster_adv_steps_kernel(const __grid_constant__ ClusterStepsArgs C) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using CS = ClusterShape<DIM, NQ>;
    constexpr int NP = CS::NP, EPB = CS::EPB, NF = 2 * DIM, TH = CS::S::THREADS;
    T* sq = reinterpret_cast<T*>(smem_raw);  // [2][EPB * NP]: the CTA's elements, by stage parity
    T* sW = sq + 2 * EPB * NP;               // W[a + NQ i]
    const StageArgs& A = C.a;
    const int tid = threadIdx.x;
    const int el = tid / NP;
    const int n = tid - el * NP;
    const int64_t e = A.e_begin + (int64_t)blockIdx.x * EPB + el;
    const bool active = e < A.E;
    int id[3];
    id[0] = n % NQ;
    id[1] = DIM > 1 ? (n / NQ) % NQ : 0;
    id[2] = DIM > 2 ? n / (NQ * NQ) : 0;
    for (int i = tid; i < NQ * NQ; i += TH) {
        const int a = i % NQ, ii = i / NQ;
        sW[i] = (T)(A.D[a + NQ * ii] * (A.w[a] / A.w[ii]));
    }
    const int dmask = A.dir_mask ? A.dir_mask : 7;
    const size_t node0 = (size_t)e * NP + n;
    double qd = 0.0, drdx[3] = {0.0, 0.0, 0.0};
    T dqv = T(0);
    int32_t nb[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) nb[f] = -1;
    if (active) {
        qd = C.q[node0];
        if (C.rka[0] != 0.0) {  // a table whose first stage reads the register
            if (sizeof(T) == 4) dqv = (T) reinterpret_cast<const float*>(A.dq)[node0];
            else dqv = (T) reinterpret_cast<const double*>(A.dq)[node0];
        }
        const double* eg = A.elem_geo + 4 * e;
#pragma unroll
        for (int d = 0; d < DIM; ++d) drdx[d] = __ldg(eg + d);
#pragma unroll
        for (int f = 0; f < NF; ++f) nb[f] = __ldg(A.nbr + (size_t)NF * e + f);
        sq[el * NP + n] = (T)qd;
    }
    cluster_barrier();  // every CTA's first-stage state is in its shared memory
    int b = 0;
    for (int32_t step = 0; step < C.nsteps; ++step) {
        for (int stg = 0; stg < C.nstages; ++stg) {
            const T* cur = sq + b * EPB * NP;
            if (active) {
                const T q0 = (T)qd;
                const T* qe = cur + el * NP;
                // ---- volume term
                T acc = T(0);
#pragma unroll
                for (int dir = 0; dir < DIM; ++dir) {
                    if (!((dmask >> dir) & 1)) continue;
                    const int stride = dir == 0 ? 1 : (dir == 1 ? NQ : NQ * NQ);
                    const int idd = id[dir];
                    const int base = n - idd * stride;
                    T sum = T(0);
#pragma unroll
                    for (int a = 0; a < NQ; ++a) sum += sW[a + NQ * idd] * qe[base + a * stride];
                    acc += ((T)drdx[dir] * (T)A.adv[dir]) * sum;
                }
                // ---- combine with dq
                const double rka = C.rka[stg];
                T v = acc;
                if (rka != 0.0) v = (T)rka * dqv + v;
                // ---- surface term, faces in the order x-, x+, y-, y+, z-, z+ (dgsem.jl:756-782)
#pragma unroll
                for (int dir = 0; dir < DIM; ++dir) {
                    const int idd = id[dir];
                    if (idd != 0 && idd != NQ - 1) continue;
                    if (!((dmask >> dir) & 1)) continue;
                    const int side = idd == 0 ? 0 : 1;
                    const int stride = dir == 0 ? 1 : (dir == 1 ? NQ : NQ * NQ);
                    const int ne = side == 0 ? nb[2 * dir] : nb[2 * dir + 1];  // registers, not a stack array
                    T qp = q0;  // default boundarystate (balancelaw.jl:77)
                    if (ne >= 0) {
                        const int nn = n + (side == 0 ? (NQ - 1) * stride : -(NQ - 1) * stride);
                        const int64_t rel = ne - A.e_begin;
                        const T* peer = cluster_peer(cur, (unsigned)(rel / EPB));
                        qp = peer[(rel % EPB) * NP + nn];
                    } else if (ne <= -kBcBase && A.bc_kind[-ne - kBcBase] == BC_PRESCRIBED) {
                        qp = (T)A.bc_state[-ne - kBcBase][0];
                    }
                    const T an = (T)A.adv[dir] * (side == 0 ? T(-1) : T(1));
                    const T fc = (an * q0 + an * qp) * T(0.5);
                    const T nf = A.surface_rusanov ? fc - (fabs(an) * (qp - q0)) * T(0.5) : fc;
                    v = v - nf * (T)(fabs(drdx[dir]) / A.w[0]);
                }
                dqv = v;
                qd = qd + C.rkb_dt[stg] * (double)v;
                sq[(b ^ 1) * EPB * NP + el * NP + n] = (T)qd;
            }
            cluster_barrier();  // this stage's reads done and the next stage's state written
            b ^= 1;
        }
    }
    if (active) {
        C.q[node0] = qd;
        if (sizeof(T) == 4) reinterpret_cast<float*>(A.dq)[node0] = (float)dqv;
        else reinterpret_cast<double*>(A.dq)[node0] = (double)dqv;
    }
}

// One cluster of `ctas` CTAs (1..kClusterCtas) runs c.nsteps steps of c.nstages stages.
template <int DIM, int NQ, typename T>
cudaError_t launch_cluster_adv(const ClusterStepsArgs& c, int ctas, cudaStream_t st) {
    using CS = ClusterShape<DIM, NQ>;
    if (ctas < 1 || ctas > kClusterCtas) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ctas, 1, 1);
    cfg.blockDim = dim3(CS::S::THREADS, 1, 1);
    cfg.dynamicSmemBytes = CS::smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)ctas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    auto kern = cluster_adv_steps_kernel<DIM, NQ, T>;
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= 64) return cudaErrorNotSupported;  // the caches below hold 64 devices
    if (kClusterCtas > 8) {  // sizes above the portable 8 need the kernel's opt-in, per device
        static std::atomic<uint64_t> opted{0};
        const uint64_t bit = uint64_t{1} << dev;
        if (!(opted.load(std::memory_order_acquire) & bit)) {
            err = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            if (err != cudaSuccess) return err;
            opted.fetch_or(bit, std::memory_order_acq_rel);
        }
    }
    // whether a cluster of this size fits the device at all, asked once per device and
    // size; cudaErrorNotSupported tells the caller to run the steps as stage launches
    static std::atomic<uint8_t> fits[64][kClusterCtas + 1];  // 0 unknown, 1 yes, 2 no
    int f = fits[dev][ctas].load(std::memory_order_relaxed);
    if (f == 0) {
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) {
            cudaGetLastError();
            n = 0;
        }
        f = n > 0 ? 1 : 2;
        fits[dev][ctas].store((uint8_t)f, std::memory_order_relaxed);
    }
    if (f != 1) return cudaErrorNotSupported;
    err = cudaLaunchKernelEx(&cfg, kern, c);
    return err != cudaSuccess ? err : cudaGetLastError();
}

}  // namespace rb200
