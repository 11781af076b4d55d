// Mortar fluxes of an adapted (non-conforming) brick grid.
//
// The reference's surfaceterm! (src/balancelaws/dgsem.jl:733-784) leaves hanging faces
// uncoupled: a non-conforming face keeps vmapP = vmapM (lobattocells.jl:2073-2074), so
// its flux sees the element's own trace on both sides.  Here each hanging face is
// coupled to its 2^(dim-1) small neighbours by a mortar:
// * the large face's trace is interpolated to the nodes of each small face with the
//   tohalves operators (lobattocells.jl:16-17);
// * the surface flux is taken there with the large element's outward normal, and the
//   small element's face gets its negative;
// * the large face gets the lumped L2 projection of the small faces' fluxes, so the
//   flux integrals match and the coupling conserves.
// On a curved (warped) grid the small face's own geometry is used: the flux at a small
// face node is taken with the negative of that face's outward normal, and what is
// projected onto the large face is the flux scaled by the small face's surface measure,
// sigma_k = 2^(dim-1) wsJ_k / W (W the tensor LGL weight of the node), which is divided
// by the large face's sJ = wsJ_C / W afterwards.  With the projection's property
// W . (P g) = (W / 2^(dim-1)) . g this keeps sum wsJ_C * flux_C = sum_k sum wsJ_k *
// flux_k, i.e. the coupling conserves on curved faces too.
// The fluxes are left in a per-face buffer that the stage kernel subtracts like any
// other face flux (wsJ * nf * MJI).
//
// One CTA per mortar, one thread per (small face, face node).  All sums are fma chains
// in a fixed order, the same as the CPU restatement's.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "rb200_internal.h"
#include "surface_fluxes.cuh"

namespace rb200 {

namespace {

template <int N, int D>
struct Pow {
    static constexpr int v = N * Pow<N, D - 1>::v;
};
template <int N>
struct Pow<N, 0> {
    static constexpr int v = 1;
};

template <typename T>
__device__ __forceinline__ T dsqrt(T x) {
    return sqrt(x);
}

// Surface flux of the stage kernel at one node, normal n = sn e_dir (affine faces).
template <int DIM, bool EULER, typename T>
__device__ __forceinline__ void face_flux(const MortarArgs& A, int dir, T sn, const T* qm, const T* qp, T* nf) {
    constexpr int NS = EULER ? DIM + 2 : 1;
    if constexpr (!EULER) {
        const T an = (T)A.adv[dir] * sn;
        const T fc = (an * qm[0] + an * qp[0]) * T(0.5);
        nf[0] = A.surface_rusanov ? fc - (fabs(an) * (qp[0] - qm[0])) * T(0.5) : fc;
    } else if (A.surface_flux == kFluxKG || A.surface_flux == kFluxEC || A.surface_flux == kFluxRoe ||
               A.surface_flux == kFluxMatrix) {
        T n[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) n[d] = d == dir ? sn : T(0);
        euler_entropy_surface_flux<DIM, T>(A.surface_flux, n, qm, qp, (T)A.gamma, nf);
    } else {
        const T gm1 = (T)(A.gamma - 1.0);
        T Fn[2][NS], ws[2];
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const T* qq = side == 0 ? qm : qp;
            const T rho = qq[0], rhoe = qq[DIM + 1];
            T u[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) u[d] = qq[1 + d] / rho;
            T rr = qq[1] * qq[1];
#pragma unroll
            for (int d = 1; d < DIM; ++d) rr = rr + qq[1 + d] * qq[1 + d];
            const T p = gm1 * (rhoe - rr / (T(2) * rho));
            const T un = u[dir] * sn, mn = qq[1 + dir] * sn;
            Fn[side][0] = mn;
#pragma unroll
            for (int b = 0; b < DIM; ++b) Fn[side][1 + b] = mn * u[b] + (b == dir ? p * sn : T(0));
            Fn[side][DIM + 1] = un * (rhoe + p);
            ws[side] = fabs(un) + dsqrt((T)A.gamma * p / rho);
        }
        const T mx = fmax(ws[0], ws[1]);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const T fc = (Fn[0][s] + Fn[1][s]) * T(0.5);
            nf[s] = A.surface_rusanov ? fc - (mx * (qp[s] - qm[s])) * T(0.5) : fc;
        }
    }
}

// Surface flux with a general unit normal n (curved faces): the same fluxes as the
// stage kernel's face phase.
template <int DIM, bool EULER, typename T>
__device__ __forceinline__ void face_flux_n(const MortarArgs& A, const T* n, const T* qm, const T* qp, T* nf) {
    constexpr int NS = EULER ? DIM + 2 : 1;
    if constexpr (!EULER) {
        T an = (T)A.adv[0] * n[0];
#pragma unroll
        for (int d = 1; d < DIM; ++d) an += (T)A.adv[d] * n[d];
        const T fc = (an * qm[0] + an * qp[0]) * T(0.5);
        nf[0] = A.surface_rusanov ? fc - (fabs(an) * (qp[0] - qm[0])) * T(0.5) : fc;
    } else if (A.surface_flux == kFluxKG || A.surface_flux == kFluxEC || A.surface_flux == kFluxRoe ||
               A.surface_flux == kFluxMatrix) {
        euler_entropy_surface_flux<DIM, T>(A.surface_flux, n, qm, qp, (T)A.gamma, nf);
    } else {
        const T gm1 = (T)(A.gamma - 1.0);
        T Fn[2][NS], ws[2];
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const T* qq = side == 0 ? qm : qp;
            const T rho = qq[0], rhoe = qq[DIM + 1];
            T u[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) u[d] = qq[1 + d] / rho;
            T rr = qq[1] * qq[1];
#pragma unroll
            for (int d = 1; d < DIM; ++d) rr = rr + qq[1 + d] * qq[1 + d];
            const T p = gm1 * (rhoe - rr / (T(2) * rho));
            T un = u[0] * n[0], mn = qq[1] * n[0];
#pragma unroll
            for (int d = 1; d < DIM; ++d) {
                un += u[d] * n[d];
                mn += qq[1 + d] * n[d];
            }
            Fn[side][0] = mn;
#pragma unroll
            for (int b = 0; b < DIM; ++b) Fn[side][1 + b] = mn * u[b] + p * n[b];
            Fn[side][DIM + 1] = un * (rhoe + p);
            ws[side] = fabs(un) + dsqrt((T)A.gamma * p / rho);
        }
        const T mx = fmax(ws[0], ws[1]);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const T fc = (Fn[0][s] + Fn[1][s]) * T(0.5);
            nf[s] = A.surface_rusanov ? fc - (mx * (qp[s] - qm[s])) * T(0.5) : fc;
        }
    }
}

// Volume node of in-face index j on face f (x-, x+, y-, y+, z-, z+), lobattocells.jl:2012-2053.
template <int DIM, int NQ>
__device__ __forceinline__ int face_vol_node(int f, int j) {
    const int d = f >> 1, c = (f & 1) ? NQ - 1 : 0;
    if (DIM == 2) return d == 0 ? c + NQ * j : j + NQ * c;
    const int j1 = j % NQ, j2 = j / NQ;
    if (d == 0) return c + NQ * (j1 + NQ * j2);
    if (d == 1) return j1 + NQ * (c + NQ * j2);
    return j1 + NQ * (j2 + NQ * c);
}

template <int DIM, int NQ, bool EULER, typename T>
__global__ void __launch_bounds__((DIM == 3 ? 4 : 2) * Pow<NQ, DIM - 1>::v)
    mortar_kernel(const __grid_constant__ MortarArgs A) {
    constexpr int NS = EULER ? DIM + 2 : 1;
    constexpr int NP = Pow<NQ, DIM>::v, NFP = Pow<NQ, DIM - 1>::v, NF = 2 * DIM;
    constexpr int NSMALL = DIM == 3 ? 4 : 2, MCOLS = 2 + NSMALL;
    constexpr int NQ2 = DIM == 3 ? NQ : 1;  // second in-face direction (none in 2-D)
    __shared__ T qC[NS][NFP];
    __shared__ T nfm[NSMALL][NS][NFP];
    const int t = threadIdx.x;
    const int k = t / NFP, j = t - k * NFP;
    const int j1 = j % NQ, j2 = j / NQ;
    grid_dependency_wait();  // the stage that wrote A.q, and read A.ncflux, has completed
    for (int64_t m = blockIdx.x; m < A.M; m += gridDim.x) {
        const int64_t* col = A.mortars + (size_t)MCOLS * m;
        const int64_t eC = col[0];
        const int fC = (int)col[1], fF = fC ^ 1, dir = fC >> 1;
        const T sn = (fC & 1) ? T(1) : T(-1);
        if (t < NFP) {
            const int v = face_vol_node<DIM, NQ>(fC, t);
#pragma unroll
            for (int s = 0; s < NS; ++s) qC[s][t] = (T)__ldg(A.q + ((size_t)eC * NS + s) * NP + v);
        }
        __syncthreads();
        {
            const int64_t eF = col[2 + k];
            const double* Ia = (k & 1) ? A.IU : A.IL;
            const double* Ib = (k >> 1) ? A.IU : A.IL;
            T qi[NS], qf[NS], nf[NS];
            const int v = face_vol_node<DIM, NQ>(fF, j);
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                T acc = T(0);
#pragma unroll
                for (int b = 0; b < NQ2; ++b) {
                    T tt = T(0);
#pragma unroll
                    for (int a = 0; a < NQ; ++a) tt = fma((T)Ia[j1 * NQ + a], qC[s][a + NQ * b], tt);
                    acc = fma(DIM == 3 ? (T)Ib[j2 * NQ + b] : T(1), tt, acc);
                }
                qi[s] = acc;
                qf[s] = (T)__ldg(A.q + ((size_t)eF * NS + s) * NP + v);
            }
            if (A.sgeo) {
                // curved: the small face's own normal, flipped to point out of the large
                // element, and its surface measure for the projection
                const double* sg = A.sgeo + (((size_t)eF * NF + fF) * NFP + j) * (DIM + 1);
                T n[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) n[d] = -(T)__ldg(sg + d);
                face_flux_n<DIM, EULER, T>(A, n, qi, qf, nf);
                const double W = DIM == 3 ? A.w[j1] * A.w[j2] : A.w[j1];
                const T sigma = (T)((double)NSMALL * __ldg(sg + DIM) / W);
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    nfm[k][s][j] = sigma * nf[s];
                    A.ncflux[(((size_t)eF * NF + fF) * NS + s) * NFP + j] = -(double)nf[s];
                }
            } else {
                face_flux<DIM, EULER, T>(A, dir, sn, qi, qf, nf);
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    nfm[k][s][j] = nf[s];
                    A.ncflux[(((size_t)eF * NF + fF) * NS + s) * NFP + j] = -(double)nf[s];
                }
            }
        }
        __syncthreads();
        if (t < NFP) {
            // curved: divide by the large face's sJ = wsJ_C / W
            T unscale = T(1);
            if (A.sgeo) {
                const double W = DIM == 3 ? A.w[j1] * A.w[j2] : A.w[j1];
                unscale = (T)(W / __ldg(A.sgeo + (((size_t)eC * NF + fC) * NFP + t) * (DIM + 1) + DIM));
            }
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                T acc = T(0);
#pragma unroll
                for (int kk = 0; kk < NSMALL; ++kk) {
                    const double* Pa = (kk & 1) ? A.PU : A.PL;
                    const double* Pb = (kk >> 1) ? A.PU : A.PL;
#pragma unroll
                    for (int b = 0; b < NQ2; ++b) {
                        T tt = T(0);
#pragma unroll
                        for (int a = 0; a < NQ; ++a) tt = fma((T)Pa[j1 * NQ + a], nfm[kk][s][a + NQ * b], tt);
                        acc = fma(DIM == 3 ? (T)Pb[j2 * NQ + b] : T(1), tt, acc);
                    }
                }
                if (A.sgeo) acc = acc * unscale;
                A.ncflux[(((size_t)eC * NF + fC) * NS + s) * NFP + t] = (double)acc;
            }
        }
        __syncthreads();  // qC and nfm are reused by the next mortar of this CTA
    }
}

template <int DIM, int NQ, bool EULER>
cudaError_t launch_t(int fp32, const MortarArgs& a, cudaStream_t s) {
    constexpr int threads = (DIM == 3 ? 4 : 2) * Pow<NQ, DIM - 1>::v;
    const int grid = (int)std::min<int64_t>(a.M, 148 * 16);
    if (grid <= 0) return cudaSuccess;
    if (fp32) return launch_pdl(mortar_kernel<DIM, NQ, EULER, float>, grid, threads, 0, s, a);
    return launch_pdl(mortar_kernel<DIM, NQ, EULER, double>, grid, threads, 0, s, a);
}

template <int DIM, bool EULER>
cudaError_t launch_nq(int nq, int fp32, const MortarArgs& a, cudaStream_t s) {
    switch (nq) {
        case 2: return launch_t<DIM, 2, EULER>(fp32, a, s);
        case 3: return launch_t<DIM, 3, EULER>(fp32, a, s);
        case 4: return launch_t<DIM, 4, EULER>(fp32, a, s);
        case 5: return launch_t<DIM, 5, EULER>(fp32, a, s);
        case 6: return launch_t<DIM, 6, EULER>(fp32, a, s);
        case 7: return launch_t<DIM, 7, EULER>(fp32, a, s);
        case 8: return launch_t<DIM, 8, EULER>(fp32, a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_mortars(int dim, int nq, int euler, int fp32, const MortarArgs& a, cudaStream_t s) {
    if (dim == 2) return euler ? launch_nq<2, true>(nq, fp32, a, s) : launch_nq<2, false>(nq, fp32, a, s);
    if (dim == 3) return euler ? launch_nq<3, true>(nq, fp32, a, s) : launch_nq<3, false>(nq, fp32, a, s);
    return cudaErrorInvalidValue;
}

}  // namespace rb200
