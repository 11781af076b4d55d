// Entropy measures and the relaxation Runge-Kutta step RLSRK(5,4)
// (src/balancelaws/measures.jl:23-33, src/balancelaws/odesolvers.jl:73-161).
//
// Per step: q0 = q; eta0 = entropyintegral(q0); five stages, each
//   k = RHS(q)                                        (the stage kernel, tendency mode)
//   dq = rka dq + k;  prod = sum MJ v(q).k;  q += rkb dt dq      (rlsrk_stage_kernel)
// then k = q - q0 and the scalar relaxation solve for gamma, whose every iterate needs
// sum MJ eta(q0 + gamma k) and sum MJ v(q0 + gamma k).k (entropy_sums_kernel); finally
// q = q0 + gamma k.  The products and integrals are deterministic: a fixed number of
// CTAs each own a fixed strided set of elements, a fixed tree combines a CTA's threads
// and one thread adds the CTA partials in index order.  The elementwise updates use
// explicitly rounded multiply and add, as the reference's broadcasts do (no fma).
#include <cuda_runtime.h>
#include <stdint.h>

#include "rb200_internal.h"

namespace rb200 {

namespace {

constexpr int kThreads = 256;

template <int DIM, bool EULER>
struct Ent {
    static constexpr int NS = EULER ? DIM + 2 : 1;
    // entropy (euler.jl:70-77; advection.jl:20)
    static __device__ __forceinline__ double eta(const double* q, double gamma) {
        if constexpr (!EULER) {
            return q[0] * q[0] / 2.0;
        } else {
            const double rho = q[0];
            double rr = q[1] * q[1];
#pragma unroll
            for (int d = 1; d < DIM; ++d) rr = rr + q[1 + d] * q[1 + d];
            const double p = (gamma - 1.0) * (q[DIM + 1] - rr / (2.0 * rho));
            const double s = log(p / pow(rho, gamma));
            return -rho * s / (gamma - 1.0);
        }
    }
    // v(q).k with the entropy variables (euler.jl:79-91; advection.jl:21)
    static __device__ __forceinline__ double vdot(const double* q, const double* k, double gamma) {
        if constexpr (!EULER) {
            return q[0] * k[0];
        } else {
            const double rho = q[0];
            double u[DIM], rr = q[1] * q[1];
#pragma unroll
            for (int d = 1; d < DIM; ++d) rr = rr + q[1 + d] * q[1 + d];
            const double p = (gamma - 1.0) * (q[DIM + 1] - rr / (2.0 * rho));
            const double s = log(p / pow(rho, gamma));
            const double b = rho / (2.0 * p);
            double uu = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                u[d] = q[1 + d] / rho;
                uu = uu + u[d] * u[d];
            }
            double acc = ((gamma - s) / (gamma - 1.0) - uu * b) * k[0];
#pragma unroll
            for (int d = 0; d < DIM; ++d) acc = acc + (2.0 * b * u[d]) * k[1 + d];
            return acc + (-2.0 * b) * k[DIM + 1];
        }
    }
};

__device__ __forceinline__ double node_mj(const RelaxGeo& G, int64_t e, int n) {
    if (G.geom == GEOM_AFFINE) {
        const int nq = G.nq;
        const int i = n % nq, j = (n / nq) % nq, k = n / (nq * nq);
        double mj = G.w[i];
        if (G.dim >= 2) mj = mj * G.w[j];
        if (G.dim == 3) mj = mj * G.w[k];
        return mj * G.elem_geo[4 * e + 3];
    }
    const int nvg = G.dim * G.dim + 2;
    return G.vgeo[((size_t)e * nvg + G.dim * G.dim + 1) * G.np + n];
}

// Writes the CTA's two sums to partial[2 * blockIdx.x + {0, 1}].
__device__ __forceinline__ void block_pair(double a, double b, double* partial) {
    __shared__ double red[2][kThreads];
    red[0][threadIdx.x] = a;
    red[1][threadIdx.x] = b;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            red[0][threadIdx.x] += red[0][threadIdx.x + w];
            red[1][threadIdx.x] += red[1][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = red[0][0];
        partial[2 * blockIdx.x + 1] = red[1][0];
    }
}

// partial: (sum MJ eta(p), sum MJ v(p).k) per CTA, p = base + c dir (dir null: p = base)
template <int DIM, bool EULER>
__global__ void __launch_bounds__(kThreads)
    entropy_sums_kernel(const RelaxGeo G, const double* __restrict__ base, const double* __restrict__ dir, double c,
                        const double* __restrict__ k, double* __restrict__ partial) {
    using L = Ent<DIM, EULER>;
    constexpr int NS = L::NS;
    double a_eta = 0.0, a_prod = 0.0;
    for (int64_t e = blockIdx.x; e < G.E; e += gridDim.x) {
        for (int n = threadIdx.x; n < G.np; n += blockDim.x) {
            const double mj = node_mj(G, e, n);
            double p[NS], kk[NS];
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const size_t i = ((size_t)e * NS + s) * G.np + n;
                p[s] = dir ? __dadd_rn(base[i], __dmul_rn(c, dir[i])) : base[i];  // @. q = q0 + γ * k
                kk[s] = k ? k[i] : 0.0;
            }
            a_eta = a_eta + mj * L::eta(p, G.gamma);
            if (k) a_prod = a_prod + mj * L::vdot(p, kk, G.gamma);
        }
    }
    block_pair(a_eta, a_prod, partial);
}

// One RLSRK stage after k = RHS(q): dq = dq rka + k; product of v(q) with k; q += rkb_dt dq.
template <int DIM, bool EULER>
__global__ void __launch_bounds__(kThreads)
    rlsrk_stage_kernel(const RelaxGeo G, double* __restrict__ q, double* __restrict__ dq,
                       const double* __restrict__ k, double rka, double rkb_dt, double* __restrict__ partial) {
    using L = Ent<DIM, EULER>;
    constexpr int NS = L::NS;
    double a_prod = 0.0;
    for (int64_t e = blockIdx.x; e < G.E; e += gridDim.x) {
        for (int n = threadIdx.x; n < G.np; n += blockDim.x) {
            const double mj = node_mj(G, e, n);
            double qq[NS], kk[NS];
            size_t idx[NS];
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                idx[s] = ((size_t)e * NS + s) * G.np + n;
                qq[s] = q[idx[s]];
                kk[s] = k[idx[s]];
            }
            a_prod = a_prod + mj * L::vdot(qq, kk, G.gamma);
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const double d = __dadd_rn(__dmul_rn(dq[idx[s]], rka), kk[s]);  // dq .*= rka; dq .+= k
                dq[idx[s]] = d;
                q[idx[s]] = __dadd_rn(qq[s], __dmul_rn(rkb_dt, d));  // @. q += rkb * dt * dq
            }
        }
    }
    block_pair(0.0, a_prod, partial);
}

__global__ void diff_kernel(const double* __restrict__ q, const double* __restrict__ q0, double* __restrict__ k,
                            int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        k[i] = __dsub_rn(q[i], q0[i]);
}

__global__ void relax_kernel(double* __restrict__ q, const double* __restrict__ q0, const double* __restrict__ k,
                             double gamma, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        q[i] = __dadd_rn(q0[i], __dmul_rn(gamma, k[i]));
}

__global__ void finish_pair_kernel(const double* __restrict__ partial, int nblocks, double* __restrict__ out) {
    const int v = threadIdx.x;
    if (v >= 2) return;
    double acc = 0.0;
    for (int b = 0; b < nblocks; ++b) acc += partial[2 * b + v];
    out[v] = acc;
}

template <int DIM, bool EULER>
cudaError_t sums_t(const RelaxGeo& G, const double* base, const double* dir, double c, const double* k,
                   double* partial, int nblocks, double* out, cudaStream_t s) {
    entropy_sums_kernel<DIM, EULER><<<nblocks, kThreads, 0, s>>>(G, base, dir, c, k, partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    finish_pair_kernel<<<1, 32, 0, s>>>(partial, nblocks, out);
    return cudaGetLastError();
}

template <int DIM, bool EULER>
cudaError_t stage_t(const RelaxGeo& G, double* q, double* dq, const double* k, double rka, double rkb_dt,
                    double* partial, int nblocks, double* out, cudaStream_t s) {
    rlsrk_stage_kernel<DIM, EULER><<<nblocks, kThreads, 0, s>>>(G, q, dq, k, rka, rkb_dt, partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    finish_pair_kernel<<<1, 32, 0, s>>>(partial, nblocks, out);
    return cudaGetLastError();
}

int grid_for(int64_t n) {
    int64_t b = (n + kThreads - 1) / kThreads;
    return (int)(b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b));
}

}  // namespace

cudaError_t launch_entropy_sums(const RelaxGeo& G, const double* base, const double* dir, double c, const double* k,
                                double* partial, int nblocks, double* out, cudaStream_t s) {
    if (G.dim == 1) return G.euler ? sums_t<1, true>(G, base, dir, c, k, partial, nblocks, out, s)
                                   : sums_t<1, false>(G, base, dir, c, k, partial, nblocks, out, s);
    if (G.dim == 2) return G.euler ? sums_t<2, true>(G, base, dir, c, k, partial, nblocks, out, s)
                                   : sums_t<2, false>(G, base, dir, c, k, partial, nblocks, out, s);
    if (G.dim == 3) return G.euler ? sums_t<3, true>(G, base, dir, c, k, partial, nblocks, out, s)
                                   : sums_t<3, false>(G, base, dir, c, k, partial, nblocks, out, s);
    return cudaErrorInvalidValue;
}

cudaError_t launch_rlsrk_stage(const RelaxGeo& G, double* q, double* dq, const double* k, double rka, double rkb_dt,
                               double* partial, int nblocks, double* out, cudaStream_t s) {
    if (G.dim == 1) return G.euler ? stage_t<1, true>(G, q, dq, k, rka, rkb_dt, partial, nblocks, out, s)
                                   : stage_t<1, false>(G, q, dq, k, rka, rkb_dt, partial, nblocks, out, s);
    if (G.dim == 2) return G.euler ? stage_t<2, true>(G, q, dq, k, rka, rkb_dt, partial, nblocks, out, s)
                                   : stage_t<2, false>(G, q, dq, k, rka, rkb_dt, partial, nblocks, out, s);
    if (G.dim == 3) return G.euler ? stage_t<3, true>(G, q, dq, k, rka, rkb_dt, partial, nblocks, out, s)
                                   : stage_t<3, false>(G, q, dq, k, rka, rkb_dt, partial, nblocks, out, s);
    return cudaErrorInvalidValue;
}

cudaError_t launch_state_diff(const double* q, const double* q0, double* k, int64_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    diff_kernel<<<grid_for(n), kThreads, 0, s>>>(q, q0, k, n);
    return cudaGetLastError();
}

cudaError_t launch_relax(double* q, const double* q0, const double* k, double gamma, int64_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    relax_kernel<<<grid_for(n), kThreads, 0, s>>>(q, q0, k, gamma, n);
    return cudaGetLastError();
}

}  // namespace rb200
