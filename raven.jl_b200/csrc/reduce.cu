// FP64 reductions behind weightednorm / conservation integrals (measures.jl:6-33) and
// the device-side rebuild of vmapP from the neighbour table.
//
// The reductions are deterministic: a fixed number of CTAs each own a fixed,
// strided set of elements, partial sums are combined in a fixed tree, and a single
// CTA adds the per-CTA partials in index order.
#include <cuda.h>  // CUcontext (cuCtxGetCurrent is reached through cudaGetDriverEntryPoint)

#include <mutex>

#include "../../include/raven_b200.h"
#include "rb200_internal.h"

namespace rb200 {

namespace {

constexpr int kRedThreads = 256;

// partial[(blockIdx.x * 2*ns) + s]       = sum MJ q_s^2
// partial[(blockIdx.x * 2*ns) + ns + s]  = sum MJ q_s
__global__ void __launch_bounds__(kRedThreads) weighted_sums_kernel(const double* __restrict__ q,
                                                                    const double* __restrict__ elem_geo,
                                                                    const double* __restrict__ vgeo,
                                                                    const double* __restrict__ wgt, int dim, int nq,
                                                                    int ns, int64_t E, int geom,
                                                                    double* __restrict__ partial) {
    __shared__ double red[kRedThreads];
    const int np = dim == 1 ? nq : dim == 2 ? nq * nq : nq * nq * nq;
    const int nvg = dim * dim + 2;
    for (int s = 0; s < ns; ++s) {
        double a2 = 0.0, a1 = 0.0;
        for (int64_t e = blockIdx.x; e < E; e += gridDim.x) {
            for (int n = threadIdx.x; n < np; n += blockDim.x) {
                double mj;
                if (geom == GEOM_AFFINE) {
                    const int i = n % nq, j = (n / nq) % nq, k = n / (nq * nq);
                    mj = wgt[i];
                    if (dim >= 2) mj = mj * wgt[j];
                    if (dim == 3) mj = mj * wgt[k];
                    mj = mj * elem_geo[4 * e + 3];
                } else {
                    mj = vgeo[((size_t)e * nvg + dim * dim + 1) * np + n];
                }
                const double v = q[((size_t)e * ns + s) * np + n];
                a2 += mj * (v * v);
                a1 += mj * v;
            }
        }
        for (int pass = 0; pass < 2; ++pass) {
            red[threadIdx.x] = pass == 0 ? a2 : a1;
            __syncthreads();
            for (int w = kRedThreads / 2; w > 0; w >>= 1) {
                if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
                __syncthreads();
            }
            if (threadIdx.x == 0) partial[(size_t)blockIdx.x * 2 * ns + pass * ns + s] = red[0];
            __syncthreads();
        }
    }
}

// max that keeps a NaN, as Julia's maximum does
__device__ __forceinline__ double nan_max(double a, double b) { return (isnan(b) || b > a) ? b : a; }

// weightednorm for p != 2 (measures.jl:9-21), same element partition and tree as
// weighted_sums_kernel.  kind 0: partial[b*ns + s] = sum MJ |q_s|^p; kind 1 (p = Inf):
// partial[b*ns + s] = max |q_s| (unweighted, as in the reference).
__global__ void __launch_bounds__(kRedThreads) weighted_pnorm_kernel(const double* __restrict__ q,
                                                                     const double* __restrict__ elem_geo,
                                                                     const double* __restrict__ vgeo,
                                                                     const double* __restrict__ wgt, int dim, int nq,
                                                                     int ns, int64_t E, int geom, double p, int kind,
                                                                     double* __restrict__ partial) {
    __shared__ double red[kRedThreads];
    const int np = dim == 1 ? nq : dim == 2 ? nq * nq : nq * nq * nq;
    const int nvg = dim * dim + 2;
    for (int s = 0; s < ns; ++s) {
        double acc = 0.0;
        for (int64_t e = blockIdx.x; e < E; e += gridDim.x) {
            for (int n = threadIdx.x; n < np; n += blockDim.x) {
                const double v = fabs(q[((size_t)e * ns + s) * np + n]);
                if (kind == 1) {
                    acc = nan_max(acc, v);
                    continue;
                }
                double mj;
                if (geom == GEOM_AFFINE) {
                    const int i = n % nq, j = (n / nq) % nq, k = n / (nq * nq);
                    mj = wgt[i];
                    if (dim >= 2) mj = mj * wgt[j];
                    if (dim == 3) mj = mj * wgt[k];
                    mj = mj * elem_geo[4 * e + 3];
                } else {
                    mj = vgeo[((size_t)e * nvg + dim * dim + 1) * np + n];
                }
                acc += mj * (p == 1.0 ? v : pow(v, p));
            }
        }
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int w = kRedThreads / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w)
                red[threadIdx.x] = kind == 1 ? nan_max(red[threadIdx.x], red[threadIdx.x + w])
                                             : red[threadIdx.x] + red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) partial[(size_t)blockIdx.x * ns + s] = red[0];
        __syncthreads();
    }
}

__global__ void finish_pnorm_kernel(const double* __restrict__ partial, int nblocks, int ns, int kind, double* out) {
    const int v = threadIdx.x;
    if (v >= ns) return;
    double acc = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        const double x = partial[(size_t)b * ns + v];
        acc = kind == 1 ? nan_max(acc, x) : acc + x;
    }
    out[v] = acc;
}

__global__ void finish_sums_kernel(const double* __restrict__ partial, int nblocks, int nvals, double* out) {
    const int v = threadIdx.x;
    if (v >= nvals) return;
    double acc = 0.0;
    for (int b = 0; b < nblocks; ++b) acc += partial[(size_t)b * nvals + v];
    out[v] = acc;
}

__global__ void face_vmapP_kernel(const int32_t* __restrict__ nbr, int dim, int nq, int64_t E,
                                  int64_t* __restrict__ out) {
    const int np = dim == 1 ? nq : dim == 2 ? nq * nq : nq * nq * nq;
    const int nfp = dim == 1 ? 1 : dim == 2 ? nq : nq * nq;
    const int nf = 2 * dim;
    const int64_t total = E * nf * nfp;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(t % nfp);
        const int f = (int)((t / nfp) % nf);
        const int64_t e = t / ((int64_t)nfp * nf);
        const int dir = f / 2, side = f % 2;
        const int ne = nbr[(size_t)nf * e + f];
        // node of face f (side) or of the opposite face (1-side) at in-face index j
        auto facenode = [&](int sd) {
            const int c = sd ? nq - 1 : 0;
            if (dim == 1) return c;
            if (dim == 2) return dir == 0 ? c + nq * j : j + nq * c;
            const int j1 = j % nq, j2 = j / nq;
            if (dir == 0) return c + nq * (j1 + nq * j2);
            if (dir == 1) return j1 + nq * (c + nq * j2);
            return j1 + nq * (j2 + nq * c);
        };
        out[t] = ne < 0 ? e * np + facenode(side) + 1 : (int64_t)ne * np + facenode(1 - side) + 1;
    }
}

// Variant of weighted_sums_kernel for rb200_weighted_sums_noalloc: the caller passes
// the nodal weights MJ (Np, E) instead of the handle's geometry.
__global__ void __launch_bounds__(kRedThreads) weighted_sums_mj_kernel(const double* __restrict__ q,
                                                                       const double* __restrict__ mj, int np,
                                                                       int ns, int64_t E,
                                                                       double* __restrict__ partial) {
    __shared__ double red[kRedThreads];
    for (int s = 0; s < ns; ++s) {
        double a2 = 0.0, a1 = 0.0;
        for (int64_t e = blockIdx.x; e < E; e += gridDim.x) {
            for (int n = threadIdx.x; n < np; n += blockDim.x) {
                const double w = mj[(size_t)e * np + n];
                const double v = q[((size_t)e * ns + s) * np + n];
                a2 += w * (v * v);
                a1 += w * v;
            }
        }
        for (int pass = 0; pass < 2; ++pass) {
            red[threadIdx.x] = pass == 0 ? a2 : a1;
            __syncthreads();
            for (int w = kRedThreads / 2; w > 0; w >>= 1) {
                if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
                __syncthreads();
            }
            if (threadIdx.x == 0) partial[(size_t)blockIdx.x * 2 * ns + pass * ns + s] = red[0];
            __syncthreads();
        }
    }
}

// Scratch of rb200_weighted_sums_noalloc: one slot per (CTA, sum).  Every CTA of a
// call writes all of its slots before the final sum reads them, so nothing has to be
// cleared between calls.  It lives in every device that loads the library, until exit.
constexpr int kNoAllocBlocks = 256;
constexpr int kNoAllocMaxFields = 5;
__device__ __align__(256) double g_noalloc_partials[kNoAllocBlocks * 2 * kNoAllocMaxFields];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};
// the context the address was looked up in: a device reset (or a destroyed and recreated
// primary context) reloads the module at another address, so a new context means a new
// lookup
CUcontext g_noalloc_ctx[kNoAllocMaxDevices] = {nullptr};

using CtxGetCurrent = CUresult (*)(CUcontext*);
CtxGetCurrent ctx_get_current() {
    static const CtxGetCurrent fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return static_cast<CtxGetCurrent>(nullptr);
        }
        return reinterpret_cast<CtxGetCurrent>(p);
    }();
    return fn;
}

CUcontext current_context() {
    CUcontext c = nullptr;
    if (CtxGetCurrent f = ctx_get_current()) {
        if (f(&c) != CUDA_SUCCESS) c = nullptr;
    }
    return c;
}

// true if p is device (or managed) memory that the current device `dev` can use
bool on_device(const void* p, int dev) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice && a.device == dev) || a.type == cudaMemoryTypeManaged;
}

}  // namespace

cudaError_t launch_weighted_sums(const double* q, const double* elem_geo, const double* vgeo, const double* w, int dim,
                                 int nq, int ns, int64_t E, int geom, double* partial, int nblocks, double* out_dev,
                                 cudaStream_t s) {
    weighted_sums_kernel<<<nblocks, kRedThreads, 0, s>>>(q, elem_geo, vgeo, w, dim, nq, ns, E, geom, partial);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    finish_sums_kernel<<<1, 32, 0, s>>>(partial, nblocks, 2 * ns, out_dev);
    return cudaGetLastError();
}

cudaError_t launch_weighted_pnorm(const double* q, const double* elem_geo, const double* vgeo, const double* w, int dim,
                                  int nq, int ns, int64_t E, int geom, double p, double* partial, int nblocks,
                                  double* out_dev, cudaStream_t s) {
    const int kind = isinf(p) ? 1 : 0;
    weighted_pnorm_kernel<<<nblocks, kRedThreads, 0, s>>>(q, elem_geo, vgeo, w, dim, nq, ns, E, geom, p, kind,
                                                          partial);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    finish_pnorm_kernel<<<1, 32, 0, s>>>(partial, nblocks, ns, kind, out_dev);
    return cudaGetLastError();
}

cudaError_t launch_face_vmapP(const int32_t* nbr, int dim, int nq, int64_t E, int64_t* out, cudaStream_t s) {
    const int nfp = dim == 1 ? 1 : dim == 2 ? nq : nq * nq;
    const int64_t total = E * 2 * dim * nfp;
    if (total == 0) return cudaSuccess;
    int64_t blocks = (total + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    face_vmapP_kernel<<<(unsigned)blocks, 256, 0, s>>>(nbr, dim, nq, E, out);
    return cudaGetLastError();
}

__global__ void copy_vmapP_kernel(const int32_t* __restrict__ v, int64_t n, int64_t* __restrict__ out) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        out[t] = (int64_t)v[t] + 1;
}

cudaError_t launch_copy_vmapP(const int32_t* vmapP0, int64_t n, int64_t* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    int64_t blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    copy_vmapP_kernel<<<(unsigned)blocks, 256, 0, s>>>(vmapP0, n, out);
    return cudaGetLastError();
}

}  // namespace rb200

// ---------------------------------------------------------------------------------
// rb200_weighted_sums_noalloc (declared in include/raven_b200.h)
// ---------------------------------------------------------------------------------
extern "C" rb200_status rb200_weighted_sums_noalloc(const double* q, const double* MJ, int32_t np, int32_t ns,
                                                    int64_t num_elements, double* sums_out, void* stream) {
    using namespace rb200;
    if (!q || !MJ || !sums_out) return RB200_ERR_BAD_ARG;
    if (np < 1 || np > 512 || num_elements < 0) return RB200_ERR_BAD_ARG;
    if (ns < 1 || ns > kNoAllocMaxFields) return RB200_ERR_UNSUPPORTED;  // beyond the scratch array
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return RB200_ERR_CUDA;
    // the arrays must be device memory of the current device (a host or foreign-device
    // pointer would otherwise fail later as an asynchronous launch error)
    if (!on_device(q, dev) || !on_device(MJ, dev) || !on_device(sums_out, dev)) return RB200_ERR_BAD_ARG;
    double* scratch;
    {
        // once per device and context, with that device current: the device address of
        // the array (looked up again when the current context changed, e.g. after a reset)
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        const CUcontext ctx = current_context();
        if (!g_noalloc_ptr[dev] || g_noalloc_ctx[dev] != ctx) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) {
                cudaGetLastError();
                return RB200_ERR_CUDA;
            }
            g_noalloc_ptr[dev] = static_cast<double*>(p);
            g_noalloc_ctx[dev] = current_context();  // current now, if it was not before the lookup
        }
        scratch = g_noalloc_ptr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    weighted_sums_mj_kernel<<<kNoAllocBlocks, kRedThreads, 0, s>>>(q, MJ, np, ns, num_elements, scratch);
    if (cudaGetLastError() != cudaSuccess) return RB200_ERR_CUDA;
    finish_sums_kernel<<<1, 32, 0, s>>>(scratch, kNoAllocBlocks, 2 * ns, sums_out);
    if (cudaGetLastError() != cudaSuccess) return RB200_ERR_CUDA;
    return RB200_OK;
}
