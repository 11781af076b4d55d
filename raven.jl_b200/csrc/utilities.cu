// Device versions of three utilities Raven.jl exports beside the DGSEM path:
//   * Kron * f            src/kron.jl:15-387
//   * scatter! / gather!  src/gatherscatter.jl:1-103 (setbuffer_kernel!,
//                         src/communication.jl:267-270; gather_kernel!)
//   * decode(facecode)    src/facecode.jl:1-140
// Each is a one-thread-per-output kernel with the reference's arithmetic order, so
// the results are bit-identical to a CPU restatement of the reference.  These are
// HBM- or latency-bound utilities, not part of the timed path.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/raven_b200.h"

namespace {

constexpr int kMaxKronDim = 16;  // rows and columns of each Kron factor

template <typename T>
struct KronArgs {
    T mats[3][kMaxKronDim * kMaxKronDim];  // column-major
    int eye[3], rows[3], cols[3];
    int nf, ndense, dense;
    const T* in;
    T* out;
    int64_t sn, sc, scol, tn, tc, tcol;
    int64_t ncol, total;
    int ncomp;
};

template <typename T>
__device__ __forceinline__ T kron_x(const KronArgs<T>& A, int d, int i, int l) {
    if (A.eye[d]) return i == l ? T(1) : T(0);
    return A.mats[d][i + A.rows[d] * l];
}

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }

// One output entry per thread.  The arithmetic is the method Julia dispatches to for
// the factor pattern (see kron.jl): copy for all-Eye, one fma chain for a single dense
// factor, else the generic nested sum with the factor products formed left to right.
template <typename T>
__global__ void kron_kernel(const __grid_constant__ KronArgs<T> A) {
    const int R0 = A.rows[0], R1 = A.nf > 1 ? A.rows[1] : 1, R2 = A.nf > 2 ? A.rows[2] : 1;
    const int C0 = A.cols[0], C1 = A.nf > 1 ? A.cols[1] : 1, C2 = A.nf > 2 ? A.cols[2] : 1;
    const int64_t nout = (int64_t)R0 * R1 * R2;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < A.total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t onode = t % nout;
        const int64_t rest = t / nout;
        const int c = (int)(rest % A.ncomp);
        const int64_t col = rest / A.ncomp;
        const int i = (int)(onode % R0), j = (int)((onode / R0) % R1), k = (int)(onode / ((int64_t)R0 * R1));
        const T* g = A.in + (int64_t)c * A.sc + col * A.scol;
        auto G = [&](int l, int m, int n) { return g[(l + (int64_t)C0 * (m + (int64_t)C1 * n)) * A.sn]; };
        T acc = T(0);
        if (A.nf > 1 && A.ndense == 0) {
            acc = G(i, j, k);
        } else if (A.nf == 1) {
            for (int l = 0; l < C0; ++l) acc = fma(kron_x(A, 0, i, l), G(l, j, k), acc);
        } else if (A.ndense == 1) {
            const int d = A.dense;
            const int od = d == 0 ? i : (d == 1 ? j : k);
            for (int l = 0; l < A.cols[d]; ++l)
                acc = fma(kron_x(A, d, od, l), d == 0 ? G(l, j, k) : (d == 1 ? G(i, l, k) : G(i, j, l)), acc);
        } else if (A.nf == 2) {
            for (int m = 0; m < C1; ++m)
                for (int l = 0; l < C0; ++l) acc = fma(mul_rn(kron_x(A, 1, j, m), kron_x(A, 0, i, l)), G(l, m, k), acc);
        } else {
            for (int l = 0; l < C0; ++l)
                for (int m = 0; m < C1; ++m)
                    for (int n = 0; n < C2; ++n)
                        acc = fma(mul_rn(mul_rn(kron_x(A, 2, k, n), kron_x(A, 1, j, m)), kron_x(A, 0, i, l)),
                                  G(l, m, n), acc);
        }
        A.out[onode * A.tn + (int64_t)c * A.tc + col * A.tcol] = acc;
    }
}

struct Layout {
    int64_t block, node_stride, block_stride, comp_stride;
};

__device__ __forceinline__ int64_t loff(const Layout& L, int64_t i, int c) {
    return (i % L.block) * L.node_stride + (i / L.block) * L.block_stride + (int64_t)c * L.comp_stride;
}

template <typename T>
__global__ void scatter_kernel(T* dest, Layout dl, const T* src, Layout sl, const int64_t* dtoc, int64_t n,
                               int ncomp) {
    const int64_t total = n * ncomp;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / ncomp;
        const int c = (int)(t % ncomp);
        dest[loff(dl, i, c)] = src[loff(sl, dtoc[i] - 1, c)];
    }
}

// Julia's min/max on floats: NaN propagates and -0.0 < 0.0.
template <typename T>
__device__ __forceinline__ T jl_min(T v, T x) {
    if (v != v) return v;
    if (x != x) return x;
    return (x < v || (x == v && signbit(x) && !signbit(v))) ? x : v;
}
template <typename T>
__device__ __forceinline__ T jl_max(T v, T x) {
    if (v != v) return v;
    if (x != x) return x;
    return (x > v || (x == v && !signbit(x) && signbit(v))) ? x : v;
}
__device__ __forceinline__ int64_t jl_min(int64_t v, int64_t x) { return x < v ? x : v; }
__device__ __forceinline__ int64_t jl_max(int64_t v, int64_t x) { return x > v ? x : v; }
__device__ __forceinline__ int32_t jl_min(int32_t v, int32_t x) { return x < v ? x : v; }
__device__ __forceinline__ int32_t jl_max(int32_t v, int32_t x) { return x > v ? x : v; }

template <typename T>
__global__ void gather_kernel(T* dest, Layout dl, const T* src, Layout sl, const int64_t* colptr,
                              const int64_t* rowval, int64_t ncols, int ncomp, int op, T init) {
    const int64_t total = ncols * ncomp;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = t / ncomp;
        const int c = (int)(t % ncomp);
        T v = init;
        for (int64_t p = colptr[j] - 1; p < colptr[j + 1] - 1; ++p) {
            const T x = src[loff(sl, rowval[p] - 1, c)];
            v = op == 0 ? v + x : (op == 1 ? jl_min(v, x) : jl_max(v, x));
        }
        dest[loff(dl, j, c)] = v;
    }
}

__global__ void decode8_kernel(const uint8_t* codes, int64_t n, uint8_t* out) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const unsigned code = codes[t];
        const unsigned corner = code & 3u;
        const bool xh = (code >> 2) & 1u, yh = (code >> 3) & 1u;
        uint8_t* o = out + 4 * t;
        o[0] = (xh && corner == 0) ? 1 : (xh && corner == 2) ? 2 : 0;
        o[1] = (xh && corner == 1) ? 1 : (xh && corner == 3) ? 2 : 0;
        o[2] = (yh && corner == 0) ? 1 : (yh && corner == 1) ? 2 : 0;
        o[3] = (yh && corner == 2) ? 1 : (yh && corner == 3) ? 2 : 0;
    }
}

// UInt16 codes: bits 0-2 the octant's corner in its parent, 3-5 hanging x/y/z faces,
// 6-8 hanging x/y/z edges.  out: 6 hanging-face then 12 hanging-edge values.
__global__ void decode16_kernel(const uint16_t* codes, int64_t n, uint8_t* out) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const unsigned code = codes[t];
        const unsigned corner = code & 7u;
        uint8_t hf[6];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            // the other two axes, in increasing order, number the quarter of the face
            const int o1 = d == 0 ? 1 : 0, o2 = d == 2 ? 1 : 2;
            const unsigned quarter = ((corner >> o1) & 1u) + 2u * ((corner >> o2) & 1u) + 1u;
            const bool hanging = (code >> (3 + d)) & 1u;
            const bool plus = (corner >> d) & 1u;
            hf[2 * d] = (hanging && !plus) ? (uint8_t)quarter : 0;
            hf[2 * d + 1] = (hanging && plus) ? (uint8_t)quarter : 0;
        }
        uint8_t* o = out + 18 * t;
#pragma unroll
        for (int f = 0; f < 6; ++f) o[f] = hf[f];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int o1 = a == 0 ? 1 : 0, o2 = a == 2 ? 1 : 2;
            const bool edge_hanging = (code >> (6 + a)) & 1u;
            const unsigned shift = (corner >> a) & 1u;
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const unsigned b1 = m & 1u, b2 = (m >> 1) & 1u;
                const bool onface = hf[2 * o1 + b1] > 0 || hf[2 * o2 + b2] > 0;
                const bool onedge = edge_hanging && ((corner >> o1) & 1u) == b1 && ((corner >> o2) & 1u) == b2;
                o[6 + 4 * a + m] = onedge ? (uint8_t)((onface ? 3u : 1u) + shift) : (uint8_t)(onface ? 5u : 0u);
            }
        }
    }
}

int grid_for(int64_t total) {
    const int64_t b = (total + 255) / 256;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32));
}

rb200_status to_status(cudaError_t e) { return e == cudaSuccess ? RB200_OK : RB200_ERR_CUDA; }

template <typename T>
rb200_status kron_t(int32_t nf, const void* const* mats, const int32_t* rows, const int32_t* cols, const void* in,
                    const int64_t* is, void* out, const int64_t* os, int64_t ncol, int32_t ncomp, cudaStream_t s) {
    KronArgs<T> A{};
    A.nf = nf;
    int64_t nout = 1;
    for (int d = 0; d < nf; ++d) {
        if (rows[d] < 1 || cols[d] < 1 || rows[d] > kMaxKronDim || cols[d] > kMaxKronDim) return RB200_ERR_UNSUPPORTED;
        A.rows[d] = rows[d];
        A.cols[d] = cols[d];
        A.eye[d] = mats[d] == nullptr;
        if (A.eye[d] && rows[d] != cols[d]) return RB200_ERR_SHAPE;
        if (!A.eye[d]) {
            const T* m = static_cast<const T*>(mats[d]);
            for (int q = 0; q < rows[d] * cols[d]; ++q) A.mats[d][q] = m[q];
            A.ndense += 1;
            A.dense = d;
        }
        nout *= rows[d];
    }
    A.in = static_cast<const T*>(in);
    A.out = static_cast<T*>(out);
    A.sn = is[0];
    A.sc = is[1];
    A.scol = is[2];
    A.tn = os[0];
    A.tc = os[1];
    A.tcol = os[2];
    A.ncol = ncol;
    A.ncomp = ncomp;
    A.total = nout * ncomp * ncol;
    if (A.total == 0) return RB200_OK;
    kron_kernel<T><<<grid_for(A.total), 256, 0, s>>>(A);
    return to_status(cudaGetLastError());
}

}  // namespace

extern "C" {

rb200_status rb200_kron_apply(int32_t nfactors, const void* const* mats, const int32_t* rows, const int32_t* cols,
                              int32_t dtype, const void* in, const int64_t* in_strides, void* out,
                              const int64_t* out_strides, int64_t ncols, int32_t ncomp, void* stream) {
    if (nfactors < 1 || nfactors > 3 || !mats || !rows || !cols || !in_strides || !out_strides || ncols < 0 ||
        ncomp < 1)
        return RB200_ERR_BAD_ARG;
    if (ncols > 0 && (!in || !out)) return RB200_ERR_BAD_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == 0) return kron_t<double>(nfactors, mats, rows, cols, in, in_strides, out, out_strides, ncols, ncomp, s);
    if (dtype == 1) return kron_t<float>(nfactors, mats, rows, cols, in, in_strides, out, out_strides, ncols, ncomp, s);
    return RB200_ERR_BAD_ARG;
}

rb200_status rb200_scatter(void* dest, const rb200_layout* dest_layout, const void* src,
                           const rb200_layout* src_layout, const int64_t* dtoc, int64_t n, int32_t ncomp,
                           int32_t dtype, void* stream) {
    if (!dest_layout || !src_layout || n < 0 || ncomp < 1) return RB200_ERR_BAD_ARG;
    if (dest_layout->block < 1 || src_layout->block < 1) return RB200_ERR_BAD_ARG;
    if (n == 0) return RB200_OK;
    if (!dest || !src || !dtoc) return RB200_ERR_BAD_ARG;
    const Layout dl{dest_layout->block, dest_layout->node_stride, dest_layout->block_stride, dest_layout->comp_stride};
    const Layout sl{src_layout->block, src_layout->node_stride, src_layout->block_stride, src_layout->comp_stride};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int g = grid_for(n * ncomp);
    switch (dtype) {
        case 0: scatter_kernel<double><<<g, 256, 0, s>>>((double*)dest, dl, (const double*)src, sl, dtoc, n, ncomp); break;
        case 1: scatter_kernel<float><<<g, 256, 0, s>>>((float*)dest, dl, (const float*)src, sl, dtoc, n, ncomp); break;
        case 2: scatter_kernel<int64_t><<<g, 256, 0, s>>>((int64_t*)dest, dl, (const int64_t*)src, sl, dtoc, n, ncomp); break;
        case 3: scatter_kernel<int32_t><<<g, 256, 0, s>>>((int32_t*)dest, dl, (const int32_t*)src, sl, dtoc, n, ncomp); break;
        default: return RB200_ERR_BAD_ARG;
    }
    return to_status(cudaGetLastError());
}

rb200_status rb200_gather(void* dest, const rb200_layout* dest_layout, const void* src,
                          const rb200_layout* src_layout, const int64_t* colptr, const int64_t* rowval, int64_t ncols,
                          int32_t ncomp, int32_t dtype, int32_t op, double init, void* stream) {
    if (!dest_layout || !src_layout || ncols < 0 || ncomp < 1 || op < 0 || op > 2) return RB200_ERR_BAD_ARG;
    if (dest_layout->block < 1 || src_layout->block < 1) return RB200_ERR_BAD_ARG;
    if (ncols == 0) return RB200_OK;
    if (!dest || !src || !colptr || !rowval) return RB200_ERR_BAD_ARG;
    const Layout dl{dest_layout->block, dest_layout->node_stride, dest_layout->block_stride, dest_layout->comp_stride};
    const Layout sl{src_layout->block, src_layout->node_stride, src_layout->block_stride, src_layout->comp_stride};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int g = grid_for(ncols * ncomp);
    switch (dtype) {
        case 0:
            gather_kernel<double><<<g, 256, 0, s>>>((double*)dest, dl, (const double*)src, sl, colptr, rowval, ncols,
                                                    ncomp, op, init);
            break;
        case 1:
            gather_kernel<float><<<g, 256, 0, s>>>((float*)dest, dl, (const float*)src, sl, colptr, rowval, ncols,
                                                   ncomp, op, (float)init);
            break;
        case 2:
            gather_kernel<int64_t><<<g, 256, 0, s>>>((int64_t*)dest, dl, (const int64_t*)src, sl, colptr, rowval,
                                                     ncols, ncomp, op, (int64_t)init);
            break;
        case 3:
            gather_kernel<int32_t><<<g, 256, 0, s>>>((int32_t*)dest, dl, (const int32_t*)src, sl, colptr, rowval,
                                                     ncols, ncomp, op, (int32_t)init);
            break;
        default: return RB200_ERR_BAD_ARG;
    }
    return to_status(cudaGetLastError());
}

rb200_status rb200_decode_facecodes(const void* codes, int32_t bits, int64_t n, uint8_t* out, void* stream) {
    if ((bits != 8 && bits != 16) || n < 0) return RB200_ERR_BAD_ARG;
    if (n == 0) return RB200_OK;
    if (!codes || !out) return RB200_ERR_BAD_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (bits == 8) decode8_kernel<<<grid_for(n), 256, 0, s>>>((const uint8_t*)codes, n, out);
    else decode16_kernel<<<grid_for(n), 256, 0, s>>>((const uint16_t*)codes, n, out);
    return to_status(cudaGetLastError());
}

}  // extern "C"
