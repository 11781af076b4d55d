// Buffer fills of the face-trace exchange of a distributed step: the setbuffer!/getbuffer!
// kernels of Raven's comm managers (src/communication.jl:267-293) with 0-based indices
// into a state array (Np, Ns, E + ghosts).  The exchange itself (which rank sends which
// slice) is host logic over torch.distributed; these kernels only gather the values a
// rank sends into one contiguous buffer and scatter the received buffer into its ghost
// elements.  Indices outside [0, len) are skipped (the host checks every pattern when it
// builds it), so a bad pattern cannot write outside the arrays.
#include <cuda_runtime.h>

#include <algorithm>

#include "raven_b200.h"

namespace {

__global__ void pack_values_kernel(const double* __restrict__ src, int64_t src_len, const int64_t* __restrict__ idx,
                                   int64_t n, double* __restrict__ buf) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = idx[i];
        if (j >= 0 && j < src_len) buf[i] = src[j];
    }
}

__global__ void unpack_values_kernel(const double* __restrict__ buf, const int64_t* __restrict__ idx, int64_t n,
                                     double* __restrict__ dest, int64_t dest_len) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = idx[i];
        if (j >= 0 && j < dest_len) dest[j] = buf[i];
    }
}

int grid_for(int64_t n) {
    // 148 SMs x 8 CTAs of 256 threads at most; a grid-stride loop covers the rest
    return (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
}

}  // namespace

extern "C" rb200_status rb200_pack_values(const double* src, int64_t src_len, const int64_t* indices, int64_t n,
                                          double* buffer, void* stream) {
    if (n < 0 || src_len < 0) return RB200_ERR_BAD_ARG;
    if (n == 0) return RB200_OK;
    if (!src || !indices || !buffer) return RB200_ERR_BAD_ARG;
    pack_values_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(src, src_len, indices, n, buffer);
    return cudaGetLastError() == cudaSuccess ? RB200_OK : RB200_ERR_CUDA;
}

extern "C" rb200_status rb200_unpack_values(const double* buffer, const int64_t* indices, int64_t n, double* dest,
                                            int64_t dest_len, void* stream) {
    if (n < 0 || dest_len < 0) return RB200_ERR_BAD_ARG;
    if (n == 0) return RB200_OK;
    if (!buffer || !indices || !dest) return RB200_ERR_BAD_ARG;
    unpack_values_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(buffer, indices, n, dest, dest_len);
    return cudaGetLastError() == cudaSuccess ? RB200_OK : RB200_ERR_CUDA;
}
