// Diagnostics: exercises the bounded-wait path the stage kernels use on every mbarrier,
// without a fault.  One CTA initialises an mbarrier that nothing will complete and polls
// it with the same try_wait loop and a caller-given poll limit; when the limit runs out
// the kernel records RB200_ERR_TIMEOUT in a device status word and returns, so the
// context stays usable.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/raven_b200.h"
#include "pipelined_kernel.cuh"
#include "rb200_internal.h"

namespace rb200 {
namespace {

__global__ void unfinished_wait_kernel(int64_t polls, int32_t* status) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        pipe::mbar_init(&bar, 1);  // expects one arrival that never comes
        pipe::fence_mbar_init();
    }
    __syncthreads();
    int64_t it = 0;
    bool done = false;
    while (!(done = pipe::mbar_try_wait(&bar, 0))) {
        if (++it >= polls) break;
    }
    if (__syncthreads_or(!done) && threadIdx.x == 0) atomicExch(status, kStatusTimeout);
}

}  // namespace
}  // namespace rb200

extern "C" rb200_status rb200_probe_bounded_wait(int64_t polls, void* stream) {
    using namespace rb200;
    if (polls < 1 || polls > (int64_t(1) << 30)) return RB200_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int32_t* d_status = nullptr;
    if (cudaMalloc(&d_status, sizeof(int32_t)) != cudaSuccess) {
        cudaGetLastError();
        return RB200_ERR_OOM;
    }
    int32_t h_status = 0;
    cudaError_t e = cudaMemsetAsync(d_status, 0, sizeof(int32_t), s);
    if (e == cudaSuccess) {
        unfinished_wait_kernel<<<1, 32, 0, s>>>(polls, d_status);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_status, d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_status);
    if (e != cudaSuccess) return RB200_ERR_CUDA;
    return h_status == kStatusTimeout ? RB200_ERR_TIMEOUT : RB200_OK;
}
