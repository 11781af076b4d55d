// Diagnostics.
// * rb200_probe_bounded_wait exercises the bounded-wait path the stage kernels use on
//   every mbarrier, without a fault.  One CTA initialises an mbarrier that nothing will
//   complete and polls it with the same try_wait loop and a caller-given poll limit; when
//   the limit runs out the kernel records RB200_ERR_TIMEOUT in a device status word and
//   returns, so the context stays usable.
// * rb200_probe_fp64_rate measures the device's FP64 FMA throughput (the denominator of
//   the stage kernels' arithmetic roofline): every thread of a full grid runs 8
//   independent fma chains.
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

// 8 independent chains a thread, `iters` fmas each; the result is kept live by a
// store that never happens for finite inputs (acc stays in (0, 2)).
__global__ void __launch_bounds__(256) dfma_rate_kernel(int64_t iters, double b, double c, double* sink) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = 1.0 + 1e-3 * (threadIdx.x + k);
    for (int64_t i = 0; i < iters; i += 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, c);
    }
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc += a[k];
    if (acc < 0.0) sink[blockIdx.x] = acc;
}

}  // namespace
}  // namespace rb200

extern "C" rb200_status rb200_probe_fp64_rate(int64_t iters, double* tflops_out, void* stream) {
    using namespace rb200;
    if (!tflops_out || iters < 4 || iters > (int64_t(1) << 26) || (iters & 3)) return RB200_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = nsm * 8, threads = 256;
    double* sink = nullptr;
    if (cudaMalloc(&sink, sizeof(double) * blocks) != cudaSuccess) {
        cudaGetLastError();
        return RB200_ERR_OOM;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float best = 0.0f;
    // b slightly below 1 and c small: the chains converge to c / (1 - b) and stay finite
    const double b = 0.9999999, c = 1e-8;
    for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {  // the first launch is a warm-up
        e = cudaEventRecord(e0, s);
        if (e == cudaSuccess) {
            dfma_rate_kernel<<<blocks, threads, 0, s>>>(iters, b, c, sink);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess && rep > 0 && (best == 0.0f || ms < best)) best = ms;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess || best <= 0.0f) return RB200_ERR_CUDA;
    const double flops = 2.0 * 8.0 * (double)iters * (double)blocks * threads;
    *tflops_out = flops / (best * 1e-3) / 1e12;
    return RB200_OK;
}

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
