// Instantiations and launch helpers of the pipelined 3-D Nq = 8 stage kernel: one state
// (the DGSEM handle) or the chunks of a serving class (BATCH).
#include "pipelined_curved.cuh"
#include "pipelined_kernel.cuh"

namespace rb200 {

#ifndef RB200_PIPE_NPT
#define RB200_PIPE_NPT 2  // nodes per thread of the pipelined kernel
#endif
constexpr int kNPT = RB200_PIPE_NPT;

template <int COMBO, typename T, bool BATCH>
static cudaError_t launch_p(const PipeArgs& a, const PipeBatch& b, int grid, cudaStream_t s) {
    auto kern = pipelined_stage_kernel<COMBO, T, kNPT, BATCH>;
    static std::atomic<uint64_t> configured{0};
    cudaError_t err = ensure_smem_limit(kern, (int)sizeof(pipe::Smem<T>), configured);
    if (err != cudaSuccess) return err;
    kern<<<grid, 512 / kNPT, sizeof(pipe::Smem<T>), s>>>(a, b);
    return cudaGetLastError();
}

cudaError_t launch_pipelined(int combo, int fp32, const PipeArgs& a, int grid, cudaStream_t s) {
    const PipeBatch none{};
    if (combo == EUL_KG)
        return fp32 ? launch_p<EUL_KG, float, false>(a, none, grid, s) : launch_p<EUL_KG, double, false>(a, none, grid, s);
    if (combo == EUL_EC)
        return fp32 ? launch_p<EUL_EC, float, false>(a, none, grid, s) : launch_p<EUL_EC, double, false>(a, none, grid, s);
    return cudaErrorInvalidValue;
}

cudaError_t launch_pipelined_batch(int combo, int fp32, const PipeArgs& a, const PipeBatch& b, int grid,
                                   cudaStream_t s) {
    if (combo == EUL_KG)
        return fp32 ? launch_p<EUL_KG, float, true>(a, b, grid, s) : launch_p<EUL_KG, double, true>(a, b, grid, s);
    return cudaErrorInvalidValue;
}

template <int COMBO, typename T, bool BATCH>
static int occupancy_p() {
    auto kern = pipelined_stage_kernel<COMBO, T, kNPT, BATCH>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(pipe::Smem<T>)) !=
        cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, 512 / kNPT, sizeof(pipe::Smem<T>)) != cudaSuccess)
        return 0;
    return n;
}

int pipelined_blocks_per_sm(int combo, int fp32) {
    if (combo == EUL_KG) return fp32 ? occupancy_p<EUL_KG, float, false>() : occupancy_p<EUL_KG, double, false>();
    if (combo == EUL_EC) return fp32 ? occupancy_p<EUL_EC, float, false>() : occupancy_p<EUL_EC, double, false>();
    return 0;
}

int pipelined_batch_blocks_per_sm(int combo, int fp32) {
    if (combo == EUL_KG) return fp32 ? occupancy_p<EUL_KG, float, true>() : occupancy_p<EUL_KG, double, true>();
    return 0;
}

// The curved-grid kernel (FP32 bulk, Kennedy-Gruber): two CTAs per SM.
cudaError_t launch_pipelined_curved(const PipeCurvedArgs& a, int grid, cudaStream_t s) {
    auto kern = pipelined_curved_kernel<EUL_KG>;
    static std::atomic<uint64_t> configured{0};
    cudaError_t err = ensure_smem_limit(kern, (int)sizeof(pipec::Smem), configured);
    if (err != cudaSuccess) return err;
    kern<<<grid, pipec::NT, sizeof(pipec::Smem), s>>>(a);
    return cudaGetLastError();
}

int pipelined_curved_blocks_per_sm() {
    auto kern = pipelined_curved_kernel<EUL_KG>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(pipec::Smem)) !=
        cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, pipec::NT, sizeof(pipec::Smem)) != cudaSuccess)
        return 0;
    return n;
}

}  // namespace rb200
