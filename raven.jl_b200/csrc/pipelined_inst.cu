// Instantiations and launch helpers of the pipelined 3-D stage kernels (Euler flux
// differencing and weak-form advection, Nq = 4, 6, 8): one state (the DGSEM handle) or
// the chunks of a serving class (BATCH).
#include "pipelined_adv.cuh"
#include "pipelined_curved.cuh"
#include "pipelined_curved64.cuh"
#include "pipelined_kernel.cuh"

namespace rb200 {

template <int COMBO, typename T, bool BATCH, int Q>
static cudaError_t launch_p(const PipeArgs& a, const PipeBatch& b, int grid, cudaStream_t s) {
    constexpr int kNPT = pipe_npt<T, Q>();
    auto kern = pipelined_stage_kernel<COMBO, T, kNPT, BATCH, Q>;
    static std::atomic<uint64_t> configured{0};
    cudaError_t err = ensure_smem_limit(kern, (int)sizeof(pipe::Smem<T, Q>), configured);
    if (err != cudaSuccess) return err;
    if constexpr (!BATCH)  // serving ticks follow host-written chunk tables: plain order
        return launch_pdl(kern, grid, Q * Q * Q / kNPT, sizeof(pipe::Smem<T, Q>), s, a, b);
    kern<<<grid, Q * Q * Q / kNPT, sizeof(pipe::Smem<T, Q>), s>>>(a, b);
    return cudaGetLastError();
}

// The advection law: one field, pipea::npt<Q>() nodes a thread.
template <typename T, bool BATCH, int Q>
static cudaError_t launch_a(const PipeArgs& a, const PipeBatch& b, int grid, cudaStream_t s) {
    auto kern = pipelined_adv_kernel<T, BATCH, Q>;
    static std::atomic<uint64_t> configured{0};
    cudaError_t err = ensure_smem_limit(kern, (int)sizeof(pipea::Smem<T, Q>), configured);
    if (err != cudaSuccess) return err;
    kern<<<grid, Q * Q * Q / pipea::npt<Q>(), sizeof(pipea::Smem<T, Q>), s>>>(a, b);
    return cudaGetLastError();
}

template <int COMBO, typename T, bool BATCH>
static cudaError_t launch_q(int nq, const PipeArgs& a, const PipeBatch& b, int grid, cudaStream_t s) {
    if constexpr (COMBO == ADV_WEAK) {
        switch (nq) {
            case 4: return launch_a<T, BATCH, 4>(a, b, grid, s);
            case 6: return launch_a<T, BATCH, 6>(a, b, grid, s);
            case 8: return launch_a<T, BATCH, 8>(a, b, grid, s);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (nq) {
        case 4: return launch_p<COMBO, T, BATCH, 4>(a, b, grid, s);
        case 6: return launch_p<COMBO, T, BATCH, 6>(a, b, grid, s);
        case 8: return launch_p<COMBO, T, BATCH, 8>(a, b, grid, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_pipelined(int nq, int combo, int fp32, const PipeArgs& a, int grid, cudaStream_t s) {
    const PipeBatch none{};
    if (combo == EUL_KG)
        return fp32 ? launch_q<EUL_KG, float, false>(nq, a, none, grid, s)
                    : launch_q<EUL_KG, double, false>(nq, a, none, grid, s);
    if (combo == EUL_EC)
        return fp32 ? launch_q<EUL_EC, float, false>(nq, a, none, grid, s)
                    : launch_q<EUL_EC, double, false>(nq, a, none, grid, s);
    if (combo == ADV_WEAK)
        return fp32 ? launch_q<ADV_WEAK, float, false>(nq, a, none, grid, s)
                    : launch_q<ADV_WEAK, double, false>(nq, a, none, grid, s);
    return cudaErrorInvalidValue;
}

cudaError_t launch_pipelined_batch(int nq, int combo, int fp32, const PipeArgs& a, const PipeBatch& b, int grid,
                                   cudaStream_t s) {
    if (combo == EUL_KG)
        return fp32 ? launch_q<EUL_KG, float, true>(nq, a, b, grid, s) : launch_q<EUL_KG, double, true>(nq, a, b, grid, s);
    if (combo == ADV_WEAK)
        return fp32 ? launch_q<ADV_WEAK, float, true>(nq, a, b, grid, s)
                    : launch_q<ADV_WEAK, double, true>(nq, a, b, grid, s);
    return cudaErrorInvalidValue;
}

template <int COMBO, typename T, bool BATCH, int Q>
static int occupancy_p() {
    constexpr int kNPT = pipe_npt<T, Q>();
    auto kern = pipelined_stage_kernel<COMBO, T, kNPT, BATCH, Q>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(pipe::Smem<T, Q>)) !=
        cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, Q * Q * Q / kNPT, sizeof(pipe::Smem<T, Q>)) !=
        cudaSuccess)
        return 0;
    return n;
}

template <typename T, bool BATCH, int Q>
static int occupancy_a() {
    auto kern = pipelined_adv_kernel<T, BATCH, Q>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(pipea::Smem<T, Q>)) !=
        cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, Q * Q * Q / pipea::npt<Q>(), sizeof(pipea::Smem<T, Q>)) !=
        cudaSuccess)
        return 0;
    return n;
}

template <int COMBO, typename T, bool BATCH>
static int occupancy_q(int nq) {
    if constexpr (COMBO == ADV_WEAK) {
        switch (nq) {
            case 4: return occupancy_a<T, BATCH, 4>();
            case 6: return occupancy_a<T, BATCH, 6>();
            case 8: return occupancy_a<T, BATCH, 8>();
            default: return 0;
        }
    }
    switch (nq) {
        case 4: return occupancy_p<COMBO, T, BATCH, 4>();
        case 6: return occupancy_p<COMBO, T, BATCH, 6>();
        case 8: return occupancy_p<COMBO, T, BATCH, 8>();
        default: return 0;
    }
}

int pipelined_blocks_per_sm(int nq, int combo, int fp32) {
    if (combo == EUL_KG) return fp32 ? occupancy_q<EUL_KG, float, false>(nq) : occupancy_q<EUL_KG, double, false>(nq);
    if (combo == EUL_EC) return fp32 ? occupancy_q<EUL_EC, float, false>(nq) : occupancy_q<EUL_EC, double, false>(nq);
    if (combo == ADV_WEAK)
        return fp32 ? occupancy_q<ADV_WEAK, float, false>(nq) : occupancy_q<ADV_WEAK, double, false>(nq);
    return 0;
}

int pipelined_batch_blocks_per_sm(int nq, int combo, int fp32) {
    if (combo == EUL_KG) return fp32 ? occupancy_q<EUL_KG, float, true>(nq) : occupancy_q<EUL_KG, double, true>(nq);
    if (combo == ADV_WEAK)
        return fp32 ? occupancy_q<ADV_WEAK, float, true>(nq) : occupancy_q<ADV_WEAK, double, true>(nq);
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

// The curved-grid kernel in FP64 (Kennedy-Gruber): two CTAs per SM.
cudaError_t launch_pipelined_curved64(const PipeCurvedArgs& a, int grid, cudaStream_t s) {
    auto kern = pipelined_curved64_kernel<EUL_KG>;
    static std::atomic<uint64_t> configured{0};
    cudaError_t err = ensure_smem_limit(kern, (int)sizeof(pipec64::Smem), configured);
    if (err != cudaSuccess) return err;
    kern<<<grid, pipec64::NT, sizeof(pipec64::Smem), s>>>(a);
    return cudaGetLastError();
}

int pipelined_curved64_blocks_per_sm() {
    auto kern = pipelined_curved64_kernel<EUL_KG>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(pipec64::Smem)) !=
        cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, pipec64::NT, sizeof(pipec64::Smem)) != cudaSuccess)
        return 0;
    return n;
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
