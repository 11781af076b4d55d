// Instantiations of the batched serving kernel for one dimension (compiled once per
// dim with -DRB_SERVE_DIM=<dim>): Nq in {4, 6, 8} (polynomial orders 3, 5, 7),
// advection weak form and Euler Kennedy-Gruber flux differencing, unwarped bricks,
// FP64 or FP32 bulk, and the element-per-CTA tiles the autotuner chooses from.
#include "serve_kernel.cuh"

#ifndef RB_SERVE_DIM
#error "RB_SERVE_DIM must be defined"
#endif

#define RB_SCAT2(a, b) a##b
#define RB_SCAT(a, b) RB_SCAT2(a, b)

namespace rb200 {

namespace {

template <int NQ, int COMBO, typename T, int EPB>
cudaError_t launch_t(const BatchArgs& b, int grid, cudaStream_t s, int* blocks_per_sm) {
    auto kern = batched_stage_kernel<RB_SERVE_DIM, NQ, COMBO, GEOM_AFFINE, T, EPB>;
    using S = Shape<RB_SERVE_DIM, NQ, EPB>;
    using PC = PersistentCfg<RB_SERVE_DIM, NQ, COMBO, GEOM_AFFINE, T, EPB>;
    static std::atomic<uint64_t> configured{0};
    cudaError_t err = ensure_smem_limit(kern, (int)PC::smem, configured);
    if (err != cudaSuccess) return err;
    if (blocks_per_sm) {  // occupancy query only
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kern, S::THREADS, PC::smem);
    }
    kern<<<grid, S::THREADS, PC::smem, s>>>(b);
    return cudaGetLastError();
}

// Candidate tiles: half, default and double the default elements per CTA (equal where
// the 512-thread limit does not allow a variant).
template <int NQ>
struct Tiles {
    static constexpr int NP = IPow<NQ, RB_SERVE_DIM>::v;
    static constexpr int D = NP >= 256 ? 1 : 256 / NP;
    static constexpr int LO = D > 1 ? D / 2 : 1;
    static constexpr int HI = (2 * D * NP <= 512) ? 2 * D : D;
};

template <int NQ, int COMBO, typename T>
cudaError_t launch_tiles(int tile, const BatchArgs& b, int grid, cudaStream_t s, int* bps) {
    using TL = Tiles<NQ>;
    if (tile == 0) return launch_t<NQ, COMBO, T, TL::LO>(b, grid, s, bps);
    if (tile == 1) return launch_t<NQ, COMBO, T, TL::D>(b, grid, s, bps);
    return launch_t<NQ, COMBO, T, TL::HI>(b, grid, s, bps);
}

template <int NQ>
cudaError_t launch_nq(int combo, int fp32, int tile, const BatchArgs& b, int grid, cudaStream_t s, int* bps) {
    if (combo == ADV_WEAK)
        return fp32 ? launch_tiles<NQ, ADV_WEAK, float>(tile, b, grid, s, bps)
                    : launch_tiles<NQ, ADV_WEAK, double>(tile, b, grid, s, bps);
    if (combo == EUL_KG)
        return fp32 ? launch_tiles<NQ, EUL_KG, float>(tile, b, grid, s, bps)
                    : launch_tiles<NQ, EUL_KG, double>(tile, b, grid, s, bps);
    return cudaErrorInvalidValue;
}

template <int NQ>
int tiles_nq(int* epb) {
    using TL = Tiles<NQ>;
    epb[0] = TL::LO;
    epb[1] = TL::D;
    epb[2] = TL::HI;
    return 3;
}

}  // namespace

// tile: 0, 1, 2 = half, default, double the default elements per CTA.
// blocks_per_sm != nullptr: occupancy query, nothing is launched.
cudaError_t RB_SCAT(launch_batched_d, RB_SERVE_DIM)(int nq, int combo, int fp32, int tile, const BatchArgs& b,
                                                    int grid, cudaStream_t s, int* blocks_per_sm) {
    switch (nq) {
        case 4: return launch_nq<4>(combo, fp32, tile, b, grid, s, blocks_per_sm);
        case 6: return launch_nq<6>(combo, fp32, tile, b, grid, s, blocks_per_sm);
        case 8: return launch_nq<8>(combo, fp32, tile, b, grid, s, blocks_per_sm);
        default: return cudaErrorInvalidValue;
    }
}

int RB_SCAT(batched_tiles_d, RB_SERVE_DIM)(int nq, int* epb) {
    switch (nq) {
        case 4: return tiles_nq<4>(epb);
        case 6: return tiles_nq<6>(epb);
        case 8: return tiles_nq<8>(epb);
        default: return 0;
    }
}

}  // namespace rb200
