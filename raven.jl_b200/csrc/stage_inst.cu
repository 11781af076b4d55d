// Instantiates the stage kernel for one (dim, nq) pair.  The build compiles this file
// once per pair with -DRB_DIM=<dim> -DRB_NQ=<nq> so that the instantiations build in
// parallel; dispatch.cu routes (dim, nq) to the matching entry point.
#include "stage_kernel.cuh"

#ifndef RB_DIM
#error "RB_DIM must be defined"
#endif
#ifndef RB_NQ
#error "RB_NQ must be defined"
#endif

#define RB_CAT2(a, b, c, d) a##b##c##d
#define RB_CAT(a, b, c, d) RB_CAT2(a, b, c, d)
#define RB_LAUNCH_NAME RB_CAT(launch_stage_d, RB_DIM, _q, RB_NQ)
#define RB_SMEM_NAME RB_CAT(smem_stage_d, RB_DIM, _q, RB_NQ)
#define RB_CLUSTER_NAME RB_CAT(launch_cluster_d, RB_DIM, _q, RB_NQ)

namespace rb200 {

template <int COMBO, int GEOM>
static cudaError_t launch_cg(int fp32, const StageArgs& a, cudaStream_t s) {
    const bool entropy_family = a.surface_flux == kFluxEC || a.surface_flux == kFluxKG ||
                                a.surface_flux == kFluxRoe || a.surface_flux == kFluxMatrix;
    if (entropy_family) {  // Euler only, FP64 only (the host checks both)
        if constexpr (COMBO == ADV_WEAK || COMBO == ADV_FDC) return cudaErrorInvalidValue;
        else return fp32 ? cudaErrorInvalidValue : launch_one<RB_DIM, RB_NQ, COMBO, GEOM, double, 1>(a, s);
    }
    return fp32 ? launch_one<RB_DIM, RB_NQ, COMBO, GEOM, float>(a, s)
                : launch_one<RB_DIM, RB_NQ, COMBO, GEOM, double>(a, s);
}

template <int COMBO>
static cudaError_t launch_c(int geom, int fp32, const StageArgs& a, cudaStream_t s) {
    return geom == GEOM_AFFINE ? launch_cg<COMBO, GEOM_AFFINE>(fp32, a, s) : launch_cg<COMBO, GEOM_CURVED>(fp32, a, s);
}

cudaError_t RB_LAUNCH_NAME(int combo, int geom, int fp32, const StageArgs& a, cudaStream_t s) {
    switch (combo) {
        case ADV_WEAK: return launch_c<ADV_WEAK>(geom, fp32, a, s);
        case ADV_FDC: return launch_c<ADV_FDC>(geom, fp32, a, s);
        case EUL_WEAK: return launch_c<EUL_WEAK>(geom, fp32, a, s);
        case EUL_FDC: return launch_c<EUL_FDC>(geom, fp32, a, s);
        case EUL_KG: return launch_c<EUL_KG>(geom, fp32, a, s);
        case EUL_EC: return launch_c<EUL_EC>(geom, fp32, a, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int COMBO>
static size_t smem_c(int geom, int fp32) {
    if (geom == GEOM_AFFINE)
        return fp32 ? PersistentCfg<RB_DIM, RB_NQ, COMBO, GEOM_AFFINE, float>::smem
                    : PersistentCfg<RB_DIM, RB_NQ, COMBO, GEOM_AFFINE, double>::smem;
    return fp32 ? PersistentCfg<RB_DIM, RB_NQ, COMBO, GEOM_CURVED, float>::smem
                : PersistentCfg<RB_DIM, RB_NQ, COMBO, GEOM_CURVED, double>::smem;
}

cudaError_t RB_CLUSTER_NAME(int fp32, const ClusterStepsArgs& c, int ctas, cudaStream_t s) {
    return fp32 ? launch_cluster_adv<RB_DIM, RB_NQ, float>(c, ctas, s) : launch_cluster_adv<RB_DIM, RB_NQ, double>(c, ctas, s);
}

size_t RB_SMEM_NAME(int combo, int geom, int fp32) {
    switch (combo) {
        case ADV_WEAK: return smem_c<ADV_WEAK>(geom, fp32);
        case ADV_FDC: return smem_c<ADV_FDC>(geom, fp32);
        case EUL_WEAK: return smem_c<EUL_WEAK>(geom, fp32);
        case EUL_FDC: return smem_c<EUL_FDC>(geom, fp32);
        case EUL_KG: return smem_c<EUL_KG>(geom, fp32);
        case EUL_EC: return smem_c<EUL_EC>(geom, fp32);
        default: return 0;
    }
}

}  // namespace rb200
