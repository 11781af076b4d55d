// Routes (dim, nq) to the per-pair stage-kernel instantiations (stage_inst.cu).
#include "rb200_internal.h"

namespace rb200 {

#define RB_DECL(D, Q)                                                                          \
    cudaError_t launch_stage_d##D##_q##Q(int combo, int geom, int fp32, const StageArgs& a, \
                                         cudaStream_t s);                                   \
    size_t smem_stage_d##D##_q##Q(int combo, int geom, int fp32);                            \
    cudaError_t launch_cluster_d##D##_q##Q(int fp32, const ClusterStepsArgs& c, int ctas, cudaStream_t s);
#define RB_DECL_DIM(D) RB_DECL(D, 2) RB_DECL(D, 3) RB_DECL(D, 4) RB_DECL(D, 5) RB_DECL(D, 6) RB_DECL(D, 7) RB_DECL(D, 8)
RB_DECL_DIM(1)
RB_DECL_DIM(2)
RB_DECL_DIM(3)

#define RB_CASE(D, Q) \
    case Q: return launch_stage_d##D##_q##Q(combo, geom, fp32, a, s);
#define RB_SCASE(D, Q) \
    case Q: return smem_stage_d##D##_q##Q(combo, geom, fp32);

cudaError_t launch_stage(int dim, int nq, int combo, int geom, int fp32, const StageArgs& a, cudaStream_t s) {
    if (dim == 1) {
        switch (nq) { RB_CASE(1, 2) RB_CASE(1, 3) RB_CASE(1, 4) RB_CASE(1, 5) RB_CASE(1, 6) RB_CASE(1, 7) RB_CASE(1, 8) }
    } else if (dim == 2) {
        switch (nq) { RB_CASE(2, 2) RB_CASE(2, 3) RB_CASE(2, 4) RB_CASE(2, 5) RB_CASE(2, 6) RB_CASE(2, 7) RB_CASE(2, 8) }
    } else if (dim == 3) {
        switch (nq) { RB_CASE(3, 2) RB_CASE(3, 3) RB_CASE(3, 4) RB_CASE(3, 5) RB_CASE(3, 6) RB_CASE(3, 7) RB_CASE(3, 8) }
    }
    return cudaErrorInvalidValue;
}

#define RB_CCASE(D, Q) \
    case Q: return launch_cluster_d##D##_q##Q(fp32, c, ctas, s);

cudaError_t launch_cluster_steps(int dim, int nq, int fp32, const ClusterStepsArgs& c, int ctas, cudaStream_t s) {
    if (dim == 1) {
        switch (nq) { RB_CCASE(1, 2) RB_CCASE(1, 3) RB_CCASE(1, 4) RB_CCASE(1, 5) RB_CCASE(1, 6) RB_CCASE(1, 7) RB_CCASE(1, 8) }
    } else if (dim == 2) {
        switch (nq) { RB_CCASE(2, 2) RB_CCASE(2, 3) RB_CCASE(2, 4) RB_CCASE(2, 5) RB_CCASE(2, 6) RB_CCASE(2, 7) RB_CCASE(2, 8) }
    } else if (dim == 3) {
        switch (nq) { RB_CCASE(3, 2) RB_CCASE(3, 3) RB_CCASE(3, 4) RB_CCASE(3, 5) RB_CCASE(3, 6) RB_CCASE(3, 7) RB_CCASE(3, 8) }
    }
    return cudaErrorInvalidValue;
}

size_t stage_smem_bytes(int dim, int nq, int combo, int geom, int fp32) {
    if (dim == 1) {
        switch (nq) { RB_SCASE(1, 2) RB_SCASE(1, 3) RB_SCASE(1, 4) RB_SCASE(1, 5) RB_SCASE(1, 6) RB_SCASE(1, 7) RB_SCASE(1, 8) }
    } else if (dim == 2) {
        switch (nq) { RB_SCASE(2, 2) RB_SCASE(2, 3) RB_SCASE(2, 4) RB_SCASE(2, 5) RB_SCASE(2, 6) RB_SCASE(2, 7) RB_SCASE(2, 8) }
    } else if (dim == 3) {
        switch (nq) { RB_SCASE(3, 2) RB_SCASE(3, 3) RB_SCASE(3, 4) RB_SCASE(3, 5) RB_SCASE(3, 6) RB_SCASE(3, 7) RB_SCASE(3, 8) }
    }
    return 0;
}

}  // namespace rb200
