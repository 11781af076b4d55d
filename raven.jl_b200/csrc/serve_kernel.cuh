// Batched stage kernel of the serving loop: one launch advances a stage of every active
// solve of one class (same dim, Nq, law, form, precision).  Solves live anywhere in the
// server's device arena; a chunk table maps each CTA to (solve, first element, count)
// and a descriptor table gives the solve's buffers and time step.  The launch shape is
// fixed (one CTA per chunk slot, empty slots exit at once), so a whole LSRK step of a
// class is captured once as a CUDA graph and replayed while solves come and go: only
// the tables change.  Per-element arithmetic is the one of stage_element, so a solve's
// result does not depend on which solves share its launch.
#pragma once

#include "stage_kernel.cuh"

namespace rb200 {

struct BatchArgs {
    StageArgs base;               // class constants (D, w, gamma, advection velocity, mode, rka)
    const SolveDesc* solves;
    const Chunk* chunks;
    const int32_t* nchunks;       // chunk slots in use (device)
    const int64_t* tick;          // class tick counter (device), advanced after each step
    int32_t stage;                // 0..4
    double rkb;                   // LSRK b coefficient of this stage (times each solve's dt)
};

template <int DIM, int NQ, int COMBO, int GEOM, typename T, int EPBX>
__global__ void __launch_bounds__(Shape<DIM, NQ, EPBX>::THREADS, 1)
    batched_stage_kernel(const __grid_constant__ BatchArgs B) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using S = Shape<DIM, NQ, EPBX>;
    const int nch = *B.nchunks;
    const int64_t tick = *B.tick;
    const int el = threadIdx.x / S::NP;
    for (int ci = blockIdx.x; ci < nch; ci += gridDim.x) {
        const Chunk c = B.chunks[ci];
        if (c.solve < 0 || c.count <= 0) continue;
        const SolveDesc& sd = B.solves[c.solve];
        const int par = (int)((tick - sd.start_tick + B.stage) & 1);
        ElemPtrs P;
        P.q_in = sd.q[par];
        P.q_out = sd.q[par ^ 1];
        P.dq = sd.dq;
        P.elem_geo = sd.elem_geo;
        P.vgeo = nullptr;
        P.sgeo = nullptr;
        P.nbr = sd.nbr;
        P.rkb_dt = B.rkb * sd.dt;
        P.ncflux = nullptr;
        for (int g = 0; g < c.count; g += S::EPB) {
            const int64_t e = c.first + g + el;
            stage_element<DIM, NQ, COMBO, GEOM, T, EPBX>(B.base, P, e, g + el < c.count, smem_raw);
            __syncthreads();  // the shared partner values are reused by the next group
        }
    }
}

// Initial data of a brick solve evaluated on the device at its LGL nodes:
// x_d = fma(dx_d, fma(1/2, r_i + 1, 0), c1_d) as Raven's brick points (lobattocells.jl:1657-1671).
// kind 1: Euler isentropic vortex (p[0] = strength, p[1] = u0 along x, p[2..3] = centre xy,
//         invariant along z); kind 2: advection sin(2 pi x) sin(2 pi y) [sin(2 pi z)] +
//         exp(-|x - c|^2 / (2 s^2)) with p[0] = s, p[1..3] = c.
struct InitArgs {
    double* q;
    const double* corners;  // (2, dim, E): c1, dx per direction
    int64_t E;
    int dim, nq, ns, kind;
    double gamma;
    double r[kMaxNq];
    double p[8];
};

}  // namespace rb200
