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

// The CTA walks chunk slots blockIdx.x + k*gridDim.x and, within a chunk, groups of EPB
// elements.  Where the generic kernel prefetches (3-D, FP32 bulk), every thread copies
// its node's state and register in the CTA's next group (possibly the next chunk's) into
// its own shared-memory slots with cp.async while the current group runs.
template <int DIM, int NQ, int COMBO, int GEOM, typename T, int EPBX>
__global__ void __launch_bounds__(Shape<DIM, NQ, EPBX>::THREADS,
                                  (PersistentCfg<DIM, NQ, COMBO, GEOM, T, EPBX>::MIN_CTAS))
    batched_stage_kernel(const __grid_constant__ BatchArgs B) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using S = Shape<DIM, NQ, EPBX>;
    using PC = PersistentCfg<DIM, NQ, COMBO, GEOM, T, EPBX>;
    constexpr int NS = PC::NS, TH = S::THREADS, NP = S::NP;
    double* qs = reinterpret_cast<double*>(smem_raw + PC::off_q);  // [2][NS][TH]
    T* dqs = reinterpret_cast<T*>(smem_raw + PC::off_dq);           // [2][NS][TH]
    const int nch = *B.nchunks;
    const int64_t tick = *B.tick;
    const int tid = threadIdx.x, el = tid / NP, n = tid - el * NP;
    const bool pf_dq = PC::PF && B.base.mode == MODE_STAGE;
    auto live = [&](int ci) {
        while (ci < nch && (B.chunks[ci].solve < 0 || B.chunks[ci].count <= 0)) ci += gridDim.x;
        return ci;
    };
    auto elem = [&](int ci, int g, ElemPtrs& P, int64_t& e, bool& active) {
        const Chunk c = B.chunks[ci];
        const SolveDesc& sd = B.solves[c.solve];
        const int par = (int)((tick - sd.start_tick + B.stage) & 1);
        P.q_in = sd.q[par];
        P.q_out = sd.q[par ^ 1];
        P.dq = sd.dq;
        P.elem_geo = sd.elem_geo;
        P.vgeo = nullptr;
        P.sgeo = nullptr;
        P.nbr = sd.nbr;
        P.rkb_dt = B.rkb * sd.dt;
        P.ncflux = nullptr;
        P.vmapP = nullptr;
        e = c.first + g + el;
        active = g + el < c.count;
    };
    auto prefetch = [&](int ci, int g, int b) {
        if (PC::PF && ci < nch) {
            ElemPtrs P;
            int64_t e;
            bool active;
            elem(ci, g, P, e, active);
            if (active) {
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    const size_t gi = ((size_t)e * NS + s) * NP + n;
                    cpa8(qs + (b * NS + s) * TH + tid, P.q_in + gi);
                    if (pf_dq) {
                        if constexpr (sizeof(T) == 4) cpa4(dqs + (b * NS + s) * TH + tid, static_cast<const float*>(P.dq) + gi);
                        else cpa8(dqs + (b * NS + s) * TH + tid, static_cast<const double*>(P.dq) + gi);
                    }
                }
            }
        }
        cpa_commit();
    };
    int ci = live(blockIdx.x), g = 0, b = 0;
    prefetch(ci, 0, 0);
    bool tables_ready = false;
    while (ci < nch) {
        int ci2 = ci, g2 = g + S::EPB;  // the CTA's next group
        if (g2 >= B.chunks[ci].count) {
            ci2 = live(ci + gridDim.x);
            g2 = 0;
        }
        cpa_wait_all();
        prefetch(ci2, g2, b ^ 1);
        ElemPtrs P;
        int64_t e;
        bool active;
        elem(ci, g, P, e, active);
        Prefetched pf;
        if (PC::PF) {
            pf.q = qs + b * NS * TH + tid;
            pf.dq = pf_dq ? static_cast<const void*>(dqs + b * NS * TH + tid) : nullptr;
            pf.stride = TH;
        }
        pf.tables_ready = tables_ready;
        stage_element<DIM, NQ, COMBO, GEOM, T, EPBX>(B.base, P, e, active, smem_raw, pf);
        tables_ready = true;
        __syncthreads();  // the shared partner values are reused by the next group
        ci = ci2;
        g = g2;
        b ^= 1;
    }
    cpa_wait_all();
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
