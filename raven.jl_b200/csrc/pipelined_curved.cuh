// Persistent, bulk-copy-pipelined LSRK stage kernel for 3-D hexahedra with Nq = 8 on
// curved (warped) grids: Kennedy-Gruber flux differencing, FP32 bulk arithmetic, FP64
// state, metrics and LSRK state update.
//
// The curved form of esvolumeterm_dir! (src/balancelaws/dgsem.jl:514-608) contracts the
// two-point flux of nodes i and a on a line in direction dir with
//     G_d = D[a,i] l_g[a][dir][d] - D[i,a] l_g[i][dir][d],   l_g = wJ dRdX (vgeo rows),
// and the result is scaled by MJI.  The surface term (dgsem.jl:733-784) takes the
// Rusanov or central flux with the face normal n and subtracts (wsJ nf) MJI.
//
// Each CTA owns a strided set of elements; two CTAs share an SM.  Per element:
// * the state q and the face geometry (n, wsJ for the 384 face nodes) arrive by 1-D
//   bulk copies (cp.async.bulk, completion on mbarriers): q is issued one element ahead,
//   right after the partner values of the current element are built from it; the face
//   geometry after the current element's faces are done;
// * the FP32 LSRK register arrives by a bulk copy issued at the start of the element;
// * each thread loads the metric rows and MJI of its two nodes from global memory before
//   it waits for q, so that the loads overlap that wait;
// * the neighbour face traces arrive with cp.async during the volume term;
// * the element's own old q is read at the end (L2-resident: it arrived by bulk copy).
//
// A thread owns nodes t and t + 256 (same i, j; k and k + 4), so their z partners are
// loaded once.  Every wait on an mbarrier is bounded: after kWaitLimit polls the CTA
// records RB200 status TIMEOUT in *A.status and returns.
#pragma once

#include "pipelined_kernel.cuh"

// unroll factor of the curved kernels' pair loops over partners (8, full: measured 3.8 % (FP32
// bulk) and 2.6 % (FP64) faster than 2 on the warped 32^3 grid, 128 registers, no spills)
#ifndef RB200_CURVED_UNROLL
#define RB200_CURVED_UNROLL 8
#endif

namespace rb200 {

constexpr int kCurvedUnroll = RB200_CURVED_UNROLL;

struct PipeCurvedArgs {
    const double* q_in;
    double* q_out;
    float* dq;               // FP32 LSRK register (FP32-bulk kernel)
    double* dq64;            // FP64 LSRK register (FP64 kernel)
    const double* vgeo;      // (512, 11, E): wJ dRdX[dir][d] (dir-major), MJI, MJ
    const double* sgeo;      // (4, 384, E): n, wsJ per face node
    const int32_t* nbr;      // (6, E)
    int32_t* status;
    int64_t E;               // elements e_begin..E-1 are computed
    int64_t e_begin;
    int32_t mode;            // MODE_STAGE or MODE_STAGE_FIRST
    int32_t surface_rusanov;
    double rka, rkb_dt, gamma;
    double D[64];            // D[i + 8 j] = l_j'(r_i)
};

namespace pipec {

using pipe::NAUX;
using pipe::NP;
using pipe::NPP;
using pipe::NQ;
using pipe::NS;
using pipe::NSLOT;
using pipe::PAD;
constexpr int NT = 256, NVG = 11;

struct Smem {
    double q[NS][NP];                 // element state (bulk copy)
    double sg[NSLOT][4];              // face normal and wsJ per face slot (bulk copy)
    __align__(16) float dqb[NS][NP];  // the element's LSRK register (bulk copy)
    float4 auxa[NPP];                 // partner values: rho/2, u/2
    float2 auxb[NPP];                 // e/2, p/2
    float4 lgd[3][NPP];               // l_g[dir][0..2] of each node
    double slot[NS][NSLOT];           // neighbour trace, then (wsJ nf) MJI per face slot
    float mji[NP];
    float D[NQ][NQ];                  // D[i][j] = l_j'(r_i)
    int32_t nb[2][8];                 // neighbours of the current / next element
    uint64_t barq, bars, bard;        // arrivals of q, face geometry, register
};

}  // namespace pipec

template <int COMBO>
__global__ void __launch_bounds__(256, 2) pipelined_curved_kernel(const __grid_constant__ PipeCurvedArgs A) {
    using namespace pipe;
    using namespace pipec;
    static_assert(COMBO == EUL_KG, "the curved pipelined kernel implements Kennedy-Gruber");
    extern __shared__ __align__(128) unsigned char pipe_smem_raw[];
    pipec::Smem& sm = *reinterpret_cast<pipec::Smem*>(pipe_smem_raw);
    const int t = threadIdx.x;
    const int ii = t & 7, jj = (t >> 3) & 7, k0 = t >> 6;
    const bool read_dq = A.mode == MODE_STAGE;
    const uint32_t qbytes = NS * NP * sizeof(double), sgbytes = NSLOT * 4 * sizeof(double),
                   dqbytes = NS * NP * sizeof(float);
    const float gm1 = (float)(A.gamma - 1.0), gam = (float)A.gamma;

    if (t == 0) {
        mbar_init(&sm.barq, 1);
        mbar_init(&sm.bars, 1);
        mbar_init(&sm.bard, 1);
        fence_mbar_init();
    }
    for (int c = t; c < 64; c += NT) sm.D[c & 7][c >> 3] = (float)A.D[c];
    int64_t e = A.e_begin + blockIdx.x;
    if (t < 6 && e < A.E) cp_async4(&sm.nb[0][t], A.nbr + 6 * e + t);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    if (t == 0 && e < A.E) {
        mbar_expect_tx(&sm.barq, qbytes);
        bulk_g2s(&sm.q[0][0], A.q_in + (size_t)e * NS * NP, qbytes, &sm.barq);
        mbar_expect_tx(&sm.bars, sgbytes);
        bulk_g2s(&sm.sg[0][0], A.sgeo + (size_t)e * NSLOT * 4, sgbytes, &sm.bars);
    }
    uint32_t phq = 0, phs = 0, phd = 0;
    for (int buf = 0; e < A.E; buf ^= 1, e += gridDim.x) {
        const int64_t en = e + gridDim.x;  // the next element of this CTA
        // ---- metric rows and MJI of the thread's nodes (overlap the wait for q)
        double vgl[2][9], mjid[2];
        {
            const double* vg = A.vgeo + (size_t)e * NVG * NP + t;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
#pragma unroll
                for (int c = 0; c < 9; ++c) vgl[h][c] = __ldg(vg + c * NP + NT * h);
                mjid[h] = __ldg(vg + 9 * NP + NT * h);
            }
        }
        if (__syncthreads_or(!bounded_wait(&sm.barq, phq))) {
            if (t == 0) atomicExch(A.status, kStatusTimeout);
            return;
        }
        phq ^= 1;
        // ---- partner values, metric rows and MJI into shared memory
        float own[2][NAUX], lgo[2][9], mjiT[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int n = t + NT * h;
            const float rho = (float)sm.q[0][n];
            const float rinv = 1.f / rho;
            const float m0 = (float)sm.q[1][n], m1 = (float)sm.q[2][n], m2 = (float)sm.q[3][n];
            const float rhoe = (float)sm.q[4][n];
            const float u0 = m0 * rinv, u1 = m1 * rinv, u2 = m2 * rinv;
            const float p = gm1 * (rhoe - (m0 * m0 + m1 * m1 + m2 * m2) / (2.f * rho));
            own[h][0] = rho * 0.5f;
            own[h][1] = u0 * 0.5f;
            own[h][2] = u1 * 0.5f;
            own[h][3] = u2 * 0.5f;
            own[h][4] = (rhoe / rho) * 0.5f;
            own[h][5] = p * 0.5f;
            sm.auxa[PAD(n)] = make_float4(own[h][0], own[h][1], own[h][2], own[h][3]);
            sm.auxb[PAD(n)] = make_float2(own[h][4], own[h][5]);
#pragma unroll
            for (int c = 0; c < 9; ++c) lgo[h][c] = (float)vgl[h][c];
#pragma unroll
            for (int dir = 0; dir < 3; ++dir)
                sm.lgd[dir][PAD(n)] = make_float4(lgo[h][3 * dir], lgo[h][3 * dir + 1], lgo[h][3 * dir + 2], 0.f);
            mjiT[h] = (float)mjid[h];
            sm.mji[n] = mjiT[h];
        }
        __syncthreads();  // #1: partner values ready; q is free
        if (t == 0) {
            fence_proxy_async();  // q and dqb were last read by the generic proxy
            if (en < A.E) {  // the next element's state
                mbar_expect_tx(&sm.barq, qbytes);
                bulk_g2s(&sm.q[0][0], A.q_in + (size_t)en * NS * NP, qbytes, &sm.barq);
            }
            if (read_dq) {  // this element's register (the previous element's final phase is done)
                mbar_expect_tx(&sm.bard, dqbytes);
                bulk_g2s(&sm.dqb[0][0], A.dq + (size_t)e * NS * NP, dqbytes, &sm.bard);
            }
        }
        if (t < 6 && en < A.E) cp_async4(&sm.nb[buf ^ 1][t], A.nbr + 6 * en + t);
        // neighbour traces of this thread's face slots t and t + 256
#pragma unroll
        for (int sl = 0; sl < 2; ++sl) {
            const int slot = t + NT * sl;
            if (slot >= NSLOT) continue;
            int vn, opp;
            slot_nodes(slot, vn, opp);
            const int ne = sm.nb[buf][slot >> 6];
            if (ne >= 0) {
                const double* qn = A.q_in + (size_t)ne * NS * NP + opp;
#pragma unroll
                for (int s = 0; s < NS; ++s) cp_async8(&sm.slot[s][slot], qn + s * NP);
            }
        }
        cp_async_commit();

        // ---- volume term: pairs along x, y, z with the averaged metric combination G
        float acc[2][NS];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int s = 0; s < NS; ++s) acc[h][s] = 0.f;
        auto pair = [&](float (&ac)[NS], const float (&o)[NAUX], const float4 pa, const float2 pb, const float4 lp,
                        const float* lo, const float Dai, const float Dia) {
            float G[3];
            // the self pair, whose G must cancel exactly, is never formed (a != i)
            G[0] = fmaf(Dai, lp.x, -(Dia * lo[0]));
            G[1] = fmaf(Dai, lp.y, -(Dia * lo[1]));
            G[2] = fmaf(Dai, lp.z, -(Dia * lo[2]));
            const float rb = o[0] + pa.x;
            const float ub0 = o[1] + pa.y, ub1 = o[2] + pa.z, ub2 = o[3] + pa.w;
            const float eb = o[4] + pb.x, pbar = o[5] + pb.y;
            const float un = ub0 * G[0] + ub1 * G[1] + ub2 * G[2];
            const float f1 = rb * un;
            ac[0] += f1;
            ac[1] += f1 * ub0 + pbar * G[0];
            ac[2] += f1 * ub1 + pbar * G[1];
            ac[3] += f1 * ub2 + pbar * G[2];
            ac[4] += un * (rb * eb + pbar);
        };
#pragma unroll kCurvedUnroll
        for (int a = 0; a < NQ; ++a) {
            const float Dax = sm.D[a][ii], Dxa = sm.D[ii][a];
            const float Day = sm.D[a][jj], Dya = sm.D[jj][a];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int kk = k0 + 4 * h;
                if (a != ii) {
                    const int na = a + 8 * (jj + 8 * kk);
                    pair(acc[h], own[h], sm.auxa[PAD(na)], sm.auxb[PAD(na)], sm.lgd[0][PAD(na)], &lgo[h][0], Dax, Dxa);
                }
                if (a != jj) {
                    const int na = ii + 8 * (a + 8 * kk);
                    pair(acc[h], own[h], sm.auxa[PAD(na)], sm.auxb[PAD(na)], sm.lgd[1][PAD(na)], &lgo[h][3], Day, Dya);
                }
            }
            const int nz = ii + 8 * (jj + 8 * a);
            const float4 za = sm.auxa[PAD(nz)], zl = sm.lgd[2][PAD(nz)];
            const float2 zb = sm.auxb[PAD(nz)];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int kk = k0 + 4 * h;
                if (a != kk) pair(acc[h], own[h], za, zb, zl, &lgo[h][6], sm.D[a][kk], sm.D[kk][a]);
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int s = 0; s < NS; ++s) acc[h][s] = acc[h][s] * mjiT[h];

        // ---- face-slot contributions (wsJ nf) MJI, written over the slot's trace
        cp_async_wait_all();
        if (__syncthreads_or(!bounded_wait(&sm.bars, phs))) {  // also: the traces of every thread
            if (t == 0) atomicExch(A.status, kStatusTimeout);
            return;
        }
        phs ^= 1;
#pragma unroll
        for (int sl = 0; sl < 2; ++sl) {
            const int slot = t + NT * sl;
            if (slot >= NSLOT) continue;
            const int f = slot >> 6;
            int vn, opp;
            slot_nodes(slot, vn, opp);
            const bool open_face = sm.nb[buf][f] >= 0;
            const float nx = (float)sm.sg[slot][0], ny = (float)sm.sg[slot][1], nz = (float)sm.sg[slot][2];
            const float wsJ = (float)sm.sg[slot][3];
            float qm[NS], qp[NS], Fm[NS], Fp[NS], wm, wp;
            {
                const float4 a4 = sm.auxa[PAD(vn)];
                const float2 b2 = sm.auxb[PAD(vn)];
                const float rho = 2.f * a4.x;
                qm[0] = rho;
                qm[1] = rho * (2.f * a4.y);
                qm[2] = rho * (2.f * a4.z);
                qm[3] = rho * (2.f * a4.w);
                qm[4] = rho * (2.f * b2.x);
            }
            // normal flux and wave speed of one side (euler.jl:50-68)
            auto side_flux = [&](const float (&qq)[NS], float (&F)[NS], float& w) {
                const float rho = qq[0], rhoe = qq[4];
                const float u0 = qq[1] / rho, u1 = qq[2] / rho, u2 = qq[3] / rho;
                const float rr = qq[1] * qq[1] + qq[2] * qq[2] + qq[3] * qq[3];
                const float p = gm1 * (rhoe - rr / (2.f * rho));
                const float un = u0 * nx + u1 * ny + u2 * nz;
                const float mn = qq[1] * nx + qq[2] * ny + qq[3] * nz;
                F[0] = mn;
                F[1] = mn * u0 + p * nx;
                F[2] = mn * u1 + p * ny;
                F[3] = mn * u2 + p * nz;
                F[4] = un * (rhoe + p);
                w = fabsf(un) + sqrtf(gam * p / rho);
            };
            side_flux(qm, Fm, wm);
            if (open_face) {
#pragma unroll
                for (int s = 0; s < NS; ++s) qp[s] = (float)sm.slot[s][slot];
                side_flux(qp, Fp, wp);
            } else {  // boundary face: q+ = q- (balancelaw.jl:77)
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    qp[s] = qm[s];
                    Fp[s] = Fm[s];
                }
                wp = wm;
            }
            const float mx = fmaxf(wm, wp);
            const float mj = sm.mji[vn];
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const float fc = (Fm[s] + Fp[s]) * 0.5f;
                const float nf = A.surface_rusanov ? fc - (mx * (qp[s] - qm[s])) * 0.5f : fc;
                sm.slot[s][slot] = (double)((wsJ * nf) * mj);
            }
        }
        // #2: face contributions ready, and the element's register has landed
        if (__syncthreads_or(read_dq && !bounded_wait(&sm.bard, phd))) {
            if (t == 0) atomicExch(A.status, kStatusTimeout);
            return;
        }
        if (read_dq) phd ^= 1;
        if (t == 0 && en < A.E) {  // the next element's face geometry (this element's faces are done)
            fence_proxy_async();
            mbar_expect_tx(&sm.bars, sgbytes);
            bulk_g2s(&sm.sg[0][0], A.sgeo + (size_t)en * NSLOT * 4, sgbytes, &sm.bars);
        }
        // ---- own nodes: dq = rka dq + volume - faces (x, y, z order); q_out = q + rkb dt dq
        const size_t g0 = (size_t)e * NS * NP + t;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int kk = k0 + 4 * h;
            int slots[3] = {-1, -1, -1};
            if (ii == 0) slots[0] = jj + 8 * kk;
            else if (ii == NQ - 1) slots[0] = 64 + jj + 8 * kk;
            if (jj == 0) slots[1] = 128 + ii + 8 * kk;
            else if (jj == NQ - 1) slots[1] = 192 + ii + 8 * kk;
            if (kk == 0) slots[2] = 256 + ii + 8 * jj;
            else if (kk == NQ - 1) slots[2] = 320 + ii + 8 * jj;
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const size_t g = g0 + NT * h + s * NP;
                float v = acc[h][s];
                if (read_dq) v = (float)A.rka * sm.dqb[s][t + NT * h] + v;
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    if (slots[d] >= 0) v = v - (float)sm.slot[s][slots[d]];
                A.dq[g] = v;
                A.q_out[g] = __ldg(A.q_in + g) + A.rkb_dt * (double)v;
            }
        }
    }
}

}  // namespace rb200
