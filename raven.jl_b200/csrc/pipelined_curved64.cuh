// Persistent, bulk-copy-pipelined LSRK stage kernel for 3-D hexahedra with Nq = 8 on
// curved (warped) grids in FP64: Kennedy-Gruber flux differencing, Rusanov or central
// surface flux, FP64 state, metrics, arithmetic and LSRK register.
//
// The curved form of esvolumeterm_dir! (src/balancelaws/dgsem.jl:514-608) contracts the
// two-point flux of nodes i and a on a line in direction dir with
//     G_d = D[a,i] l_g[a][dir][d] - D[i,a] l_g[i][dir][d],   l_g = wJ dRdX (vgeo rows),
// and the sum is scaled by MJI.  The surface term (dgsem.jl:733-784) takes the Rusanov
// or central flux with the face normal n and subtracts (wsJ nf) MJI.
//
// Layout per CTA (two CTAs of 256 threads share an SM; ~105 KB of shared memory each):
// * the element's state q arrives by one 1-D bulk copy, issued one element ahead right
//   after the partner values of the current element have been built from it;
// * partner values (rho/2, u/2, e/2, p/2) and the nine metric rows l_g[dir][d] of every
//   node are staged in shared memory, padded so that lines along x and y do not share
//   banks; each thread loads its two nodes' metric rows from global memory before it
//   waits for q, so that those loads overlap the wait;
// * the pair loop runs direction by direction, so that only the own node's metric row of
//   the current direction is held in registers;
// * the neighbour face traces arrive with cp.async during the volume term; the face
//   normals, wsJ and MJI of a thread's face slots are read from global memory as the
//   face phase starts (the neighbour traces are waited for there anyway);
// * the element's own old state and FP64 register are read at the end, like the brick
//   kernel (staging them in shared memory costs shared-memory bandwidth, which the pair
//   loop needs).
//
// A thread owns nodes t and t + 256 (same i, j; k and k + 4), so their z partners are
// loaded once.  Every wait on an mbarrier is bounded: after kWaitLimit polls the CTA
// records RB200 status TIMEOUT in *A.status and returns.
#pragma once

#include "pipelined_curved.cuh"

namespace rb200 {

namespace pipec64 {

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
    pipe::AuxBuf<double> aux;         // partner values
    double2 lga[3][NPP];              // l_g[dir][0..1] of each node
    double lgb[3][NPP];               // l_g[dir][2]
    double slot[NS][NSLOT];           // neighbour trace, then (wsJ nf) MJI per face slot
    double D[NQ][NQ];                 // D[i][j] = l_j'(r_i)
    int32_t nb[2][8];                 // neighbours of the current / next element
    uint64_t barq;                    // arrival of q
};

}  // namespace pipec64

template <int COMBO>
__global__ void __launch_bounds__(256, 2) pipelined_curved64_kernel(const __grid_constant__ PipeCurvedArgs A) {
    using namespace pipe;
    using namespace pipec64;
    static_assert(COMBO == EUL_KG, "the curved pipelined kernel implements Kennedy-Gruber");
    extern __shared__ __align__(128) unsigned char pipe_smem_raw[];
    pipec64::Smem& sm = *reinterpret_cast<pipec64::Smem*>(pipe_smem_raw);
    const int t = threadIdx.x;
    const int ii = t & 7, jj = (t >> 3) & 7, k0 = t >> 6;
    const bool read_dq = A.mode == MODE_STAGE;
    const uint32_t qbytes = NS * NP * sizeof(double);
    const double gm1 = A.gamma - 1.0, gam = A.gamma;

    if (t == 0) {
        mbar_init(&sm.barq, 1);
        fence_mbar_init();
    }
    for (int c = t; c < 64; c += NT) sm.D[c & 7][c >> 3] = A.D[c];
    int64_t e = A.e_begin + blockIdx.x;
    if (t < 6 && e < A.E) cp_async4(&sm.nb[0][t], A.nbr + 6 * e + t);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    if (t == 0 && e < A.E) {
        mbar_expect_tx(&sm.barq, qbytes);
        bulk_g2s(&sm.q[0][0], A.q_in + (size_t)e * NS * NP, qbytes, &sm.barq);
    }
    uint32_t phq = 0;
    for (int buf = 0; e < A.E; buf ^= 1, e += gridDim.x) {
        const int64_t en = e + gridDim.x;  // the next element of this CTA
        // ---- metric rows of the thread's nodes (overlap the wait for q)
        double vgl[2][9];
        {
            const double* vg = A.vgeo + (size_t)e * NVG * NP + t;
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int c = 0; c < 9; ++c) vgl[h][c] = __ldg(vg + c * NP + NT * h);
        }
        if (__syncthreads_or(!bounded_wait(&sm.barq, phq))) {
            if (t == 0) atomicExch(A.status, kStatusTimeout);
            return;
        }
        phq ^= 1;
        // ---- partner values and metric rows into shared memory
        double own[2][NAUX];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int n = t + NT * h;
            const double rho = sm.q[0][n];
            const double rinv = 1.0 / rho;
            const double m0 = sm.q[1][n], m1 = sm.q[2][n], m2 = sm.q[3][n];
            const double rhoe = sm.q[4][n];
            const double p = gm1 * (rhoe - (m0 * m0 + m1 * m1 + m2 * m2) * (0.5 * rinv));
            own[h][0] = rho * 0.5;
            own[h][1] = m0 * rinv * 0.5;
            own[h][2] = m1 * rinv * 0.5;
            own[h][3] = m2 * rinv * 0.5;
            own[h][4] = rhoe * rinv * 0.5;
            own[h][5] = p * 0.5;
            sm.aux.put(PAD(n), own[h]);
#pragma unroll
            for (int dir = 0; dir < 3; ++dir) {
                sm.lga[dir][PAD(n)] = make_double2(vgl[h][3 * dir], vgl[h][3 * dir + 1]);
                sm.lgb[dir][PAD(n)] = vgl[h][3 * dir + 2];
            }
        }
        __syncthreads();  // #1: partner values and metric rows ready; q is free
        if (t == 0 && en < A.E) {  // the next element's state
            fence_proxy_async();   // q was last read by the generic proxy
            mbar_expect_tx(&sm.barq, qbytes);
            bulk_g2s(&sm.q[0][0], A.q_in + (size_t)en * NS * NP, qbytes, &sm.barq);
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

        // ---- volume term: pairs along x, y, z with the metric combination G, direction by
        // direction (the own node's metric row of that direction stays in registers)
        double acc[2][NS];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int s = 0; s < NS; ++s) acc[h][s] = 0.0;
        auto pair = [&](double (&ac)[NS], const double (&o)[NAUX], const double (&pv)[NAUX], const double2 la,
                        const double lb, const double (&lo)[3], const double Dai, const double Dia) {
            double G[3];
            G[0] = fma(Dai, la.x, -(Dia * lo[0]));
            G[1] = fma(Dai, la.y, -(Dia * lo[1]));
            G[2] = fma(Dai, lb, -(Dia * lo[2]));
            const double rb = o[0] + pv[0];
            const double ub0 = o[1] + pv[1], ub1 = o[2] + pv[2], ub2 = o[3] + pv[3];
            const double eb = o[4] + pv[4], pbar = o[5] + pv[5];
            const double un = ub0 * G[0] + ub1 * G[1] + ub2 * G[2];
            const double f1 = rb * un;
            ac[0] += f1;
            ac[1] += f1 * ub0 + pbar * G[0];
            ac[2] += f1 * ub1 + pbar * G[1];
            ac[3] += f1 * ub2 + pbar * G[2];
            ac[4] += un * (rb * eb + pbar);
        };
#pragma unroll
        for (int dir = 0; dir < 2; ++dir) {  // x, y: a partner of its own for each node
            double lo[2][3];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int n = t + NT * h;
                const double2 la = sm.lga[dir][PAD(n)];
                lo[h][0] = la.x;
                lo[h][1] = la.y;
                lo[h][2] = sm.lgb[dir][PAD(n)];
            }
            const int id = dir == 0 ? ii : jj;
#pragma unroll kCurvedUnroll
            for (int a = 0; a < NQ; ++a) {
                const double Dai = sm.D[a][id], Dia = sm.D[id][a];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    if (a == id) continue;  // the self pair, whose G cancels exactly, is never formed
                    const int kk = k0 + 4 * h;
                    const int na = dir == 0 ? a + 8 * (jj + 8 * kk) : ii + 8 * (a + 8 * kk);
                    double pv[NAUX];
                    sm.aux.get(PAD(na), pv);
                    pair(acc[h], own[h], pv, sm.lga[dir][PAD(na)], sm.lgb[dir][PAD(na)], lo[h], Dai, Dia);
                }
            }
        }
        {  // z: both nodes of the thread share the partner
            double lo[2][3];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int n = t + NT * h;
                const double2 la = sm.lga[2][PAD(n)];
                lo[h][0] = la.x;
                lo[h][1] = la.y;
                lo[h][2] = sm.lgb[2][PAD(n)];
            }
#pragma unroll kCurvedUnroll
            for (int a = 0; a < NQ; ++a) {
                const int nz = ii + 8 * (jj + 8 * a);
                double pv[NAUX];
                sm.aux.get(PAD(nz), pv);
                const double2 la = sm.lga[2][PAD(nz)];
                const double lb = sm.lgb[2][PAD(nz)];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int kk = k0 + 4 * h;
                    if (a != kk) pair(acc[h], own[h], pv, la, lb, lo[h], sm.D[a][kk], sm.D[kk][a]);
                }
            }
        }
        // MJI of the own nodes (vgeo row 9)
        {
            const double* mj = A.vgeo + ((size_t)e * NVG + 9) * NP + t;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const double m = __ldg(mj + NT * h);
#pragma unroll
                for (int s = 0; s < NS; ++s) acc[h][s] = acc[h][s] * m;
            }
        }

        // ---- face-slot contributions (wsJ nf) MJI, written over the slot's trace
        double sg[2][4], mjf[2];
#pragma unroll
        for (int sl = 0; sl < 2; ++sl) {  // face geometry of the thread's slots (global memory)
            const int slot = t + NT * sl;
            if (slot >= NSLOT) continue;
            int vn, opp;
            slot_nodes(slot, vn, opp);
            const double* g = A.sgeo + ((size_t)e * NSLOT + slot) * 4;
#pragma unroll
            for (int c = 0; c < 4; ++c) sg[sl][c] = __ldg(g + c);
            mjf[sl] = __ldg(A.vgeo + ((size_t)e * NVG + 9) * NP + vn);
        }
        cp_async_wait_all();  // this thread's traces (each thread fluxes the slots it fetched)
#pragma unroll
        for (int sl = 0; sl < 2; ++sl) {
            const int slot = t + NT * sl;
            if (slot >= NSLOT) continue;
            const int f = slot >> 6;
            int vn, opp;
            slot_nodes(slot, vn, opp);
            const bool open_face = sm.nb[buf][f] >= 0;
            const double nx = sg[sl][0], ny = sg[sl][1], nz = sg[sl][2], wsJ = sg[sl][3];
            double qm[NS], qp[NS], Fm[NS], Fp[NS], wm, wp;
            {
                double v[NAUX];
                sm.aux.get(PAD(vn), v);
                const double rho = 2.0 * v[0];
                qm[0] = rho;
                qm[1] = rho * (2.0 * v[1]);
                qm[2] = rho * (2.0 * v[2]);
                qm[3] = rho * (2.0 * v[3]);
                qm[4] = rho * (2.0 * v[4]);
            }
            // normal flux and wave speed of one side (euler.jl:50-68)
            auto side_flux = [&](const double (&qq)[NS], double (&F)[NS], double& w) {
                const double rho = qq[0], rhoe = qq[4];
                const double rinv = 1.0 / rho;
                const double u0 = qq[1] * rinv, u1 = qq[2] * rinv, u2 = qq[3] * rinv;
                const double p = gm1 * (rhoe - (qq[1] * qq[1] + qq[2] * qq[2] + qq[3] * qq[3]) * (0.5 * rinv));
                const double un = u0 * nx + u1 * ny + u2 * nz;
                const double mn = qq[1] * nx + qq[2] * ny + qq[3] * nz;
                F[0] = mn;
                F[1] = mn * u0 + p * nx;
                F[2] = mn * u1 + p * ny;
                F[3] = mn * u2 + p * nz;
                F[4] = un * (rhoe + p);
                w = fabs(un) + sqrt(gam * p * rinv);
            };
            side_flux(qm, Fm, wm);
            if (open_face) {
#pragma unroll
                for (int s = 0; s < NS; ++s) qp[s] = sm.slot[s][slot];
                side_flux(qp, Fp, wp);
            } else {  // boundary face: q+ = q- (balancelaw.jl:77)
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    qp[s] = qm[s];
                    Fp[s] = Fm[s];
                }
                wp = wm;
            }
            const double mx = fmax(wm, wp);
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const double fc = (Fm[s] + Fp[s]) * 0.5;
                const double nf = A.surface_rusanov ? fc - (mx * (qp[s] - qm[s])) * 0.5 : fc;
                sm.slot[s][slot] = (wsJ * nf) * mjf[sl];
            }
        }
        __syncthreads();  // #2: face contributions ready
        // ---- own nodes: dq = rka dq + volume - faces (x, y, z order); q_out = q + rkb dt dq
        const size_t g0 = (size_t)e * NS * NP + t;
        double qold[2][NS], dqold[2][NS];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const size_t g = g0 + NT * h + s * NP;
                qold[h][s] = __ldg(A.q_in + g);
                dqold[h][s] = read_dq ? __ldg(A.dq64 + g) : 0.0;
            }
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
                double v = acc[h][s];
                if (read_dq) v = A.rka * dqold[h][s] + v;
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    if (slots[d] >= 0) v = v - sm.slot[s][slots[d]];
                A.dq64[g] = v;
                A.q_out[g] = qold[h][s] + A.rkb_dt * v;
            }
        }
    }
}

}  // namespace rb200
