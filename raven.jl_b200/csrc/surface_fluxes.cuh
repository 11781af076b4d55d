// Entropy-family surface fluxes of the Euler law at one face node, for the generic stage
// kernel (FP64):
// * entropy conservative and Kennedy-Gruber: the two-point flux contracted with the
//   normal, the default surfaceflux (src/balancelaws/numericalfluxes.jl:27-37) of
//   twopointflux (balancelaws/euler.jl:150-216);
// * Roe (euler.jl:93-149);
// * matrix dissipation (euler.jl:218-300), including its u2_bar built from norms (not
//   squared norms), as the reference writes it.
#pragma once

#include "rb200_internal.h"

namespace rb200 {

template <typename T>
__device__ __forceinline__ T sf_logavg(T a, T b) {  // numericalfluxes.jl:9-22
    const T zeta = a / b;
    const T f = (zeta - T(1)) / (zeta + T(1));
    const T u = f * f;
    const T eps = sizeof(T) == 8 ? T(2.220446049250313e-16) : T(1.1920929e-07f);
    T F;
    if (u < eps) F = fma(u, fma(u, fma(u, fma(u, T(1) / T(9), T(1) / T(7)), T(1) / T(5)), T(1) / T(3)), T(1));
    else F = log(zeta) / (T(2) * f);
    return (a + b) / (T(2) * F);
}

template <int DIM, typename T>
struct SfState {
    T rho, u[DIM], rhoe, e, p, b, uu, unorm;
    __device__ __forceinline__ SfState(const T* q, T gm1) {
        rho = q[0];
        rhoe = q[DIM + 1];
        T rr = T(0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            u[d] = q[1 + d] / rho;
            rr += q[1 + d] * q[1 + d];
        }
        p = gm1 * (rhoe - rr / (T(2) * rho));
        e = rhoe / rho;
        b = rho / (T(2) * p);
        uu = T(0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) uu += u[d] * u[d];
        unorm = sqrt(uu);
    }
};

// Two-point entropy-conservative flux of (1, 2) contracted with n (euler.jl:150-184).
template <int DIM, typename T>
__device__ __forceinline__ void sf_ec(const SfState<DIM, T>& s1, const SfState<DIM, T>& s2, const T* n, T gamma,
                                      T* nf) {
    const T rho_avg = (s1.rho + s2.rho) / T(2);
    const T b_avg = (s1.b + s2.b) / T(2);
    const T u2_avg = (s1.uu + s2.uu) / T(2);
    const T rho_log = sf_logavg(s1.rho, s2.rho);
    const T b_log = sf_logavg(s1.b, s2.b);
    T ua[DIM], fr[DIM], un = T(0), fu = T(0), fn = T(0);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        ua[d] = (s1.u[d] + s2.u[d]) / T(2);
        fr[d] = ua[d] * rho_log;
        un += ua[d] * n[d];
        fu += fr[d] * ua[d];
        fn += fr[d] * n[d];
    }
    const T pt = rho_avg / (T(2) * b_avg);
    const T c = T(1) / (T(2) * (gamma - T(1)) * b_log) - u2_avg / T(2);
    nf[0] = fn;
#pragma unroll
    for (int k = 0; k < DIM; ++k) nf[1 + k] = un * fr[k] + pt * n[k];
    nf[DIM + 1] = c * fn + un * fu + pt * un;
}

template <int DIM, typename T>
__device__ __forceinline__ void euler_entropy_surface_flux(int kind, const T* n, const T* qm, const T* qp, T gamma,
                                                           T* nf) {
    const T gm1 = gamma - T(1);
    const SfState<DIM, T> sm(qm, gm1), sp(qp, gm1);
    if (kind == kFluxEC) {
        sf_ec<DIM, T>(sm, sp, n, gamma, nf);
    } else if (kind == kFluxKG) {  // euler.jl:186-216
        const T rho_avg = (sm.rho + sp.rho) / T(2);
        const T e_avg = (sm.e + sp.e) / T(2);
        const T p_avg = (sm.p + sp.p) / T(2);
        T ua[DIM], un = T(0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            ua[d] = (sm.u[d] + sp.u[d]) / T(2);
            un += ua[d] * n[d];
        }
        nf[0] = rho_avg * un;
#pragma unroll
        for (int k = 0; k < DIM; ++k) nf[1 + k] = un * (ua[k] * rho_avg) + p_avg * n[k];
        nf[DIM + 1] = un * (rho_avg * e_avg + p_avg);
    } else if (kind == kFluxRoe) {  // euler.jl:93-149
        const T hm = sm.e + sm.p / sm.rho, hp = sp.e + sp.p / sp.rho;
        const T cm = sqrt(gamma * sm.p / sm.rho), cp = sqrt(gamma * sp.p / sp.rho);
        const T sqm = sqrt(sm.rho), sqp = sqrt(sp.rho);
        auto roe = [&](T a, T b) { return (sqm * a + sqp * b) / (sqm + sqp); };
        const T rho = sqrt(sm.rho * sp.rho);
        T u[DIM], du[DIM], un = T(0), dun = T(0), uu = T(0), udu = T(0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            u[d] = roe(sm.u[d], sp.u[d]);
            du[d] = sp.u[d] - sm.u[d];
            un += u[d] * n[d];
            dun += du[d] * n[d];
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            uu += u[d] * u[d];
            udu += u[d] * du[d];
        }
        const T h = roe(hm, hp), c = roe(cm, cp);
        const T drho = sp.rho - sm.rho, dp = sp.p - sm.p;
        const T ci2 = T(1) / (c * c);
        const T w1 = fabs(un - c) * (dp - rho * c * dun) * ci2 / T(2);
        const T w2 = fabs(un + c) * (dp + rho * c * dun) * ci2 / T(2);
        const T w3 = fabs(un) * (drho - dp * ci2);
        const T w4 = fabs(un) * rho;
        // central part: (f- + f+)' n / 2 with the physical fluxes (euler.jl:50-61)
        T fm[DIM + 2], fp[DIM + 2];
        const SfState<DIM, T>* st[2] = {&sm, &sp};
        const T* qs[2] = {qm, qp};
        for (int side = 0; side < 2; ++side) {
            const SfState<DIM, T>& s = *st[side];
            T* f = side ? fp : fm;
            T mn = T(0), vn = T(0);
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                mn += qs[side][1 + d] * n[d];
                vn += s.u[d] * n[d];
            }
            f[0] = mn;
#pragma unroll
            for (int k = 0; k < DIM; ++k) f[1 + k] = vn * qs[side][1 + k] + s.p * n[k];
            f[DIM + 1] = vn * (s.rhoe + s.p);
        }
        nf[0] = (fm[0] + fp[0]) / T(2) - (w1 + w2 + w3) / T(2);
#pragma unroll
        for (int k = 0; k < DIM; ++k)
            nf[1 + k] = (fm[1 + k] + fp[1 + k]) / T(2) -
                        (w1 * (u[k] - c * n[k]) + w2 * (u[k] + c * n[k]) + w3 * u[k] + w4 * (du[k] - dun * n[k])) / T(2);
        nf[DIM + 1] = (fm[DIM + 1] + fp[DIM + 1]) / T(2) -
                      (w1 * (h - c * un) + w2 * (h + c * un) + w3 * uu / T(2) + w4 * (udu - un * dun)) / T(2);
    } else {  // matrix dissipation, euler.jl:218-300
        sf_ec<DIM, T>(sm, sp, n, gamma, nf);
        const T rho_log = sf_logavg(sm.rho, sp.rho);
        const T b_log = sf_logavg(sm.b, sp.b);
        T ua[DIM], un = T(0), uaa = T(0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            ua[d] = (sm.u[d] + sp.u[d]) / T(2);
            un += ua[d] * n[d];
            uaa += ua[d] * ua[d];
        }
        const T p_avg = ((sm.rho + sp.rho) / T(2)) / (T(2) * ((sm.b + sp.b) / T(2)));
        const T u2_bar = T(2) * sqrt(uaa) - (sm.unorm + sp.unorm) / T(2);
        const T h_bar = gamma / (T(2) * b_log * (gamma - T(1))) + u2_bar / T(2);
        const T c_bar = sqrt(gamma * p_avg / rho_log);
        // entropy variables (euler.jl:79-91) and their jump
        auto ent = [&](const SfState<DIM, T>& s, T* v) {
            const T sv = log(s.p / pow(s.rho, gamma));
            v[0] = (gamma - sv) / (gamma - T(1)) - s.uu * s.b;
#pragma unroll
            for (int d = 0; d < DIM; ++d) v[1 + d] = T(2) * s.b * s.u[d];
            v[DIM + 1] = -T(2) * s.b;
        };
        T vm[DIM + 2], vp[DIM + 2], dv[DIM + 2];
        ent(sm, vm);
        ent(sp, vp);
#pragma unroll
        for (int s = 0; s < DIM + 2; ++s) dv[s] = vp[s] - vm[s];
        const T l1 = fabs(un - c_bar) * rho_log / (T(2) * gamma);
        const T l2 = fabs(un) * rho_log * (gamma - T(1)) / gamma;
        const T l3 = fabs(un + c_bar) * rho_log / (T(2) * gamma);
        const T l4 = fabs(un) * p_avg;
        T umc[DIM], upc[DIM], ut[DIM], dvn = T(0), umcdv = T(0), upcdv = T(0), uadv = T(0), utdv = T(0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            umc[d] = ua[d] - c_bar * n[d];
            upc[d] = ua[d] + c_bar * n[d];
            ut[d] = ua[d] - un * n[d];
            dvn += n[d] * dv[1 + d];
            umcdv += umc[d] * dv[1 + d];
            upcdv += upc[d] * dv[1 + d];
            uadv += ua[d] * dv[1 + d];
            utdv += ut[d] * dv[1 + d];
        }
        const T dve = dv[DIM + 1];
        const T w1 = l1 * (dv[0] + umcdv + (h_bar - c_bar * un) * dve);
        const T w2 = l2 * (dv[0] + uadv + u2_bar / T(2) * dve);
        const T w3 = l3 * (dv[0] + upcdv + (h_bar + c_bar * un) * dve);
        nf[0] = nf[0] - (w1 + w2 + w3) / T(2);
#pragma unroll
        for (int k = 0; k < DIM; ++k)
            nf[1 + k] = nf[1 + k] - (w1 * umc[k] + w2 * ua[k] + w3 * upc[k] +
                                     l4 * (dv[1 + k] - dvn * n[k] + dve * ut[k])) / T(2);
        nf[DIM + 1] = nf[DIM + 1] - (w1 * (h_bar - c_bar * un) + w2 * u2_bar / T(2) + w3 * (h_bar + c_bar * un) +
                                     l4 * (utdv + dve * (uaa - un * un))) / T(2);
    }
}

}  // namespace rb200
