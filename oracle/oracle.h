/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of Raven.jl's DGSEM tendency + LSRK(5,4) path and of the
 * brick grid generation it consumes.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load this library; the product path
 * (raven.jl_b200) never does.
 *
 * Parity is pinned against the reference's own known-answer values
 * (tests/golden/reference_goldens.json: the golden L2 errors of
 * test/balancelaws/{advection,euler}/*.jl and the vmapP vectors of
 * test/gridnumbering.jl:369-386).
 */
#ifndef RAVEN_ORACLE_H
#define RAVEN_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct og_grid og_grid;

/* Law / scheme selection (mirrors Raven's types; see oracle.cpp for citations). */
enum { OG_LAW_ADVECTION = 0, OG_LAW_EULER = 1 };
enum { OG_FORM_WEAK = 0, OG_FORM_FLUXDIFF = 1 };
enum { OG_FLUX_CENTRAL = 0, OG_FLUX_KG = 1, OG_FLUX_EC = 2, OG_FLUX_RUSANOV = 3, OG_FLUX_ROE = 4, OG_FLUX_MATRIX = 5 };
enum { OG_WARP_NONE = 0, OG_WARP_SINE = 1, OG_WARP_IDENTITY_CURVED = 2 };

typedef struct {
    int law;          /* OG_LAW_* */
    int form;         /* OG_FORM_* */
    int volume_flux;  /* two-point flux for OG_FORM_FLUXDIFF */
    int surface_flux; /* OG_FLUX_*: Rusanov, central, or (Euler) KG, EC, Roe, matrix */
    double gamma;     /* Euler */
    double adv[3];    /* advection velocity */
} og_law;

/* Brick grid: dim in 1..3, nq nodes per direction, K elements per direction on
 * [lo, hi] (Julia `range(lo, stop=hi, length=K+1)` vertices), periodic flags.
 * warp: OG_WARP_NONE (unwarped brick metrics), OG_WARP_SINE
 * (x += amp*L*sin(pi*xi)sin(pi*eta)sin(pi*zeta) per component, xi=(x-lo)/L),
 * OG_WARP_IDENTITY_CURVED (no displacement, but curved-metric formulas). */
og_grid* og_grid_create(int dim, int nq, const int* K, const double* lo, const double* hi,
                        const int* periodic, int warp, double warp_amp);
void og_grid_destroy(og_grid* g);

/* sizes[0]=dim, [1]=nq, [2]=Np, [3]=Nfp, [4]=nfaces, [5]=E, [6]=number of volume
 * metric fields, [7]=number of surface metric fields */
void og_grid_sizes(const og_grid* g, int64_t* sizes);
void og_grid_lgl(const og_grid* g, double* r, double* w, double* D); /* D column-major (Nq,Nq) */
void og_grid_points(const og_grid* g, double* out);  /* (Np, dim, E) */
void og_grid_vmet(const og_grid* g, double* out);    /* (Np, dim*dim+2, E): dRdX, J, wJ */
void og_grid_smet(const og_grid* g, double* out);    /* (dim+2, nfaces*Nfp, E): n, sJ, wsJ */
void og_grid_vmapM(const og_grid* g, int64_t* out);  /* (nfaces*Nfp, E), 1-based */
void og_grid_vmapP(const og_grid* g, int64_t* out);
void og_grid_boundary(const og_grid* g, int64_t* out); /* (nfaces, E) */
void og_grid_tree_coords(const og_grid* g, int32_t* out); /* (3, E) lattice coordinates */

/* A grid from the arrays of a generated grid (used for adapted grids, which the product's
 * forest module builds): points (Np, dim, E), volume metrics (Np, dim*dim+2, E), surface
 * metrics (dim+2, nfaces*Nfp, E), vmapM/vmapP (nfaces*Nfp, E) 1-based, boundary codes
 * (nfaces, E). */
og_grid* og_grid_from_arrays(int dim, int nq, int64_t E, const double* points, const double* vmet,
                             const double* smet, const int64_t* vmapM, const int64_t* vmapP,
                             const int64_t* bc);
/* Mortars coupling the hanging faces of an adapted grid: (2 + 2^(dim-1), M) int64 0-based
 * columns (large element, its face, small elements by position on the face) and the
 * (nq, nq) row-major interpolation to / projection from the two halves. */
void og_grid_set_mortars(og_grid* g, const int64_t* mortars, int64_t M, const double* IL, const double* IU,
                         const double* PL, const double* PU);
/* Warped adapted grid: mortar fluxes with the small faces' own normals and surface
 * measures, projected so that the coupling conserves (a project-defined extension). */
void og_grid_set_curved_mortars(og_grid* g, int curved);
/* DGSEM(; directions): volume and surface terms of the directions in `mask` only (bit d =
 * direction d + 1; all when mask covers every direction). */
void og_grid_set_directions(og_grid* g, int mask);
/* boundarystate of the faces with boundary code `tag` (1..8): kind 0 q+ = q-, 1 q+ =
 * state (Ns doubles), 2 a reflecting wall (Euler). */
void og_grid_set_boundary_condition(og_grid* g, int tag, int kind, const double* state);
/* One step of LSRK / RLSRK with a caller's low-storage table (nstages <= 32). */
void og_lsrk_step_coeffs(const og_grid* g, const og_law* law, double* q, double* dq, const double* rka,
                         const double* rkb, int nstages, double time, double dt);
int og_rlsrk_step_coeffs(const og_grid* g, const og_law* law, double* q, double* dq, double* gamma,
                         const double* rka, const double* rkb, int nstages, double time, double dt);

/* Standalone LGL operators for nq points (computed in __float128, rounded). */
void og_lgl(int nq, double* r, double* w, double* D);

/* Fill q (Np, Ns, E) with an initial condition.
 * kind 0: advection wave  2 + sin(pi*(sum(x) - sum(a)*t))
 * kind 1: Euler density wave (u=1 each direction, p=1)
 * kind 2: 2D isentropic vortex of the reference test (center (5,0), u0=(1,0), beta=5)
 * kind 3: sin(2pi x)sin(2pi y) + exp(-|x-c|^2/(2 sigma^2)), params[0]=sigma, c=params[1..3]
 * kind 4: z-invariant isentropic vortex: params: [0]=beta, [1]=u0x, [2]=cx, [3]=cy
 * kind 5: Euler density pulse rho=1+0.2exp(-|x-c|^2/0.01) at p=1, c=params[0..2] */
void og_initial_condition(const og_grid* g, const og_law* law, int kind, const double* params,
                          double t, double* q);

/* dq = (increment ? dq : 0) + RHS(q) on elements [e0, e1) (full grid: 0, E). */
void og_tendency(const og_grid* g, const og_law* law, double* dq, const double* q, double t,
                 int increment, int64_t e0, int64_t e1);

/* One LSRK(5,4) step on elements [e0,e1) -- used by the CPU baseline sample.  For the
 * full grid pass 0, E. */
void og_lsrk54_step(const og_grid* g, const og_law* law, double* q, double* dq, double time,
                    double dt);
/* One LSRK(14,4) step (odesolvers.jl:191-239), same arguments. */
void og_lsrk144_step(const og_grid* g, const og_law* law, double* q, double* dq, double time, double dt);

/* Raven's solve!(q, timeend, LSRK54(dg, q, dt)) with adjust_final; returns steps taken. */
int64_t og_solve(const og_grid* g, const og_law* law, double* q, double dt, double timeend);

/* weightednorm(dg, q, p=2): componentwise sqrt(sum(MJ |q_s|^2)), then the 2-norm. */
double og_weightednorm(const og_grid* g, const double* q, int ns, double* componentwise);
/* weightednorm(dg, q, p; componentwise) for p >= 1 or p = INFINITY (measures.jl:6-21):
 * componentwise[s] = (sum MJ |q_s|^p)^(1/p), max |q_s| for p = Inf; returns norm(., p). */
double og_weightednorm_p(const og_grid* g, const double* q, int ns, double p, double* componentwise);

/* sum(MJ .* q_s) per field (conservation integrals). */
void og_integrals(const og_grid* g, const double* q, int ns, double* out);

/* entropyintegral / entropyproduct (measures.jl:23-33) in one pass over p = base + c*dir
 * (dir NULL: p = base): out[0] = sum MJ eta(p), out[1] = sum MJ v(p).k (0 when k is NULL). */
void og_entropy_sums(const og_grid* g, const og_law* law, const double* base, const double* dir, double c,
                     const double* k, double* out);

/* One RLSRK(5,4) step (odesolvers.jl:118-151); *gamma carries the relaxation parameter
 * between steps (1 at the start).  Returns the Newton iterations taken. */
int og_rlsrk54_step(const og_grid* g, const og_law* law, double* q, double* dq, double* gamma, double time,
                    double dt);
/* One RLSRK(14,4) step (odesolvers.jl:158-161), same arguments. */
int og_rlsrk144_step(const og_grid* g, const og_law* law, double* q, double* dq, double* gamma, double time,
                     double dt);

/* solve!(q, timeend, RLSRK54(dg, q, dt)) with adjust_final; returns steps taken. */
int64_t og_solve_rlsrk(const og_grid* g, const og_law* law, double* q, double dt, double timeend, double* gamma);

int og_num_threads(void);
void og_set_num_threads(int n);

#ifdef __cplusplus
}
#endif

#endif
