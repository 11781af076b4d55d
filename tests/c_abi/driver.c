/* A C host of libravenb200 (include/raven_b200.h), as a non-Python caller binds it.
 *
 * Builds, in plain C, a periodic K^3 brick of Nq = 4 Lobatto elements on [0, L]^3 in
 * Raven's array layouts (lobattocells.jl:3182-3295 brick metrics, :1992-2295 face maps;
 * elements in x-fastest order, which the library accepts as it checks the face maps
 * node by node), then through the C ABI:
 *   1. free stream: a constant state has a zero tendency (max |dq| <= 1e-12 of the flux
 *      scale) - rb200_create, rb200_tendency on device buffers;
 *   2. conservation: 10 LSRK(5,4) steps of a smooth state through the host-buffer entry
 *      point keep sum(MJ q_s) to 1e-13 relative - rb200_lsrk54_step_host, rb200_integrals;
 *   3. the step of the device entry point equals the host entry point bit for bit;
 *   4. argument errors come back as status codes with a message.
 * Prints one line per check and exits 0 when all pass. */
#include <cuda_runtime_api.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "raven_b200.h"

#define NQ 4
#define K 4
#define DIM 3
#define NP (NQ * NQ * NQ)
#define NFP (NQ * NQ)
#define NF 6
#define NS 5

static int failures = 0;

static void check(int ok, const char* what) {
    printf("%s: %s\n", ok ? "ok" : "FAIL", what);
    if (!ok) failures++;
}

static double legendre(int n, double x, double* dp) {
    double p0 = 1.0, p1 = x;
    for (int k = 2; k <= n; ++k) {
        const double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
    }
    *dp = n * (x * p1 - p0) / (x * x - 1.0);
    return p1;
}

/* Lobatto nodes (Newton on P_N'), weights 2 / (N (N+1) P_N(x)^2), and the derivative
 * matrix D[i + nq j] = l_j'(r_i). */
static void lobatto(double* r, double* w, double* D) {
    const int N = NQ - 1;
    r[0] = -1.0;
    r[N] = 1.0;
    for (int i = 1; i < N; ++i) {
        double x = -cos(M_PI * i / N);
        for (int it = 0; it < 100; ++it) {  /* Newton on q = (1 - x^2) P_N' */
            double dp;
            const double p = legendre(N, x, &dp);
            const double q = (1 - x * x) * dp, dq = -N * (N + 1) * p;
            const double dx = q / dq;
            x -= dx;
            if (fabs(dx) < 1e-16) break;
        }
        r[i] = x;
    }
    double pn[NQ];
    for (int i = 0; i < NQ; ++i) {
        double dp;
        pn[i] = legendre(N, r[i], &dp);
        w[i] = 2.0 / (N * (N + 1) * pn[i] * pn[i]);
    }
    for (int i = 0; i < NQ; ++i)
        for (int j = 0; j < NQ; ++j) {
            double v;
            if (i != j) v = pn[i] / (pn[j] * (r[i] - r[j]));
            else if (i == 0) v = -N * (N + 1) / 4.0;
            else if (i == N) v = N * (N + 1) / 4.0;
            else v = 0.0;
            D[i + NQ * j] = v;
        }
}

static int face_node(int f, int j) {
    const int d = f / 2, c = (f % 2) ? NQ - 1 : 0, j1 = j % NQ, j2 = j / NQ;
    if (d == 0) return c + NQ * (j1 + NQ * j2);
    if (d == 1) return j1 + NQ * (c + NQ * j2);
    return j1 + NQ * (j2 + NQ * c);
}

int main(void) {
    const int64_t E = (int64_t)K * K * K;
    const double L = 2.0, dx = L / K;
    double r[NQ], w[NQ], D[NQ * NQ];
    lobatto(r, w, D);

    /* brick metrics: dRdX = (2/dx) I, J = (dx/2)^3, wJ = w_i w_j w_k J */
    const int nvm = DIM * DIM + 2, nsm = DIM + 2;
    double* vm = calloc((size_t)NP * nvm * E, sizeof(double));
    double* sm = calloc((size_t)nsm * NF * NFP * E, sizeof(double));
    int64_t* vmapM = malloc(sizeof(int64_t) * NF * NFP * E);
    int64_t* vmapP = malloc(sizeof(int64_t) * NF * NFP * E);
    double* pts = malloc(sizeof(double) * NP * DIM * E);
    const double drdx = 2.0 / dx, J = (dx / 2) * (dx / 2) * (dx / 2), sJ = fabs(J * drdx);
    for (int64_t e = 0; e < E; ++e) {
        const int ex = (int)(e % K), ey = (int)((e / K) % K), ez = (int)(e / (K * K));
        const int ec[3] = {ex, ey, ez};
        for (int n = 0; n < NP; ++n) {
            const int id[3] = {n % NQ, (n / NQ) % NQ, n / (NQ * NQ)};
            double* m = vm + (size_t)nvm * NP * e;
            for (int a = 0; a < DIM; ++a) {
                for (int b = 0; b < DIM; ++b) m[n + (size_t)NP * (a + DIM * b)] = a == b ? drdx : 0.0;
                pts[n + (size_t)NP * (a + DIM * e)] = dx * ec[a] + dx * 0.5 * (r[id[a]] + 1.0);
            }
            m[n + (size_t)NP * (DIM * DIM)] = J;
            m[n + (size_t)NP * (DIM * DIM + 1)] = ((w[id[0]] * w[id[1]]) * w[id[2]]) * J;
        }
        for (int f = 0; f < NF; ++f) {
            const int d = f / 2, side = f % 2;
            int nc[3] = {ex, ey, ez};
            nc[d] = (nc[d] + (side ? 1 : K - 1)) % K;
            const int64_t ne = nc[0] + (int64_t)K * (nc[1] + (int64_t)K * nc[2]);
            for (int j = 0; j < NFP; ++j) {
                const size_t k = (size_t)NF * NFP * e + (size_t)f * NFP + j;
                vmapM[k] = NP * e + face_node(f, j) + 1;
                vmapP[k] = NP * ne + face_node(f ^ 1, j) + 1;
                double* s = sm + (size_t)nsm * k;
                for (int c = 0; c < DIM; ++c) s[c] = c == d ? (side ? 1.0 : -1.0) : 0.0;
                s[DIM] = sJ;
                s[DIM + 1] = (sJ * w[j % NQ]) * w[j / NQ];
            }
        }
    }

    rb200_desc desc;
    memset(&desc, 0, sizeof(desc));
    desc.abi_version = RB200_ABI_VERSION;
    desc.dim = DIM;
    desc.nq = NQ;
    desc.law = RB200_LAW_EULER;
    desc.num_elements = E;
    desc.volume_form = RB200_FORM_FLUXDIFF;
    desc.volume_flux = RB200_FLUX_KENNEDY_GRUBER;
    desc.surface_flux = RB200_FLUX_RUSANOV;
    desc.precision = RB200_PRECISION_FP64;
    desc.gamma = 1.4;
    desc.D = D;
    desc.w = w;
    desc.volume_metrics = vm;
    desc.surface_metrics = sm;
    desc.vmapM = vmapM;
    desc.vmapP = vmapP;
    desc.boundary_codes = NULL;
    desc.device = 0;
    rb200_handle* h = NULL;
    rb200_status st = rb200_create(&desc, &h);
    check(st == RB200_OK && h != NULL, "rb200_create on a periodic 4^3 brick, Nq = 4, Euler KG");
    if (st != RB200_OK) {
        printf("  %s\n", rb200_last_error(h));
        return 1;
    }

    const size_t n = (size_t)NP * NS * E;
    double* q = malloc(n * sizeof(double));
    double* q2 = malloc(n * sizeof(double));
    double* dq = malloc(n * sizeof(double));
    double *d_q = NULL, *d_dq = NULL;
    if (cudaMalloc((void**)&d_q, n * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&d_dq, n * sizeof(double)) != cudaSuccess) {
        check(0, "cudaMalloc");
        return 1;
    }

    /* 1. free stream */
    for (int64_t e = 0; e < E; ++e)
        for (int s = 0; s < NS; ++s)
            for (int k = 0; k < NP; ++k) {
                const double v[NS] = {1.2, 0.3, -0.2, 0.1, 3.0};
                q[k + (size_t)NP * (s + (size_t)NS * e)] = v[s];
            }
    cudaMemcpy(d_q, q, n * sizeof(double), cudaMemcpyHostToDevice);
    st = rb200_tendency(h, d_dq, d_q, 0.0, 0, NULL);
    cudaMemcpy(dq, d_dq, n * sizeof(double), cudaMemcpyDeviceToHost);
    double mx = 0.0;
    for (size_t i = 0; i < n; ++i) mx = fmax(mx, fabs(dq[i]));
    check(st == RB200_OK && mx <= 1e-12 * 9.0 / (dx / NQ), "free stream: zero tendency");

    /* 2. conservation through the host-buffer entry point */
    for (int64_t e = 0; e < E; ++e)
        for (int k = 0; k < NP; ++k) {
            const double x = pts[k + (size_t)NP * (0 + DIM * e)], y = pts[k + (size_t)NP * (1 + DIM * e)],
                         z = pts[k + (size_t)NP * (2 + DIM * e)];
            const double rho = 1.0 + 0.1 * sin(M_PI * x) * sin(M_PI * y) * cos(M_PI * z);
            const double u[3] = {0.2 * sin(M_PI * y), 0.1 * cos(M_PI * z), -0.1 * sin(M_PI * x)};
            const double p = 1.0 + 0.05 * cos(M_PI * (x + y));
            double* qe = q + (size_t)NP * NS * e;
            qe[k] = rho;
            for (int c = 0; c < 3; ++c) qe[k + NP * (1 + c)] = rho * u[c];
            qe[k + NP * 4] = p / 0.4 + 0.5 * rho * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        }
    memcpy(q2, q, n * sizeof(double));
    double I0[NS], I1[NS];
    cudaMemcpy(d_q, q, n * sizeof(double), cudaMemcpyHostToDevice);
    st = rb200_integrals(h, d_q, I0, NULL);
    const double dt = 2e-3;
    if (st == RB200_OK) st = rb200_lsrk54_step_host(h, q, 0.0, dt, 10, NULL);
    cudaMemcpy(d_q, q, n * sizeof(double), cudaMemcpyHostToDevice);
    if (st == RB200_OK) st = rb200_integrals(h, d_q, I1, NULL);
    int cons = st == RB200_OK;
    for (int s = 0; s < NS; ++s) cons = cons && fabs(I1[s] - I0[s]) <= 1e-13 * fmax(fabs(I0[s]), fabs(I0[0]));
    check(cons, "10 LSRK(5,4) steps through rb200_lsrk54_step_host conserve sum(MJ q)");

    /* 3. the device entry point gives the same steps bit for bit */
    cudaMemcpy(d_q, q2, n * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemset(d_dq, 0, n * sizeof(double));
    st = rb200_lsrk54_step(h, d_q, d_dq, 0.0, dt, 10, NULL);
    cudaMemcpy(q2, d_q, n * sizeof(double), cudaMemcpyDeviceToHost);
    check(st == RB200_OK && memcmp(q, q2, n * sizeof(double)) == 0,
          "rb200_lsrk54_step on device buffers equals the host-buffer path bit for bit");

    /* 4. errors are status codes */
    st = rb200_tendency(h, NULL, d_q, 0.0, 0, NULL);
    check(st == RB200_ERR_BAD_ARG && strlen(rb200_last_error(h)) > 0, "a null state pointer is BAD_ARG");
    st = rb200_lsrk54_step(h, d_q, d_dq, 0.0, NAN, 1, NULL);
    check(st == RB200_ERR_BAD_ARG, "a NaN time step is BAD_ARG");

    cudaFree(d_q);
    cudaFree(d_dq);
    check(rb200_destroy(h) == RB200_OK, "rb200_destroy");
    free(q);
    free(q2);
    free(dq);
    free(vm);
    free(sm);
    free(vmapM);
    free(vmapP);
    free(pts);
    printf("%d failure(s)\n", failures);
    return failures ? 1 : 0;
}
