// oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product path).
//
// A plain C++ FP64 restatement of the Raven.jl path that the CUDA library replaces:
// the brick grid (element order, node points, metrics, face maps) and the DGSEM
// tendency with the LSRK(5,4) time stepper.  Citations are to the reference tree
// (Raven.jl 0.2.4-pre).  Build with -ffp-contract=off so that, like Julia, no
// multiply-add is fused unless the reference writes `muladd` (those sites use fma()).
//
// Parity pins: the golden L2 errors of test/balancelaws/{advection,euler}/*.jl and
// the golden vmapP vectors of test/gridnumbering.jl:369-386
// (tests/test_oracle_golden.py).
//
// Third-party algorithms restated here (not vendored in the reference):
//  * OneDimensionalNodes.jl 1.x `legendregausslobatto` / `spectralderivative`
//    (called at src/lobattocells.jl:9-11 at 256-bit precision, then rounded).
//    Restated as Newton iteration on P'_N in __float128 plus the barycentric
//    derivative matrix; every value is rounded once to double.
//  * P4estTypes 0.2.0 / p4est `p4est_connectivity_new_brick` tree order
//    (src/coarsegrids.jl:297): trees of a brick are numbered along a Morton curve of
//    the power-of-two bounding box, dimensions ranked by their bit counts, cells
//    outside the brick skipped.  The degree-3 `lnodes` numbering that the face maps
//    use (src/gridmanager.jl:480) is replaced by a lattice numbering of the brick's
//    degree-3 nodes with the same sharing pattern; the face maps only depend on
//    which nodes are shared and on their relative order.

#include "oracle.h"

#include <quadmath.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef __float128 f128;

// ---------------------------------------------------------------------------------
// 1-D Legendre-Gauss-Lobatto operators (src/lobattocells.jl:1-47)
// ---------------------------------------------------------------------------------

static void legendre_f128(int n, f128 x, f128& P, f128& dP) {
    // P_n(x) and P_n'(x) by the three-term recurrence.
    f128 p0 = 1, p1 = x;
    if (n == 0) { P = 1; dP = 0; return; }
    for (int k = 2; k <= n; ++k) {
        f128 p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
    }
    P = p1;
    // (1-x^2) P_n' = n (P_{n-1} - x P_n)
    dP = n * (p0 - x * p1) / (1 - x * x);
}

extern "C" void og_lgl(int nq, double* r, double* w, double* D) {
    const int N = nq - 1;
    std::vector<f128> x(nq), wt(nq);
    x[0] = -1;
    x[N] = 1;
    for (int j = 1; j < N; ++j) {
        // Newton on P_N'(x) = 0 from the Chebyshev-Gauss-Lobatto guess.
        f128 xj = -cosq(M_PIq * j / N);
        for (int it = 0; it < 100; ++it) {
            f128 P, dP;
            legendre_f128(N, xj, P, dP);
            // P'' from the Legendre equation
            f128 d2P = (2 * xj * dP - N * (N + 1) * P) / (1 - xj * xj);
            f128 dx = dP / d2P;
            xj -= dx;
            if (fabsq(dx) < 1e-33Q) break;
        }
        x[j] = xj;
    }
    for (int j = 0; j < nq / 2; ++j) {  // exact symmetry of the node set
        f128 s = (x[N - j] - x[j]) / 2;
        x[j] = -s;
        x[N - j] = s;
    }
    if (nq % 2 == 1) x[N / 2] = 0;
    for (int j = 0; j < nq; ++j) {
        f128 P, dP;
        legendre_f128(N, x[j], P, dP);
        wt[j] = (f128)2 / (N * (N + 1) * P * P);
    }
    // barycentric weights and spectral derivative D[i,j] = l_j'(x_i)
    std::vector<f128> lam(nq);
    for (int j = 0; j < nq; ++j) {
        f128 p = 1;
        for (int k = 0; k < nq; ++k)
            if (k != j) p *= (x[j] - x[k]);
        lam[j] = 1 / p;
    }
    for (int i = 0; i < nq; ++i) {
        if (r) r[i] = (double)x[i];
        if (w) w[i] = (double)wt[i];
    }
    if (D) {
        for (int i = 0; i < nq; ++i)
            for (int j = 0; j < nq; ++j)
                D[i + nq * j] = (i == j) ? 0.0 : (double)((lam[j] / lam[i]) / (x[i] - x[j]));
        // exact diagonal: -N(N+1)/4, N(N+1)/4 at the end points, 0 inside
        D[0] = -N * (N + 1) / 4.0;
        D[N + nq * N] = N * (N + 1) / 4.0;
    }
}

// ---------------------------------------------------------------------------------
// Grid
// ---------------------------------------------------------------------------------

struct og_grid {
    int dim, nq, np, nfp, nfaces, nvmet, nsmet;
    int64_t E;
    int K[3];
    int periodic[3];
    int warp;
    std::vector<double> r, w, D;   // 1-D operators, D column-major
    std::vector<double> vx[3];     // vertex coordinates per direction
    std::vector<std::array<int, 3>> tree;  // lattice coordinates per element
    std::vector<double> points;    // (np, dim, E)
    std::vector<double> vmet;      // (np, nvmet, E)
    std::vector<double> smet;      // (nsmet, nfaces*nfp, E)
    std::vector<int64_t> vmapM, vmapP, bc;
    std::vector<double> MJI;       // DGSEM's MJI = 1 ./ MJ (dgsem.jl:56)
    // mortars of an adapted grid: (2 + 2^(dim-1), M) columns (large element, its face,
    // small elements); operators to and from the halves, (nq, nq) row-major [i][j]
    std::vector<int64_t> mortars;
    std::vector<double> IL, IU, PL, PU;
    std::vector<uint8_t> ncface;   // (nfaces, E): 1 on faces coupled through a mortar
    int curved_mortars = 0;        // 1: warped grid, mortar fluxes with the small faces' geometry
    int dir_mask = 0;              // DGSEM(; directions) as a bit mask (dgsem.jl:46-81); 0 = all
    // boundarystate per boundary tag 1..8 (balancelaw.jl:22 and its overloads in the
    // reference's examples): 0 q+ = q-, 1 a prescribed state, 2 a reflecting wall
    int bc_kind[9] = {0};
    double bc_state[9][5] = {{0}};
};

// Correctly rounded value of lo + (hi-lo)*i/K (Julia `range(lo, stop=hi, length=K+1)`).
static double range_value(double lo, double hi, int i, int K) {
    if (i == 0) return lo;
    if (i == K) return hi;
    f128 v = (f128)lo + ((f128)hi - (f128)lo) * (f128)i / (f128)K;
    return (double)v;
}

static int sc_log2_32(int x) {  // floor(log2(x)), -1 for 0
    int l = -1;
    while (x > 0) { ++l; x >>= 1; }
    return l;
}

// Morton order of a p4est brick connectivity.
static void brick_tree_order(int dim, const int* K, std::vector<std::array<int, 3>>& out) {
    out.clear();
    if (dim == 1) {
        for (int i = 0; i < K[0]; ++i) out.push_back({i, 0, 0});
        return;
    }
    int logx[3] = {0, 0, 0};
    for (int d = 0; d < dim; ++d) logx[d] = sc_log2_32(K[d] - 1) + 1;
    int rankx[3] = {0, 1, 2};
    if (dim == 2) {
        if (logx[0] <= logx[1]) { rankx[0] = 0; rankx[1] = 1; }
        else { rankx[0] = 1; rankx[1] = 0; }
    } else {
        if (logx[0] <= logx[1]) {
            if (logx[1] <= logx[2]) { rankx[0] = 0; rankx[1] = 1; rankx[2] = 2; }
            else if (logx[0] <= logx[2]) { rankx[0] = 0; rankx[1] = 2; rankx[2] = 1; }
            else { rankx[0] = 2; rankx[1] = 0; rankx[2] = 1; }
        } else {
            if (logx[0] <= logx[2]) { rankx[0] = 1; rankx[1] = 0; rankx[2] = 2; }
            else if (logx[1] <= logx[2]) { rankx[0] = 1; rankx[1] = 2; rankx[2] = 0; }
            else { rankx[0] = 2; rankx[1] = 1; rankx[2] = 0; }
        }
    }
    int64_t n_iter = 1;
    for (int d = 0; d < dim; ++d) n_iter <<= logx[d];
    for (int64_t t = 0; t < n_iter; ++t) {
        int64_t ti = t;
        int64_t tx[3] = {0, 0, 0};
        int lastlog = 0;
        for (int i = 0; i < dim - 1; ++i) {
            int logi = logx[rankx[i]] - lastlog;
            bool active[3] = {false, false, false};
            for (int k = i; k < dim; ++k) active[rankx[k]] = true;
            int na = dim - i;
            for (int j = 0; j < logi; ++j) {
                int c = 0;
                for (int k = 0; k < dim; ++k) {
                    if (!active[k]) continue;
                    int64_t bit = (ti >> (na * j + c)) & 1;
                    tx[k] |= bit << (lastlog + j);
                    ++c;
                }
            }
            lastlog += logi;
            ti >>= na * logi;
        }
        tx[rankx[dim - 1]] += ti << lastlog;
        bool inside = true;
        for (int d = 0; d < dim; ++d) inside = inside && tx[d] < K[d];
        if (inside) out.push_back({(int)tx[0], (int)tx[1], (int)tx[2]});
    }
}

// ----- orientation algebra (src/orientation.jl) -----
static int orient2(int64_t a, int64_t b) { return a <= b ? 1 : 2; }  // :167-171
static int orient4(const int64_t* s) {                               // :173-187
    int i = 0;
    for (int k = 1; k < 4; ++k)
        if (s[k] < s[i]) i = k;
    if (i == 0) return s[1] <= s[2] ? 1 : 5;
    if (i == 1) return s[3] <= s[0] ? 6 : 2;
    if (i == 2) return s[0] <= s[3] ? 7 : 3;
    return s[2] <= s[1] ? 4 : 8;
}
static int inv4(int k) { static const int m[8] = {1, 2, 3, 4, 5, 7, 6, 8}; return m[k - 1]; }  // :147-150
static int compose4(int p, int q) {  // :153-165
    static const int t[8][8] = {{1, 2, 3, 4, 5, 6, 7, 8}, {2, 1, 4, 3, 7, 8, 5, 6},
                                {3, 4, 1, 2, 6, 5, 8, 7}, {4, 3, 2, 1, 8, 7, 6, 5},
                                {5, 6, 7, 8, 1, 2, 3, 4}, {6, 5, 8, 7, 3, 4, 1, 2},
                                {7, 8, 5, 6, 2, 1, 4, 3}, {8, 7, 6, 5, 4, 3, 2, 1}};
    return t[p - 1][q - 1];
}
static int compose2(int p, int q) { return p == q ? 1 : 2; }
// orientindex (orientation.jl:63-98), 1-based indices in, 1-based out
static void orientindex4(int kind, int d1, int d2, int i1, int i2, int& o1, int& o2) {
    int dv = (kind - 1) / 4, rm = (kind - 1) % 4;
    if (dv != 0) {
        int li = (i1 - 1) + d1 * (i2 - 1);  // LinearIndices(dims)
        int c1 = li % d2, c2 = li / d2;     // CartesianIndices(reverse(dims))
        i1 = c2 + 1;
        i2 = c1 + 1;
    }
    o1 = (rm & 1) ? d1 - i1 + 1 : i1;
    o2 = (rm & 2) ? d2 - i2 + 1 : i2;
}

// Local (1-based, column-major) node index list of face f (src/lobattocells.jl:2012-2053).
static void cell_face_indices(int dim, int nq, int f, std::vector<int>& out) {
    out.clear();
    auto lin = [&](int i, int j, int k) { return i + nq * (j - 1) + nq * nq * (k - 1); };
    if (dim == 1) {
        out.push_back(f == 0 ? 1 : nq);
    } else if (dim == 2) {
        for (int a = 1; a <= nq; ++a) {
            if (f == 0) out.push_back(lin(1, a, 1));
            if (f == 1) out.push_back(lin(nq, a, 1));
            if (f == 2) out.push_back(lin(a, 1, 1));
            if (f == 3) out.push_back(lin(a, nq, 1));
        }
    } else {
        for (int b = 1; b <= nq; ++b)
            for (int a = 1; a <= nq; ++a) {
                if (f == 0) out.push_back(lin(1, a, b));
                if (f == 1) out.push_back(lin(nq, a, b));
                if (f == 2) out.push_back(lin(a, 1, b));
                if (f == 3) out.push_back(lin(a, nq, b));
                if (f == 4) out.push_back(lin(a, b, 1));
                if (f == 5) out.push_back(lin(a, b, nq));
            }
    }
}

static void build_points_warp(og_grid& g, double amp) {
    if (g.warp != OG_WARP_SINE) return;
    const int dim = g.dim, np = g.np;
    for (int64_t e = 0; e < g.E; ++e)
        for (int n = 0; n < np; ++n) {
            double x[3], s = 1.0;
            for (int d = 0; d < dim; ++d) {
                x[d] = g.points[n + (size_t)np * (d + dim * e)];
                double lo = g.vx[d].front(), L = g.vx[d].back() - lo;
                s *= sin(M_PI * ((x[d] - lo) / L));
            }
            for (int d = 0; d < dim; ++d) {
                double L = g.vx[d].back() - g.vx[d].front();
                g.points[n + (size_t)np * (d + dim * e)] = x[d] + (amp * L) * s;
            }
        }
}

static inline double& P(og_grid& g, int n, int d, int64_t e) {
    return g.points[n + (size_t)g.np * (d + g.dim * e)];
}

static void build_brick_metrics(og_grid& g) {
    const int dim = g.dim, nq = g.nq, np = g.np, nv = g.nvmet;
    g.vmet.assign((size_t)np * nv * g.E, 0.0);
    // hexvolumebrickmetrics! reads the corner points of element p = local workgroup
    // index (src/lobattocells.jl:3202-3206), i.e. element ((q-1) mod Q) + 1 with
    // Q = max(512 / (Nq*Nq), 1); the 2-D and 1-D kernels read element q itself.
    const int64_t Qw = std::max(512 / (nq * nq), 1);
    for (int64_t e = 0; e < g.E; ++e) {
        int64_t src = (dim == 3) ? (e % Qw) : e;
        double dX[3], drdx[3];
        for (int d = 0; d < dim; ++d) {
            int nlast = (d == 0) ? nq - 1 : (d == 1 ? nq * (nq - 1) : nq * nq * (nq - 1));
            dX[d] = P(g, nlast, d, src) - P(g, 0, d, src);
            drdx[d] = 2.0 / dX[d];
        }
        double J = dX[0] / 2.0;
        for (int d = 1; d < dim; ++d) J = J * (dX[d] / 2.0);
        for (int n = 0; n < np; ++n) {
            int idx[3] = {n % nq, (n / nq) % nq, n / (nq * nq)};
            double* m = &g.vmet[(size_t)np * nv * e];
            for (int a = 0; a < dim; ++a)
                for (int b = 0; b < dim; ++b) m[n + (size_t)np * (a + dim * b)] = (a == b) ? drdx[a] : -0.0;
            double wJ = g.w[idx[0]];
            for (int d = 1; d < dim; ++d) wJ = wJ * g.w[idx[d]];
            wJ = wJ * J;
            m[n + (size_t)np * (dim * dim)] = J;
            m[n + (size_t)np * (dim * dim + 1)] = wJ;
        }
    }
}

static inline void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

static void build_curved_metrics(og_grid& g) {
    const int dim = g.dim, nq = g.nq, np = g.np, nv = g.nvmet;
    g.vmet.assign((size_t)np * nv * g.E, 0.0);
    const double* D = g.D.data();
    auto Dm = [&](int i, int m) { return D[i + nq * m]; };
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < g.E; ++e) {
        double* m = &g.vmet[(size_t)np * nv * e];
        if (dim == 1) {  // linevolumemetrics! (src/lobattocells.jl:2545-2588)
            for (int i = 0; i < nq; ++i) {
                double dxdr = -0.0;
                for (int k = 0; k < nq; ++k) dxdr += Dm(i, k) * P(g, k, 0, e);
                double G = dxdr * dxdr, invG = 1.0 / G;
                m[i] = invG * dxdr;
                double J = std::fabs(dxdr);
                m[i + np] = J;
                m[i + 2 * np] = g.w[i] * J;
            }
        } else if (dim == 2) {  // quadvolumemetrics! (src/lobattocells.jl:2756-2813)
            for (int j = 0; j < nq; ++j)
                for (int i = 0; i < nq; ++i) {
                    double xr[2] = {-0.0, -0.0}, xs[2] = {-0.0, -0.0};
                    for (int k = 0; k < nq; ++k)
                        for (int c = 0; c < 2; ++c) xr[c] += Dm(i, k) * P(g, k + nq * j, c, e);
                    for (int k = 0; k < nq; ++k)
                        for (int c = 0; c < 2; ++c) xs[c] += Dm(j, k) * P(g, i + nq * k, c, e);
                    double G11 = xr[0] * xr[0] + xr[1] * xr[1];
                    double G12 = xr[0] * xs[0] + xr[1] * xs[1];
                    double G22 = xs[0] * xs[0] + xs[1] * xs[1];
                    double det = G11 * G22 - G12 * G12;
                    double iG11 = G22 / det, iG21 = -G12 / det, iG12 = -G12 / det, iG22 = G11 / det;
                    // dRdX = invG * [xr'; xs']
                    double R[2][2];
                    for (int c = 0; c < 2; ++c) {
                        R[0][c] = iG11 * xr[c] + iG12 * xs[c];
                        R[1][c] = iG21 * xr[c] + iG22 * xs[c];
                    }
                    int n = i + nq * j;
                    for (int a = 0; a < 2; ++a)
                        for (int b = 0; b < 2; ++b) m[n + (size_t)np * (a + 2 * b)] = R[a][b];
                    double J = std::fabs(xr[0] * xs[1] - xr[1] * xs[0]);
                    m[n + (size_t)np * 4] = J;
                    m[n + (size_t)np * 5] = (g.w[i] * g.w[j]) * J;
                }
        } else {  // hexvolumemetrics! (src/lobattocells.jl:3038-3180), curl-invariant form
            std::vector<double> X(3 * np), Xr(3 * np), Xs(3 * np), Xt(3 * np);
            auto at = [&](std::vector<double>& A, int i, int j, int k) { return &A[3 * (i + nq * (j + nq * k))]; };
            for (int n = 0; n < np; ++n)
                for (int c = 0; c < 3; ++c) X[3 * n + c] = P(g, n, c, e);
            std::fill(Xr.begin(), Xr.end(), -0.0);
            std::fill(Xs.begin(), Xs.end(), -0.0);
            std::fill(Xt.begin(), Xt.end(), -0.0);
            for (int k = 0; k < nq; ++k)
                for (int j = 0; j < nq; ++j)
                    for (int i = 0; i < nq; ++i)
                        for (int c = 0; c < 3; ++c) {
                            double sr = Xr[3 * (i + nq * (j + nq * k)) + c];
                            for (int mm = 0; mm < nq; ++mm) sr += Dm(i, mm) * at(X, mm, j, k)[c];
                            Xr[3 * (i + nq * (j + nq * k)) + c] = sr;
                            double ss = Xs[3 * (i + nq * (j + nq * k)) + c];
                            for (int mm = 0; mm < nq; ++mm) ss += Dm(j, mm) * at(X, i, mm, k)[c];
                            Xs[3 * (i + nq * (j + nq * k)) + c] = ss;
                        }
            // dXdt[o] += Dt[o,k] * X[k] accumulated in k order
            for (int j = 0; j < nq; ++j)
                for (int i = 0; i < nq; ++i)
                    for (int k = 0; k < nq; ++k)
                        for (int o = 0; o < nq; ++o)
                            for (int c = 0; c < 3; ++c) at(Xt, i, j, o)[c] += Dm(o, k) * at(X, i, j, k)[c];
            // cross products
            std::vector<double> CXs(3 * np), CXt(3 * np), CXr(3 * np);
            for (int n = 0; n < np; ++n) {
                cross3(&X[3 * n], &Xs[3 * n], &CXs[3 * n]);
                cross3(&X[3 * n], &Xt[3 * n], &CXt[3 * n]);
                cross3(&X[3 * n], &Xr[3 * n], &CXr[3 * n]);
            }
            for (int k = 0; k < nq; ++k)
                for (int j = 0; j < nq; ++j)
                    for (int i = 0; i < nq; ++i) {
                        double a1[3] = {-0.0, -0.0, -0.0}, a2[3] = {-0.0, -0.0, -0.0},
                               a3[3] = {-0.0, -0.0, -0.0};
                        for (int c = 0; c < 3; ++c) {
                            for (int mm = 0; mm < nq; ++mm) a3[c] += Dm(i, mm) * at(CXs, mm, j, k)[c];
                            for (int mm = 0; mm < nq; ++mm) a2[c] -= Dm(i, mm) * at(CXt, mm, j, k)[c];
                            for (int mm = 0; mm < nq; ++mm) a1[c] += Dm(j, mm) * at(CXt, i, mm, k)[c];
                            for (int mm = 0; mm < nq; ++mm) a3[c] -= Dm(j, mm) * at(CXr, i, mm, k)[c];
                            for (int o = 0; o < nq; ++o) a2[c] += Dm(k, o) * at(CXr, i, j, o)[c];
                            for (int o = 0; o < nq; ++o) a1[c] -= Dm(k, o) * at(CXs, i, j, o)[c];
                        }
                        const double* xr = at(Xr, i, j, k);
                        const double* xs = at(Xs, i, j, k);
                        const double* xt = at(Xt, i, j, k);
                        double cst[3];
                        cross3(xs, xt, cst);
                        double detJ = xr[0] * cst[0] + xr[1] * cst[1] + xr[2] * cst[2];
                        double den = 2 * detJ;
                        int n = i + nq * (j + nq * k);
                        // dRdX = [a1 a2 a3]' ./ 2detJ : row a = a_{a+1}
                        for (int b = 0; b < 3; ++b) {
                            m[n + (size_t)np * (0 + 3 * b)] = a1[b] / den;
                            m[n + (size_t)np * (1 + 3 * b)] = a2[b] / den;
                            m[n + (size_t)np * (2 + 3 * b)] = a3[b] / den;
                        }
                        m[n + (size_t)np * 9] = detJ;
                        m[n + (size_t)np * 10] = ((g.w[i] * g.w[j]) * g.w[k]) * detJ;
                    }
        }
    }
}

static void build_face_maps(og_grid& g) {
    const int dim = g.dim, nq = g.nq, np = g.np, nfp = g.nfp, nf = g.nfaces;
    const int64_t E = g.E;
    g.vmapM.assign((size_t)nf * nfp * E, 0);
    g.vmapP.assign((size_t)nf * nfp * E, 0);
    g.bc.assign((size_t)nf * E, 0);
    std::vector<std::vector<int>> cfi(nf);
    for (int f = 0; f < nf; ++f) cell_face_indices(dim, nq, f, cfi[f]);
    for (int64_t e = 0; e < E; ++e)  // src/lobattocells.jl:2278-2287
        for (int f = 0; f < nf; ++f)
            for (int j = 0; j < nfp; ++j)
                g.vmapM[(size_t)nf * nfp * e + (size_t)f * nfp + j] = cfi[f][j] + (int64_t)np * e;
    std::vector<int64_t> mapP((size_t)nf * nfp * E);
    for (size_t n = 0; n < mapP.size(); ++n) mapP[n] = (int64_t)n + 1;

    if (dim == 1) {
        // _get_quadrant_data(::Any1DBrickGridManager) (src/gridmanager.jl:918-1016)
        for (int64_t e = 0; e < E; ++e) {
            for (int f = 0; f < 2; ++f) {
                int64_t e2 = (f == 0) ? e - 1 : e + 1;
                int f2 = 1 - f;
                if (e2 < 0 || e2 >= E) {
                    if (g.periodic[0]) e2 = (e2 + E) % E;
                    else { e2 = e; f2 = f; g.bc[2 * e + f] = f + 1; }
                }
                mapP[2 * e + f] = 2 * e2 + f2 + 1;
            }
        }
    } else {
        // materializefacemaps, conforming branch (src/lobattocells.jl:1992-2206) on the
        // brick's degree-3 node lattice.
        const int n3 = (dim == 2) ? 16 : 64;
        auto gid = [&](int64_t e, const int* abc) -> int64_t {
            int64_t id = 0, stride = 1;
            for (int d = 0; d < dim; ++d) {
                int64_t L = 3 * (int64_t)g.K[d];
                int64_t c = 3 * (int64_t)g.tree[e][d] + (abc[d] - 1);
                if (g.periodic[d]) c %= L;
                id += c * stride;
                stride *= (L + 1);
            }
            return id;
        };
        static const int f3d[6][4][3] = {{{1, 2, 2}, {1, 3, 2}, {1, 2, 3}, {1, 3, 3}},
                                         {{4, 2, 2}, {4, 3, 2}, {4, 2, 3}, {4, 3, 3}},
                                         {{2, 1, 2}, {3, 1, 2}, {2, 1, 3}, {3, 1, 3}},
                                         {{2, 4, 2}, {3, 4, 2}, {2, 4, 3}, {3, 4, 3}},
                                         {{2, 2, 1}, {3, 2, 1}, {2, 3, 1}, {3, 3, 1}},
                                         {{2, 2, 4}, {3, 2, 4}, {2, 3, 4}, {3, 3, 4}}};
        static const int f2d[4][2][3] = {{{1, 2, 0}, {1, 3, 0}}, {{4, 2, 0}, {4, 3, 0}},
                                         {{2, 1, 0}, {3, 1, 0}}, {{2, 4, 0}, {3, 4, 0}}};
        static const int i2f3[6][4] = {{21, 25, 37, 41}, {24, 28, 40, 44}, {18, 19, 34, 35},
                                       {30, 31, 46, 47}, {6, 7, 10, 11},   {54, 55, 58, 59}};
        static const int i2f2[4][2] = {{5, 9}, {8, 12}, {2, 3}, {14, 15}};
        const int nc = (dim == 2) ? 2 : 4;
        auto facenode = [&](int f, int n) -> const int* { return dim == 2 ? f2d[f][n] : f3d[f][n]; };
        auto loc3 = [&](const int* abc) { return abc[0] + 4 * (abc[1] - 1) + (dim == 3 ? 16 * (abc[2] - 1) : 0); };
        auto indextoface = [&](int pi) {
            for (int f = 0; f < nf; ++f)
                for (int n = 0; n < nc; ++n)
                    if ((dim == 2 ? i2f2[f][n] : i2f3[f][n]) == pi) return f;
            return -1;
        };
        // face orientations (src/lobattocells.jl:2061-2070)
        std::vector<int> orient((size_t)nf * E);
        for (int64_t e = 0; e < E; ++e)
            for (int f = 0; f < nf; ++f) {
                int64_t s[4];
                for (int n = 0; n < nc; ++n) s[n] = gid(e, facenode(f, n));
                orient[(size_t)nf * e + f] = (dim == 2) ? orient2(s[0], s[1]) : orient4(s);
            }
        // continuous -> discontinuous rows for the first degree-3 node of every face
        std::unordered_map<int64_t, std::vector<int64_t>> ctod;
        ctod.reserve((size_t)E * nf);
        for (int64_t e = 0; e < E; ++e)
            for (int f = 0; f < nf; ++f) {
                const int* abc = facenode(f, 0);
                ctod[gid(e, abc)].push_back((int64_t)n3 * e + loc3(abc));
            }
        for (auto& kv : ctod) std::sort(kv.second.begin(), kv.second.end());
        int fdims[6][2];
        for (int f = 0; f < nf; ++f) {
            if (dim == 2) { fdims[f][0] = nq; fdims[f][1] = 1; }
            else { fdims[f][0] = nq; fdims[f][1] = nq; }
        }
        for (int64_t e = 0; e < E; ++e)
            for (int f = 0; f < nf; ++f) {
                const auto& rows = ctod[gid(e, facenode(f, 0))];
                size_t kind = rows.size();
                if (kind == 1) { g.bc[(size_t)nf * e + f] = 1; continue; }
                if (kind != 2) continue;  // non-conforming faces keep mapP = self
                int64_t nqe = -1;
                int nfc = -1;
                for (int64_t row : rows) {
                    nqe = (row - 1) / n3;
                    int pi = (int)((row - 1) % n3) + 1;
                    nfc = indextoface(pi);
                    if (nqe != e || nfc != f) break;
                }
                int o = (dim == 2) ? compose2(orient[(size_t)nf * e + f], orient[(size_t)nf * nqe + nfc])
                                   : compose4(inv4(orient[(size_t)nf * e + f]), orient[(size_t)nf * nqe + nfc]);
                for (int j = 0; j < nfp; ++j) {
                    int fi;
                    if (dim == 2) {
                        int i1 = j + 1;
                        fi = (o == 1) ? i1 : nq - i1 + 1;
                    } else {
                        int i1 = j % nq + 1, i2 = j / nq + 1, o1, o2;
                        orientindex4(o, fdims[f][0], fdims[f][1], i1, i2, o1, o2);
                        fi = (o1 - 1) + nq * (o2 - 1) + 1;
                    }
                    mapP[(size_t)nf * nfp * e + (size_t)f * nfp + j] =
                        (int64_t)nf * nfp * nqe + (int64_t)nfc * nfp + fi;
                }
            }
    }
    for (size_t n = 0; n < mapP.size(); ++n) g.vmapP[n] = g.vmapM[mapP[n] - 1];
}

static void build_surface_metrics(og_grid& g) {
    // hexsurfacemetrics! / quadsurfacemetrics! / linesurfacemetrics!
    // (src/lobattocells.jl:3253-3295, 2862-2900, 2630-2664)
    const int dim = g.dim, np = g.np, nfp = g.nfp, nf = g.nfaces, ns = g.nsmet, nv = g.nvmet, nq = g.nq;
    g.smet.assign((size_t)ns * nf * nfp * g.E, 0.0);
    for (int64_t e = 0; e < g.E; ++e)
        for (int f = 0; f < nf; ++f)
            for (int j = 0; j < nfp; ++j) {
                size_t sk = (size_t)nf * nfp * e + (size_t)f * nfp + j;
                int64_t k = g.vmapM[sk] - 1;
                int64_t ke = k / np;
                int kn = (int)(k % np);
                const double* m = &g.vmet[(size_t)np * nv * ke];
                int fg = f / 2, fn = f % 2;
                double sn = fn == 0 ? -1.0 : 1.0;
                double J = m[kn + (size_t)np * (dim * dim)];
                double n[3], sJ2 = 0;
                for (int d = 0; d < dim; ++d) n[d] = (sn * J) * m[kn + (size_t)np * (fg + dim * d)];
                for (int d = 0; d < dim; ++d) sJ2 += n[d] * n[d];
                double sJ = std::sqrt(sJ2);
                for (int d = 0; d < dim; ++d) n[d] = n[d] / sJ;
                double wsJ;
                if (dim == 1) wsJ = sJ;
                else if (dim == 2) wsJ = sJ * (fg == 0 ? g.w[j] : g.w[j]);
                else {
                    int i1 = j % nq, i2 = j / nq;
                    wsJ = (sJ * g.w[i1]) * g.w[i2];
                }
                double* s = &g.smet[(size_t)ns * sk];
                for (int d = 0; d < dim; ++d) s[d] = n[d];
                s[dim] = sJ;
                s[dim + 1] = wsJ;
            }
}

extern "C" og_grid* og_grid_create(int dim, int nq, const int* K, const double* lo, const double* hi,
                                   const int* periodic, int warp, double warp_amp) {
    og_grid* g = new og_grid();
    g->dim = dim;
    g->nq = nq;
    g->np = 1;
    for (int d = 0; d < dim; ++d) g->np *= nq;
    g->nfp = g->np / nq;
    g->nfaces = 2 * dim;
    g->nvmet = dim * dim + 2;
    g->nsmet = dim + 2;
    g->warp = warp;
    for (int d = 0; d < 3; ++d) {
        g->K[d] = d < dim ? K[d] : 1;
        g->periodic[d] = d < dim ? periodic[d] : 0;
    }
    g->r.resize(nq);
    g->w.resize(nq);
    g->D.resize(nq * nq);
    og_lgl(nq, g->r.data(), g->w.data(), g->D.data());
    for (int d = 0; d < dim; ++d) {
        g->vx[d].resize(g->K[d] + 1);
        for (int i = 0; i <= g->K[d]; ++i) g->vx[d][i] = range_value(lo[d], hi[d], i, g->K[d]);
    }
    brick_tree_order(dim, g->K, g->tree);
    g->E = (int64_t)g->tree.size();
    // points (unwarped), then the warp
    {
        const int np = g->np;
        g->points.assign((size_t)np * dim * g->E, 0.0);
        for (int64_t e = 0; e < g->E; ++e) {
            const auto& t = g->tree[e];
            for (int d = 0; d < dim; ++d) {
                double c1 = g->vx[d][t[d]];
                double dx = g->vx[d][t[d] + 1] - c1;
                for (int n = 0; n < np; ++n) {
                    int idx[3] = {n % nq, (n / nq) % nq, n / (nq * nq)};
                    double rr = fma(0.5, g->r[idx[d]] + 1, 0.0);
                    g->points[n + (size_t)np * (d + dim * e)] = fma(dx, rr, c1);
                }
            }
        }
        build_points_warp(*g, warp_amp);
    }
    if (warp == OG_WARP_NONE) build_brick_metrics(*g);
    else build_curved_metrics(*g);
    build_face_maps(*g);
    build_surface_metrics(*g);
    g->MJI.resize((size_t)g->np * g->E);
    for (int64_t e = 0; e < g->E; ++e)
        for (int n = 0; n < g->np; ++n)
            g->MJI[(size_t)g->np * e + n] = 1.0 / g->vmet[n + (size_t)g->np * (g->nvmet - 1 + (size_t)g->nvmet * e)];
    return g;
}

extern "C" void og_grid_destroy(og_grid* g) { delete g; }

extern "C" void og_grid_sizes(const og_grid* g, int64_t* s) {
    s[0] = g->dim; s[1] = g->nq; s[2] = g->np; s[3] = g->nfp; s[4] = g->nfaces; s[5] = g->E;
    s[6] = g->nvmet; s[7] = g->nsmet;
}
extern "C" void og_grid_lgl(const og_grid* g, double* r, double* w, double* D) {
    std::copy(g->r.begin(), g->r.end(), r);
    std::copy(g->w.begin(), g->w.end(), w);
    std::copy(g->D.begin(), g->D.end(), D);
}
extern "C" void og_grid_points(const og_grid* g, double* o) { std::copy(g->points.begin(), g->points.end(), o); }
extern "C" void og_grid_vmet(const og_grid* g, double* o) { std::copy(g->vmet.begin(), g->vmet.end(), o); }
extern "C" void og_grid_smet(const og_grid* g, double* o) { std::copy(g->smet.begin(), g->smet.end(), o); }
extern "C" void og_grid_vmapM(const og_grid* g, int64_t* o) { std::copy(g->vmapM.begin(), g->vmapM.end(), o); }
extern "C" void og_grid_vmapP(const og_grid* g, int64_t* o) { std::copy(g->vmapP.begin(), g->vmapP.end(), o); }
extern "C" void og_grid_boundary(const og_grid* g, int64_t* o) { std::copy(g->bc.begin(), g->bc.end(), o); }
extern "C" void og_grid_tree_coords(const og_grid* g, int32_t* o) {
    for (int64_t e = 0; e < g->E; ++e)
        for (int d = 0; d < 3; ++d) o[3 * e + d] = g->tree[e][d];
}

// ---------------------------------------------------------------------------------
// Physics (src/balancelaws/balancelaws/{advection,euler}.jl, numericalfluxes.jl)
// ---------------------------------------------------------------------------------

static const int MAXS = 5;

struct Phys {
    int dim, ns;
    og_law L;
};

static inline double dotv(const double* a, const double* b, int n) {
    double s = a[0] * b[0];
    for (int i = 1; i < n; ++i) s = s + a[i] * b[i];
    return s;
}

static inline double pressure(const Phys& P, const double* q) {  // euler.jl:34-37
    const int dim = P.dim;
    double rho = q[0], rhoe = q[dim + 1];
    return (P.L.gamma - 1) * (rhoe - dotv(q + 1, q + 1, dim) / (2 * rho));
}

// F[d*MAXS + s]: physical flux (euler.jl:50-61, advection.jl:18)
static void flux(const Phys& P, const double* q, double* F) {
    const int dim = P.dim;
    if (P.L.law == OG_LAW_ADVECTION) {
        for (int d = 0; d < dim; ++d) F[d * MAXS] = P.L.adv[d] * q[0];
        return;
    }
    double rho = q[0], rhoe = q[dim + 1];
    double u[3];
    for (int d = 0; d < dim; ++d) u[d] = q[1 + d] / rho;
    double p = pressure(P, q);
    for (int d = 0; d < dim; ++d) {
        F[d * MAXS + 0] = q[1 + d];
        for (int b = 0; b < dim; ++b) F[d * MAXS + 1 + b] = (d == b) ? q[1 + d] * u[b] + p : q[1 + d] * u[b];
        F[d * MAXS + dim + 1] = u[d] * (rhoe + p);
    }
}

static double wavespeed(const Phys& P, const double* n, const double* q) {  // euler.jl:63-68
    const int dim = P.dim;
    if (P.L.law == OG_LAW_ADVECTION) return std::fabs(dotv(n, P.L.adv, dim));
    double rho = q[0];
    double u[3];
    for (int d = 0; d < dim; ++d) u[d] = q[1 + d] / rho;
    double p = pressure(P, q);
    return std::fabs(dotv(n, u, dim)) + std::sqrt(P.L.gamma * p / rho);
}

static double logavg(double a, double b) {  // numericalfluxes.jl:9-22
    double zeta = a / b;
    double f = (zeta - 1) / (zeta + 1);
    double u = f * f;
    const double eps = 2.220446049250313e-16;
    double F;
    if (u < eps) {
        // @evalpoly(u, 1, 1/3, 1/5, 1/7, 1/9) (Horner with muladd)
        F = fma(u, fma(u, fma(u, fma(u, 1.0 / 9, 1.0 / 7), 1.0 / 5), 1.0 / 3), 1.0);
    } else {
        F = std::log(zeta) / (2 * f);
    }
    return (a + b) / (2 * F);
}

static void twopointflux(const Phys& P, int which, const double* q1, const double* q2, double* F) {
    const int dim = P.dim, ns = P.ns;
    if (which == OG_FLUX_CENTRAL || P.L.law == OG_LAW_ADVECTION) {  // numericalfluxes.jl:40-42
        double F1[3 * MAXS], F2[3 * MAXS];
        flux(P, q1, F1);
        flux(P, q2, F2);
        for (int d = 0; d < dim; ++d)
            for (int s = 0; s < ns; ++s) F[d * MAXS + s] = (F1[d * MAXS + s] + F2[d * MAXS + s]) / 2;
        return;
    }
    double r1 = q1[0], r2 = q2[0];
    double u1[3], u2[3], ua[3];
    for (int d = 0; d < dim; ++d) { u1[d] = q1[1 + d] / r1; u2[d] = q2[1 + d] / r2; }
    double p1 = pressure(P, q1), p2 = pressure(P, q2);
    for (int d = 0; d < dim; ++d) ua[d] = (u1[d] + u2[d]) / 2;
    if (which == OG_FLUX_KG) {  // euler.jl:186-216
        double e1 = q1[dim + 1] / r1, e2 = q2[dim + 1] / r2;
        double ra = (r1 + r2) / 2, ea = (e1 + e2) / 2, pa = (p1 + p2) / 2;
        double fr[3];
        for (int d = 0; d < dim; ++d) fr[d] = ua[d] * ra;
        for (int d = 0; d < dim; ++d) {
            F[d * MAXS] = fr[d];
            for (int b = 0; b < dim; ++b) F[d * MAXS + 1 + b] = (d == b) ? ua[d] * fr[b] + pa : ua[d] * fr[b];
            F[d * MAXS + dim + 1] = ua[d] * (ra * ea + pa);
        }
        return;
    }
    // entropy conservative (euler.jl:150-184)
    double b1 = r1 / (2 * p1), b2 = r2 / (2 * p2);
    double ra = (r1 + r2) / 2, ba = (b1 + b2) / 2;
    double u2a = (dotv(u1, u1, dim) + dotv(u2, u2, dim)) / 2;
    double rlog = logavg(r1, r2), blog = logavg(b1, b2);
    double fr[3], M[3][3];
    for (int d = 0; d < dim; ++d) fr[d] = ua[d] * rlog;
    double pt = ra / (2 * ba);
    for (int a = 0; a < dim; ++a)
        for (int b = 0; b < dim; ++b) M[a][b] = (a == b) ? ua[a] * fr[b] + pt : ua[a] * fr[b];
    double c = 1 / ((2 * (P.L.gamma - 1)) * blog) - u2a / 2;
    for (int d = 0; d < dim; ++d) {
        F[d * MAXS] = fr[d];
        for (int b = 0; b < dim; ++b) F[d * MAXS + 1 + b] = M[d][b];
        double mu = M[d][0] * ua[0];
        for (int b = 1; b < dim; ++b) mu = mu + M[d][b] * ua[b];
        F[d * MAXS + dim + 1] = c * fr[d] + mu;
    }
}

// F' * n for a (dim, ns) flux
static void contract(const Phys& P, const double* F, const double* n, double* nf) {
    for (int s = 0; s < P.ns; ++s) {
        double v = F[s] * n[0];
        for (int d = 1; d < P.dim; ++d) v = v + F[d * MAXS + s] * n[d];
        nf[s] = v;
    }
}

// entropyvariables (euler.jl:79-91)
static void entropyvariables(const Phys& P, const double* q, double* v) {
    const int dim = P.dim;
    const double g = P.L.gamma, rho = q[0], p = pressure(P, q);
    const double sv = std::log(p / std::pow(rho, g)), b = rho / (2 * p);
    double u[3];
    for (int d = 0; d < dim; ++d) u[d] = q[1 + d] / rho;
    v[0] = (g - sv) / (g - 1) - dotv(u, u, dim) * b;
    for (int d = 0; d < dim; ++d) v[1 + d] = 2 * b * u[d];
    v[dim + 1] = -2 * b;
}

// Roe flux (euler.jl:93-149)
static void roeflux(const Phys& P, const double* n, const double* qm, const double* qp, double* nf) {
    const int dim = P.dim, ns = P.ns;
    const double g = P.L.gamma;
    double Fm[3 * MAXS], Fp[3 * MAXS], fm[MAXS], fp[MAXS];
    flux(P, qm, Fm);
    flux(P, qp, Fp);
    contract(P, Fm, n, fm);
    contract(P, Fp, n, fp);
    const double rm = qm[0], rp = qp[0], pm = pressure(P, qm), pp = pressure(P, qp);
    double um[3], up[3];
    for (int d = 0; d < dim; ++d) { um[d] = qm[1 + d] / rm; up[d] = qp[1 + d] / rp; }
    const double hm = qm[dim + 1] / rm + pm / rm, hp = qp[dim + 1] / rp + pp / rp;
    const double cm = std::sqrt(g * pm / rm), cp = std::sqrt(g * pp / rp);
    const double sm = std::sqrt(rm), sp = std::sqrt(rp);
    auto roe_avg = [&](double a, double b) { return (sm * a + sp * b) / (sm + sp); };  // numericalfluxes.jl:23
    const double rho = std::sqrt(rm * rp), h = roe_avg(hm, hp), c = roe_avg(cm, cp);
    double u[3], du[3];
    for (int d = 0; d < dim; ++d) { u[d] = roe_avg(um[d], up[d]); du[d] = up[d] - um[d]; }
    const double un = dotv(u, n, dim), dun = dotv(du, n, dim);
    const double drho = rp - rm, dp = pp - pm, ci2 = 1 / (c * c);
    const double w1 = std::fabs(un - c) * (dp - rho * c * dun) * ci2 / 2;
    const double w2 = std::fabs(un + c) * (dp + rho * c * dun) * ci2 / 2;
    const double w3 = std::fabs(un) * (drho - dp * ci2);
    const double w4 = std::fabs(un) * rho;
    double D[MAXS];
    D[0] = (w1 + w2 + w3) / 2;
    for (int k = 0; k < dim; ++k)
        D[1 + k] = (w1 * (u[k] - c * n[k]) + w2 * (u[k] + c * n[k]) + w3 * u[k] + w4 * (du[k] - dun * n[k])) / 2;
    D[dim + 1] = (w1 * (h - c * un) + w2 * (h + c * un) + w3 * dotv(u, u, dim) / 2 + w4 * (dotv(u, du, dim) - un * dun)) / 2;
    for (int s = 0; s < ns; ++s) nf[s] = (fm[s] + fp[s]) / 2 - D[s];
}

// matrix-dissipation flux (euler.jl:218-300): the entropy-conservative flux minus a
// dissipation built on the jump of the entropy variables
static void matrixflux(const Phys& P, const double* n, const double* qm, const double* qp, double* nf) {
    const int dim = P.dim, ns = P.ns;
    const double g = P.L.gamma;
    double F[3 * MAXS];
    twopointflux(P, OG_FLUX_EC, qm, qp, F);
    contract(P, F, n, nf);
    const double rm = qm[0], rp = qp[0], pm = pressure(P, qm), pp = pressure(P, qp);
    double um[3], up[3], ua[3];
    for (int d = 0; d < dim; ++d) {
        um[d] = qm[1 + d] / rm;
        up[d] = qp[1 + d] / rp;
        ua[d] = (um[d] + up[d]) / 2;
    }
    const double bm = rm / (2 * pm), bp = rp / (2 * pp);
    const double rlog = logavg(rm, rp), blog = logavg(bm, bp);
    const double pavg = ((rm + rp) / 2) / (2 * ((bm + bp) / 2));
    const double u2bar = 2 * std::sqrt(dotv(ua, ua, dim)) - (std::sqrt(dotv(um, um, dim)) + std::sqrt(dotv(up, up, dim))) / 2;
    const double hbar = g / (2 * blog * (g - 1)) + u2bar / 2;
    const double cbar = std::sqrt(g * pavg / rlog);
    const double un = dotv(ua, n, dim);
    double umc[3], upc[3], ut[3], vm[MAXS], vp[MAXS], dv[MAXS];
    for (int d = 0; d < dim; ++d) {
        umc[d] = ua[d] - cbar * n[d];
        upc[d] = ua[d] + cbar * n[d];
        ut[d] = ua[d] - un * n[d];
    }
    entropyvariables(P, qm, vm);
    entropyvariables(P, qp, vp);
    for (int s = 0; s < ns; ++s) dv[s] = vp[s] - vm[s];
    const double l1 = std::fabs(un - cbar) * rlog / (2 * g);
    const double l2 = std::fabs(un) * rlog * (g - 1) / g;
    const double l3 = std::fabs(un + cbar) * rlog / (2 * g);
    const double l4 = std::fabs(un) * pavg;
    const double* dvm = dv + 1;
    const double dve = dv[dim + 1];
    const double w1 = l1 * (dv[0] + dotv(umc, dvm, dim) + (hbar - cbar * un) * dve);
    const double w2 = l2 * (dv[0] + dotv(ua, dvm, dim) + u2bar / 2 * dve);
    const double w3 = l3 * (dv[0] + dotv(upc, dvm, dim) + (hbar + cbar * un) * dve);
    const double ndv = dotv(n, dvm, dim);
    double D[MAXS];
    D[0] = w1 + w2 + w3;
    for (int k = 0; k < dim; ++k)
        D[1 + k] = w1 * umc[k] + w2 * ua[k] + w3 * upc[k] + l4 * (dvm[k] - ndv * n[k] + dve * ut[k]);
    D[dim + 1] = w1 * (hbar - cbar * un) + w2 * u2bar / 2 + w3 * (hbar + cbar * un) +
                 l4 * (dotv(ut, dvm, dim) + dve * (dotv(ua, ua, dim) - un * un));
    for (int s = 0; s < ns; ++s) nf[s] = nf[s] - D[s] / 2;
}

// surfaceflux (numericalfluxes.jl:27-37, 44-50; euler.jl:93-149, 218-300)
static void surfaceflux(const Phys& P, const double* n, const double* qm, const double* qp, double* nf) {
    const int dim = P.dim, ns = P.ns;
    const int which = P.L.surface_flux;
    if (P.L.law == OG_LAW_EULER && which == OG_FLUX_ROE) return roeflux(P, n, qm, qp, nf);
    if (P.L.law == OG_LAW_EULER && which == OG_FLUX_MATRIX) return matrixflux(P, n, qm, qp, nf);
    double Fc[3 * MAXS];
    // the default surfaceflux: the flux's two-point form contracted with n
    twopointflux(P, which == OG_FLUX_RUSANOV ? OG_FLUX_CENTRAL : which, qm, qp, Fc);
    for (int s = 0; s < ns; ++s) {
        double v = Fc[s] * n[0];
        for (int d = 1; d < dim; ++d) v = v + Fc[d * MAXS + s] * n[d];
        nf[s] = v;
    }
    if (which == OG_FLUX_RUSANOV) {
        double wm = wavespeed(P, n, qm), wp = wavespeed(P, n, qp);
        double mx = std::max(wm, wp);
        for (int s = 0; s < ns; ++s) nf[s] = nf[s] - (mx * (qp[s] - qm[s])) / 2;
    }
}

static int num_states(const og_grid* g, const og_law* L) { return L->law == OG_LAW_ADVECTION ? 1 : g->dim + 2; }

// ---------------------------------------------------------------------------------
// DGSEM tendency (src/balancelaws/dgsem.jl)
// ---------------------------------------------------------------------------------

static void element_tendency(const og_grid* g, const Phys& Ph, double* dq, const double* q, bool increment,
                             int64_t e, std::vector<double>& scratch, const double* ncflux) {
    const int dim = g->dim, nq = g->nq, np = g->np, ns = Ph.ns, nv = g->nvmet;
    const double* D = g->D.data();
    auto Dm = [&](int i, int j) { return D[i + nq * j]; };
    const double* m = &g->vmet[(size_t)np * nv * e];
    auto dRdX = [&](int n, int a, int b) { return m[n + (size_t)np * (a + dim * b)]; };
    auto MJ = [&](int n) { return m[n + (size_t)np * (dim * dim + 1)]; };
    const double* MJI = &g->MJI[(size_t)np * e];
    const double* qe = q + (size_t)np * ns * e;
    double* dqe = dq + (size_t)np * ns * e;
    auto qnode = [&](int n, double* out) {
        for (int s = 0; s < ns; ++s) out[s] = qe[n + (size_t)np * s];
    };
    auto ijk = [&](int n, int* idx) { idx[0] = n % nq; idx[1] = (n / nq) % nq; idx[2] = n / (nq * nq); };
    auto lin = [&](int i, int j, int k) { return i + nq * (j + nq * k); };
    // `d in directions` (dgsem.jl:257-348, 203-227, 756-782)
    const int dmask = g->dir_mask ? g->dir_mask : (1 << dim) - 1;
    auto in_dirs = [&](int d) { return ((dmask >> d) & 1) != 0; };

    if (Ph.L.form == OG_FORM_WEAK) {
        // volumeterm! (dgsem.jl:257-348)
        scratch.resize((size_t)np * dim * ns);
        double* lF = scratch.data();  // lF[(n*dim + d)*ns + s]
        for (int n = 0; n < np; ++n) {
            double qn[MAXS], F[3 * MAXS];
            qnode(n, qn);
            flux(Ph, qn, F);
            double mj = MJ(n);
            for (int s = 0; s < ns; ++s)
                for (int d = 0; d < dim; ++d) {
                    double v = 0.0;
                    for (int dd = 0; dd < dim; ++dd) v += dRdX(n, d, dd) * F[dd * MAXS + s];
                    v *= mj;
                    lF[((size_t)n * dim + d) * ns + s] = v;
                }
        }
        for (int n = 0; n < np; ++n) {
            int id[3];
            ijk(n, id);
            double acc[MAXS];
            for (int s = 0; s < ns; ++s) acc[s] = -0.0;
            double mji = MJI[n];
            for (int a = 0; a < nq; ++a) {
                double Dd[3];
                for (int d = 0; d < dim; ++d) Dd[d] = Dm(a, id[d]) * mji;
                for (int s = 0; s < ns; ++s) {
                    for (int d = 0; d < dim; ++d) {
                        if (!in_dirs(d)) continue;
                        int nb = (d == 0) ? lin(a, id[1], id[2]) : (d == 1 ? lin(id[0], a, id[2]) : lin(id[0], id[1], a));
                        acc[s] += Dd[d] * lF[((size_t)nb * dim + d) * ns + s];
                    }
                }
            }
            for (int s = 0; s < ns; ++s) {
                double& t = dqe[n + (size_t)np * s];
                t = increment ? t + acc[s] : acc[s];
            }
        }
    } else {
        // esvolumeterm_dir! per direction (dgsem.jl:203-227, 514-608)
        scratch.resize((size_t)np * 3);
        double* lg = scratch.data();
        int first_dir = 0;
        while (!in_dirs(first_dir)) ++first_dir;
        for (int dir = 0; dir < dim; ++dir) {
            if (!in_dirs(dir)) continue;
            for (int n = 0; n < np; ++n)
                for (int d = 0; d < dim; ++d) lg[n * 3 + d] = MJ(n) * dRdX(n, dir, d);
            bool inc = (dir == first_dir) ? increment : true;
            for (int n = 0; n < np; ++n) {
                int id3[3];
                ijk(n, id3);
                double q1[MAXS];
                qnode(n, q1);
                double acc[MAXS];
                for (int s = 0; s < ns; ++s) acc[s] = -0.0;
                double mji = MJI[n];
                int id = id3[dir];
                for (int a = 0; a < nq; ++a) {
                    int ild = (dir == 0) ? lin(a, id3[1], id3[2]) : (dir == 1 ? lin(id3[0], a, id3[2]) : lin(id3[0], id3[1], a));
                    double q2[MAXS], F[3 * MAXS];
                    qnode(ild, q2);
                    twopointflux(Ph, Ph.L.volume_flux, q1, q2, F);
                    for (int s = 0; s < ns; ++s) {
                        double Ddn = mji * Dm(id, a);
                        double Dnd = mji * Dm(a, id);
                        for (int d = 0; d < dim; ++d) {
                            acc[s] -= (Ddn * lg[n * 3 + d]) * F[d * MAXS + s];
                            acc[s] += (F[d * MAXS + s] * lg[ild * 3 + d]) * Dnd;
                        }
                    }
                }
                for (int s = 0; s < ns; ++s) {
                    double& t = dqe[n + (size_t)np * s];
                    t = inc ? t + acc[s] : acc[s];
                }
            }
        }
    }
    // surfaceterm! (dgsem.jl:733-784): faces in order x-, x+, y-, y+, z-, z+
    const int nfp = g->nfp, nf = g->nfaces, nsm = g->nsmet;
    for (int face = 0; face < nf; ++face) {
        if (!in_dirs(face / 2)) continue;
        for (int i = 0; i < nfp; ++i) {
            size_t j = (size_t)nf * nfp * e + (size_t)face * nfp + i;
            int64_t idm = g->vmapM[j] - 1;
            const double* sm = &g->smet[(size_t)nsm * j];
            double n[3];
            for (int d = 0; d < dim; ++d) n[d] = sm[d];
            double fMJ = sm[dim + 1];
            int64_t em = idm / np, nm = idm % np;
            double qm[MAXS], qp[MAXS];
            for (int s = 0; s < ns; ++s) qm[s] = q[(size_t)np * ns * em + (size_t)np * s + nm];
            if (ncflux && g->ncface[(size_t)nf * e + face]) {  // mortar face: its flux comes precomputed
                const double mji = g->MJI[idm];
                for (int s = 0; s < ns; ++s) {
                    const double nfl = ncflux[(((size_t)nf * e + face) * ns + s) * nfp + i];
                    double& t = dq[(size_t)np * ns * em + (size_t)np * s + nm];
                    t = t - (fMJ * nfl) * mji;
                }
                continue;
            }
            if (g->bc[(size_t)nf * e + face] == 0) {
                int64_t idp = g->vmapP[j] - 1;
                int64_t ep = idp / np, npn = idp % np;
                for (int s = 0; s < ns; ++s) qp[s] = q[(size_t)np * ns * ep + (size_t)np * s + npn];
            } else {
                for (int s = 0; s < ns; ++s) qp[s] = qm[s];  // balancelaw.jl:77 default boundarystate
                const int64_t tag = g->bc[(size_t)nf * e + face];
                const int kind = (tag >= 1 && tag <= 8) ? g->bc_kind[tag] : 0;
                if (kind == 1) {
                    for (int s = 0; s < ns; ++s) qp[s] = g->bc_state[tag][s];
                } else if (kind == 2 && ns == dim + 2) {
                    // rho u+ = rho u- - 2 (n' rho u-) n (examples/balancelaws/euler_gravity/gravitywave.jl:16-21)
                    double mn = 0.0;
                    for (int d = 0; d < dim; ++d) mn = d == 0 ? n[0] * qm[1] : mn + n[d] * qm[1 + d];
                    for (int d = 0; d < dim; ++d) qp[1 + d] = qm[1 + d] - (2 * mn) * n[d];
                }
            }
            double nfl[MAXS];
            surfaceflux(Ph, n, qm, qp, nfl);
            double mji = g->MJI[idm];
            for (int s = 0; s < ns; ++s) {
                double& t = dq[(size_t)np * ns * em + (size_t)np * s + nm];
                t = t - (fMJ * nfl[s]) * mji;
            }
        }
    }
}

// Face-node index j of face f (x-, x+, y-, y+, z-, z+): volume node (lobattocells.jl:2012-2053).
static int face_vol_node(int dim, int nq, int f, int j) {
    const int d = f / 2, c = (f % 2) ? nq - 1 : 0;
    if (dim == 2) return d == 0 ? c + nq * j : j + nq * c;
    const int j1 = j % nq, j2 = j / nq;
    if (d == 0) return c + nq * (j1 + nq * j2);
    if (d == 1) return j1 + nq * (c + nq * j2);
    return j1 + nq * (j2 + nq * c);
}

// Mortar fluxes of an adapted grid (a project-defined restatement: the reference's
// surfaceterm! leaves non-conforming faces uncoupled).  For each mortar, the large
// face's trace is interpolated to the nodes of each small face, the surface flux is
// taken there with the large element's outward normal, the small element gets its
// negative, and the large element gets the lumped L2 projection of the small faces'
// fluxes back onto its face nodes.  ncflux: (nfaces, E) faces x (ns, nfp), only mortar
// faces written.
static void mortar_fluxes(const og_grid* g, const Phys& Ph, const double* q, double* ncflux) {
    const int dim = g->dim, nq = g->nq, np = g->np, nfp = g->nfp, nf = g->nfaces, ns = Ph.ns;
    const int nsmall = dim == 3 ? 4 : 2, mcols = 2 + nsmall;
    const int nq2 = dim == 3 ? nq : 1;  // second in-face direction (none in 2-D)
    const int64_t M = (int64_t)g->mortars.size() / mcols;
    const double one = 1.0;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t m = 0; m < M; ++m) {
        const int64_t* col = &g->mortars[(size_t)mcols * m];
        const int64_t eC = col[0];
        const int fC = (int)col[1], fF = fC ^ 1;
        const int nsm = g->nsmet;
        double n[3] = {0, 0, 0};
        n[fC / 2] = (fC % 2) ? 1.0 : -1.0;
        std::vector<double> qC((size_t)ns * nfp), nfm((size_t)nsmall * ns * nfp);
        for (int j = 0; j < nfp; ++j) {
            const int v = face_vol_node(dim, nq, fC, j);
            for (int s = 0; s < ns; ++s) qC[(size_t)s * nfp + j] = q[(size_t)np * ns * eC + (size_t)np * s + v];
        }
        for (int k = 0; k < nsmall; ++k) {
            const int64_t eF = col[2 + k];
            const double* Ia = (k & 1) ? g->IU.data() : g->IL.data();
            const double* Ib = (k >> 1) ? g->IU.data() : g->IL.data();
            for (int j = 0; j < nfp; ++j) {
                const int j1 = j % nq, j2 = j / nq;
                double qi[MAXS], qf[MAXS], nfl[MAXS];
                const int v = face_vol_node(dim, nq, fF, j);
                for (int s = 0; s < ns; ++s) {
                    double acc = 0.0;
                    for (int b = 0; b < nq2; ++b) {
                        double t = 0.0;
                        for (int a = 0; a < nq; ++a) t = std::fma(Ia[j1 * nq + a], qC[(size_t)s * nfp + a + nq * b], t);
                        acc = std::fma(dim == 3 ? Ib[j2 * nq + b] : one, t, acc);
                    }
                    qi[s] = acc;
                    qf[s] = q[(size_t)np * ns * eF + (size_t)np * s + v];
                }
                double sigma = 1.0;
                if (g->curved_mortars) {
                    // warped grid: the small face's own normal (flipped to point out of the
                    // large element) and surface measure 2^(dim-1) wsJ / W (mortar.cu)
                    const double* sm = &g->smet[(size_t)nsm * ((size_t)nf * nfp * eF + (size_t)fF * nfp + j)];
                    for (int d = 0; d < dim; ++d) n[d] = -sm[d];
                    const double W = dim == 3 ? g->w[j1] * g->w[j2] : g->w[j1];
                    sigma = (double)nsmall * sm[dim + 1] / W;
                }
                surfaceflux(Ph, n, qi, qf, nfl);
                for (int s = 0; s < ns; ++s) {
                    nfm[((size_t)k * ns + s) * nfp + j] = g->curved_mortars ? sigma * nfl[s] : nfl[s];
                    ncflux[(((size_t)nf * eF + fF) * ns + s) * nfp + j] = -nfl[s];
                }
            }
        }
        for (int j = 0; j < nfp; ++j) {
            const int j1 = j % nq, j2 = j / nq;
            double unscale = 1.0;  // curved: 1 / sJ of the large face = W / wsJ_C
            if (g->curved_mortars) {
                const double W = dim == 3 ? g->w[j1] * g->w[j2] : g->w[j1];
                unscale = W / g->smet[(size_t)nsm * ((size_t)nf * nfp * eC + (size_t)fC * nfp + j) + dim + 1];
            }
            for (int s = 0; s < ns; ++s) {
                double acc = 0.0;
                for (int k = 0; k < nsmall; ++k) {
                    const double* Pa = (k & 1) ? g->PU.data() : g->PL.data();
                    const double* Pb = (k >> 1) ? g->PU.data() : g->PL.data();
                    for (int b = 0; b < nq2; ++b) {
                        double t = 0.0;
                        for (int a = 0; a < nq; ++a)
                            t = std::fma(Pa[j1 * nq + a], nfm[((size_t)k * ns + s) * nfp + a + nq * b], t);
                        acc = std::fma(dim == 3 ? Pb[j2 * nq + b] : one, t, acc);
                    }
                }
                if (g->curved_mortars) acc = acc * unscale;
                ncflux[(((size_t)nf * eC + fC) * ns + s) * nfp + j] = acc;
            }
        }
    }
}

extern "C" void og_tendency(const og_grid* g, const og_law* law, double* dq, const double* q, double t,
                            int increment, int64_t e0, int64_t e1) {
    (void)t;
    Phys Ph{g->dim, num_states(g, law), *law};
    std::vector<double> ncflux;
    if (!g->mortars.empty()) {
        ncflux.assign((size_t)g->nfaces * g->E * Ph.ns * g->nfp, 0.0);
        mortar_fluxes(g, Ph, q, ncflux.data());
    }
    const double* nc = ncflux.empty() ? nullptr : ncflux.data();
#pragma omp parallel
    {
        std::vector<double> scratch;
#pragma omp for schedule(dynamic, 16)
        for (int64_t e = e0; e < e1; ++e) element_tendency(g, Ph, dq, q, increment != 0, e, scratch, nc);
    }
}

// A grid from the arrays of a generated Raven grid (adapted grids are built on the host
// by the product's forest module; their arrays are the oracle's input here).
extern "C" og_grid* og_grid_from_arrays(int dim, int nq, int64_t E, const double* points, const double* vmet,
                                        const double* smet, const int64_t* vmapM, const int64_t* vmapP,
                                        const int64_t* bc) {
    og_grid* g = new og_grid();
    g->dim = dim;
    g->nq = nq;
    g->np = 1;
    for (int d = 0; d < dim; ++d) g->np *= nq;
    g->nfp = g->np / nq;
    g->nfaces = 2 * dim;
    g->nvmet = dim * dim + 2;
    g->nsmet = dim + 2;
    g->warp = OG_WARP_NONE;
    g->E = E;
    for (int d = 0; d < 3; ++d) {
        g->K[d] = 1;
        g->periodic[d] = 0;
    }
    g->r.resize(nq);
    g->w.resize(nq);
    g->D.resize(nq * nq);
    og_lgl(nq, g->r.data(), g->w.data(), g->D.data());
    g->tree.assign(E, {0, 0, 0});
    const size_t np = g->np, nfp = g->nfp, nf = g->nfaces;
    g->points.assign(points, points + np * dim * E);
    g->vmet.assign(vmet, vmet + np * g->nvmet * E);
    g->smet.assign(smet, smet + (size_t)g->nsmet * nf * nfp * E);
    g->vmapM.assign(vmapM, vmapM + nf * nfp * E);
    g->vmapP.assign(vmapP, vmapP + nf * nfp * E);
    g->bc.assign(bc, bc + nf * E);
    g->MJI.resize(np * E);
    for (int64_t e = 0; e < E; ++e)
        for (size_t n = 0; n < np; ++n) g->MJI[np * e + n] = 1.0 / g->vmet[n + np * (g->nvmet - 1 + (size_t)g->nvmet * e)];
    return g;
}

// Mortars of an adapted grid: (2 + 2^(dim-1), M) int64 0-based, and the (nq, nq)
// row-major operators I_lower, I_upper, P_lower, P_upper.
extern "C" void og_grid_set_mortars(og_grid* g, const int64_t* mortars, int64_t M, const double* IL,
                                    const double* IU, const double* PL, const double* PU) {
    const int mcols = 2 + (g->dim == 3 ? 4 : 2);
    g->mortars.assign(mortars, mortars + (size_t)mcols * M);
    const size_t q2 = (size_t)g->nq * g->nq;
    g->IL.assign(IL, IL + q2);
    g->IU.assign(IU, IU + q2);
    g->PL.assign(PL, PL + q2);
    g->PU.assign(PU, PU + q2);
    g->ncface.assign((size_t)g->nfaces * g->E, 0);
    for (int64_t m = 0; m < M; ++m) {
        const int64_t* col = &g->mortars[(size_t)mcols * m];
        g->ncface[(size_t)g->nfaces * col[0] + col[1]] = 1;
        for (int k = 2; k < mcols; ++k) g->ncface[(size_t)g->nfaces * col[k] + (col[1] ^ 1)] = 1;
    }
}

extern "C" void og_grid_set_curved_mortars(og_grid* g, int curved) { g->curved_mortars = curved != 0; }

extern "C" void og_grid_set_boundary_condition(og_grid* g, int tag, int kind, const double* state) {
    if (tag < 1 || tag > 8) return;
    g->bc_kind[tag] = kind;
    for (int s = 0; s < 5; ++s) g->bc_state[tag][s] = (kind == 1 && state) ? state[s] : 0.0;
}

extern "C" void og_grid_set_directions(og_grid* g, int mask) {
    const int all = (1 << g->dim) - 1;
    g->dir_mask = (mask == all) ? 0 : (mask & all);
}

// ---------------------------------------------------------------------------------
// LSRK(5,4) (src/balancelaws/odesolvers.jl:9-66, 163-189)
// ---------------------------------------------------------------------------------

static const double RKA[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                              -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
static const double RKB[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                              1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                              2277821191437.0 / 14882151754819.0};

// LSRK(14,4) (odesolvers.jl:191-239, coefficients_lsrk144): the reference's Float64
// literals (rka[1] is the integer 0)
static const double RKA144[14] = {0.0,
                                  -0.7188012108672410,
                                  -0.7785331173421570,
                                  -0.0053282796654044,
                                  -0.8552979934029281,
                                  -3.9564138245774565,
                                  -1.5780575380587385,
                                  -2.0837094552574054,
                                  -0.7483334182761610,
                                  -0.7032861106563359,
                                  0.0013917096117681,
                                  -0.0932075369637460,
                                  -0.9514200470875948,
                                  -7.1151571693922548};
static const double RKB144[14] = {0.0367762454319673, 0.3136296607553959, 0.1531848691869027,
                                  0.0030097086818182, 0.3326293790646110, 0.2440251405350864,
                                  0.3718879239592277, 0.6204126221582444, 0.1524043173028741,
                                  0.0760894927419266, 0.0077604214040978, 0.0024647284755382,
                                  0.0780348340049386, 5.5059777270269628};

struct LsrkScheme {
    int stages;
    const double* a;
    const double* b;
};
static const LsrkScheme kScheme54{5, RKA, RKB}, kScheme144{14, RKA144, RKB144};

// dostep!(q, lsrk, after_stage) (odesolvers.jl:51-61): per stage dq .*= a; rhs!(dq, q);
// q .+= b dt dq
static void lsrk_step(const og_grid* g, const og_law* law, const LsrkScheme& sc, double* q, double* dq,
                      double time, double dt) {
    const int64_t n = (int64_t)g->np * num_states(g, law) * g->E;
    for (int st = 0; st < sc.stages; ++st) {
        const double a = sc.a[st];
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) dq[i] = dq[i] * a;
        og_tendency(g, law, dq, q, time, 1, 0, g->E);
        const double c = sc.b[st] * dt;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) q[i] = q[i] + c * dq[i];
    }
}

extern "C" void og_lsrk54_step(const og_grid* g, const og_law* law, double* q, double* dq, double time,
                               double dt) {
    lsrk_step(g, law, kScheme54, q, dq, time, dt);
}

extern "C" void og_lsrk144_step(const og_grid* g, const og_law* law, double* q, double* dq, double time,
                                double dt) {
    lsrk_step(g, law, kScheme144, q, dq, time, dt);
}

extern "C" int64_t og_solve(const og_grid* g, const og_law* law, double* q, double dt, double timeend) {
    const int64_t n = (int64_t)g->np * num_states(g, law) * g->E;
    std::vector<double> dq(n, 0.0);
    double time = 0.0;
    int64_t steps = 0;
    while (true) {
        ++steps;
        bool final = false;
        if (time + dt >= timeend) {
            dt = timeend - time;
            final = true;
        }
        og_lsrk54_step(g, law, q, dq.data(), time, dt);
        time += dt;
        if (final) break;
    }
    return steps;
}

extern "C" double og_weightednorm(const og_grid* g, const double* q, int ns, double* comp) {
    // measures.jl:6-21
    const int np = g->np;
    long double tot = 0;
    for (int s = 0; s < ns; ++s) {
        long double acc = 0;
        for (int64_t e = 0; e < g->E; ++e)
            for (int n = 0; n < np; ++n) {
                double mj = g->vmet[n + (size_t)np * (g->nvmet - 1 + (size_t)g->nvmet * e)];
                double v = q[(size_t)np * ns * e + (size_t)np * s + n];
                acc += (long double)(mj * (v * v));
            }
        double ns_ = std::sqrt((double)acc);
        if (comp) comp[s] = ns_;
        tot += (long double)ns_ * ns_;
    }
    return std::sqrt((double)tot);
}

// weightednorm(dg, q, p; componentwise) for any p >= 1 (measures.jl:6-14) and p = Inf
// (measures.jl:16-21).  comp[s] = (sum MJ |q_s|^p)^(1/p), or max |q_s| for p = Inf
// (no weights, as in the reference); the return value is norm(comp, p).
extern "C" double og_weightednorm_p(const og_grid* g, const double* q, int ns, double p, double* comp) {
    const int np = g->np;
    const bool inf = std::isinf(p);
    double tot = 0.0, mx = 0.0;
    for (int s = 0; s < ns; ++s) {
        long double acc = 0;
        double m = 0.0;
        for (int64_t e = 0; e < g->E; ++e)
            for (int n = 0; n < np; ++n) {
                const double v = std::fabs(q[(size_t)np * ns * e + (size_t)np * s + n]);
                if (inf) {
                    if (std::isnan(v) || v > m) m = v;
                    continue;
                }
                const double mj = g->vmet[n + (size_t)np * (g->nvmet - 1 + (size_t)g->nvmet * e)];
                const double vp = p == 1.0 ? v : (p == 2.0 ? v * v : std::pow(v, p));
                acc += (long double)(mj * vp);
            }
        const double c = inf ? m : (p == 2.0 ? std::sqrt((double)acc) : std::pow((double)acc, 1.0 / p));
        if (comp) comp[s] = c;
        if (std::isnan(c) || c > mx) mx = c;
        tot += p == 1.0 ? c : (p == 2.0 ? c * c : std::pow(c, p));
    }
    // norm(n, p) of LinearAlgebra: maximum for Inf, the sum for 1, (sum n^p)^(1/p) else
    if (inf) return mx;
    if (p == 1.0) return tot;
    return p == 2.0 ? std::sqrt(tot) : std::pow(tot, 1.0 / p);
}

extern "C" void og_integrals(const og_grid* g, const double* q, int ns, double* out) {
    const int np = g->np;
    for (int s = 0; s < ns; ++s) {
        long double acc = 0;
        for (int64_t e = 0; e < g->E; ++e)
            for (int n = 0; n < np; ++n) {
                double mj = g->vmet[n + (size_t)np * (g->nvmet - 1 + (size_t)g->nvmet * e)];
                acc += (long double)(mj * q[(size_t)np * ns * e + (size_t)np * s + n]);
            }
        out[s] = (double)acc;
    }
}

// ---------------------------------------------------------------------------------
// Entropy measures and the relaxation Runge-Kutta step
// (src/balancelaws/measures.jl:23-33, odesolvers.jl:73-161)
// ---------------------------------------------------------------------------------

static double entropy_at(const Phys& P, const double* q) {  // euler.jl:70-77, advection.jl:20
    if (P.L.law == OG_LAW_ADVECTION) return q[0] * q[0] / 2;
    const double g = P.L.gamma, rho = q[0], p = pressure(P, q);
    const double sv = std::log(p / std::pow(rho, g));
    return -rho * sv / (g - 1);
}

extern "C" void og_entropy_sums(const og_grid* g, const og_law* law, const double* base, const double* dir,
                                double c, const double* k, double* out) {
    Phys P{g->dim, num_states(g, law), *law};
    const int np = g->np, ns = P.ns;
    long double eta = 0, prod = 0;
    for (int64_t e = 0; e < g->E; ++e)
        for (int n = 0; n < np; ++n) {
            const double mj = g->vmet[n + (size_t)np * (g->nvmet - 1 + (size_t)g->nvmet * e)];
            double q[MAXS], v[MAXS];
            for (int s = 0; s < ns; ++s) {
                const size_t i = (size_t)np * ns * e + (size_t)np * s + n;
                q[s] = dir ? base[i] + c * dir[i] : base[i];  // @. q = q0 + γ * k
            }
            eta += (long double)(mj * entropy_at(P, q));
            if (k) {
                if (P.L.law == OG_LAW_ADVECTION) v[0] = q[0];  // advection.jl:21
                else entropyvariables(P, q, v);
                double vk = v[0] * k[(size_t)np * ns * e + n];
                for (int s = 1; s < ns; ++s) vk = vk + v[s] * k[(size_t)np * ns * e + (size_t)np * s + n];
                prod += (long double)(mj * vk);
            }
        }
    out[0] = (double)eta;
    out[1] = (double)prod;
}

// rkb_full: the b coefficients of the standard Butcher form (odesolvers.jl:91-97)
static void rkb_full(const LsrkScheme& sc, double* bf) {
    const int n = sc.stages;
    bf[n - 1] = sc.b[n - 1];
    for (int i = n - 2; i >= 0; --i) bf[i] = sc.a[i + 1] * bf[i + 1] + sc.b[i];
}

// The relaxation solve r(γ) = η(q0 + γk) - η0 - γ dη = 0 with r'(γ) = v(q0 + γk).k - dη
// (odesolvers.jl:137-148).  The reference calls NLsolve's default trust-region method
// with ftol = 10 eps; for this scalar problem its steps are Newton steps, accepted when
// they reduce r^2 by more than the 1e-4 fraction of the predicted reduction.  A rejected
// step ends the solve here (the residual is at round-off), where NLsolve would retry
// shorter steps until its 1000-iteration limit.
template <class Eval>
static int relaxation_newton(Eval eval, double* gamma) {
    const double ftol = 10 * 2.220446049250313e-16;
    double gm = *gamma, F, J;
    eval(gm, &F, &J);
    int it = 0;
    if (std::fabs(F) <= ftol) return it;
    while (it < 1000) {
        ++it;
        if (!(J != 0)) break;
        const double step = -F / J;
        const double gn = gm + step;
        double Fn, Jn;
        eval(gn, &Fn, &Jn);
        if (!(Fn * Fn < F * F * (1 - 1e-4))) break;
        gm = gn;
        F = Fn;
        J = Jn;
        if (std::fabs(F) <= ftol || step == 0) break;
    }
    *gamma = gm;
    return it;
}

static int rlsrk_step(const og_grid* g, const og_law* law, const LsrkScheme& sc, double* q, double* dq,
                      double* gamma, double time, double dt) {
    const int64_t n = (int64_t)g->np * num_states(g, law) * g->E;
    std::vector<double> q0(q, q + n), k(n);
    double bf[32], sums[2];
    rkb_full(sc, bf);
    og_entropy_sums(g, law, q0.data(), nullptr, 0.0, nullptr, sums);
    const double eta0 = sums[0];
    double deta = -0.0;
    for (int st = 0; st < sc.stages; ++st) {
        const double a = sc.a[st];
        for (int64_t i = 0; i < n; ++i) dq[i] = dq[i] * a;
        og_tendency(g, law, k.data(), q, time, 0, 0, g->E);
        for (int64_t i = 0; i < n; ++i) dq[i] = dq[i] + k[i];
        og_entropy_sums(g, law, q, nullptr, 0.0, k.data(), sums);
        deta = deta + bf[st] * dt * sums[1];
        const double c = sc.b[st] * dt;
        for (int64_t i = 0; i < n; ++i) q[i] = q[i] + c * dq[i];
    }
    for (int64_t i = 0; i < n; ++i) k[i] = q[i] - q0[i];
    auto eval = [&](double gm, double* F, double* J) {
        double s2[2];
        og_entropy_sums(g, law, q0.data(), k.data(), gm, k.data(), s2);
        *F = s2[0] - eta0 - gm * deta;
        *J = s2[1] - deta;
    };
    const int its = relaxation_newton(eval, gamma);
    for (int64_t i = 0; i < n; ++i) q[i] = q0[i] + *gamma * k[i];
    return its;
}

extern "C" int og_rlsrk54_step(const og_grid* g, const og_law* law, double* q, double* dq, double* gamma,
                               double time, double dt) {
    return rlsrk_step(g, law, kScheme54, q, dq, gamma, time, dt);
}

extern "C" int og_rlsrk144_step(const og_grid* g, const og_law* law, double* q, double* dq, double* gamma,
                                double time, double dt) {
    return rlsrk_step(g, law, kScheme144, q, dq, gamma, time, dt);
}

// LSRK(rhs!, rka, rkb, rkc, q, dt, t0) and RLSRK(...) with a caller's table
// (odesolvers.jl:32-61, 73-151)
extern "C" void og_lsrk_step_coeffs(const og_grid* g, const og_law* law, double* q, double* dq, const double* rka,
                                    const double* rkb, int nstages, double time, double dt) {
    lsrk_step(g, law, LsrkScheme{nstages, rka, rkb}, q, dq, time, dt);
}

extern "C" int og_rlsrk_step_coeffs(const og_grid* g, const og_law* law, double* q, double* dq, double* gamma,
                                    const double* rka, const double* rkb, int nstages, double time, double dt) {
    return rlsrk_step(g, law, LsrkScheme{nstages, rka, rkb}, q, dq, gamma, time, dt);
}

extern "C" int64_t og_solve_rlsrk(const og_grid* g, const og_law* law, double* q, double dt, double timeend,
                                  double* gamma) {
    const int64_t n = (int64_t)g->np * num_states(g, law) * g->E;
    std::vector<double> dq(n, 0.0);
    double time = 0.0;
    int64_t steps = 0;
    while (true) {
        ++steps;
        bool final = false;
        if (time + dt >= timeend) {
            dt = timeend - time;
            final = true;
        }
        og_rlsrk54_step(g, law, q, dq.data(), gamma, time, dt);
        time += dt;
        if (final) break;
    }
    return steps;
}

// ---------------------------------------------------------------------------------
// Initial conditions (test/balancelaws/{advection,euler}/*.jl and the benchmark setups)
// ---------------------------------------------------------------------------------

static double energy(double gamma, double rho, const double* rhou, int dim, double p) {  // euler.jl:38-41
    return p / (gamma - 1) + dotv(rhou, rhou, dim) / (2 * rho);
}

extern "C" void og_initial_condition(const og_grid* g, const og_law* law, int kind, const double* prm,
                                     double t, double* q) {
    const int dim = g->dim, np = g->np, ns = num_states(g, law);
    const double pi = M_PI;
    for (int64_t e = 0; e < g->E; ++e)
        for (int n = 0; n < np; ++n) {
            double x[3] = {0, 0, 0};
            for (int d = 0; d < dim; ++d) x[d] = g->points[n + (size_t)np * (d + dim * e)];
            double v[MAXS] = {0, 0, 0, 0, 0};
            double gm = law->gamma;
            if (kind == 0) {  // advection/wave_{1,2,3}d.jl:18-21
                double sx = x[0], sa = law->adv[0];
                for (int d = 1; d < dim; ++d) { sx = sx + x[d]; sa = sa + law->adv[d]; }
                v[0] = 2 + std::sin(pi * (sx - sa * t));
            } else if (kind == 1) {  // euler/wave_{1,2,3}d.jl:18-26
                double sx = x[0], su = 1.0;
                for (int d = 1; d < dim; ++d) { sx = sx + x[d]; su = su + 1.0; }
                double rho = 2 + std::sin(pi * (sx - su * t));
                double ru[3];
                for (int d = 0; d < dim; ++d) ru[d] = rho * 1.0;
                v[0] = rho;
                for (int d = 0; d < dim; ++d) v[1 + d] = ru[d];
                v[dim + 1] = energy(gm, rho, ru, dim, 1.0);
            } else if (kind == 2 || kind == 4) {
                // euler/isentropicvortex.jl:18-34 (kind 2); z-invariant extension (kind 4)
                double beta = (kind == 2) ? 5.0 : prm[0];
                double u0x = (kind == 2) ? 1.0 : prm[1];
                double cx = (kind == 2) ? 5.0 : prm[2], cy = (kind == 2) ? 0.0 : prm[3];
                double r0 = (x[0] - cx) - u0x * t, r1 = (x[1] - cy) - 0.0 * t;
                double f = beta * std::exp(1 - (r0 * r0 + r1 * r1));
                double pi2 = pi * pi;
                double rho = std::pow(1 - ((gm - 1) * (f * f)) / ((16 * gm) * pi2), 1 / (gm - 1));
                double c = f / (2 * pi);
                double u[3] = {u0x + c * (-r1), 0.0 + c * r0, 0.0};
                double ru[3];
                for (int d = 0; d < dim; ++d) ru[d] = rho * u[d];
                double p = std::pow(rho, gm);
                v[0] = rho;
                for (int d = 0; d < dim; ++d) v[1 + d] = ru[d];
                v[dim + 1] = energy(gm, rho, ru, dim, p);
            } else if (kind == 3) {  // sin(2pi x) sin(2pi y) + Gaussian bump
                double sigma = prm[0];
                double r2 = 0;
                for (int d = 0; d < dim; ++d) r2 += (x[d] - prm[1 + d]) * (x[d] - prm[1 + d]);
                double s = 1.0;
                for (int d = 0; d < dim; ++d) s *= std::sin(2 * pi * x[d]);
                v[0] = s + std::exp(-r2 / (2 * sigma * sigma));
            } else if (kind == 5) {  // density pulse at uniform pressure
                double r2 = 0;
                for (int d = 0; d < dim; ++d) r2 += (x[d] - prm[d]) * (x[d] - prm[d]);
                double rho = 1 + 0.2 * std::exp(-r2 / 0.01);
                double ru[3] = {0, 0, 0};
                v[0] = rho;
                v[dim + 1] = energy(gm, rho, ru, dim, 1.0);
            }
            for (int s = 0; s < ns; ++s) q[(size_t)np * ns * e + (size_t)np * s + n] = v[s];
        }
}

extern "C" int og_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

extern "C" void og_set_num_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}
