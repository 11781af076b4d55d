// utilities.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of three utilities Raven.jl exports beside the DGSEM path:
//   * Kron * f           src/kron.jl:15-387 (tensor-product operators, muladd = fma)
//   * scatter! / gather! src/gatherscatter.jl:1-103 (+ setbuffer_kernel!,
//                        src/communication.jl:267-270)
//   * decode(facecode)   src/facecode.jl:1-140 (hanging face / edge codes)
// Only tests/ load this library (it is linked into liboracle.so).
#include <stdint.h>
#include <string.h>

#include <cmath>

// ------------------------------------------------------------------------------ decode

// decode(facecode::UInt8) (facecode.jl:1-26): out[0..3] = hangingface.
extern "C" void og_decode8(const uint8_t* codes, int64_t n, uint8_t* out) {
    for (int64_t t = 0; t < n; ++t) {
        const unsigned code = codes[t];
        const unsigned corner = code & 0x3u;
        const bool xh = ((code >> 2) & 1u) == 1u;
        const bool yh = ((code >> 3) & 1u) == 1u;
        uint8_t* o = out + 4 * t;
        o[0] = (corner == 0 && xh) ? 1 : (corner == 2 && xh) ? 2 : 0;
        o[1] = (corner == 1 && xh) ? 1 : (corner == 3 && xh) ? 2 : 0;
        o[2] = (corner == 0 && yh) ? 1 : (corner == 1 && yh) ? 2 : 0;
        o[3] = (corner == 2 && yh) ? 1 : (corner == 3 && yh) ? 2 : 0;
    }
}

// decode(facecode::UInt16) (facecode.jl:28-140): out[0..5] = hangingface,
// out[6..17] = hangingedge.
extern "C" void og_decode16(const uint16_t* codes, int64_t n, uint8_t* out) {
    for (int64_t t = 0; t < n; ++t) {
        const unsigned code = codes[t];
        const bool fh[3] = {((code >> 3) & 1u) == 1u, ((code >> 4) & 1u) == 1u, ((code >> 5) & 1u) == 1u};
        const bool eh[3] = {((code >> 6) & 1u) == 1u, ((code >> 7) & 1u) == 1u, ((code >> 8) & 1u) == 1u};
        const unsigned corner = code & 0x7u;
        const bool shift[3] = {(corner & 1u) != 0, ((corner >> 1) & 1u) != 0, ((corner >> 2) & 1u) != 0};
        uint8_t hf[6];
        // face pair d (x, y, z): the corner's bit d selects the - or + face; the other two
        // bits, in increasing order, give the quarter 1..4
        for (int d = 0; d < 3; ++d) {
            const int o1 = d == 0 ? 1 : 0, o2 = d == 2 ? 1 : 2;
            const unsigned q = ((corner >> o1) & 1u) + 2u * ((corner >> o2) & 1u) + 1u;
            const bool plus = ((corner >> d) & 1u) != 0;
            hf[2 * d] = (fh[d] && !plus) ? (uint8_t)q : 0;
            hf[2 * d + 1] = (fh[d] && plus) ? (uint8_t)q : 0;
        }
        // edges: four parallel to each axis a, ordered by the other two corner bits
        bool onface[12], onedge[12];
        for (int a = 0; a < 3; ++a) {
            const int o1 = a == 0 ? 1 : 0, o2 = a == 2 ? 1 : 2;
            for (int m = 0; m < 4; ++m) {
                const unsigned b1 = m & 1u, b2 = (m >> 1) & 1u;
                const int n12 = 4 * a + m;
                // the edge lies on face (o1, side b1) and face (o2, side b2)
                onface[n12] = hf[2 * o1 + b1] > 0 || hf[2 * o2 + b2] > 0;
                onedge[n12] = eh[a] && ((corner >> o1) & 1u) == b1 && ((corner >> o2) & 1u) == b2;
            }
        }
        uint8_t* o = out + 18 * t;
        memcpy(o, hf, 6);
        for (int n12 = 0; n12 < 12; ++n12) {
            const int a = n12 / 4;
            o[6 + n12] = onedge[n12] ? (uint8_t)((onface[n12] ? 3 : 1) + (shift[a] ? 1 : 0))
                                     : (uint8_t)(onface[n12] ? 5 : 0);
        }
    }
}

// ---------------------------------------------------------------------------- Kron * f

// Kron(args) * f with args = (X_nf, ..., X_1): X_1 acts on the fastest index.  mats[d]
// is X_{d+1} (column-major rows[d] x cols[d]), or NULL for Eye(rows[d]).  f and r are
// addressed as  f[node, comp, col] = in[node*sn + comp*sc + col*scol]  (same for out
// with tn, tc, tcol), node = l + L*(m + M*n) over the factors' column (input) or row
// (output) extents.  The arithmetic follows the method Julia dispatches to:
//   all Eye -> copy; exactly one dense factor with the others Eye (the specialised
//   kernels for that pattern) -> one fma chain over that factor's index; otherwise
//   the generic kernel over every factor, Eye entries used as 0/1 values, with the
//   factor products formed left to right in the argument order (X_nf * ... * X_1)
//   and the loops nested as in kron_B_A_kernel (m outer, l inner) and
//   kron_C_B_A_kernel (l outer, m, n inner).
template <typename T>
static void kron_apply(int nf, const T* const* mats, const int* rows, const int* cols, const T* in, int64_t sn,
                       int64_t sc, int64_t scol, T* out, int64_t tn, int64_t tc, int64_t tcol, int64_t ncol,
                       int ncomp) {
    auto X = [&](int d, int i, int l) -> T {
        if (!mats[d]) return i == l ? T(1) : T(0);
        return mats[d][i + (int64_t)rows[d] * l];
    };
    int ndense = 0, dense = -1;
    for (int d = 0; d < nf; ++d)
        if (mats[d]) {
            ++ndense;
            dense = d;
        }
    const int R0 = rows[0], R1 = nf > 1 ? rows[1] : 1, R2 = nf > 2 ? rows[2] : 1;
    const int C0 = cols[0], C1 = nf > 1 ? cols[1] : 1, C2 = nf > 2 ? cols[2] : 1;
    for (int64_t col = 0; col < ncol; ++col)
        for (int c = 0; c < ncomp; ++c)
            for (int k = 0; k < R2; ++k)
                for (int j = 0; j < R1; ++j)
                    for (int i = 0; i < R0; ++i) {
                        const int64_t onode = i + (int64_t)R0 * (j + (int64_t)R1 * k);
                        auto g = [&](int l, int m, int n) -> T {
                            const int64_t inode = l + (int64_t)C0 * (m + (int64_t)C1 * n);
                            return in[inode * sn + c * sc + col * scol];
                        };
                        T acc = T(0);
                        if (nf > 1 && ndense == 0) {
                            acc = g(i, j, k);
                        } else if (nf == 1) {
                            for (int l = 0; l < C0; ++l) acc = std::fma(X(0, i, l), g(l, j, k), acc);
                        } else if (ndense == 1) {
                            const int oi[3] = {i, j, k};
                            for (int l = 0; l < cols[dense]; ++l) {
                                int a[3] = {i, j, k};
                                a[dense] = l;
                                acc = std::fma(X(dense, oi[dense], l), g(a[0], a[1], a[2]), acc);
                            }
                        } else if (nf == 2) {
                            for (int m = 0; m < C1; ++m)
                                for (int l = 0; l < C0; ++l)
                                    acc = std::fma(X(1, j, m) * X(0, i, l), g(l, m, k), acc);
                        } else {
                            for (int l = 0; l < C0; ++l)
                                for (int m = 0; m < C1; ++m)
                                    for (int n = 0; n < C2; ++n)
                                        acc = std::fma(X(2, k, n) * X(1, j, m) * X(0, i, l), g(l, m, n), acc);
                        }
                        out[onode * tn + c * tc + col * tcol] = acc;
                    }
}

extern "C" void og_kron_apply_f64(int nf, const double* const* mats, const int* rows, const int* cols, const double* in,
                       const int64_t* in_strides, double* out, const int64_t* out_strides, int64_t ncol, int ncomp) {
    kron_apply<double>(nf, mats, rows, cols, in, in_strides[0], in_strides[1], in_strides[2], out, out_strides[0],
                       out_strides[1], out_strides[2], ncol, ncomp);
}

extern "C" void og_kron_apply_f32(int nf, const float* const* mats, const int* rows, const int* cols, const float* in,
                       const int64_t* in_strides, float* out, const int64_t* out_strides, int64_t ncol, int ncomp) {
    kron_apply<float>(nf, mats, rows, cols, in, in_strides[0], in_strides[1], in_strides[2], out, out_strides[0],
                      out_strides[1], out_strides[2], ncol, ncomp);
}

// --------------------------------------------------------------------- gather / scatter

// Element i, component c of an array described by (block, node stride, block stride,
// component stride): Raven's GridArray parent layouts are (Np, Ns, E) -> (Np, 1,
// Np*Ns, Np) and, for continuous arrays, (Ns, Nc) -> (Nc, Ns, 0, 1).
static inline int64_t off(const int64_t* L, int64_t i, int c) {
    return (i % L[0]) * L[1] + (i / L[0]) * L[2] + (int64_t)c * L[3];
}

// scatter!: dest[i] = src[dtoc[i]] for every i of dest (setbuffer_kernel!).
extern "C" void og_scatter_f64(double* dest, const int64_t* dl, const double* src, const int64_t* sl, const int64_t* dtoc,
                    int64_t n, int ncomp) {
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < ncomp; ++c) dest[off(dl, i, c)] = src[off(sl, dtoc[i] - 1, c)];
}

// gather!: dest[j] = op(...op(op(init, src[r1]), src[r2])..., src[rk]) over the rows of
// column j of the CSC matrix ctod, in stored order (gather_kernel!).  op: 0 +, 1 min,
// 2 max (Julia's min/max on floats: NaN propagates and -0.0 < 0.0).
extern "C" void og_gather_f64(double* dest, const int64_t* dl, const double* src, const int64_t* sl, const int64_t* colptr,
                   const int64_t* rowval, int64_t ncols, int ncomp, int op, double init) {
    for (int64_t j = 0; j < ncols; ++j)
        for (int c = 0; c < ncomp; ++c) {
            double v = init;
            for (int64_t p = colptr[j] - 1; p < colptr[j + 1] - 1; ++p) {
                const double x = src[off(sl, rowval[p] - 1, c)];
                if (op == 0) v = v + x;
                else if (std::isnan(v)) continue;
                else if (std::isnan(x)) v = x;
                else if (op == 1) v = (x < v || (x == v && std::signbit(x) && !std::signbit(v))) ? x : v;
                else v = (x > v || (x == v && !std::signbit(x) && std::signbit(v))) ? x : v;
            }
            dest[off(dl, j, c)] = v;
        }
}

