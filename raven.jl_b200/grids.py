"""Host-side grid generation mirroring Raven.jl's brick path (run once, outside the hot path).

Produces exactly the arrays a Raven ``Grid`` holds for a brick: the p4est brick element
order, LGL node points, first-order volume metrics, surface metrics, ``vmapM``/``vmapP``
and boundary codes, in Raven's GridArray parent layouts (column-major numpy arrays).

Reference behaviour restated (Raven.jl 0.2.4-pre):
  * LGL operators            src/lobattocells.jl:1-47 (OneDimensionalNodes at 256 bits)
  * brick tree order         src/coarsegrids.jl:294-305 (p4est_connectivity_new_brick)
  * brick points             src/lobattocells.jl:1590-1674, 801-872
  * brick / curved metrics   src/lobattocells.jl:3182-3251, 2815-2860, 3038-3180, 2756-2813
  * surface metrics          src/lobattocells.jl:3253-3295, 2862-2900
  * face maps                src/lobattocells.jl:1992-2295 (conforming, aligned bricks)
"""

from decimal import Decimal, getcontext
from fractions import Fraction
import math

import numpy as np

# ---------------------------------------------------------------------------- 1-D operators


def _legendre(n, x):
    p0, p1 = Decimal(1), x
    if n == 0:
        return Decimal(1), Decimal(0)
    for k in range(2, n + 1):
        p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
    if abs(x) == 1:  # P_n'(+-1) is not needed by the callers
        return p1, None
    dp = n * (p0 - x * p1) / (1 - x * x)
    return p1, dp


def _lgl_decimal(nq):
    """LGL points of nq nodes in 80-digit decimal arithmetic."""
    getcontext().prec = 80
    N = nq - 1
    x = [Decimal(-1)] + [None] * (N - 1) + [Decimal(1)]
    for j in range(1, N):
        xj = Decimal(-math.cos(math.pi * j / N))
        for _ in range(200):
            P, dP = _legendre(N, xj)
            d2P = (2 * xj * dP - N * (N + 1) * P) / (1 - xj * xj)
            dx = dP / d2P
            xj -= dx
            if abs(dx) < Decimal("1e-75"):
                break
        x[j] = xj
    for j in range(nq // 2):
        s = (x[N - j] - x[j]) / 2
        x[j], x[N - j] = -s, s
    if nq % 2 == 1:
        x[N // 2] = Decimal(0)
    return x


def lobatto_operators(nq):
    """LGL points, weights and derivative matrix D[i, j] = l_j'(r_i) for nq points.

    Computed with 80-digit decimal arithmetic and rounded once to double, as Raven does
    with BigFloat (src/lobattocells.jl:1-47)."""
    x = _lgl_decimal(nq)
    N = nq - 1
    w = []
    for j in range(nq):
        P, _ = _legendre(N, x[j])
        w.append(Decimal(2) / (N * (N + 1) * P * P))
    lam = []
    for j in range(nq):
        p = Decimal(1)
        for k in range(nq):
            if k != j:
                p *= x[j] - x[k]
        lam.append(1 / p)
    D = np.zeros((nq, nq))
    for i in range(nq):
        for j in range(nq):
            if i != j:
                D[i, j] = float((lam[j] / lam[i]) / (x[i] - x[j]))
    # exact diagonal: -N(N+1)/4 and N(N+1)/4 at the end points, 0 inside (the
    # high-precision row sums leave only sub-1e-30 residuals of these values)
    D[0, 0] = -N * (N + 1) / 4
    D[N, N] = N * (N + 1) / 4
    return np.array([float(v) for v in x]), np.array([float(v) for v in w]), D


def tohalves_operators(nq):
    """Interpolation from the LGL nodes of [-1, 1] to those of the lower and upper halves
    (tohalves of lobattooperators_1d, src/lobattocells.jl:16-17, 30), I[i, j] =
    l_j((r_i -+ 1) / 2), and the matching lumped L2 projections back,
    P[j, i] = I[i, j] w_i / (2 w_j).  All in 80-digit decimals, rounded once.

    Returns (I_lower, I_upper, P_lower, P_upper), each (nq, nq)."""
    x = _lgl_decimal(nq)
    N = nq - 1
    w = []
    for j in range(nq):
        P, _ = _legendre(N, x[j])
        w.append(Decimal(2) / (N * (N + 1) * P * P))

    def lagrange(j, t):
        v = Decimal(1)
        for k in range(nq):
            if k != j:
                v *= (t - x[k]) / (x[j] - x[k])
        return v

    out = []
    for shift in (-1, 1):
        Id = [[lagrange(j, (x[i] + shift) / 2) for j in range(nq)] for i in range(nq)]
        I = np.array([[float(v) for v in row] for row in Id])
        P = np.array([[float(Id[i][j] * w[i] / (2 * w[j])) for i in range(nq)] for j in range(nq)])
        out.append((I, P))
    return out[0][0], out[1][0], out[0][1], out[1][1]


def jl_range(lo, hi, length):
    """Values of Julia's ``range(lo, stop=hi, length=length)`` (correctly rounded)."""
    K = length - 1
    a, b = Fraction(lo), Fraction(hi)
    return np.array([float(a + (b - a) * i / K) for i in range(length)])


def _fma_exact(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


# ------------------------------------------------------------------------------ brick order


def brick_tree_order(K):
    """Lattice coordinates (3, E) of a brick's trees in p4est's brick numbering.

    p4est numbers the trees of an m x n (x p) brick along a Morton curve of the
    power-of-two box: dimensions are ranked by their bit counts, each level of the
    curve interleaves the bits of the dimensions still active (x lowest), and lattice
    cells outside the brick are skipped."""
    dim = len(K)
    if dim == 1:
        return np.array([np.arange(K[0]), np.zeros(K[0], int), np.zeros(K[0], int)])
    logx = [0 if k <= 1 else int(k - 1).bit_length() for k in K]
    if dim == 2:
        rankx = [0, 1] if logx[0] <= logx[1] else [1, 0]
    else:
        if logx[0] <= logx[1]:
            if logx[1] <= logx[2]:
                rankx = [0, 1, 2]
            elif logx[0] <= logx[2]:
                rankx = [0, 2, 1]
            else:
                rankx = [2, 0, 1]
        else:
            if logx[0] <= logx[2]:
                rankx = [1, 0, 2]
            elif logx[1] <= logx[2]:
                rankx = [1, 2, 0]
            else:
                rankx = [2, 1, 0]
    n_iter = 1 << sum(logx)
    ti = np.arange(n_iter, dtype=np.int64)
    tx = np.zeros((3, n_iter), dtype=np.int64)
    last = 0
    for i in range(dim - 1):
        logi = logx[rankx[i]] - last
        active = sorted(rankx[i:])
        na = dim - i
        for j in range(logi):
            for c, k in enumerate(active):
                tx[k] |= ((ti >> (na * j + c)) & 1) << (last + j)
        last += logi
        ti = ti >> (na * logi)
    tx[rankx[dim - 1]] += ti << last
    inside = np.all([tx[d] < K[d] for d in range(dim)], axis=0)
    return tx[:, inside]


# ---------------------------------------------------------------------------------- the grid


def face_node(dim, nq, f, j):
    """0-based volume node of face f at in-face index j (lobattocells.jl:2012-2053)."""
    d, c = f // 2, (nq - 1 if f % 2 else 0)
    if dim == 1:
        return c
    if dim == 2:
        return c + nq * j if d == 0 else j + nq * c
    j1, j2 = j % nq, j // nq
    if d == 0:
        return c + nq * (j1 + nq * j2)
    if d == 1:
        return j1 + nq * (c + nq * j2)
    return j1 + nq * (j2 + nq * c)


class Grid:
    """A generated brick grid (Raven's ``Grid`` for one rank, host arrays).

    Attributes (Raven parent layouts, column-major):
      points          (Np, dim, E)
      volume_metrics  (Np, dim*dim+2, E): dRdX (col-major), J, wJ
      surface_metrics (dim+2, 2*dim*Nfp, E): n, sJ, wsJ
      vmapM, vmapP    (2*dim*Nfp, E) int64, 1-based
      boundarycodes   (2*dim, E) int64
    """

    def __init__(self, cell, coarse, warp=None, level=0):
        self.cell = cell
        dim, nq = cell.dim, cell.nq
        if dim == 1:
            self._init_line(cell, coarse, warp, level)
            return
        self.dim, self.nq = dim, nq
        self.np = nq**dim
        self.nfp = nq ** (dim - 1)
        self.nfaces = 2 * dim
        coords = coarse.coordinates
        K = [len(c) - 1 for c in coords]
        periodic = list(coarse.periodic)
        tree = brick_tree_order(K)
        self.tree = tree
        E = tree.shape[1]
        self.E = E
        r, w = cell.r, cell.w
        # --- points: x = muladd(dx, muladd(1/2, r+1, 0), c1), evaluated exactly once per
        # (tree coordinate, node index) pair and broadcast
        pts = np.zeros((self.np, dim, E), order="F")
        idx = np.indices((nq,) * dim).reshape(dim, -1, order="F")  # idx[d, n]
        for d in range(dim):
            c = np.asarray(coords[d], dtype=np.float64)
            table = np.zeros((K[d], nq))
            for t in range(K[d]):
                dx = c[t + 1] - c[t]
                for i in range(nq):
                    table[t, i] = _fma_exact(dx, 0.5 * (r[i] + 1), c[t])
            pts[:, d, :] = table[tree[d][None, :], idx[d][:, None]]
        if warp is not None:
            xs = [pts[:, d, :] for d in range(dim)]
            out = warp(*xs)
            for d in range(dim):
                pts[:, d, :] = out[d]
        self.points = pts
        self.isunwarpedbrick = warp is None
        self.volume_metrics = (self._brick_metrics() if warp is None else self._curved_metrics())
        self._face_maps(K, periodic)
        self._surface_metrics()

    def _init_line(self, cell, coarse, warp, level):
        """A 1-D brick refined uniformly to `level` (gridmanager.jl:918-1000, 1-D
        connectivity; points by linebrickpoints!, lobattocells.jl:695-755): trees in
        order, 2^level quadrants each; boundary code 1 on the x- end and 2 on the x+ end
        of a non-periodic line."""
        if warp is not None:
            raise NotImplementedError("warped 1-D grids are not generated")
        nq = cell.nq
        self.dim, self.nq, self.np, self.nfp, self.nfaces = 1, nq, nq, 1, 2
        c = np.asarray(coarse.coordinates[0], dtype=np.float64)
        per = bool(coarse.periodic[0])
        T = len(c) - 1
        nq_t = 1 << int(level)
        self.E = E = T * nq_t
        self.tree = np.array([np.arange(E) // nq_t, np.zeros(E, int), np.zeros(E, int)])
        r = cell.r
        h = 1.0 / (1 << (int(level) + 1))
        pts = np.zeros((nq, 1, E), order="F")
        for e in range(E):
            t, qq = divmod(e, nq_t)
            cr = qq / nq_t  # ix / 2^30 with ix = qq 2^(30 - level): exact
            dx = c[t + 1] - c[t]
            for i in range(nq):
                pts[i, 0, e] = _fma_exact(dx, _fma_exact(h, r[i] + 1, cr), c[t])
        self.points = pts
        self.isunwarpedbrick = True
        self.volume_metrics = self._brick_metrics()
        fn = np.array([[0], [nq - 1]])
        e = np.arange(E)
        vmapM = (fn[:, :, None] + nq * e[None, None, :] + 1).reshape(2, E)
        vmapP = vmapM.copy()
        bc = np.zeros((2, E), dtype=np.int64)
        left, right = (e - 1) % E, (e + 1) % E
        vmapP[0, :] = nq * left + (nq - 1) + 1
        vmapP[1, :] = nq * right + 1
        if not per:
            vmapP[0, 0], vmapP[1, E - 1] = vmapM[0, 0], vmapM[1, E - 1]
            bc[0, 0], bc[1, E - 1] = 1, 2
        self.vmapM = np.asfortranarray(vmapM.astype(np.int64))
        self.vmapP = np.asfortranarray(vmapP.astype(np.int64))
        self.boundarycodes = np.asfortranarray(bc)
        self._surface_metrics()

    # ------------------------------------------------------------------ metrics
    def _brick_metrics(self):
        dim, nq, np_, E = self.dim, self.nq, self.np, self.E
        pts = self.points
        # 3-D reads the corners of element p = local workgroup index
        # (lobattocells.jl:3202-3206); 2-D reads element q itself
        Qw = max(512 // (nq * nq), 1)
        src = np.arange(E) % Qw if dim == 3 else np.arange(E)
        last = [nq - 1, nq * (nq - 1), nq * nq * (nq - 1)]
        dX = np.stack([pts[last[d], d, src] - pts[0, d, src] for d in range(dim)])
        drdx = 2.0 / dX
        J = dX[0] / 2.0
        for d in range(1, dim):
            J = J * (dX[d] / 2.0)
        idx = np.indices((nq,) * dim).reshape(dim, -1, order="F")
        W = self.cell.w[idx[0]]
        for d in range(1, dim):
            W = W * self.cell.w[idx[d]]
        m = np.zeros((np_, dim * dim + 2, E), order="F")
        for a in range(dim):
            for b in range(dim):
                m[:, a + dim * b, :] = drdx[a][None, :] if a == b else -0.0
        m[:, dim * dim, :] = J[None, :]
        m[:, dim * dim + 1, :] = W[:, None] * J[None, :]
        return m

    def _curved_metrics(self):
        dim, nq, np_, E = self.dim, self.nq, self.np, self.E
        D = self.cell.D
        X = self.points.reshape((nq,) * dim + (dim, E), order="F")  # X[i,j,(k),c,e]
        m = np.zeros((np_, dim * dim + 2, E), order="F")
        w = self.cell.w
        if dim == 2:
            xr = np.einsum("im,mjce->ijce", D, X)
            xs = np.einsum("jm,imce->ijce", D, X)
            G11 = (xr * xr).sum(2)
            G12 = (xr * xs).sum(2)
            G22 = (xs * xs).sum(2)
            det = G11 * G22 - G12 * G12
            i11, i12, i22 = G22 / det, -G12 / det, G11 / det
            R = np.zeros((nq, nq, 2, 2, E))
            for c in range(2):
                R[:, :, 0, c] = i11 * xr[:, :, c] + i12 * xs[:, :, c]
                R[:, :, 1, c] = i12 * xr[:, :, c] + i22 * xs[:, :, c]
            J = np.abs(xr[:, :, 0] * xs[:, :, 1] - xr[:, :, 1] * xs[:, :, 0])
            W = w[:, None] * w[None, :]
            for a in range(2):
                for b in range(2):
                    m[:, a + 2 * b, :] = R[:, :, a, b].reshape(np_, E, order="F")
            m[:, 4, :] = J.reshape(np_, E, order="F")
            m[:, 5, :] = (W[:, :, None] * J).reshape(np_, E, order="F")
            return m
        # 3-D: curl-invariant metric terms (Kopriva 2006, eq. 37; lobattocells.jl:3038-3180)
        xr = np.einsum("im,mjkce->ijkce", D, X)
        xs = np.einsum("jm,imkce->ijkce", D, X)
        xt = np.einsum("km,ijmce->ijkce", D, X)
        cs, ct, cr = np.cross(X, xs, axis=3), np.cross(X, xt, axis=3), np.cross(X, xr, axis=3)
        a1 = np.einsum("jm,imkce->ijkce", D, ct) - np.einsum("km,ijmce->ijkce", D, cs)
        a2 = np.einsum("km,ijmce->ijkce", D, cr) - np.einsum("im,mjkce->ijkce", D, ct)
        a3 = np.einsum("im,mjkce->ijkce", D, cs) - np.einsum("jm,imkce->ijkce", D, cr)
        detJ = (xr * np.cross(xs, xt, axis=3)).sum(3)
        for b in range(3):
            m[:, 0 + 3 * b, :] = (a1[:, :, :, b] / (2 * detJ)).reshape(np_, E, order="F")
            m[:, 1 + 3 * b, :] = (a2[:, :, :, b] / (2 * detJ)).reshape(np_, E, order="F")
            m[:, 2 + 3 * b, :] = (a3[:, :, :, b] / (2 * detJ)).reshape(np_, E, order="F")
        W = (w[:, None, None] * w[None, :, None]) * w[None, None, :]
        m[:, 9, :] = detJ.reshape(np_, E, order="F")
        m[:, 10, :] = (W[..., None] * detJ).reshape(np_, E, order="F")
        return m

    # --------------------------------------------------------------- face maps
    def _face_maps(self, K, periodic):
        dim, nq, np_, nfp, nf, E = self.dim, self.nq, self.np, self.nfp, self.nfaces, self.E
        tree = self.tree
        lookup = -np.ones(tuple(K), dtype=np.int64)
        lookup[tuple(tree[d] for d in range(dim))] = np.arange(E)
        fn = np.array([[face_node(dim, nq, f, j) for j in range(nfp)] for f in range(nf)])  # (nf, nfp)
        e = np.arange(E)
        vmapM = (fn[:, :, None] + np_ * e[None, None, :] + 1).reshape(nf * nfp, E)
        vmapP = vmapM.copy()
        bc = np.zeros((nf, E), dtype=np.int64)
        for f in range(nf):
            d, side = f // 2, f % 2
            nb = [tree[k].copy() for k in range(dim)]
            nb[d] = nb[d] + (1 if side else -1)
            inside = (nb[d] >= 0) & (nb[d] < K[d])
            if periodic[d]:
                nb[d] = nb[d] % K[d]
                inside[:] = True
            else:
                bc[f, ~inside] = 1
                nb[d] = np.clip(nb[d], 0, K[d] - 1)
            ne = lookup[tuple(nb)]
            opp = fn[f ^ 1]
            vp = opp[:, None] + np_ * ne[None, :] + 1
            rows = slice(f * nfp, (f + 1) * nfp)
            vmapP[rows, :] = np.where(inside[None, :], vp, vmapM[rows, :])
        self.vmapM = np.asfortranarray(vmapM.astype(np.int64))
        self.vmapP = np.asfortranarray(vmapP.astype(np.int64))
        self.boundarycodes = np.asfortranarray(bc)

    def _surface_metrics(self):
        dim, nq, np_, nfp, nf, E = self.dim, self.nq, self.np, self.nfp, self.nfaces, self.E
        m = self.volume_metrics
        w = self.cell.w
        s = np.zeros((dim + 2, nf * nfp, E), order="F")
        for f in range(nf):
            fg, side = f // 2, f % 2
            sn = 1.0 if side else -1.0
            nodes = np.array([face_node(dim, nq, f, j) for j in range(nfp)])
            J = m[nodes, dim * dim, :]
            n = np.stack([(sn * J) * m[nodes, fg + dim * d, :] for d in range(dim)])
            sJ = np.sqrt((n * n).sum(0))
            n = n / sJ
            j = np.arange(nfp)
            if dim == 1:
                wsJ = sJ  # one node a face: weight 1 (lobattocells.jl:2656)
            elif dim == 2:
                wsJ = sJ * w[j][:, None]
            else:
                wsJ = (sJ * w[j % nq][:, None]) * w[j // nq][:, None]
            rows = slice(f * nfp, (f + 1) * nfp)
            for d in range(dim):
                s[d, rows, :] = n[d]
            s[dim, rows, :] = sJ
            s[dim + 1, rows, :] = wsJ
        self.surface_metrics = s

    # ----------------------------------------------------------------- helpers
    def volume_weights(self):
        """MJ = wJ per node, (Np, E)."""
        return self.volume_metrics[:, self.dim * self.dim + 1, :]

    def min_node_distance(self):
        """Smallest distance between neighbouring nodes along each direction (grids.jl:122-145)."""
        nq, dim = self.nq, self.dim
        X = self.points.reshape((nq,) * dim + (dim, self.E), order="F")
        best = np.inf
        for d in range(dim):
            a = np.take(X, range(1, nq), axis=d)
            b = np.take(X, range(0, nq - 1), axis=d)
            best = min(best, float(np.sqrt(((a - b) ** 2).sum(axis=dim)).min()))
        return best
