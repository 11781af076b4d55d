"""Adapted (non-conforming) brick grids: a p4est-style forest of quadtrees/octrees on a
brick, 2:1 face balance, and the mortars of its hanging faces.

Raven builds such grids with P4estTypes (GridManager with min_level, adapt!, balance!,
src/gridmanager.jl:53-175).  p4est is not available here, so this module restates the
parts the DGSEM path needs:
* the forest: leaves in tree order, Morton order inside a tree;
* refinement and coarsening by flags (AdaptRefine, AdaptNone, AdaptCoarsen);
* 2:1 balance across faces;
* the grid arrays (points, metrics, face maps), with the hanging faces of the reference
  (vmapP = vmapM on a non-conforming face, lobattocells.jl:2073-2074);
* the mortar table that couples each hanging face to its 2^(dim-1) small neighbours.

Two things differ from the reference on adapted grids:
* Brick metrics come from each element's own corner points.  The reference's brick
  metric kernel reads the corners of another element
  (hexvolumebrickmetrics!, lobattocells.jl:3202-3206).  That is harmless on a uniform
  brick but wrong when element sizes differ.
* The reference's surfaceterm! ignores non-conforming faces.  Here they are coupled
  by mortars (see raven.jl_b200/csrc/mortar.cu).
"""

from fractions import Fraction

import numpy as np

from .grids import brick_tree_order, face_node, lobatto_operators, tohalves_operators

AdaptCoarsen, AdaptNone, AdaptRefine = 0x00, 0x01, 0x10  # src/gridmanager.jl:25-27

LMAX = 20  # finest level of the integer leaf coordinates


def _morton(coords, dim):
    """Interleaved bits of integer coordinates (x lowest), LMAX bits each."""
    key = 0
    for b in range(LMAX):
        for d in range(dim):
            key |= ((coords[d] >> b) & 1) << (dim * b + d)
    return key


class Forest:
    """Leaves of a forest on a brick of K trees per direction.

    A leaf is (tree index, level, anchor); the anchor holds the integer coordinates of
    the leaf's lower corner inside its tree, in units of 2^-LMAX of a tree."""

    def __init__(self, dim, K, periodic, min_level=0):
        self.dim = dim
        self.K = tuple(int(k) for k in K)
        self.periodic = tuple(bool(p) for p in periodic)
        self.tree = brick_tree_order(self.K)  # (3, ntrees) lattice coordinates
        self.ntrees = self.tree.shape[1]
        size = 1 << (LMAX - min_level)
        self.leaves = []
        for t in range(self.ntrees):
            for idx in np.ndindex(*(1 << min_level,) * dim):
                self.leaves.append((t, min_level, tuple(i * size for i in reversed(idx))))
        self._sort()

    # ---------------------------------------------------------------- bookkeeping
    def _sort(self):
        self.leaves.sort(key=lambda L: (L[0], _morton(L[2], self.dim)))
        self._index = {(L[0], L[1], L[2]): i for i, L in enumerate(self.leaves)}

    def __len__(self):
        return len(self.leaves)

    def global_anchor(self, leaf):
        t, _, a = leaf
        return tuple(int(self.tree[d, t]) * (1 << LMAX) + a[d] for d in range(self.dim))

    def _locate(self, level, g):
        """Leaf at `level` with global anchor g (wrapped if periodic), or None."""
        gg = list(g)
        for d in range(self.dim):
            n = self.K[d] << LMAX
            if gg[d] < 0 or gg[d] >= n:
                if not self.periodic[d]:
                    return None
                gg[d] %= n
        tc = [gg[d] >> LMAX for d in range(self.dim)]
        t = self._tree_of(tc)
        a = tuple(gg[d] - (tc[d] << LMAX) for d in range(self.dim))
        return self._index.get((t, level, a))

    def _tree_of(self, tc):
        if not hasattr(self, "_treemap"):
            self._treemap = {tuple(int(self.tree[d, t]) for d in range(self.dim)): t for t in range(self.ntrees)}
        return self._treemap[tuple(tc)]

    def _outside(self, g):
        return any(not self.periodic[d] and (g[d] < 0 or g[d] >= (self.K[d] << LMAX)) for d in range(self.dim))

    def face_neighbours(self, i, f):
        """('same', j) | ('coarser', j) | ('finer', [j...]) | ('boundary', None) for face f
        (x-, x+, y-, y+, z-, z+) of leaf i.  'finer' lists the 2^(dim-1) small leaves in
        the order of their position along the face's in-face directions (first fastest).
        Unbalanced forests also give ('muchcoarser', j) (a neighbour two or more levels
        coarser) and ('deeper', None) (neighbours two or more levels finer)."""
        t, lev, a = self.leaves[i]
        size = 1 << (LMAX - lev)
        g = list(self.global_anchor(self.leaves[i]))
        d, side = f // 2, f % 2
        n = list(g)
        n[d] += size if side else -size
        if self._outside(n):
            return ("boundary", None)
        j = self._locate(lev, n)
        if j is not None:
            return ("same", j)
        for up in range(1, lev + 1):  # an ancestor-level leaf across the face
            s2 = size << up
            pn = [c - (c % s2) for c in n]
            j = self._locate(lev - up, pn)
            if j is not None:
                return ("coarser" if up == 1 else "muchcoarser", j)
        half = size // 2
        small = []
        inface = [e for e in range(self.dim) if e != d]
        for b in range(1 << (self.dim - 1)):
            c = list(n)
            if side == 0:
                c[d] += half  # the layer of small leaves next to the face
            for k, e in enumerate(inface):
                c[e] += half * ((b >> k) & 1)
            j = self._locate(lev + 1, c)
            if j is None:
                return ("deeper", None)
            small.append(j)
        return ("finer", small)

    # ------------------------------------------------------------------ adaptation
    def adapt(self, flags):
        """adapt!(gm, flags) (gridmanager.jl:160-173): coarsen complete families flagged
        AdaptCoarsen, refine leaves flagged AdaptRefine, then balance 2:1 across faces."""
        if len(flags) != len(self.leaves):
            raise ValueError("one flag per leaf")
        flags = list(flags)
        nchild = 1 << self.dim
        # coarsening: a family is 2^dim consecutive siblings, all flagged
        keep = []
        i = 0
        while i < len(self.leaves):
            t, lev, a = self.leaves[i]
            if lev > 0 and flags[i] == AdaptCoarsen and i + nchild <= len(self.leaves):
                psize = 1 << (LMAX - lev + 1)
                pa = tuple(c - (c % psize) for c in a)
                fam = self.leaves[i:i + nchild]
                if (all(L[0] == t and L[1] == lev and tuple(c - (c % psize) for c in L[2]) == pa for L in fam)
                        and all(flags[i + k] == AdaptCoarsen for k in range(nchild))):
                    keep.append(((t, lev - 1, pa), AdaptNone))
                    i += nchild
                    continue
            keep.append((self.leaves[i], flags[i]))
            i += 1
        leaves = []
        for L, fl in keep:
            if fl == AdaptRefine:
                leaves.extend(self._children(L))
            else:
                leaves.append(L)
        self.leaves = leaves
        self._sort()
        self.balance()

    def _children(self, leaf):
        t, lev, a = leaf
        half = 1 << (LMAX - lev - 1)
        out = []
        for b in range(1 << self.dim):
            out.append((t, lev + 1, tuple(a[d] + half * ((b >> d) & 1) for d in range(self.dim))))
        return out

    def balance(self):
        """2:1 balance across faces (balance! with face connectivity)."""
        while True:
            refine = set()
            for i in range(len(self.leaves)):
                for f in range(2 * self.dim):
                    kind, j = self.face_neighbours(i, f)
                    if kind == "deeper":
                        refine.add(i)
                    elif kind == "muchcoarser":
                        refine.add(j)
            if not refine:
                return
            leaves = []
            for i, L in enumerate(self.leaves):
                leaves.extend(self._children(L) if i in refine else [L])
            self.leaves = leaves
            self._sort()


# ---------------------------------------------------------------------------- the grid


def _fma_exact(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


class ForestGrid:
    """A generated adapted brick grid (Raven's Grid for one rank), host arrays.

    Same attributes as grids.Grid (points, volume_metrics, surface_metrics, vmapM,
    vmapP, boundarycodes in Raven's parent layouts), plus:
      mortars  (2 + 2^(dim-1), M) int64, 0-based: large element, its face, then the
               small elements in the order of their position on the face;
      tohalves (I_lower, I_upper, P_lower, P_upper), the mortar operators.

    With `warp` (a function of the coordinate arrays, as for Grid) the points are warped
    after they are generated and the metrics are the curved ones (gridmanager.jl:1159-1174);
    the mortars then couple the hanging faces with the small faces' own geometry."""

    def __init__(self, cell, forest, coordinates, warp=None):
        dim, nq = cell.dim, cell.nq
        self.cell, self.forest = cell, forest
        self.dim, self.nq = dim, nq
        self.np = nq**dim
        self.nfp = nq ** (dim - 1)
        self.nfaces = 2 * dim
        self.E = E = len(forest)
        self.isunwarpedbrick = warp is None
        r, w = cell.r, cell.w
        coords = [np.asarray(c, dtype=np.float64) for c in coordinates]
        # points: x = muladd(dx, muladd(h, r + 1, cr), c1) with h = 2^-(level+1) and cr the
        # leaf corner in the tree's reference coordinates (hexbrickpoints!,
        # lobattocells.jl:1590-1674)
        idx = np.indices((nq,) * dim).reshape(dim, -1, order="F")
        pts = np.zeros((self.np, dim, E), order="F")
        for e, (t, lev, a) in enumerate(forest.leaves):
            h = Fraction(1, 1 << (lev + 1))
            for d in range(dim):
                tc = int(forest.tree[d, t])
                c1 = coords[d][tc]
                dx = coords[d][tc + 1] - coords[d][tc]
                cr = Fraction(a[d], 1 << LMAX)
                line = np.array([_fma_exact(dx, float(h * Fraction(r[i] + 1) + cr), c1) for i in range(nq)])
                pts[:, d, e] = line[idx[d]]
        if warp is not None:
            out = warp(*[pts[:, d, :] for d in range(dim)])
            for d in range(dim):
                pts[:, d, :] = out[d]
        self.points = pts
        if warp is not None:
            from .grids import Grid

            self.volume_metrics = Grid._curved_metrics(self)
            self._face_maps()
            self._surface_metrics()
            self.tohalves = tohalves_operators(nq)
            return
        # brick metrics from the element's own corners
        last = [nq - 1, nq * (nq - 1), nq * nq * (nq - 1)]
        dX = np.stack([pts[last[d], d, :] - pts[0, d, :] for d in range(dim)])
        drdx = 2.0 / dX
        J = dX[0] / 2.0
        for d in range(1, dim):
            J = J * (dX[d] / 2.0)
        W = w[idx[0]]
        for d in range(1, dim):
            W = W * w[idx[d]]
        m = np.zeros((self.np, dim * dim + 2, E), order="F")
        for a_ in range(dim):
            for b in range(dim):
                m[:, a_ + dim * b, :] = drdx[a_][None, :] if a_ == b else -0.0
        m[:, dim * dim, :] = J[None, :]
        m[:, dim * dim + 1, :] = W[:, None] * J[None, :]
        self.volume_metrics = m
        self._face_maps()
        self._surface_metrics()
        self.tohalves = tohalves_operators(nq)

    def _face_maps(self):
        dim, nq, np_, nfp, nf, E = self.dim, self.nq, self.np, self.nfp, self.nfaces, self.E
        fn = np.array([[face_node(dim, nq, f, j) for j in range(nfp)] for f in range(nf)])
        vmapM = np.zeros((nf * nfp, E), dtype=np.int64)
        for e in range(E):
            for f in range(nf):
                vmapM[f * nfp:(f + 1) * nfp, e] = fn[f] + np_ * e + 1
        vmapP = vmapM.copy()
        bc = np.zeros((nf, E), dtype=np.int64)
        mortars = []
        for e in range(E):
            for f in range(nf):
                kind, nb = self.forest.face_neighbours(e, f)
                rows = slice(f * nfp, (f + 1) * nfp)
                if kind == "same":
                    vmapP[rows, e] = fn[f ^ 1] + np_ * nb + 1
                elif kind == "boundary":
                    bc[f, e] = 1
                elif kind == "finer":
                    mortars.append([e, f] + list(nb))
                # "coarser": the small side of a mortar; vmapP stays vmapM
        self.vmapM = np.asfortranarray(vmapM)
        self.vmapP = np.asfortranarray(vmapP)
        self.boundarycodes = np.asfortranarray(bc)
        ncol = 2 + (1 << (dim - 1))
        self.mortars = np.asfortranarray(np.array(mortars, dtype=np.int64).reshape(-1, ncol).T)

    def _surface_metrics(self):
        dim, nq, nfp, nf, E = self.dim, self.nq, self.nfp, self.nfaces, self.E
        m = self.volume_metrics
        w = self.cell.w
        s = np.zeros((dim + 2, nf * nfp, E), order="F")
        for f in range(nf):
            fg, side = f // 2, f % 2
            sn = 1.0 if side else -1.0
            nodes = np.array([face_node(dim, nq, f, j) for j in range(nfp)])
            Jn = m[nodes, dim * dim, :]
            n = np.stack([(sn * Jn) * m[nodes, fg + dim * d, :] for d in range(dim)])
            sJ = np.sqrt((n * n).sum(0))
            n = n / sJ
            j = np.arange(nfp)
            if dim == 2:
                wsJ = sJ * w[j][:, None]
            else:
                wsJ = (sJ * w[j % nq][:, None]) * w[j // nq][:, None]
            rows = slice(f * nfp, (f + 1) * nfp)
            for d in range(dim):
                s[d, rows, :] = n[d]
            s[dim, rows, :] = sJ
            s[dim + 1, rows, :] = wsJ
        self.surface_metrics = s

    def volume_weights(self):
        return self.volume_metrics[:, self.dim * self.dim + 1, :]

    def min_node_distance(self):
        nq, dim = self.nq, self.dim
        X = self.points.reshape((nq,) * dim + (dim, self.E), order="F")
        best = np.inf
        for d in range(dim):
            a = np.take(X, range(1, nq), axis=d)
            b = np.take(X, range(0, nq - 1), axis=d)
            best = min(best, float(np.sqrt(((a - b) ** 2).sum(axis=dim)).min()))
        return best


def sphere_refinement_flags(grid_or_forest, coordinates, center, radius):
    """AdaptRefine for the leaves whose box comes within `radius` of `center` (strictly),
    AdaptNone otherwise."""
    F = grid_or_forest if isinstance(grid_or_forest, Forest) else grid_or_forest.forest
    coords = [np.asarray(c, dtype=np.float64) for c in coordinates]
    flags = []
    for t, lev, a in F.leaves:
        d2 = 0.0
        for d in range(F.dim):
            tc = int(F.tree[d, t])
            c1, dx = coords[d][tc], coords[d][tc + 1] - coords[d][tc]
            lo = c1 + dx * a[d] / (1 << LMAX)
            hi = lo + dx / (1 << lev)
            q = min(max(center[d], lo), hi)
            d2 += (center[d] - q) ** 2
        flags.append(AdaptRefine if d2 < radius * radius else AdaptNone)
    return flags
