"""Unstructured coarse grids: Raven's CoarseGrid (src/coarsegrids.jl:47-232) and the grid
generated from it.

A coarse grid is a list of vertices and a list of cells, each cell a tuple of 1-based
vertex ids in p4est's corner order (corner c = i + 2j + 4k for the tree coordinates
(i, j, k) in {0, 1}^dim).  Every cell is a tree of the forest; ``min_level`` refines
each tree uniformly.  Unlike a brick, two trees may share a face in any of the 2
(2-D) or 8 (3-D) relative orientations, and a tree's face x- may meet the other
tree's face z+: the face maps then pair nodes through that orientation, which is what
the orientation algebra of the reference computes (src/orientation.jl,
lobattocells.jl:2177-2206).

Here the pairing is derived from the vertex ids of the shared coarse face: the tree
faces whose corner vertex sets coincide are glued, and the correspondence of their
corners gives the orientation (a swap of the two face directions and a flip of
each).  Face node (U, V) of the tree face, counted over all quadrants of the face at
the refinement level, maps to (U', V') on the other tree's face with U' = U or
M - 1 - U and so on (M nodes per face direction; the Lobatto nodes are symmetric, so
a flip maps node i of quadrant q to node nq - 1 - i of quadrant 2^L - 1 - q).
"""

import numpy as np

P4EST_ROOT_LEN = 1 << 30  # P4EST_MAXLEVEL = 30 (lobattocells.jl:390-391)


class CoarseGrid:
    """CoarseGrid(vertices, cells, warp, unwarp) (src/coarsegrids.jl:47-88).

    vertices: (nv, dim) array; cells: sequence of tuples of 2^dim 1-based vertex ids;
    warp / unwarp: functions of the coordinate arrays (x, y[, z]) returning the new
    arrays (identity when None)."""

    def __init__(self, vertices, cells, warp=None, unwarp=None):
        self.vertices = np.asarray(vertices, dtype=np.float64)
        if self.vertices.ndim != 2:
            raise ValueError("vertices must be an (nv, dim) array")
        ncorner = {len(c) for c in cells}
        if len(ncorner) != 1 or ncorner.pop() not in (4, 8):
            raise ValueError("cells must all have 4 (quadrilaterals) or 8 (hexahedra) vertices")
        self.cells = np.asarray(cells, dtype=np.int64)
        self.dim = 2 if self.cells.shape[1] == 4 else 3
        if self.vertices.shape[1] != self.dim:
            raise NotImplementedError("cells embedded in a space of another dimension (manifold grids) "
                                      "are not generated")
        if self.cells.min() < 1 or self.cells.max() > len(self.vertices):
            raise ValueError("cell vertex ids must be 1-based indices into vertices")
        self.warp = warp
        self.unwarp = unwarp

    def __len__(self):
        return len(self.cells)


def coarsegrid(vertices, cells, warp=None, unwarp=None):
    """coarsegrid(vertices, cells, warp, unwarp) (src/coarsegrids.jl:86-88)."""
    return CoarseGrid(vertices, cells, warp, unwarp)


def _cubesphere_warp(x, y, z):
    """The cube-to-sphere map of cubeshellgrid (coarsegrids.jl:122-144), vectorised: on
    each point the coordinate of largest magnitude becomes the radius and the other two
    equiangular coordinates."""
    P = np.stack([x, y, z], axis=-1)
    p = np.argsort(np.abs(P), axis=-1, kind="stable")  # sortperm(abs.(point))
    S = np.take_along_axis(P, p, axis=-1)
    xi = np.pi * S[..., 1] / (4 * S[..., 2])
    eta = np.pi * S[..., 0] / (4 * S[..., 2])
    y_x = np.tan(xi)
    z_x = np.tan(eta)
    xx = S[..., 2] / np.sqrt(1.0 + y_x * y_x + z_x * z_x)
    new = np.stack([xx * z_x, xx * y_x, xx], axis=-1)  # SVector(z, y, x)
    out = np.empty_like(new)
    np.put_along_axis(out, p, new, axis=-1)  # [sortperm(p)]
    return out[..., 0], out[..., 1], out[..., 2]


def _cubesphere_unwarp(x, y, z):
    """cubesphereunwarp (coarsegrids.jl:146-165)."""
    P = np.stack([x, y, z], axis=-1)
    p = np.argsort(np.abs(P), axis=-1, kind="stable")
    S = np.take_along_axis(P, p, axis=-1)
    xi = 4 * np.arctan(S[..., 1] / S[..., 2]) / np.pi
    eta = 4 * np.arctan(S[..., 0] / S[..., 2]) / np.pi
    R = np.sign(S[..., 2]) * np.sqrt((S * S).sum(-1))
    new = np.stack([R * eta, R * xi, R], axis=-1)
    out = np.empty_like(new)
    np.put_along_axis(out, p, new, axis=-1)
    return out[..., 0], out[..., 1], out[..., 2]


def cubeshellgrid(R, r):
    """cubeshellgrid(R, r) (src/coarsegrids.jl:90-172): six hexahedral trees between the
    cubes of half-widths r < R, warped onto the spherical shell."""
    if not R > r:
        raise ValueError("R (outer radius) must be greater than r (inner radius)")
    v = []
    for s in (R, r):
        v += [(+s, +s, -s), (+s, -s, -s), (+s, +s, +s), (+s, -s, +s),
              (-s, +s, -s), (-s, -s, -s), (-s, +s, +s), (-s, -s, +s)]
    cells = [(1, 2, 3, 4, 9, 10, 11, 12), (2, 6, 4, 8, 10, 14, 12, 16), (6, 5, 8, 7, 14, 13, 16, 15),
             (5, 1, 7, 3, 13, 9, 15, 11), (3, 4, 7, 8, 11, 12, 15, 16), (1, 2, 5, 6, 9, 10, 13, 14)]
    return coarsegrid(np.array(v, dtype=np.float64), cells, _cubesphere_warp, _cubesphere_unwarp)


def _morton_coords(dim, level):
    """Quadrant coordinates (dim, 2^(dim*level)) in Morton order (x the lowest bit)."""
    n = 1 << (dim * level)
    m = np.arange(n, dtype=np.int64)
    c = np.zeros((dim, n), dtype=np.int64)
    for b in range(level):
        for d in range(dim):
            c[d] |= ((m >> (dim * b + d)) & 1) << b
    return c


def _face_corners(dim, f):
    """Tree corners of face f (x-, x+, y-, y+, z-, z+), ordered over the tangential
    directions, the lower one fastest."""
    d, s = f // 2, f % 2
    tang = [a for a in range(dim) if a != d]
    out = []
    for b in range(1 << (dim - 1)):
        bits = [0] * dim
        bits[d] = s
        for t, a in enumerate(tang):
            bits[a] = (b >> t) & 1
        out.append(sum(bits[k] << k for k in range(dim)))
    return out


def tree_face_connections(cg):
    """For every tree face, its partner (tree, face, swap, flips) or None on the boundary."""
    dim, nf = cg.dim, 2 * cg.dim
    corners = [_face_corners(dim, f) for f in range(nf)]
    faces = {}
    for t, cell in enumerate(cg.cells):
        for f in range(nf):
            ids = tuple(int(cell[c]) for c in corners[f])
            if len(set(ids)) != len(ids):
                raise ValueError(f"tree {t + 1} face {f + 1} has repeated vertices")
            faces.setdefault(tuple(sorted(ids)), []).append((t, f, ids))
    conn = [[None] * nf for _ in range(len(cg.cells))]
    for key, lst in faces.items():
        if len(lst) == 1:
            continue
        if len(lst) != 2:
            raise ValueError(f"a coarse face is shared by {len(lst)} trees")
        for (tA, fA, idsA), (tB, fB, idsB) in (lst, lst[::-1]):
            posB = {v: b for b, v in enumerate(idsB)}
            img = [posB[v] for v in idsA]  # B corner (tangential bits) of each A corner
            if dim == 2:
                fu = img[0] & 1
                if img[1] != 1 ^ fu:
                    raise ValueError("inconsistent face corners")
                conn[tA][fA] = (tB, fB, False, fu, 0)
                continue
            fu, fv = img[0] & 1, img[0] >> 1
            swap = (img[1] >> 1) != fv  # A's first direction moves B's second one
            for b in range(4):
                u, v = b & 1, b >> 1
                uB, vB = ((v ^ fu), (u ^ fv)) if swap else ((u ^ fu), (v ^ fv))
                if img[b] != uB + 2 * vB:
                    raise ValueError("inconsistent face corners")
            conn[tA][fA] = (tB, fB, swap, fu, fv)
    return conn


class UnstructuredGrid:
    """The grid generated from a CoarseGrid refined uniformly to ``level``
    (gridmanager.jl:1084-1208 with materializepoints, lobattocells.jl:305-1053):
    elements tree by tree, Morton order inside each tree.  Same attributes as Grid."""

    def __init__(self, cell, cg, level=0, warp=None):
        from .grids import Grid, face_node

        if cell.dim != cg.dim:
            raise ValueError("cell and coarse grid dimensions differ")
        dim, nq = cell.dim, cell.nq
        self.cell, self.dim, self.nq = cell, dim, nq
        self.np, self.nfp, self.nfaces = nq**dim, nq ** (dim - 1), 2 * dim
        self.level = int(level)
        T = len(cg.cells)
        nqt = 1 << (dim * self.level)
        self.E = E = T * nqt
        self.quadranttotreeid = np.repeat(np.arange(1, T + 1), nqt)
        qc = _morton_coords(dim, self.level)  # (dim, nqt)
        self.quadrantcoords = np.tile(qc, (1, T))
        self.isunwarpedbrick = False

        # ---- points: quadpoints!/hexpoints! (lobattocells.jl:305-380, 919-1010)
        r = cell.r
        h = 1.0 / (1 << (self.level + 1))
        idx = np.indices((nq,) * dim).reshape(dim, -1, order="F")  # idx[d, n]
        ref = []
        for d in range(dim):
            cr = (qc[d] * (P4EST_ROOT_LEN >> self.level)).astype(np.float64) / P4EST_ROOT_LEN
            ref.append(cr[None, :] + h * (r[idx[d]][:, None] + 1))  # (Np, nqt)
        one = 1.0
        if dim == 2:
            rr, ss = ref
            wts = [(one - rr) * (one - ss), rr * (one - ss), (one - rr) * ss, rr * ss]
        else:
            rr, ss, tt = ref
            wts = [(one - rr) * (one - ss) * (one - tt), rr * (one - ss) * (one - tt), (one - rr) * ss * (one - tt),
                   rr * ss * (one - tt), (one - rr) * (one - ss) * tt, rr * (one - ss) * tt, (one - rr) * ss * tt,
                   rr * ss * tt]
        pts = np.zeros((self.np, dim, E), order="F")
        V = cg.vertices
        for t in range(T):
            vt = V[cg.cells[t] - 1]  # (2^dim, dim)
            sl = slice(t * nqt, (t + 1) * nqt)
            for d in range(dim):
                acc = wts[0] * vt[0, d]
                for c in range(1, len(wts)):
                    acc = acc + wts[c] * vt[c, d]
                pts[:, d, sl] = acc
        # points = warp.(coarsegrid_warp.(points)) (gridmanager.jl:1159-1160)
        for wf in (cg.warp, warp):
            if wf is not None:
                out = wf(*[pts[:, d, :] for d in range(dim)])
                for d in range(dim):
                    pts[:, d, :] = out[d]
        self.points = pts
        self.volume_metrics = Grid._curved_metrics(self)
        self._face_maps(cg, qc, nqt, face_node)
        Grid._surface_metrics(self)

    def _face_maps(self, cg, qc, nqt, face_node):
        dim, nq, np_, nfp, nf, E = self.dim, self.nq, self.np, self.nfp, self.nfaces, self.E
        L = self.level
        n2 = 1 << L
        M = n2 * nq
        conn = tree_face_connections(cg)
        # Morton index of a quadrant inside its tree
        mort = np.zeros((n2,) * dim, dtype=np.int64)
        mort[tuple(qc)] = np.arange(nqt)
        fn = np.array([[face_node(dim, nq, f, j) for j in range(nfp)] for f in range(nf)])
        e = np.arange(E)
        vmapM = (fn[:, :, None] + np_ * e[None, None, :] + 1).reshape(nf * nfp, E)
        vmapP = vmapM.copy()
        bc = np.zeros((nf, E), dtype=np.int64)
        tree = e // nqt
        q = np.asarray(self.quadrantcoords)  # (dim, E)
        nid = np.indices((nq,) * dim).reshape(dim, -1, order="F")  # node index per volume node
        for f in range(nf):
            d, s = f // 2, f % 2
            tang = [a for a in range(dim) if a != d]
            edge = 0 if s == 0 else n2 - 1
            rows = slice(f * nfp, (f + 1) * nfp)
            nodes = fn[f]  # (nfp,)
            # interior of the tree: the neighbour quadrant, aligned
            inner = q[d] != edge
            if inner.any():
                qn = q[:, inner].copy()
                qn[d] += -1 if s == 0 else 1
                ne = tree[inner] * nqt + mort[tuple(qn)]
                vmapP[rows, inner] = fn[f ^ 1][:, None] + np_ * ne[None, :] + 1
            # on the tree face: through the coarse connectivity
            for ee in np.nonzero(~inner)[0]:
                c = conn[tree[ee]][f]
                if c is None:
                    bc[f, ee] = 1
                    continue
                tB, fB, swap, fu, fv = c
                dB, sB = fB // 2, fB % 2
                tangB = [a for a in range(dim) if a != dB]
                U = q[tang[0], ee] * nq + nid[tang[0], nodes]
                if dim == 3:
                    Vv = q[tang[1], ee] * nq + nid[tang[1], nodes]
                    a_ = Vv if swap else U
                    b_ = U if swap else Vv
                    Up = M - 1 - a_ if fu else a_
                    Vp = M - 1 - b_ if fv else b_
                    coords = [(Up, tangB[0]), (Vp, tangB[1])]
                else:
                    Up = M - 1 - U if fu else U
                    coords = [(Up, tangB[0])]
                qB = [None] * dim
                iB = [None] * dim
                qB[dB] = np.full(nfp, 0 if sB == 0 else n2 - 1)
                iB[dB] = np.full(nfp, 0 if sB == 0 else nq - 1)
                for W, a in coords:
                    qB[a] = W // nq
                    iB[a] = W % nq
                eB = tB * nqt + mort[tuple(qB)]
                nB = iB[0] + nq * iB[1] + (nq * nq * iB[2] if dim == 3 else 0)
                vmapP[rows, ee] = np_ * eB + nB + 1
        self.vmapM = np.asfortranarray(vmapM.astype(np.int64))
        self.vmapP = np.asfortranarray(vmapP.astype(np.int64))
        self.boundarycodes = np.asfortranarray(bc)

    def volume_weights(self):
        return self.volume_metrics[:, self.dim * self.dim + 1, :]

    def min_node_distance(self):
        from .grids import Grid

        return Grid.min_node_distance(self)
