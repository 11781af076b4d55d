"""The curved metrics of the grid generator against the reference's own known answers
(test/grids.jl:272-425 "2D metrics", 427-600 "3D metrics"): a polynomial warp whose
Jacobian is known in closed form.  The reference tests non-cubic cells (L, M[, N] nodes);
DGSEM needs cubic cells (dgsem.jl:92), so the same maps run here with cubic cells of 8
nodes a direction (degree 7), on which the discrete metrics of these maps (degree <= 4
in each variable) are exact too.

Checks and tolerance as the reference's (`≈`, rtol sqrt(eps) in the norm of each
quantity): J = det(dx/dr), wJ = w J, dRdX = inv(dx/dr), and on each face n wsJ / w and
n sJ equal the cofactor column of the face direction, |n| = 1.
"""

import numpy as np
import pytest

RTOL = np.sqrt(np.finfo(float).eps)


def _close(a, b):
    """isapprox in the 2-norm over the trailing component axis (Julia's ≈ on SArrays)."""
    a, b = np.asarray(a), np.asarray(b)
    d = np.linalg.norm((a - b).reshape(a.shape[0], -1), axis=1)
    s = np.maximum(np.linalg.norm(a.reshape(a.shape[0], -1), axis=1), np.linalg.norm(b.reshape(b.shape[0], -1), axis=1))
    return bool(np.all(d <= RTOL * s))


def _f2(x, y):  # test/grids.jl:274-277
    return [9 * x - (1 + x) * y**2 + (x - 1) ** 2 * (1 - y**2 + y**3),
            10 * y + x * x**3 * (1 - y) + x**2 * y * (1 + y)]


def _J2(x, y, dx, level):  # test/grids.jl:278-286
    s = [d / 2 ** (level + 1) for d in dx]
    f11 = 7 + y**2 - 2 * y**3 + 2 * x * (1 - y**2 + y**3)
    f12 = -2 * (1 + x) * y + (-1 + x) ** 2 * y * (-2 + 3 * y)
    f21 = -4 * x**3 * (-1 + y) + 2 * x * y * (1 + y)
    f22 = 10 - x * x**3 + x**2 * (1 + 2 * y)
    return np.stack([np.stack([f11 * s[0], f12 * s[1]], -1), np.stack([f21 * s[0], f22 * s[1]], -1)], -2)


def _f3(x, y, z):  # test/grids.jl:429-433
    return [3 * x + y / 5 + z / 10 + x * y**2 * z**3 / 3, 4 * y + x**3 * y**2 * z / 4, 2 * z + x**2 * y * z**3 / 2]


def _J3(x, y, z, dx, level):  # test/grids.jl:434-448
    s = [d / 2 ** (level + 1) for d in dx]
    rows = [[3 + y**2 * z**3 / 3, 1 / 5 + 2 * x * y * z**3 / 3, 1 / 10 + 3 * x * y**2 * z**2 / 3],
            [3 * x**2 * y**2 * z / 4, 4 + 2 * x**3 * y * z / 4, x**3 * y**2 / 4],
            [2 * x * y * z**3 / 2, x**2 * z**3 / 2, 2 + 3 * x**2 * y * z**2 / 2]]
    return np.stack([np.stack([np.broadcast_to(r[c] * s[c], x.shape) for c in range(3)], -1) for r in rows], -2)


def _check(g, ug, Jf, dim):
    nq, E = g.nq, g.E
    X = [ug.points[:, d, :] for d in range(dim)]
    uJ = Jf(*X)  # (Np, E, dim, dim)
    det = np.linalg.det(uJ)
    w = g.cell.w
    idx = np.indices((nq,) * dim).reshape(dim, -1, order="F")
    W = w[idx[0]]
    for d in range(1, dim):
        W = W * w[idx[d]]
    m = g.volume_metrics
    J = m[:, dim * dim, :]
    assert _close(J.reshape(-1, 1), det.reshape(-1, 1))
    assert _close(m[:, dim * dim + 1, :].reshape(-1, 1), (W[:, None] * det).reshape(-1, 1))
    inv = np.linalg.inv(uJ)
    got = np.stack([np.stack([m[:, a + dim * b, :] for b in range(dim)], -1) for a in range(dim)], -2)
    assert _close(got.reshape(-1, dim * dim), inv.reshape(-1, dim * dim))
    cof = det[..., None, None] * inv  # b = det(uJ) inv(uJ)
    s = g.surface_metrics  # (dim+2, nf*nfp, E): n, sJ, wsJ
    nfp = nq ** (dim - 1)
    from raven_b200.grids import face_node

    for f in range(2 * dim):
        d, side = f // 2, f % 2
        rows = slice(f * nfp, (f + 1) * nfp)
        nodes = np.array([face_node(dim, nq, f, j) for j in range(nfp)])
        want = (1 if side else -1) * cof[nodes][..., d, :]  # (nfp, E, dim)
        n = np.moveaxis(s[:dim, rows, :], 0, -1)  # (nfp, E, dim)
        j = np.arange(nfp)
        wf = w[j] if dim == 2 else w[j % nq] * w[j // nq]
        a = n * s[dim + 1, rows, :][..., None] / wf[:, None, None]
        assert _close(a.reshape(-1, dim), want.reshape(-1, dim)), f
        a = n * s[dim, rows, :][..., None]
        assert _close(a.reshape(-1, dim), want.reshape(-1, dim)), f
        assert np.allclose(np.linalg.norm(n, axis=-1), 1, rtol=RTOL, atol=0)


def test_2d_metrics_known_answers(rb):
    """test/grids.jl:272-425: a 5 x 4 brick on [-1, 1]^2 refined twice, warped by f."""
    coords = (rb.jl_range(-1.0, 1.0, 6), rb.jl_range(-1.0, 1.0, 5))
    level = 2
    gm = rb.GridManager(rb.LobattoCell(8, 8), rb.brick(coords), min_level=level)
    ug = rb.generate(gm)
    g = rb.generate(lambda x, y: _f2(x, y), gm)
    dx = [c[1] - c[0] for c in coords]
    _check(g, ug, lambda x, y: _J2(x, y, dx, level), 2)


def test_3d_metrics_known_answers(rb):
    """test/grids.jl:427-600: a 2 x 1 x 3 brick on [-1, 1]^3 warped by f."""
    coords = (rb.jl_range(-1.0, 1.0, 3), rb.jl_range(-1.0, 1.0, 2), rb.jl_range(-1.0, 1.0, 4))
    gm = rb.GridManager(rb.LobattoCell(8, 8, 8), rb.brick(coords), min_level=0)
    ug = rb.generate(gm)
    g = rb.generate(lambda x, y, z: _f3(x, y, z), gm)
    dx = [c[1] - c[0] for c in coords]
    _check(g, ug, lambda x, y, z: _J3(x, y, z, dx, 0), 3)
