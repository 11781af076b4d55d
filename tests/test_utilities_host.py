"""The utilities' oracle and host logic (no GPU).

* decode: the oracle reproduces every known answer of the reference's
  test/facecode.jl (tests/golden/facecode_goldens.json), exactly.
* Kron: the oracle equals the dense kron(args...) * f for the factor patterns of the
  reference's test/kron.jl, to 1e-14 (FP64) / 1e-5 (FP32) relative.
* gather/scatter: the continuous maps built from a brick's face maps join exactly the
  nodes at equal points, and the reference's gather-scatter round trip of the node
  points (test/mpitest_n3_gatherscatter.jl) holds to 10 eps.
"""

import json
import os

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def _goldens():
    with open(os.path.join(HERE, "golden", "facecode_goldens.json")) as f:
        return json.load(f)


def test_decode_oracle_pinned_to_reference_goldens():
    d = _goldens()
    assert len(d["uint8"]) == 16 and len(d["uint16"]) == 1024
    c8 = np.array([x[0] for x in d["uint8"]], dtype=np.uint8)
    v8 = np.array([x[1] for x in d["uint8"]], dtype=np.uint8)
    assert np.array_equal(O.decode(c8), v8)
    c16 = np.array([x[0] for x in d["uint16"]], dtype=np.uint16)
    v16 = np.array([x[1] + x[2] for x in d["uint16"]], dtype=np.uint8)
    assert np.array_equal(O.decode(c16), v16)


def _eye(n):
    return ("eye", n)


def _mats(args, dt):
    """args in Julia order (X_n, ..., X_1) -> oracle mats (X_1 first) and dense kron."""
    facs = list(reversed(args))
    mats = [None if isinstance(a, tuple) else a.astype(dt) for a in facs]
    sizes = [a[1] if isinstance(a, tuple) else a.shape[0] for a in facs]
    K = np.ones((1, 1))
    for a in args:
        K = np.kron(K, np.eye(a[1]) if isinstance(a, tuple) else a.astype(np.float64))
    return mats, sizes, K


def kron_cases(rng):
    a, b, c = rng.random((3, 2)), rng.random((4, 5)), rng.random((1, 7))
    A, B, C = rng.random((5, 2)), rng.random((2, 3)), rng.random((3, 5))
    return [
        (a,), (a, _eye(5)), (_eye(2), b), (a, b), (_eye(3), _eye(2), c), (_eye(2), b, _eye(7)),
        (a, _eye(4), _eye(7)), (a, b, c),  # test/kron.jl kron_testsuite
        (_eye(3), A), (B, _eye(2)), (B, A),  # kron2dgridarray_testsuite
        (_eye(5), _eye(3), A), (_eye(5), B, _eye(2)), (C, _eye(3), _eye(2)), (_eye(5), B, A),
        (C, _eye(3), A), (C, B, _eye(2)), (C, B, A),  # kron3dgridarray_testsuite
        (_eye(3), _eye(2)),
    ]


@pytest.mark.parametrize("dt,tol", [(np.float64, 1e-14), (np.float32, 1e-5)])
def test_kron_oracle_matches_dense(dt, tol):
    rng = np.random.default_rng(37)
    for args in kron_cases(rng):
        mats, sizes, K = _mats(args, dt)
        ncol, ncomp = 12, 2
        # SVector{2} columns: f[comp, node, col]
        f = rng.random((ncol, K.shape[1], ncomp)).astype(dt)
        out = O.kron_apply(mats, sizes, f.ravel(), ncomp=ncomp, in_strides=(ncomp, 1, ncomp * K.shape[1]),
                           out_strides=(ncomp, 1, ncomp * K.shape[0]), ncol=ncol)
        got = out.reshape(ncol, K.shape[0], ncomp)
        ref = np.einsum("ij,cjs->cis", K, f.astype(np.float64))
        assert np.abs(got - ref).max() <= tol * max(1.0, np.abs(ref).max()), args


def _brick(rb, dim, nq, K, per):
    coords = tuple(rb.jl_range(0.0, float(k), k + 1) for k in K)
    return rb.generate(rb.GridManager(rb.LobattoCell(*(nq,) * dim), rb.brick(coords, per)))


@pytest.mark.parametrize("dim,nq,K,per", [(2, 3, (3, 2), (False, False)), (2, 4, (3, 3), (True, False)),
                                         (3, 3, (2, 2, 3), (False, False, False)),
                                         (3, 4, (2, 3, 2), (True, True, False))])
def test_continuous_maps_join_equal_points(rb, dim, nq, K, per):
    from raven_b200.utilities import continuous_maps

    grid = _brick(rb, dim, nq, K, per)
    dtoc, colptr, rowval = continuous_maps(grid)
    n = grid.np * grid.E
    nc = colptr.size - 1
    # continuous node count of a (partly periodic) brick of degree nq-1
    expect = 1
    for d in range(dim):
        expect *= K[d] * (nq - 1) + (0 if per[d] else 1)
    assert nc == expect
    assert dtoc.shape == (grid.np, grid.E) and dtoc.min() == 1 and dtoc.max() == nc
    assert np.array_equal(np.sort(rowval), np.arange(1, n + 1))
    pts = np.stack([grid.points[:, d, :].ravel(order="F") for d in range(dim)], axis=1)
    for j in range(nc):
        rows = rowval[colptr[j] - 1:colptr[j + 1] - 1] - 1
        assert np.all(np.diff(rows) > 0)
        assert np.all(dtoc.ravel(order="F")[rows] == j + 1)
        if not any(per):
            assert np.all(pts[rows] == pts[rows[0]])


def test_gather_scatter_points_round_trip(rb):
    """gatherscatterpoints of test/mpitest_n3_gatherscatter.jl on the oracle."""
    from raven_b200.utilities import continuous_maps

    grid = _brick(rb, 2, 4, (3, 2), (False, False))  # LobattoCell(3, 4) in the reference
    dtoc, colptr, rowval = continuous_maps(grid)
    n, nc, dim = grid.np * grid.E, colptr.size - 1, grid.dim
    x = np.asfortranarray(grid.points)  # (Np, dim, E): a GridArray of SVector{dim}
    dl = (grid.np, 1, grid.np * dim, grid.np)
    cl = (nc, dim, 0, 1)
    ones = np.ones(n)
    degree = O.gather(np.zeros(nc), (nc, 1, 0, 1), ones, (grid.np, 1, grid.np, grid.np), colptr, rowval, 1)
    ca = O.gather(np.zeros(nc * dim), cl, x.ravel(order="F"), dl, colptr, rowval, dim)
    ca = ca.reshape(nc, dim) / degree[:, None]
    back = O.scatter(np.zeros(n * dim), dl, ca.ravel(), cl, dtoc.ravel(order="F"), dim)
    back = back.reshape((grid.np, dim, grid.E), order="F")
    assert np.abs(back - x).max() < 10 * np.finfo(float).eps * np.abs(x).max()
    assert degree.min() == 1 and degree.max() == 4
