"""Host side of the serving loop (no GPU): the per-element brick arrays a request
carries, and the seeded request stream."""

import math
from fractions import Fraction

import numpy as np
import pytest


def _fma_exact(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


@pytest.fixture(scope="module")
def S(rb):
    from raven_b200 import serving

    return serving


BRICKS = [
    # dim, nq, K, periodic
    (2, 4, (5, 3), (True, True)),
    (2, 6, (4, 4), (True, False)),
    (2, 8, (3, 7), (False, True)),
    (3, 4, (3, 2, 5), (True, True, True)),
    (3, 6, (2, 3, 2), (True, False, True)),
    (3, 8, (4, 4, 3), (True, True, False)),
    (3, 4, (6, 6, 6), (True, True, True)),  # more elements than the metric quirk's period
]


@pytest.mark.parametrize("case", BRICKS, ids=lambda c: f"{c[0]}d-nq{c[1]}-K{'x'.join(map(str, c[2]))}")
def test_brick_arrays_match_grid(rb, S, case):
    """elem_geo and the neighbour table equal what the DGSEM handle derives from the full
    Grid (its volume metrics and its vmapP), bit for bit; corners reproduce the grid's
    node points through fma(width, (r+1)/2, corner)."""
    dim, nq, K, per = case
    lo, hi = (0.0, -1.0, 2.0)[:dim], (3.0, 2.5, 7.0)[:dim]
    coords = tuple(rb.jl_range(lo[d], hi[d], K[d] + 1) for d in range(dim))
    grid = rb.generate(rb.GridManager(rb.LobattoCell(*(nq,) * dim), rb.brick(coords, per)))
    geo, nbr, corners = S.brick_arrays(dim, nq, coords, per)
    E = grid.E
    vm = grid.volume_metrics
    for d in range(dim):
        assert np.all(vm[:, d + dim * d, :] == geo[d][None, :])
    assert np.array_equal(geo[3], vm[0, dim * dim, :])
    if dim == 2:
        assert np.all(geo[2] == 0.0)
    # neighbour across face f: element of vmapP's first face node, -1 on a boundary
    nfp = grid.nfp
    for f in range(2 * dim):
        p0 = grid.vmapP[f * nfp, :] - 1
        m0 = grid.vmapM[f * nfp, :] - 1
        expect = np.where(grid.boundarycodes[f] != 0, -1, p0 // grid.np)
        expect = np.where(p0 == m0, -1, expect)
        assert np.array_equal(nbr[f], expect.astype(np.int32)), f
    r = grid.cell.r
    idx = np.indices((nq,) * dim).reshape(dim, -1, order="F")
    for d in range(dim):
        c1, dx = corners[0, d], corners[1, d]
        x = np.array([[_fma_exact(dx[e], 0.5 * (r[i] + 1), c1[e]) for e in range(E)] for i in range(nq)])
        assert np.array_equal(grid.points[:, d, :], x[idx[d], :])


def test_poisson_mix_is_seeded_and_in_range(rb, S):
    a = S.poisson_mix(7, 300)
    b = S.poisson_mix(7, 300)
    c = S.poisson_mix(8, 300)
    key = lambda arr: [(x.t, x.spec.dim, x.spec.nq, x.spec.law, x.spec.K, x.spec.nsteps) for x in arr]
    assert key(a) == key(b)
    assert key(a) != key(c)
    t = np.array([x.t for x in a])
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert 1 / 300 < gaps.mean() < 1 / 120  # rate 200/s
    for x in a:
        s = x.spec
        assert s.dim in (2, 3) and s.nq in (4, 6, 8)
        k = s.K[0]
        assert all(kk == k for kk in s.K)
        assert (8 <= k <= 64) if s.dim == 2 else (4 <= k <= 32)
        assert 50 <= s.nsteps <= 500
        assert s.precision == rb._lib.PRECISION_FP32_BULK
        assert s.dt > 0
    assert {x.spec.dim for x in a} == {2, 3}
    assert {x.spec.nq for x in a} == {4, 6, 8}
    assert {x.spec.law for x in a} == {0, 1}


def test_spec_cfl_steps(rb, S):
    """dt = 0.4 * min node distance / (bound on the wave speed)."""
    for nq in (4, 6, 8):
        r = rb.LobattoCell(nq, nq).r
        v = S.vortex_spec(3, nq, (8, 8, 8), 10)
        assert v.dt == pytest.approx(0.4 * (10 / 8) * (r[1] - r[0]) / 2 / 2.8)
        w = S.wave_spec(2, nq, (16, 16), 10)
        assert w.dt == pytest.approx(0.4 * (1 / 16) * (r[1] - r[0]) / 2 / math.hypot(1.0, 0.5))
    assert S.vortex_spec(2, 4, (4, 4), 3).dof_updates() == 16 * 4 * 16 * 3 * 5
    with pytest.raises(ValueError):
        S.vortex_spec(2, 4, (4, 4), 3, strength=6.0)
