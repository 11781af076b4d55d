"""1-D grids on the host (no GPU): the product's line grids against the oracle's, which
the reference's 1-D golden errors pin (test/balancelaws/*/wave_1d.jl).

Tolerance: bit-exact (points, metrics, face maps, boundary codes)."""

import numpy as np
import pytest

import oracle as O


@pytest.mark.parametrize("nq,K,per", [(5, 5, True), (5, 7, False), (2, 3, True), (8, 4, False), (4, 1, True)])
def test_line_grid_equals_oracle(rb, nq, K, per):
    g = rb.generate(rb.GridManager(rb.LobattoCell(nq), rb.brick((rb.jl_range(-1.0, 1.0, K + 1),), (per,))))
    og = O.Grid(1, nq, [K], [-1.0], [1.0], [per])
    assert np.array_equal(g.points, og.points())
    assert np.array_equal(g.volume_metrics, og.volume_metrics())
    assert np.array_equal(g.surface_metrics, og.surface_metrics())
    assert np.array_equal(g.vmapM, og.vmapM())
    assert np.array_equal(g.vmapP, og.vmapP())
    assert np.array_equal(g.boundarycodes, og.boundary())


@pytest.mark.parametrize("level", [1, 2, 3])
def test_line_uniform_refinement(rb, level):
    """min_level on a line (gridmanager.jl:918-1000): 2^level quadrants a tree, in order,
    tiling each tree; codes 1 and 2 on the x- and x+ ends."""
    K, nq = 3, 4
    gm = rb.GridManager(rb.LobattoCell(nq), rb.brick((rb.jl_range(0.0, 3.0, K + 1),), (False,)), min_level=level)
    g = rb.generate(gm)
    assert g.E == len(gm) == K << level
    x = g.points[:, 0, :]
    assert np.all(np.diff(x, axis=0) > 0) and np.all(x[0, 1:] == x[-1, :-1])
    assert x[0, 0] == 0.0 and x[-1, -1] == 3.0
    assert np.allclose(x[-1] - x[0], 1.0 / (1 << level), rtol=1e-15)
    assert g.boundarycodes[0, 0] == 1 and g.boundarycodes[1, -1] == 2 and g.boundarycodes.sum() == 3
    with pytest.raises(NotImplementedError):
        rb.adapt(gm, [rb.AdaptRefine] * len(gm))
