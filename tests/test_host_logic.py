"""Host-side logic of the product package that needs no GPU: the solve! step loop,
the LSRK coefficients, Julia ranges and the brick generator against the oracle."""

import math
from fractions import Fraction

import numpy as np
import pytest

import oracle as O


class FakeSolver:
    """Records the dt of every dostep call; mirrors LSRK's time bookkeeping."""

    def __init__(self, dt, t0=0.0):
        self.dt, self.time, self.calls = dt, t0, []

    def dostep(self, q, nsteps=1):
        for _ in range(nsteps):
            self.calls.append(self.dt)
            self.time += self.dt


def reference_solve(timeend, dt, adjust_final=True):
    """odesolvers.jl:9-30 verbatim in Python."""
    time, dts = 0.0, []
    while True:
        final = False
        if time + dt >= timeend:
            if adjust_final:
                dt = timeend - time
            final = True
        dts.append(dt)
        time += dt
        if final:
            return dts


@pytest.mark.parametrize("timeend,dt", [(0.7, 0.017677669529663688), (5.0, 0.125), (0.05, 0.05), (1.0, 0.3),
                                         (0.7, 0.7 / 3)])
def test_solve_loop_matches_reference(rb, timeend, dt):
    s = FakeSolver(dt)
    n = rb.solve(None, timeend, s)
    want = reference_solve(timeend, dt)
    assert n == len(want) and s.calls == want


def test_solve_with_after_step_visits_every_step(rb):
    s = FakeSolver(0.1)
    seen = []
    rb.solve(None, 0.55, s, after_step=lambda k, t, q: seen.append((k, t)))
    assert [k for k, _ in seen] == list(range(1, 7))
    assert s.calls == reference_solve(0.55, 0.1)


def test_julia_range(rb):
    v = rb.jl_range(-1, 1, 6)
    assert v.tolist() == [-1.0, -0.6, -0.2, 0.2, 0.6, 1.0]
    assert rb.jl_range(0, 10, 33)[1] == float(Fraction(10, 32))


def test_lobatto_operators_match_oracle(rb):
    for nq in range(2, 9):
        r, w, D = rb.grids.lobatto_operators(nq)
        ro, wo, Do = O.lgl(nq)
        assert np.array_equal(r, ro) and np.array_equal(w, wo) and np.array_equal(D, Do)


@pytest.mark.parametrize(
    "dim,nq,K,per,lo,hi",
    [
        (2, 5, (5, 5), (1, 1), (-1, -1), (1, 1)),
        (2, 3, (6, 3), (0, 1), (0, -5), (20, 5)),
        (3, 4, (3, 2, 5), (1, 0, 1), (0, 0, 0), (1, 2, 3)),
        (3, 8, (4, 4, 4), (1, 1, 1), (0, 0, 0), (10, 10, 10)),
        (3, 2, (1, 1, 1), (1, 1, 1), (0, 0, 0), (1, 1, 1)),
        (3, 6, (9, 3, 5), (1, 1, 0), (0, 0, 0), (1, 1, 1)),
    ],
)
def test_brick_grid_matches_oracle_bit_for_bit(rb, dim, nq, K, per, lo, hi):
    cell = rb.LobattoCell(*([nq] * dim))
    cg = rb.brick(tuple(rb.jl_range(lo[d], hi[d], K[d] + 1) for d in range(dim)), tuple(bool(p) for p in per))
    g = rb.generate(rb.GridManager(cell, cg))
    og = O.Grid(dim, nq, K, lo, hi, per)
    assert np.array_equal(g.tree, og.tree_coords())
    assert np.array_equal(g.points, og.points())
    assert np.array_equal(g.volume_metrics, og.volume_metrics())
    assert np.array_equal(g.surface_metrics, og.surface_metrics())
    assert np.array_equal(g.vmapM, og.vmapM())
    assert np.array_equal(g.vmapP, og.vmapP())
    assert np.array_equal(g.boundarycodes, og.boundary())


@pytest.mark.parametrize("dim,nq,K", [(2, 5, (4, 3)), (3, 5, (3, 3, 2))])
def test_warped_grid_matches_oracle(rb, dim, nq, K):
    cell = rb.LobattoCell(*([nq] * dim))
    L = [10.0] * dim
    cg = rb.brick(tuple(rb.jl_range(0, L[d], K[d] + 1) for d in range(dim)), (True,) * dim)

    def warp(*x):
        s = 1.0
        for d in range(dim):
            s = s * np.sin(np.pi * (x[d] / L[d]))
        return [x[d] + (0.1 * L[d]) * s for d in range(dim)]

    g = rb.generate(warp, rb.GridManager(cell, cg))
    og = O.Grid(dim, nq, K, [0.0] * dim, L, [1] * dim, O.WARP_SINE, 0.1)
    assert np.array_equal(g.points, og.points())
    vm = og.volume_metrics()
    assert np.abs(g.volume_metrics - vm).max() <= 1e-13 * np.abs(vm).max()
    assert np.abs(g.surface_metrics - og.surface_metrics()).max() <= 1e-11
    assert np.array_equal(g.vmapP, og.vmapP())


def test_flux_differencing_kernel_types(rb):
    """FluxDifferencingForm takes the reference's three kernel types (dgsem.jl:163-255),
    with or without the Julia symbol colon, and rejects others as the reference does."""
    for kt in ("naive", "per_dir", ":per_dir_symmetric"):
        assert rb.FluxDifferencingForm(rb.KennedyGruberFlux(), kt).kernel_type == kt.lstrip(":")
    with pytest.raises(ValueError, match="Unknown kernel type"):
        rb.FluxDifferencingForm(rb.KennedyGruberFlux(), "per_node")
