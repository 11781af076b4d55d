"""Edge cases of the grid against the oracle: the fewest elements (one element whose
faces all meet itself on a periodic grid), the lowest order (Nq = 2), grids that are one
element thick, anisotropic elements, grids with every face on the boundary, fewer
elements than the pipelined kernels' CTAs, and zero steps.

Tolerances: FP64 tendency 1e-12 and LSRK steps 1e-12 relative per field (max norm),
as the other parity tests; zero steps leave the state bit for bit.
"""

import numpy as np
import pytest

import oracle as O
from gpu_util import initial_state, oracle_law, product_scheme, rel_err, wrap_oracle_grid

pytestmark = pytest.mark.gpu


def _build(rb, dim, nq, K, per, scheme, hi=None, warp=O.WARP_NONE):
    lo = [0.0] * dim
    hi = hi or [10.0] * dim
    og = O.Grid(dim, nq, K, lo, hi, per, warp, 0.1 if warp == O.WARP_SINE else 0.0)
    g = wrap_oracle_grid(og)
    adv = [1.0, 0.5, 0.25][:dim]
    law, form = product_scheme(rb, scheme, dim, adv)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux())
    return og, dg, oracle_law(scheme, dim, adv), law


def _tendency_and_steps(rb, og, dg, olaw, law, scheme, steps=3):
    q = initial_state(og, olaw, scheme, seed=31, amp=0.01)
    ref = og.tendency(olaw, q)
    qg = rb.GridArray.from_numpy(q)
    dqg = rb.GridArray.from_numpy(np.zeros_like(q))
    dg(dqg, qg, 0.0, increment=False)
    dg.sync_status()
    got = dqg.numpy()
    for s in range(law.ns):
        assert rel_err(got[:, s], ref[:, s]) <= 1e-12, ("tendency", s)
    dt = 1e-3
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(steps):
        og.lsrk54_step(olaw, qo, dqo, i * dt, dt)
    rb.LSRK54(dg, qg, dt).dostep(qg, steps)
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(qg.numpy()[:, s], qo[:, s]) <= 1e-12, ("steps", s)


@pytest.mark.parametrize("nq", range(2, 9))
@pytest.mark.parametrize("dim", [2, 3])
def test_single_periodic_element(rb, cuda_ok, dim, nq):
    """One element whose every face meets itself (the reference's 1-element goldens)."""
    scheme = "eul_kg"
    og, dg, olaw, law = _build(rb, dim, nq, (1,) * dim, (1,) * dim, scheme)
    _tendency_and_steps(rb, og, dg, olaw, law, scheme)


@pytest.mark.parametrize("scheme", ["eul_weak", "eul_kg", "adv_weak"])
@pytest.mark.parametrize("dim", [2, 3])
def test_lowest_order(rb, cuda_ok, dim, scheme):
    og, dg, olaw, law = _build(rb, dim, 2, (3,) * dim, (1,) * dim, scheme)
    _tendency_and_steps(rb, og, dg, olaw, law, scheme)


@pytest.mark.parametrize("nq", [4, 6, 8])
@pytest.mark.parametrize("K", [(5, 1, 1), (1, 4, 1), (1, 1, 3)], ids=lambda k: "x".join(map(str, k)))
def test_one_element_thick(rb, cuda_ok, K, nq):
    """Grids one element thick in two directions: neighbours across those faces are the
    element itself (pipelined kernels for Nq = 4, 6, 8)."""
    og, dg, olaw, law = _build(rb, 3, nq, K, (1, 1, 1), "eul_kg")
    assert dg.pipelined_ctas > 0
    _tendency_and_steps(rb, og, dg, olaw, law, "eul_kg")


@pytest.mark.parametrize("scheme", ["eul_kg", "eul_ec", "adv_weak"])
def test_anisotropic_elements(rb, cuda_ok, scheme):
    """Different element sizes per direction: the per-direction metric folded into the
    pipelined kernel's tables."""
    og, dg, olaw, law = _build(rb, 3, 8, (3, 2, 2), (1, 1, 1), scheme, hi=[10.0, 3.0, 7.0])
    _tendency_and_steps(rb, og, dg, olaw, law, scheme)


@pytest.mark.parametrize("nq", [4, 8])
@pytest.mark.parametrize("scheme", ["eul_kg", "adv_weak"])
def test_all_faces_on_the_boundary(rb, cuda_ok, scheme, nq):
    """No periodic direction: every outer face takes the default boundary state."""
    og, dg, olaw, law = _build(rb, 3, nq, (2, 2, 2), (0, 0, 0), scheme)
    _tendency_and_steps(rb, og, dg, olaw, law, scheme)


def test_fewer_elements_than_ctas(rb, cuda_ok):
    og, dg, olaw, law = _build(rb, 3, 8, (2, 1, 1), (1, 1, 1), "eul_kg")
    assert 0 < og.E < dg.pipelined_ctas
    _tendency_and_steps(rb, og, dg, olaw, law, "eul_kg", steps=5)


def test_zero_steps_leave_the_state(rb, cuda_ok):
    og, dg, olaw, law = _build(rb, 3, 8, (2, 2, 2), (1, 1, 1), "eul_kg")
    q = initial_state(og, olaw, "eul_kg", seed=32)
    qg = rb.GridArray.from_numpy(q)
    solver = rb.LSRK54(dg, qg, 1e-3)
    solver.dostep(qg, 0)
    dg.sync_status()
    assert np.array_equal(qg.numpy(), q)
    assert solver.time == 0.0
