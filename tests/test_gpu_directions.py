"""DGSEM(; directions) (dgsem.jl:46-81, 203-227, 257-348, 756-782) on the GPU against
the oracle: the volume and surface terms of a subset of the directions only.

Tolerances: FP64 tendency and LSRK steps 1e-12 relative per field (max norm); the
single-direction tendencies add up to the full one to 1e-13 of its scale.
"""

import numpy as np
import pytest

import oracle as O
from gpu_util import initial_state, oracle_law, product_scheme, rel_err, wrap_oracle_grid

pytestmark = pytest.mark.gpu

CASES = [
    # dim, nq, K, scheme, warp, directions
    (3, 8, (2, 2, 2), "eul_kg", O.WARP_NONE, (1, 2)),
    (3, 8, (2, 2, 2), "eul_kg", O.WARP_NONE, (3,)),
    (3, 5, (2, 2, 2), "eul_weak", O.WARP_NONE, (2, 3)),
    (3, 4, (2, 2, 2), "adv_weak", O.WARP_NONE, (1,)),
    (3, 6, (2, 2, 2), "eul_ec", O.WARP_NONE, (1, 3)),
    (2, 5, (3, 3), "eul_kg", O.WARP_SINE, (2,)),
    (3, 8, (2, 2, 2), "eul_kg", O.WARP_SINE, (1, 2)),
    (3, 4, (2, 2, 2), "eul_weak", O.WARP_SINE, (3,)),
]


def _build(rb, dim, nq, K, scheme, warp, directions, precision="fp64"):
    og = O.Grid(dim, nq, K, [0.0] * dim, [10.0] * dim, [True] * dim, warp, 0.1 if warp == O.WARP_SINE else 0.0)
    g = wrap_oracle_grid(og)
    adv = [1.0, 0.5, 0.25][:dim]
    law, form = product_scheme(rb, scheme, dim, adv)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux(), directions=directions,
                  precision=precision)
    return og, dg, oracle_law(scheme, dim, adv), law


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}d-nq{c[1]}-{c[3]}-warp{c[4]}-dirs{''.join(map(str, c[5]))}"
                                             for c in CASES])
def test_directions_tendency_and_steps(rb, cuda_ok, case):
    dim, nq, K, scheme, warp, dirs = case
    og, dg, olaw, law = _build(rb, *case)
    assert dg.pipelined_ctas == 0  # a subset of the directions runs the generic kernel
    og.set_directions(dirs)
    q = initial_state(og, olaw, scheme, seed=41, amp=0.01)
    ref = og.tendency(olaw, q)
    qg = rb.GridArray.from_numpy(q)
    dqg = rb.GridArray.from_numpy(np.zeros_like(q))
    dg(dqg, qg, 0.0, increment=False)
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(dqg.numpy()[:, s], ref[:, s]) <= 1e-12, s
    dt = 1e-3
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(5):
        og.lsrk54_step(olaw, qo, dqo, i * dt, dt)
    rb.LSRK54(dg, qg, dt).dostep(qg, 5)
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(qg.numpy()[:, s], qo[:, s]) <= 1e-12, s


@pytest.mark.parametrize("scheme", ["eul_kg", "adv_weak"])
def test_single_directions_add_up(rb, cuda_ok, scheme):
    """Full tendency (the pipelined kernel) = sum of the single-direction tendencies
    (the generic kernel), FP64 and FP32 bulk."""
    for precision, tol in (("fp64", 1e-13), ("fp32_bulk", 5e-6)):
        og, dg, olaw, law = _build(rb, 3, 8, (2, 2, 2), scheme, O.WARP_NONE, None, precision)
        assert dg.pipelined_ctas > 0
        q = initial_state(og, olaw, scheme, seed=42, amp=0.01)
        qg = rb.GridArray.from_numpy(q)
        full = rb.GridArray.from_numpy(np.zeros_like(q))
        dg(full, qg, 0.0, increment=False)
        parts = np.zeros_like(q)
        for d in (1, 2, 3):
            _, dgd, _, _ = _build(rb, 3, 8, (2, 2, 2), scheme, O.WARP_NONE, (d,), precision)
            dd = rb.GridArray.from_numpy(np.zeros_like(q))
            dgd(dd, qg, 0.0, increment=False)
            parts += dd.numpy()
        f = full.numpy()
        assert np.abs(parts - f).max() <= tol * np.abs(f).max(), precision


def test_directions_rejected(rb, cuda_ok):
    with pytest.raises(ValueError):
        _build(rb, 3, 4, (2, 2, 2), "eul_kg", O.WARP_NONE, (0,))
    with pytest.raises(ValueError):
        _build(rb, 2, 4, (2, 2), "eul_kg", O.WARP_NONE, (3,))
