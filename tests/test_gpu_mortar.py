"""Adapted grids on the GPU: the mortar kernel plus the generic stage kernel against the
oracle's mortar restatement.

Tolerances: FP64 tendency and LSRK steps 1e-12 relative (max norm per field); FP32 bulk
tendency 5e-5; conservation on the GPU (sum of MJ * dq per field, FP64) 1e-13 of
sum |MJ * dq|; the conserved integrals after 10 FP64 steps 1e-13 relative.
"""

import numpy as np
import pytest

import oracle as O
from gpu_util import rel_err
from test_forest_host import LAWS, _adapted, _oracle, _state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F(rb, cuda_ok):
    from raven_b200 import forest

    return forest


GRIDS = [(2, 4, (3, 2), (True, True), 2), (2, 6, (2, 2), (False, True), 2), (3, 4, (2, 2, 2), (True, True, True), 2),
         (3, 6, (2, 1, 2), (True, True, False), 2), (3, 8, (2, 2, 1), (True, True, True), 2)]


def _product(rb, grid, lw, precision="fp64"):
    dim = grid.dim
    adv = [1.0, 0.5, 0.25][:dim]
    if lw[1] == O.LAW_ADVECTION:
        law, form = rb.AdvectionLaw(dim, adv), rb.WeakForm()
    else:
        law = rb.EulerLaw(dim)
        form = rb.FluxDifferencingForm(rb.KennedyGruberFlux()) if lw[2] == O.FORM_FLUXDIFF else rb.WeakForm()
    dg = rb.DGSEM(law=law, grid=grid, volume_form=form, surface_numericalflux=rb.RusanovFlux(), precision=precision)
    return dg, law, O.Law(lw[1], dim, form=lw[2], volume_flux=lw[3], adv=adv)


@pytest.mark.parametrize("lw", LAWS, ids=lambda l: l[0])
@pytest.mark.parametrize("case", GRIDS, ids=lambda c: f"{c[0]}d-nq{c[1]}")
def test_mortar_tendency_fp64(rb, F, case, lw):
    dim, nq, K, per, levels = case
    grid, _ = _adapted(rb, F, dim, nq, K, per, levels)
    assert grid.mortars.size > 0
    dg, law, olaw = _product(rb, grid, lw)
    q = _state(grid, olaw, 5)
    ref = _oracle(grid).tendency(olaw, q)
    qg, dqg = rb.GridArray.from_numpy(q), rb.GridArray.from_numpy(np.zeros_like(q))
    dg(dqg, qg, 0.0, increment=False)
    dg.sync_status()
    got = dqg.numpy()
    for s in range(olaw.ns):
        assert rel_err(got[:, s], ref[:, s]) <= 1e-12, s
    if per == (True,) * dim:  # periodic: the tendency conserves every field
        MJ = grid.volume_weights()
        for s in range(olaw.ns):
            assert abs((MJ * got[:, s]).sum()) <= 1e-13 * np.abs(MJ * got[:, s]).sum()


@pytest.mark.parametrize("case", GRIDS[2:], ids=lambda c: f"{c[0]}d-nq{c[1]}")
def test_mortar_steps_fp64(rb, F, case):
    dim, nq, K, per, levels = case
    grid, _ = _adapted(rb, F, dim, nq, K, (True,) * dim, levels)
    dg, law, olaw = _product(rb, grid, LAWS[0])
    q0 = _state(grid, olaw, 6)
    dt, steps = 2e-3, 10
    og = _oracle(grid)
    qo, dqo = np.asfortranarray(q0.copy()), og.state(olaw)
    for i in range(steps):
        og.lsrk54_step(olaw, qo, dqo, i * dt, dt)
    qg = rb.GridArray.from_numpy(q0)
    dqg = qg.similar()
    dg.lsrk54_steps(qg, dqg, 0.0, dt, steps)  # more than 4 steps: replayed from a CUDA graph
    dg.sync_status()
    got = qg.numpy()
    for s in range(olaw.ns):
        assert rel_err(got[:, s], qo[:, s]) <= 1e-12, s
    I0, I1 = rb.integrals(dg, rb.GridArray.from_numpy(q0)), rb.integrals(dg, qg)
    for a, b in zip(I0, I1):
        assert abs(a - b) <= 1e-13 * max(abs(a), 1.0)


@pytest.mark.parametrize("case", [GRIDS[0], GRIDS[2]], ids=lambda c: f"{c[0]}d-nq{c[1]}")
def test_mortar_tendency_fp32_bulk(rb, F, case):
    dim, nq, K, per, levels = case
    grid, _ = _adapted(rb, F, dim, nq, K, per, levels)
    dg, law, olaw = _product(rb, grid, LAWS[0], precision="fp32_bulk")
    q = _state(grid, olaw, 7)
    ref = _oracle(grid).tendency(olaw, q)
    qg, dqg = rb.GridArray.from_numpy(q), rb.GridArray.from_numpy(np.zeros_like(q))
    dg(dqg, qg, 0.0, increment=False)
    got = dqg.numpy()
    for s in range(olaw.ns):
        assert rel_err(got[:, s], ref[:, s]) <= 5e-5, s


@pytest.mark.parametrize("lw", LAWS, ids=lambda l: l[0])
@pytest.mark.parametrize("case", [GRIDS[0], GRIDS[2], GRIDS[4]], ids=lambda c: f"{c[0]}d-nq{c[1]}")
def test_warped_mortar_tendency_and_steps(rb, F, case, lw):
    """Warped adapted grids (curved mortars): tendency 1e-12 and conservation on the GPU,
    FP64 steps 1e-12, FP32-bulk tendency 5e-5."""
    from test_forest_host import periodic_warp

    dim, nq, K, per, levels = case
    grid, _ = _adapted(rb, F, dim, nq, K, (True,) * dim, levels, warp=periodic_warp(K, 0.05))
    assert grid.mortars.size > 0 and not grid.isunwarpedbrick
    dg, law, olaw = _product(rb, grid, lw)
    og = _oracle(grid)
    q = _state(grid, olaw, 8)
    ref = og.tendency(olaw, q)
    qg, dqg = rb.GridArray.from_numpy(q), rb.GridArray.from_numpy(np.zeros_like(q))
    dg(dqg, qg, 0.0, increment=False)
    dg.sync_status()
    got = dqg.numpy()
    MJ = grid.volume_weights()
    for s in range(olaw.ns):
        assert rel_err(got[:, s], ref[:, s]) <= 1e-12, s
        assert abs((MJ * got[:, s]).sum()) <= 1e-13 * np.abs(MJ * got[:, s]).sum()
    dt, steps = 1e-3, 6
    qo, dqo = np.asfortranarray(q.copy()), og.state(olaw)
    for i in range(steps):
        og.lsrk54_step(olaw, qo, dqo, i * dt, dt)
    qs = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, qs, dt).dostep(qs, steps)
    dg.sync_status()
    for s in range(olaw.ns):
        assert rel_err(qs.numpy()[:, s], qo[:, s]) <= 1e-12, s
    dg32, _, _ = _product(rb, grid, lw, precision="fp32_bulk")
    d32 = rb.GridArray.from_numpy(np.zeros_like(q))
    dg32(d32, rb.GridArray.from_numpy(q), 0.0, increment=False)
    for s in range(olaw.ns):
        assert rel_err(d32.numpy()[:, s], ref[:, s]) <= 5e-5, s


def test_mortar_setup_errors(rb, F):
    grid, _ = _adapted(rb, F, 2, 4, (3, 2), (True, True), 2)
    bad = grid.mortars.copy()
    bad[1, 0] = bad[1, 0] ^ 1  # a face that is connected in the face maps
    grid.mortars = bad
    with pytest.raises(rb.RB200Error) as ei:
        _product(rb, grid, LAWS[0])
    assert ei.value.status in (1, 2)
