"""Boundary conditions on the GPU against the oracle: the exterior state of the boundary
faces per boundary tag, the reference's `boundarystate` hook (balancelaw.jl:22) as its
examples overload it - a prescribed state per tag (examples/balancelaws/euler/sod.jl:15-21)
and a reflecting wall (examples/balancelaws/euler_gravity/gravitywave.jl:16-21).

Tolerances: FP64 tendency and LSRK steps 1e-12 relative per field (max norm); mass and
energy of a closed box with reflecting walls 1e-13 relative after the steps.
"""

import numpy as np
import pytest

import oracle as O
from gpu_util import initial_state, oracle_law, product_scheme, rel_err, wrap_oracle_grid

pytestmark = pytest.mark.gpu


def _build(rb, dim, nq, K, scheme, conds, hi=None):
    og = O.Grid(dim, nq, K, [0.0] * dim, hi or [1.0] * dim, [False] * dim)
    g = wrap_oracle_grid(og)
    adv = [1.0, 0.5, 0.25][:dim]
    law, form = product_scheme(rb, scheme, dim, adv)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux(),
                  boundary_conditions=conds)
    for tag, c in conds.items():
        og.set_boundary_condition(tag, 2 if c == "wall" else 1, None if c == "wall" else c)
    return og, dg, oracle_law(scheme, dim, adv), law


def _compare(rb, og, dg, olaw, law, q, steps=5, dt=1e-3):
    ref = og.tendency(olaw, q)
    qg = rb.GridArray.from_numpy(q)
    dqg = rb.GridArray.from_numpy(np.zeros_like(q))
    dg(dqg, qg, 0.0, increment=False)
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(dqg.numpy()[:, s], ref[:, s]) <= 1e-12, ("tendency", s)
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(steps):
        og.lsrk54_step(olaw, qo, dqo, i * dt, dt)
    rb.LSRK54(dg, qg, dt).dostep(qg, steps)
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(qg.numpy()[:, s], qo[:, s]) <= 1e-12, ("steps", s)
    return qg


def test_sod_shock_tube_prescribed_states(rb, cuda_ok):
    """The reference's Sod example: a 1-D line with the left state on tag 1 and the right
    state on tag 2 (rho = 1, p = 1 | rho = 1/8, p = 1/10, at rest), Rusanov flux.  The
    jump is smoothed over a tanh of width 0.03: unlimited DG (here and in the oracle, as
    in the reference) rings on the sharp jump and loses positivity within 40 steps."""
    nq, K = 5, 32
    og = O.Grid(1, nq, [K], [0.0], [1.0], [False])
    g = wrap_oracle_grid(og)
    law = rb.EulerLaw(1)
    left, right = np.array([1.0, 0.0, 1.0 / 0.4]), np.array([0.125, 0.0, 0.1 / 0.4])
    dg = rb.DGSEM(law=law, grid=g, volume_form=rb.WeakForm(), surface_numericalflux=rb.RusanovFlux(),
                  boundary_conditions={1: left, 2: right})
    assert tuple(og.boundary()[:, 0]) == (1, 0) and tuple(og.boundary()[:, -1]) == (0, 2)
    og.set_boundary_condition(1, 1, left)
    og.set_boundary_condition(2, 1, right)
    olaw = O.Law(O.LAW_EULER, 1)
    x = og.points()[:, 0, :]
    wl = 0.5 * (1 - np.tanh((x - 0.5) / 0.03))
    q = np.zeros((nq, 3, K), order="F")
    for s in range(3):
        q[:, s, :] = right[s] + (left[s] - right[s]) * wl
    dt = 0.25 * (1.0 / K) / (nq - 1) / np.sqrt(1.4)
    qg = _compare(rb, og, dg, olaw, law, q, steps=40, dt=dt)
    rho = qg.numpy()[:, 0]
    assert rho.min() > 0.1 and rho.max() < 1.05


@pytest.mark.parametrize("scheme", ["eul_kg", "eul_weak", "eul_ec"])
@pytest.mark.parametrize("dim,nq,K", [(2, 5, (3, 2)), (3, 4, (2, 2, 2)), (3, 8, (2, 2, 1))])
def test_reflecting_walls_closed_box(rb, cuda_ok, dim, nq, K, scheme):
    og, dg, olaw, law = _build(rb, dim, nq, K, scheme, {1: "wall"})
    assert dg.pipelined_ctas == 0
    q = initial_state(og, olaw, scheme, seed=61, amp=0.02)
    qg = _compare(rb, og, dg, olaw, law, q)
    I0 = rb.integrals(dg, rb.GridArray.from_numpy(q))
    I1 = rb.integrals(dg, qg)
    for s in (0, dim + 1):  # mass and energy: no flux through a reflecting wall
        assert abs(I1[s] - I0[s]) <= 1e-13 * abs(I0[s]), s


def test_prescribed_inflow_advection(rb, cuda_ok):
    og, dg, olaw, law = _build(rb, 2, 6, (3, 3), "adv_weak", {1: [0.7]})
    q = initial_state(og, olaw, "adv_weak", seed=62)
    _compare(rb, og, dg, olaw, law, q)


def test_prescribed_state_free_stream(rb, cuda_ok):
    """A uniform flow with its own state prescribed on the boundary stays uniform."""
    og, dg, olaw, law = _build(rb, 3, 6, (2, 2, 2), "eul_kg", {1: [1.2, 0.3, -0.1, 0.2, 3.0]})
    q = np.zeros((og.np, 5, og.E), order="F")
    q[:, 0], q[:, 1], q[:, 2], q[:, 3], q[:, 4] = 1.2, 0.3, -0.1, 0.2, 3.0
    qg = rb.GridArray.from_numpy(q)
    dqg = rb.GridArray.from_numpy(np.zeros_like(q))
    dg(dqg, qg, 0.0, increment=False)
    # flux scale max|q|^2 / (smallest node spacing, about 0.05 here) = 180: 1e-12 of it
    assert np.abs(dqg.numpy()).max() <= 1e-12 * 180.0


def test_conditions_switch_kernels_and_errors(rb, cuda_ok):
    og, dg, olaw, law = _build(rb, 3, 8, (2, 2, 2), "eul_kg", {})
    assert dg.pipelined_ctas > 0
    dg.set_boundary_condition(1, "wall")
    assert dg.pipelined_ctas == 0
    dg.set_boundary_condition(1, None)
    assert dg.pipelined_ctas > 0
    with pytest.raises(rb.RB200Error) as ei:
        dg.set_boundary_condition(9, "wall")
    assert ei.value.status == 1
    with pytest.raises(ValueError):
        dg.set_boundary_condition(1, [1.0, 2.0])
    og2, dga, _, _ = _build(rb, 2, 4, (2, 2), "adv_weak", {})
    with pytest.raises(rb.RB200Error) as ei:
        dga.set_boundary_condition(1, "wall")
    assert ei.value.status == 6


def test_snapshot_knows_directions_and_boundary_conditions(rb, cuda_ok):
    """A snapshot taken with a direction subset or boundary conditions restores only into
    a handle with the same ones (the fingerprint covers them)."""
    og, dg, olaw, law = _build(rb, 3, 4, (2, 2, 2), "eul_kg", {1: "wall"})
    q = rb.GridArray.from_numpy(initial_state(og, olaw, "eul_kg", seed=63))
    solver = rb.LSRK54(dg, q, 1e-3)
    solver.dostep(q, 2)
    snap = rb.snapshot(dg, q, solver)
    _, same, _, _ = _build(rb, 3, 4, (2, 2, 2), "eul_kg", {1: "wall"})
    q2 = q.similar()
    rb.restore(same, snap, q2, rb.LSRK54(same, q2, 1.0))
    assert np.array_equal(q2.numpy(), q.numpy())
    _, plain, _, _ = _build(rb, 3, 4, (2, 2, 2), "eul_kg", {})
    with pytest.raises(rb.RB200Error) as ei:
        rb.restore(plain, snap, q2, rb.LSRK54(plain, q2, 1.0))
    assert ei.value.status == 2


@pytest.mark.parametrize("conds", [{1: "wall"}, {1: [1.1, 0.2, -0.1, 0.05, 2.8]}], ids=["wall", "state"])
def test_boundary_conditions_fp32_bulk(rb, cuda_ok, conds):
    og = O.Grid(3, 5, [2, 2, 2], [0.0] * 3, [1.0] * 3, [False] * 3)
    g = wrap_oracle_grid(og)
    law, form = product_scheme(rb, "eul_kg", 3)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux(),
                  boundary_conditions=conds, precision="fp32_bulk")
    c = conds[1]
    og.set_boundary_condition(1, 2 if c == "wall" else 1, None if c == "wall" else c)
    olaw = oracle_law("eul_kg", 3)
    q = initial_state(og, olaw, "eul_kg", seed=64, amp=0.02)
    ref = og.tendency(olaw, q)
    qg = rb.GridArray.from_numpy(q)
    dqg = rb.GridArray.from_numpy(np.zeros_like(q))
    dg(dqg, qg, 0.0, increment=False)
    for s in range(law.ns):
        assert rel_err(dqg.numpy()[:, s], ref[:, s]) <= 5e-5, s
