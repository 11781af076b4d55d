"""LSRK144 and RLSRK144 (src/balancelaws/odesolvers.jl:68-71, 158-161, 191-239) on the GPU
against the oracle's restatement of the same 14-stage schemes.

Tolerances: FP64 state 1e-12 relative per field and register 1e-11 (as for LSRK54);
FP32 bulk 1e-6 after two steps; RLSRK144 state 1e-12 and relaxation parameter 1e-9
absolute.  The fused steps replay a captured CUDA graph from the fourth step on; a handle
that alternates LSRK54 and LSRK144 calls recaptures it for the other scheme, which the
last test checks bit for bit against fresh handles.
"""

import numpy as np
import pytest

import oracle as O
from gpu_util import initial_state, oracle_law, product_scheme, rel_err, wrap_oracle_grid

pytestmark = pytest.mark.gpu

CASES = [
    # dim, nq, K, scheme, warp: the pipelined brick kernel, the generic kernel, the
    # curved FP64 pipelined kernel
    (3, 8, (3, 2, 2), "eul_kg", O.WARP_NONE),
    (2, 5, (4, 3), "adv_weak", O.WARP_NONE),
    (3, 8, (2, 2, 3), "eul_kg", O.WARP_SINE),
    (2, 6, (3, 4), "eul_ec", O.WARP_NONE),
]


def _build(rb, dim, nq, K, scheme, warp, precision="fp64"):
    og = O.Grid(dim, nq, K, [0.0] * dim, [10.0] * dim, [True] * dim, warp, 0.1 if warp == O.WARP_SINE else 0.0)
    g = wrap_oracle_grid(og)
    adv = [1.0, 0.5, 0.25][:dim]
    law, form = product_scheme(rb, scheme, dim, adv)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux(), precision=precision)
    return og, dg, oracle_law(scheme, dim, adv), law


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}d-nq{c[1]}-{c[3]}-warp{c[4]}" for c in CASES])
def test_lsrk144_steps_fp64(rb, cuda_ok, case):
    og, dg, olaw, law = _build(rb, *case)
    q = initial_state(og, olaw, case[3], seed=21, amp=0.01)
    dt = 1e-3
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(5):
        og.lsrk144_step(olaw, qo, dqo, i * dt, dt)
    qg = rb.GridArray.from_numpy(q)
    solver = rb.LSRK144(dg, qg, dt)
    solver.dostep(qg, 5)  # two eager steps, then the captured graph
    dg.sync_status()
    got = qg.numpy()
    for s in range(law.ns):
        assert rel_err(got[:, s], qo[:, s]) <= 1e-12, s
    assert rel_err(solver.dq.numpy(), dqo) <= 1e-11
    assert solver.time == pytest.approx(5 * dt)


def test_lsrk144_fp32_bulk(rb, cuda_ok):
    og, dg, olaw, law = _build(rb, 3, 8, (3, 2, 2), "eul_kg", O.WARP_NONE, precision="fp32_bulk")
    q = initial_state(og, olaw, "eul_kg", seed=22, amp=0.01)
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(2):
        og.lsrk144_step(olaw, qo, dqo, i * 1e-3, 1e-3)
    qg = rb.GridArray.from_numpy(q)
    rb.LSRK144(dg, qg, 1e-3).dostep(qg, 2)
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(qg.numpy()[:, s], qo[:, s]) <= 1e-6, s


def test_rlsrk144_steps(rb, cuda_ok):
    og, dg, olaw, law = _build(rb, 2, 6, (3, 4), "eul_ec", O.WARP_NONE)
    q = initial_state(og, olaw, "eul_ec", seed=23, amp=0.01)
    qo, dqo = q.copy(order="F"), og.state(olaw)
    gamma = np.ones(1)
    dt = 2e-2
    for i in range(3):
        og.rlsrk144_step(olaw, qo, dqo, gamma, i * dt, dt)
    qg = rb.GridArray.from_numpy(q)
    solver = rb.RLSRK144(dg, qg, dt)
    solver.dostep(qg, 1)
    solver.dostep(qg, 2)
    for s in range(law.ns):
        assert rel_err(qg.numpy()[:, s], qo[:, s]) <= 1e-12, s
    assert abs(solver.gamma - gamma[0]) <= 1e-9
    assert solver.gamma != 1.0


def test_schemes_alternate_on_one_handle(rb, cuda_ok):
    """LSRK54 and LSRK144 calls on the same handle (each long enough to capture its graph)
    give exactly what fresh handles give."""
    case = CASES[0]
    og, dg, olaw, law = _build(rb, *case)
    q0 = initial_state(og, olaw, case[3], seed=24, amp=0.01)
    qa = rb.GridArray.from_numpy(q0)
    rb.LSRK54(dg, qa, 1e-3).dostep(qa, 4)
    rb.LSRK144(dg, qa, 1e-3).dostep(qa, 4)
    rb.LSRK54(dg, qa, 1e-3).dostep(qa, 4)
    og2, dg2, _, _ = _build(rb, *case)
    og3, dg3, _, _ = _build(rb, *case)
    qb = rb.GridArray.from_numpy(q0)
    rb.LSRK54(dg2, qb, 1e-3).dostep(qb, 4)
    rb.LSRK144(dg3, qb, 1e-3).dostep(qb, 4)
    rb.LSRK54(dg2, qb, 1e-3).dostep(qb, 4)
    assert np.array_equal(qa.numpy(), qb.numpy())


def test_rlsrk144_after_stage_is_refused(rb, cuda_ok):
    """The relaxation step runs its stages fused: a stage callback raises."""
    og, dg, olaw, law = _build(rb, 2, 6, (3, 4), "eul_ec", O.WARP_NONE)
    q = rb.GridArray.from_numpy(initial_state(og, olaw, "eul_ec"))
    with pytest.raises(NotImplementedError):
        rb.RLSRK144(dg, q, 1e-3).dostep(q, 1, after_stage=lambda t, q: None)


# Williamson's three-stage third-order low-storage scheme (J. Comput. Phys. 35 (1980), 48-56)
RK3_A = (0.0, -5.0 / 9.0, -153.0 / 128.0)
RK3_B = (1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0)
RK3_C = (0.0, 1.0 / 3.0, 3.0 / 4.0)


@pytest.mark.parametrize("case", CASES[:3], ids=[f"{c[0]}d-nq{c[1]}-{c[3]}-warp{c[4]}" for c in CASES[:3]])
def test_lsrk_any_table(rb, cuda_ok, case):
    """LSRK(rhs!, rka, rkb, rkc, q, dt, t0) with a table of the caller's (a three-stage
    scheme) against the oracle, and then a different table on the same handle."""
    og, dg, olaw, law = _build(rb, *case)
    q = initial_state(og, olaw, case[3], seed=25, amp=0.01)
    dt = 1e-3
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(5):
        og.lsrk_step(olaw, qo, dqo, RK3_A, RK3_B, i * dt, dt)
    qg = rb.GridArray.from_numpy(q)
    solver = rb.LSRK(dg, RK3_A, RK3_B, RK3_C, qg, dt)
    solver.dostep(qg, 5)  # two eager steps, then the captured graph
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(qg.numpy()[:, s], qo[:, s]) <= 1e-12, s
    # another table of the same length on the same handle: the graph is recaptured
    A2 = (0.0, -0.5, -1.0)
    B2 = (0.25, 0.5, 0.4)
    for i in range(5):
        og.lsrk_step(olaw, qo, dqo, A2, B2, (5 + i) * dt, dt)
    s2 = rb.LSRK(dg, A2, B2, RK3_C, qg, dt, t0=5 * dt)
    s2.dq = solver.dq
    s2.dostep(qg, 5)
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(qg.numpy()[:, s], qo[:, s]) <= 1e-12, s


def test_lsrk_generic_table_equals_lsrk54(rb, cuda_ok):
    og, dg, olaw, law = _build(rb, *CASES[0])
    q = initial_state(og, olaw, CASES[0][3], seed=26, amp=0.01)
    a, b = rb.GridArray.from_numpy(q), rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, a, 1e-3).dostep(a, 6)
    A = (0.0, -567301805773 / 1357537059087, -2404267990393 / 2016746695238, -3550918686646 / 2091501179385,
         -1275806237668 / 842570457699)
    B = (1432997174477 / 9575080441755, 5161836677717 / 13612068292357, 1720146321549 / 2090206949498,
         3134564353537 / 4481467310338, 2277821191437 / 14882151754819)
    rb.LSRK(dg, A, B, rb.LSRK54_RKC, b, 1e-3).dostep(b, 6)
    assert np.array_equal(a.numpy(), b.numpy())


def test_lsrk144_stage_callbacks(rb, cuda_ok):
    """LSRK144 with after_stage: its 14 stages one by one, the callback at time + c_i dt,
    and the same state as the fused steps, bit for bit."""
    og, dg, olaw, law = _build(rb, *CASES[1])
    q = initial_state(og, olaw, CASES[1][3], seed=27, amp=0.01)
    a, b = rb.GridArray.from_numpy(q), rb.GridArray.from_numpy(q)
    dt = 1e-3
    rb.LSRK144(dg, a, dt).dostep(a, 2)
    times = []
    rb.LSRK144(dg, b, dt).dostep(b, 2, after_stage=lambda t, qq: times.append(t))
    assert np.array_equal(a.numpy(), b.numpy())
    want = [i * dt + c * dt for i in range(2) for c in rb.LSRK144_RKC]
    assert times == pytest.approx(want, rel=0, abs=1e-15)


def test_rlsrk_any_table(rb, cuda_ok):
    og, dg, olaw, law = _build(rb, 2, 6, (3, 4), "eul_ec", O.WARP_NONE)
    q = initial_state(og, olaw, "eul_ec", seed=28, amp=0.01)
    dt = 2e-2
    qo, dqo, gamma = q.copy(order="F"), og.state(olaw), np.ones(1)
    for i in range(3):
        og.rlsrk_step(olaw, qo, dqo, gamma, RK3_A, RK3_B, i * dt, dt)
    qg = rb.GridArray.from_numpy(q)
    solver = rb.RLSRK(dg, RK3_A, RK3_B, RK3_C, qg, dt)
    solver.dostep(qg, 3)
    for s in range(law.ns):
        assert rel_err(qg.numpy()[:, s], qo[:, s]) <= 1e-12, s
    assert abs(solver.gamma - gamma[0]) <= 1e-9
