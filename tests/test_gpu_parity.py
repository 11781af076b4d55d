"""GPU parity: the CUDA kernels (through the C ABI) against the oracle.

Tolerances (stated here and in the assertion messages):
  * FP64 plain form: max |gpu - oracle| <= 1e-12 * max |oracle| per array, for one
    tendency evaluation and for several LSRK(5,4) steps;
  * FP32-bulk form: max |gpu - oracle| <= 5e-5 * max |oracle| for one tendency;
  * face indexing (vmapP rebuilt from the device neighbour table): bit-exact;
  * reductions: 1e-13 relative.
"""

import json
import math
import os

import numpy as np
import pytest

import oracle as O
from gpu_util import LAWS, initial_state, oracle_law, product_scheme, rel_err, wrap_oracle_grid

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 5e-5

CASES = [
    # dim, nq, K, periodic, scheme, warp
    (2, 5, (4, 3), (1, 1), "adv_weak", O.WARP_NONE),
    (2, 5, (4, 3), (1, 0), "adv_fdc", O.WARP_NONE),
    (2, 4, (3, 5), (1, 1), "eul_weak", O.WARP_NONE),
    (2, 6, (3, 3), (1, 1), "eul_fdc", O.WARP_NONE),
    (2, 8, (3, 2), (1, 1), "eul_kg", O.WARP_NONE),
    (2, 5, (3, 4), (1, 1), "eul_ec", O.WARP_NONE),
    (3, 4, (3, 2, 2), (1, 1, 1), "adv_weak", O.WARP_NONE),
    (3, 3, (2, 3, 2), (1, 1, 0), "adv_fdc", O.WARP_NONE),
    (3, 5, (2, 2, 3), (1, 1, 1), "eul_weak", O.WARP_NONE),
    (3, 4, (2, 3, 2), (1, 1, 1), "eul_fdc", O.WARP_NONE),
    (3, 8, (3, 2, 2), (1, 1, 1), "eul_kg", O.WARP_NONE),
    (3, 7, (2, 2, 2), (1, 0, 1), "eul_kg", O.WARP_NONE),
    (3, 6, (2, 2, 2), (1, 1, 1), "eul_ec", O.WARP_NONE),
    (2, 5, (4, 3), (1, 1), "eul_kg", O.WARP_SINE),
    (2, 4, (3, 3), (1, 1), "adv_weak", O.WARP_SINE),
    (3, 5, (2, 2, 2), (1, 1, 1), "eul_kg", O.WARP_SINE),
    (3, 4, (2, 2, 3), (1, 1, 1), "eul_weak", O.WARP_SINE),
    (3, 4, (2, 2, 2), (1, 1, 1), "eul_ec", O.WARP_SINE),
    (3, 8, (2, 2, 2), (1, 1, 1), "eul_kg", O.WARP_IDENTITY_CURVED),
]


def _build(rb, dim, nq, K, per, scheme, warp, precision="fp64"):
    lo, hi = [0.0] * dim, [10.0] * dim
    og = O.Grid(dim, nq, K, lo, hi, per, warp, 0.1 if warp == O.WARP_SINE else 0.0)
    g = wrap_oracle_grid(og)
    adv = [1.0, 0.5, 0.25][:dim]
    law, form = product_scheme(rb, scheme, dim, adv)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux(), precision=precision)
    return og, g, dg, oracle_law(scheme, dim, adv), law


def _id(c):
    return f"{c[0]}d-nq{c[1]}-{c[4]}-warp{c[5]}"


@pytest.mark.parametrize("case", CASES, ids=[_id(c) for c in CASES])
@pytest.mark.parametrize("increment", [False, True])
def test_tendency_fp64(rb, cuda_ok, case, increment):
    dim, nq, K, per, scheme, warp = case
    og, g, dg, olaw, law = _build(rb, *case)
    assert dg.geometry == ("affine" if warp == O.WARP_NONE else "curved")
    q = initial_state(og, olaw, scheme, seed=1)
    dq0 = initial_state(og, olaw, scheme, seed=2) if increment else og.state(olaw)
    ref = og.tendency(olaw, q, dq=np.asfortranarray(dq0.copy()), increment=increment)
    qg = rb.GridArray.from_numpy(q)
    dqg = rb.GridArray.from_numpy(dq0)
    dg(dqg, qg, 0.0, increment=increment)
    got = dqg.numpy()
    for s in range(law.ns):
        assert rel_err(got[:, s], ref[:, s]) <= FP64_TOL, f"field {s}: FP64 tendency beyond {FP64_TOL}"


@pytest.mark.parametrize("case", CASES[::2], ids=[_id(c) for c in CASES[::2]])
def test_lsrk54_steps_fp64(rb, cuda_ok, case):
    dim, nq, K, per, scheme, warp = case
    og, g, dg, olaw, law = _build(rb, *case)
    q = initial_state(og, olaw, scheme, seed=3, amp=0.01)
    dt = 1e-3
    qo = q.copy(order="F")
    dqo = og.state(olaw)
    for step in range(3):
        og.lsrk54_step(olaw, qo, dqo, step * dt, dt)
    qg = rb.GridArray.from_numpy(q)
    solver = rb.LSRK54(dg, qg, dt)
    solver.dostep(qg, 3)
    got = qg.numpy()
    for s in range(law.ns):
        assert rel_err(got[:, s], qo[:, s]) <= FP64_TOL
    # the LSRK register after the last stage matches too (absolute scale of dq)
    assert rel_err(solver.dq.numpy(), dqo) <= 1e-11


@pytest.mark.parametrize("case", CASES, ids=[_id(c) for c in CASES])
def test_face_indexing_bit_exact(rb, cuda_ok, case):
    og, g, dg, olaw, law = _build(rb, *case)
    assert np.array_equal(dg.face_vmapP(), og.vmapP())


@pytest.mark.parametrize("case", CASES[::3], ids=[_id(c) for c in CASES[::3]])
def test_norms_and_integrals(rb, cuda_ok, case):
    og, g, dg, olaw, law = _build(rb, *case)
    q = initial_state(og, olaw, case[4], seed=4)
    qg = rb.GridArray.from_numpy(q)
    tot, comp = og.weightednorm(q, law.ns)
    assert rb.weightednorm(dg, qg) == pytest.approx(tot, rel=1e-13)
    assert np.allclose(rb.weightednorm(dg, qg, componentwise=True), comp, rtol=1e-13, atol=0)
    ints = og.integrals(q, law.ns)
    assert np.allclose(rb.integrals(dg, qg), ints, rtol=1e-12, atol=1e-12 * np.abs(ints).max())


@pytest.mark.parametrize("case", CASES[::3], ids=[_id(c) for c in CASES[::3]])
@pytest.mark.parametrize("p", [1, 3, 2.5, math.inf])
def test_weightednorm_p(rb, cuda_ok, case, p):
    """weightednorm(dg, q, p; componentwise) for p != 2 (measures.jl:6-21): the weighted
    p-sums per field and the unweighted max-norm for p = Inf, 1e-13 against the oracle;
    the max-norm is an exact maximum, so it matches bit for bit."""
    og, g, dg, olaw, law = _build(rb, *case)
    q = initial_state(og, olaw, case[4], seed=6)
    qg = rb.GridArray.from_numpy(q)
    tot, comp = og.weightednorm_p(q, law.ns, p)
    got = rb.weightednorm(dg, qg, p, componentwise=True)
    if math.isinf(p):
        assert got == list(comp) and rb.weightednorm(dg, qg, p) == tot
        assert tot == float(np.abs(q).max())
    else:
        assert np.allclose(got, comp, rtol=1e-13, atol=0)
        assert rb.weightednorm(dg, qg, p) == pytest.approx(tot, rel=1e-13)


def test_weightednorm_p_rejects(rb, cuda_ok):
    og, g, dg, olaw, law = _build(rb, *CASES[0])
    qg = rb.GridArray.from_numpy(initial_state(og, olaw, CASES[0][4]))
    for bad in (0, -1, float("nan"), -math.inf):
        with pytest.raises(rb.RB200Error):
            rb.weightednorm(dg, qg, bad)


@pytest.mark.parametrize("case", CASES[2::2], ids=[_id(c) for c in CASES[2::2]])
def test_tendency_fp32_bulk(rb, cuda_ok, case):
    dim, nq, K, per, scheme, warp = case
    og, g, dg, olaw, law = _build(rb, *case, precision="fp32_bulk")
    q = initial_state(og, olaw, scheme, seed=5)
    ref = og.tendency(olaw, q)
    qg = rb.GridArray.from_numpy(q)
    dqg = qg.similar()
    dg(dqg, qg, 0.0, increment=False)
    got = dqg.numpy()
    for s in range(law.ns):
        assert rel_err(got[:, s], ref[:, s]) <= FP32_TOL, f"field {s}: FP32-bulk tendency beyond {FP32_TOL}"


def test_host_buffer_path_equals_device_path(rb, cuda_ok):
    og, g, dg, olaw, law = _build(rb, 3, 5, (2, 2, 2), (1, 1, 1), "eul_kg", O.WARP_NONE)
    q = initial_state(og, olaw, "eul_kg", seed=6, amp=0.01)
    qh = np.asfortranarray(q.copy())
    dg.lsrk54_steps_host(qh, 0.0, 1e-3, 2)
    qg = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, qg, 1e-3).dostep(qg, 2)
    assert np.array_equal(qh, qg.numpy())


# ------------------------------------------------------------ reference goldens on the GPU

GOLD = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_goldens.json")))


@pytest.mark.parametrize("entry", GOLD["errors"],
                         ids=[f"{e['law']}-{e['test']}-{e['form']}-L{e['level']}" for e in GOLD["errors"]])
def test_reference_goldens_through_product_api(rb, cuda_ok, entry):
    """Every golden L2 error of the reference's balance-law tests (test/balancelaws/*/*.jl,
    all refinement levels, 1-D to 3-D), run end to end through the product API: grid
    generation, DGSEM on the GPU, solve, weightednorm; to the tolerance the reference
    test applies."""
    law_name, test, form, lev = entry["law"], entry["test"], entry["form"], entry["level"]
    N, K = 4, 5 * 2 ** (lev - 1)
    vf = {"weak": None, "fd_central": rb.CentralFlux(), "fd_ec": rb.EntropyConservativeFlux()}[form]
    vform = rb.WeakForm() if vf is None else rb.FluxDifferencingForm(vf)
    if test == "isentropicvortex":
        dim, lo, hi = 2, (0.0, -5.0), (20.0, 5.0)
    else:
        dim = int(test[-2])
        lo, hi = (-1.0,) * dim, (1.0,) * dim
    cell = rb.LobattoCell(*([N + 1] * dim))
    grid = rb.generate(rb.GridManager(cell, rb.brick(tuple(rb.jl_range(lo[d], hi[d], K + 1) for d in range(dim)),
                                                     (True,) * dim)))
    law = rb.AdvectionLaw(dim) if law_name == "advection" else rb.EulerLaw(dim)
    dg = rb.DGSEM(law=law, grid=grid, volume_form=vform, surface_numericalflux=rb.RusanovFlux())
    og_law = O.Law(O.LAW_ADVECTION if law_name == "advection" else O.LAW_EULER, dim)
    og = O.Grid(dim, N + 1, [K] * dim, lo, hi, [True] * dim)  # only to evaluate initial/exact data
    cfl = 0.5 if dim == 1 else 0.25
    if test == "isentropicvortex":
        dt, T, kind = 0.25 * (10.0 / K) / N, 5.0, 2
    elif law_name == "advection":
        dt, T, kind = cfl * (2.0 / K) / N / math.sqrt(dim), 0.7, 0
    else:
        dt = cfl * (2.0 / K) / N / math.sqrt(1.4)
        T, kind = (dt if dim == 3 else 0.7), 1
    q = rb.GridArray.from_numpy(og.initial_condition(og_law, kind))
    rb.solve(q, T, rb.LSRK54(dg, q, dt))
    qe = rb.GridArray.from_numpy(og.initial_condition(og_law, kind, t=T))
    qe.data.sub_(q.data)
    err = rb.weightednorm(dg, qe)
    assert err == pytest.approx(entry["expected"], rel=entry["rtol"]), entry["source"]


@pytest.mark.parametrize("case", [CASES[0], CASES[10]], ids=[_id(CASES[0]), _id(CASES[10])])
def test_graph_replay_equals_eager_steps(rb, cuda_ok, case):
    """rb200_lsrk54_step replays a captured two-step CUDA graph for long runs; the result
    is bit-identical to stepping one call at a time, and a new dt is re-captured."""
    og, g, dg, olaw, law = _build(rb, *case)
    q = initial_state(og, olaw, case[4], seed=21, amp=0.01)
    for dt in (1e-3, 7e-4):
        qa, qb = rb.GridArray.from_numpy(q), rb.GridArray.from_numpy(q)
        sa, sb = rb.LSRK54(dg, qa, dt), rb.LSRK54(dg, qb, dt)
        sa.dostep(qa, 7)
        for _ in range(7):
            sb.dostep(qb, 1)
        assert np.array_equal(qa.numpy(), qb.numpy())
        assert np.array_equal(sa.dq.numpy(), sb.dq.numpy())


@pytest.mark.parametrize("nq,K", [(4, (12, 12, 13)), (6, (10, 10, 9)), (5, (12, 12, 10))], ids=["nq4", "nq6", "nq5"])
def test_generic_fp32_bulk_steps_walk_groups(rb, cuda_ok, nq, K):
    """3-D FP32-bulk stages on the generic kernel, whose CTAs walk several element groups
    each (more elements than resident CTAs) and prefetch the next group's state and
    register: two steps against the oracle (1e-6 relative on the state), and five steps,
    the last three graph-replayed, against a run restarted from a snapshot after two."""
    og, g, dg, olaw, law = _build(rb, 3, nq, K, (1, 1, 1), "eul_kg", O.WARP_NONE, precision="fp32_bulk")
    dg.set_kernel_path("generic")  # even Nq also has the pipelined kernel
    q = initial_state(og, olaw, "eul_kg", seed=21, amp=0.01)
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(2):
        og.lsrk54_step(olaw, qo, dqo, i * 1e-3, 1e-3)
    qg = rb.GridArray.from_numpy(q)
    solver = rb.LSRK54(dg, qg, 1e-3)
    solver.dostep(qg, 2)
    for s in range(law.ns):
        assert rel_err(qg.numpy()[:, s], qo[:, s]) <= 1e-6, s
    snap = rb.snapshot(dg, qg, solver)
    solver.dostep(qg, 3)
    q2 = rb.GridArray.from_numpy(np.zeros_like(q))
    s2 = rb.LSRK54(dg, q2, 1.0)
    rb.restore(dg, snap, q2, s2)
    s2.dostep(q2, 3)
    assert np.array_equal(q2.numpy(), qg.numpy())
