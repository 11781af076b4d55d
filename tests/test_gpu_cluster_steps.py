"""The cluster step kernel: on small weak-form advection bricks every stage of every step
of an LSRK call runs in one launch of one thread-block cluster (hardware cluster barrier
between stages, the state read through L2).  Its arithmetic per node is the one-stage
kernel's, so its states must equal the per-stage launches' bit for bit; and they must
match the oracle's LSRK steps (odesolvers.jl:51-61, 163-189) at 1e-12 relative.

Cases: the 16^2, N=4 advection grid, a 3-D and a 1-D grid, FP64 and FP32 bulk, odd and
even stage counts (the result lands in the second buffer and is copied back), the
14-stage table and a caller's 3-stage table, directions and a prescribed boundary state;
grids too large for one cluster, grids whose Nq has a pipelined kernel and Euler grids
keep the stage launches.
"""

import numpy as np
import pytest

import oracle as O
from gpu_util import initial_state, oracle_law, product_scheme, rel_err, wrap_oracle_grid

pytestmark = pytest.mark.gpu

ADV = [1.0, 0.5, 0.25]


def _build(rb, dim, nq, K, precision="fp64", per=None, hi=None, **kw):
    per = per if per is not None else [True] * dim
    og = O.Grid(dim, nq, K, [0.0] * dim, hi or [1.0] * dim, per)
    g = wrap_oracle_grid(og)
    law, form = product_scheme(rb, "adv_weak", dim, ADV[:dim])
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux(), precision=precision,
                  **kw)
    return og, dg


def _steps(rb, dg, q, dt, nsteps, path):
    dg.set_kernel_path(path)
    qg = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, qg, dt).dostep(qg, nsteps)
    dg.sync_status()
    out = qg.numpy()
    dg.set_kernel_path("auto")
    return out


CASES = [(2, 5, (16, 16)), (3, 5, (3, 3, 3)), (1, 6, (40,))]


@pytest.mark.parametrize("nsteps", [7, 8])
@pytest.mark.parametrize("precision", ["fp64", "fp32_bulk"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"d{c[0]}q{c[1]}")
def test_cluster_equals_stage_launches(rb, cuda_ok, case, precision, nsteps):
    dim, nq, K = case
    og, dg = _build(rb, dim, nq, K, precision)
    assert dg.cluster_ctas > 0
    q = initial_state(og, oracle_law("adv_weak", dim, ADV[:dim]), "adv_weak", seed=5)
    dt = 0.2 / (nq * max(K))
    got = _steps(rb, dg, q, dt, nsteps, "auto")
    ref = _steps(rb, dg, q, dt, nsteps, "generic")
    assert np.array_equal(got, ref)
    dg.set_kernel_path("generic")
    assert dg.cluster_ctas == 0
    dg.set_kernel_path("auto")
    assert dg.cluster_ctas > 0


def test_cluster_against_oracle(rb, cuda_ok):
    """The 16^2, N=4 grid with a = (1, 0.5): 10 steps against the oracle's."""
    og, dg = _build(rb, 2, 5, (16, 16))
    olaw = oracle_law("adv_weak", 2, ADV[:2])
    q = initial_state(og, olaw, "adv_weak", seed=6)
    dt = 0.5 * (1.0 / 16) / 4 / np.hypot(1.0, 0.5)
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(10):
        og.lsrk54_step(olaw, qo, dqo, i * dt, dt)
    got = _steps(rb, dg, q, dt, 10, "auto")
    assert rel_err(got[:, 0], qo[:, 0]) <= 1e-12


@pytest.mark.parametrize("table", ["lsrk144", "three_stage"])
def test_cluster_other_tables(rb, cuda_ok, table):
    og, dg = _build(rb, 2, 5, (12, 10))
    q = initial_state(og, oracle_law("adv_weak", 2, ADV[:2]), "adv_weak", seed=7)
    dt = 0.01
    outs = []
    for path in ("auto", "generic"):
        dg.set_kernel_path(path)
        qg = rb.GridArray.from_numpy(q)
        if table == "lsrk144":
            rb.LSRK144(dg, qg, dt).dostep(qg, 3)
        else:  # Williamson's 3-stage, 3rd-order low-storage table
            rk = rb.LSRK(dg, [0.0, -5 / 9, -153 / 128], [1 / 3, 15 / 16, 8 / 15], [0.0, 1 / 3, 3 / 4], qg, dt)
            rk.dostep(qg, 3)
        dg.sync_status()
        outs.append(qg.numpy())
    dg.set_kernel_path("auto")
    assert np.array_equal(outs[0], outs[1])


def test_cluster_directions_and_boundary_state(rb, cuda_ok):
    """x only, no periodic direction, a prescribed exterior state on the boundary faces."""
    og, dg = _build(rb, 2, 5, (10, 8), per=[False, False], directions=(1,), boundary_conditions={1: [0.7]})
    assert dg.cluster_ctas > 0
    q = initial_state(og, oracle_law("adv_weak", 2, ADV[:2]), "adv_weak", seed=8)
    got = _steps(rb, dg, q, 0.005, 5, "auto")
    ref = _steps(rb, dg, q, 0.005, 5, "generic")
    assert np.array_equal(got, ref)


def test_large_pipelined_and_euler_grids_keep_stage_launches(rb, cuda_ok):
    _, dg = _build(rb, 2, 5, (64, 64))
    assert dg.cluster_ctas == 0  # 205 groups of 20 elements: more than the cluster holds
    _, dg = _build(rb, 3, 6, (3, 3, 2))
    assert dg.cluster_ctas == 0 and dg.pipelined_ctas > 0  # the pipelined advection kernel
    og = O.Grid(2, 5, (4, 4), [0.0, 0.0], [1.0, 1.0], [True, True])
    law, form = product_scheme(rb, "eul_kg", 2)
    dg = rb.DGSEM(law=law, grid=wrap_oracle_grid(og), volume_form=form, surface_numericalflux=rb.RusanovFlux())
    assert dg.cluster_ctas == 0


@pytest.mark.parametrize("case", [(2, 8, (1, 1)), (2, 5, (16, 20)), (3, 2, (4, 4, 4)), (1, 2, (1,))],
                         ids=["one-element", "16-ctas", "3d-nq2", "1d-one-element"])
def test_cluster_edges(rb, cuda_ok, case):
    """One periodic element (every face meets the element itself, in its own CTA), a grid
    that fills all 16 CTAs (320 elements of 25 nodes), Nq = 2."""
    dim, nq, K = case
    og, dg = _build(rb, dim, nq, K)
    assert dg.cluster_ctas > 0
    if K == (16, 20):
        assert dg.cluster_ctas == 16
    q = initial_state(og, oracle_law("adv_weak", dim, ADV[:dim]), "adv_weak", seed=9)
    dt = 0.1 / (nq * max(K))
    got = _steps(rb, dg, q, dt, 9, "auto")
    ref = _steps(rb, dg, q, dt, 9, "generic")
    assert np.array_equal(got, ref)


def test_one_group_too_many_keeps_stage_launches(rb, cuda_ok):
    _, dg = _build(rb, 2, 5, (17, 20))  # 340 elements: 17 groups of 20
    assert dg.cluster_ctas == 0
