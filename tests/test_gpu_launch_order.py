"""Launch order on one stream without a host synchronisation in between.  The stage and
mortar kernels are launched with programmatic dependent launch: they may start while
the previous kernel of the stream drains, and wait for it (griddepcontrol.wait) before
they read or write the state.  A torch kernel that writes the state right before a
tendency or a sequence of steps, and one that reads the result right after, must see
exactly what they see with synchronisations in between.

Grids: a 3-D brick on the pipelined kernel (FP64 KG, Nq = 8) and an adapted 3-D grid
(mortar kernel, then the pipelined kernel).  Tolerance: 1e-12 relative per field against
the oracle, and bit-equal to the synchronised run.
"""

import numpy as np
import pytest

import oracle as O
from gpu_util import initial_state, oracle_law, product_scheme, rel_err, wrap_oracle_grid

pytestmark = pytest.mark.gpu


def _brick(rb):
    og = O.Grid(3, 8, (4, 3, 3), [0.0] * 3, [10.0] * 3, [True] * 3)
    law, form = product_scheme(rb, "eul_kg", 3)
    dg = rb.DGSEM(law=law, grid=wrap_oracle_grid(og), volume_form=form, surface_numericalflux=rb.RusanovFlux())
    assert dg.pipelined_ctas > 0
    olaw = oracle_law("eul_kg", 3)
    return og, dg, olaw, law.ns, initial_state(og, olaw, "eul_kg", seed=41, amp=0.01)


def _adapted_grid(rb):
    from raven_b200 import forest
    from test_forest_host import LAWS, _adapted, _oracle, _state

    lw = [l for l in LAWS if l[1] == O.LAW_EULER and l[2] == O.FORM_FLUXDIFF][0]
    grid, _ = _adapted(rb, forest, 3, 6, (2, 2, 1), (True, True, True), 2)
    assert grid.mortars.size > 0
    law = rb.EulerLaw(3)
    dg = rb.DGSEM(law=law, grid=grid, volume_form=rb.FluxDifferencingForm(rb.KennedyGruberFlux()),
                  surface_numericalflux=rb.RusanovFlux())
    assert dg.pipelined_ctas > 0
    olaw = O.Law(lw[1], 3, form=lw[2], volume_flux=lw[3])
    return _oracle(grid), dg, olaw, law.ns, _state(grid, olaw, 7)


def _run(rb, dg, q0, dt, nsteps, sync):
    import torch

    qg = rb.GridArray.from_numpy(0.5 * q0)  # halved exactly: doubled back by a torch kernel
    dqg = rb.GridArray.from_numpy(np.zeros_like(q0))
    torch.cuda.synchronize()
    qg.data.mul_(2.0)
    if sync:
        torch.cuda.synchronize()
    dg(dqg, qg, 0.0, increment=False)
    tend = dqg.data.clone()
    if sync:
        torch.cuda.synchronize()
    qg.data.mul_(0.5)
    qg.data.mul_(2.0)
    if sync:
        torch.cuda.synchronize()
    dg.lsrk54_steps(qg, dqg, 0.0, dt, nsteps)
    state = qg.data.clone()
    torch.cuda.synchronize()
    dg.sync_status()
    # (E, Ns, Np) tensors -> Raven's (Np, Ns, E) layout, as GridArray.numpy() does
    return tuple(np.asfortranarray(t.cpu().numpy().transpose(2, 1, 0)) for t in (tend, state))


@pytest.mark.parametrize("grid", ["brick", "adapted"])
def test_torch_kernels_before_and_after(rb, cuda_ok, grid):
    og, dg, olaw, ns, q0 = _brick(rb) if grid == "brick" else _adapted_grid(rb)
    dt, nsteps = 1e-3, 6  # 6 steps: the captured two-step graph replays twice
    tend, state = _run(rb, dg, q0, dt, nsteps, sync=False)
    tend_s, state_s = _run(rb, dg, q0, dt, nsteps, sync=True)
    assert np.array_equal(tend, tend_s) and np.array_equal(state, state_s)
    ref = og.tendency(olaw, q0)
    qo, dqo = q0.copy(order="F"), og.state(olaw)
    for i in range(nsteps):
        og.lsrk54_step(olaw, qo, dqo, i * dt, dt)
    for s in range(ns):
        assert rel_err(tend[:, s], ref[:, s]) <= 1e-12, ("tendency", s)
        assert rel_err(state[:, s], qo[:, s]) <= 1e-12, ("steps", s)
