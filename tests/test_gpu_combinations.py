"""Seeded combinations of the options of the tendency against the oracle: dimension,
order, grid size, periodicity, warping, scheme, surface flux, direction subset and
boundary conditions, drawn together so that the options are exercised jointly (each is
also tested on its own elsewhere).

Tolerance: FP64 tendency and two LSRK(5,4) steps 1e-12 relative per field (max norm);
FP32-bulk tendency 5e-5.
"""

import numpy as np
import pytest

import oracle as O
from gpu_util import initial_state, oracle_law, product_scheme, rel_err, wrap_oracle_grid

pytestmark = pytest.mark.gpu

SCHEMES = ["adv_weak", "adv_fdc", "eul_weak", "eul_fdc", "eul_kg", "eul_ec"]


def _draw(seed):
    rng = np.random.default_rng(1000 + seed)
    dim = int(rng.integers(1, 4))
    nq = int(rng.integers(2, 9)) if dim < 3 else int(rng.choice([2, 3, 4, 5, 6, 8]))
    K = [int(rng.integers(1, 5)) for _ in range(dim)]
    per = [bool(rng.random() < 0.6) for _ in range(dim)]
    scheme = str(rng.choice(SCHEMES))
    warp = O.WARP_SINE if dim > 1 and rng.random() < 0.4 else O.WARP_NONE
    if warp == O.WARP_SINE:
        per = [True] * dim  # the sine warp keeps periodic faces matched
    sflux = "rusanov"
    if scheme.startswith("eul") and rng.random() < 0.4:
        sflux = str(rng.choice(["central", "ec", "kg", "roe", "matrix"]))
    elif rng.random() < 0.3:
        sflux = "central"
    dirs = None
    if dim > 1 and rng.random() < 0.3:
        sub = [d for d in range(1, dim + 1) if rng.random() < 0.5]
        dirs = tuple(sub) if sub else (int(rng.integers(1, dim + 1)),)
    bc = {}
    if not all(per) and rng.random() < 0.5:
        if scheme.startswith("eul") and rng.random() < 0.5:
            bc[1] = "wall"
        else:
            bc[1] = "state"
    return dim, nq, K, per, scheme, warp, sflux, dirs, bc


CASES = list(range(40))


@pytest.mark.parametrize("seed", CASES)
def test_combination(rb, cuda_ok, seed):
    dim, nq, K, per, scheme, warp, sflux, dirs, bc = _draw(seed)
    og = O.Grid(dim, nq, K, [0.0] * dim, [3.0] * dim, per, warp, 0.1 if warp == O.WARP_SINE else 0.0)
    g = wrap_oracle_grid(og)
    adv = [1.0, 0.5, 0.25][:dim]
    law, form = product_scheme(rb, scheme, dim, adv)
    sf = {"rusanov": rb.RusanovFlux(), "central": rb.CentralFlux(), "ec": rb.EntropyConservativeFlux(),
          "kg": rb.KennedyGruberFlux(), "roe": rb.RoeFlux(), "matrix": rb.MatrixFlux()}[sflux]
    olaw = oracle_law(scheme, dim, adv)
    olaw.c.surface_flux = {"rusanov": O.FLUX_RUSANOV, "central": O.FLUX_CENTRAL, "ec": O.FLUX_EC,
                           "kg": O.FLUX_KG, "roe": O.FLUX_ROE, "matrix": O.FLUX_MATRIX}[sflux]
    q = initial_state(og, olaw, scheme, seed=seed, amp=0.01)
    conds = {}
    for tag, kind in bc.items():
        if kind == "wall":
            conds[tag] = "wall"
            og.set_boundary_condition(tag, 2)
        else:
            state = q[:, :, 0].mean(axis=0)
            conds[tag] = state
            og.set_boundary_condition(tag, 1, state)
    if dirs is not None:
        og.set_directions(dirs)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=sf, directions=dirs,
                  boundary_conditions=conds)
    ref = og.tendency(olaw, q)
    qg = rb.GridArray.from_numpy(q)
    dqg = rb.GridArray.from_numpy(np.zeros_like(q))
    dg(dqg, qg, 0.0, increment=False)
    dg.sync_status()
    label = (dim, nq, K, per, scheme, warp, sflux, dirs, bc)
    for s in range(law.ns):
        assert rel_err(dqg.numpy()[:, s], ref[:, s]) <= 1e-12, (label, "tendency", s)
    dt = 1e-3
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(2):
        og.lsrk54_step(olaw, qo, dqo, i * dt, dt)
    rb.LSRK54(dg, qg, dt).dostep(qg, 2)
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(qg.numpy()[:, s], qo[:, s]) <= 1e-12, (label, "steps", s)


@pytest.mark.parametrize("seed", range(40, 60))
def test_combination_fp32_bulk(rb, cuda_ok, seed):
    """The same draws in FP32 bulk (Rusanov or central surface flux: the entropy-family
    surface fluxes are FP64 only): tendency within 5e-5 of the oracle."""
    dim, nq, K, per, scheme, warp, sflux, dirs, bc = _draw(seed)
    if sflux not in ("rusanov", "central"):
        sflux = "rusanov"
    og = O.Grid(dim, nq, K, [0.0] * dim, [3.0] * dim, per, warp, 0.1 if warp == O.WARP_SINE else 0.0)
    g = wrap_oracle_grid(og)
    adv = [1.0, 0.5, 0.25][:dim]
    law, form = product_scheme(rb, scheme, dim, adv)
    sf = rb.RusanovFlux() if sflux == "rusanov" else rb.CentralFlux()
    olaw = oracle_law(scheme, dim, adv)
    olaw.c.surface_flux = O.FLUX_RUSANOV if sflux == "rusanov" else O.FLUX_CENTRAL
    q = initial_state(og, olaw, scheme, seed=seed, amp=0.01)
    conds = {}
    for tag, kind in bc.items():
        if kind == "wall":
            conds[tag] = "wall"
            og.set_boundary_condition(tag, 2)
        else:
            state = q[:, :, 0].mean(axis=0)
            conds[tag] = state
            og.set_boundary_condition(tag, 1, state)
    if dirs is not None:
        og.set_directions(dirs)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=sf, directions=dirs,
                  boundary_conditions=conds, precision="fp32_bulk")
    ref = og.tendency(olaw, q)
    qg = rb.GridArray.from_numpy(q)
    dqg = rb.GridArray.from_numpy(np.zeros_like(q))
    dg(dqg, qg, 0.0, increment=False)
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(dqg.numpy()[:, s], ref[:, s]) <= 5e-5, ((dim, nq, K, per, scheme, warp, sflux, dirs, bc), s)
