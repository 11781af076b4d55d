"""1-D grids on the GPU: the generic stage kernel on lines against the oracle, and the
reference's 1-D entropy-conservation tests (test/balancelaws/euler/entropy_conservation_1d.jl,
advection's counterpart) natively in 1-D.

Tolerances: FP64 tendency and LSRK steps 1e-12 relative per field (max norm); FP32 bulk
tendency 5e-5; RLSRK54 entropy drift 40 eps, the bound of the reference tests.
"""

import numpy as np
import pytest

import oracle as O
from gpu_util import initial_state, oracle_law, product_scheme, rel_err, wrap_oracle_grid

pytestmark = pytest.mark.gpu

EPS = np.finfo(float).eps
SCHEMES = ["adv_weak", "adv_fdc", "eul_weak", "eul_fdc", "eul_kg", "eul_ec"]


def _build(rb, nq, K, per, scheme, sflux=None, precision="fp64"):
    og = O.Grid(1, nq, [K], [-1.0], [1.0], [per])
    g = wrap_oracle_grid(og)
    law, form = product_scheme(rb, scheme, 1, [1.0])
    sf = sflux or rb.RusanovFlux()
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=sf, precision=precision)
    return og, dg, oracle_law(scheme, 1, [1.0]), law


@pytest.mark.parametrize("per", [True, False])
@pytest.mark.parametrize("nq", [2, 5, 8])
@pytest.mark.parametrize("scheme", SCHEMES)
def test_line_tendency_and_steps(rb, cuda_ok, scheme, nq, per):
    og, dg, olaw, law = _build(rb, nq, 7, per, scheme)
    q = initial_state(og, olaw, scheme, seed=51, amp=0.01)
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


@pytest.mark.parametrize("sflux", ["ec", "kg", "roe", "matrix"])
def test_line_entropy_surface_fluxes(rb, cuda_ok, sflux):
    flux = {"ec": rb.EntropyConservativeFlux(), "kg": rb.KennedyGruberFlux(), "roe": rb.RoeFlux(),
            "matrix": rb.MatrixFlux()}[sflux]
    og, dg, olaw, law = _build(rb, 6, 5, True, "eul_ec", flux)
    olaw = O.Law(O.LAW_EULER, 1, form=O.FORM_FLUXDIFF, volume_flux=O.FLUX_EC,
                 surface_flux={"ec": O.FLUX_EC, "kg": O.FLUX_KG, "roe": O.FLUX_ROE, "matrix": O.FLUX_MATRIX}[sflux])
    q = initial_state(og, olaw, "eul_ec", seed=52, amp=0.01)
    ref = og.tendency(olaw, q)
    qg = rb.GridArray.from_numpy(q)
    dqg = rb.GridArray.from_numpy(np.zeros_like(q))
    dg(dqg, qg, 0.0, increment=False)
    for s in range(law.ns):
        assert rel_err(dqg.numpy()[:, s], ref[:, s]) <= 1e-12, s


def test_line_fp32_bulk(rb, cuda_ok):
    og, dg, olaw, law = _build(rb, 6, 9, True, "eul_kg", precision="fp32_bulk")
    q = initial_state(og, olaw, "eul_kg", seed=53, amp=0.01)
    ref = og.tendency(olaw, q)
    qg = rb.GridArray.from_numpy(q)
    dqg = rb.GridArray.from_numpy(np.zeros_like(q))
    dg(dqg, qg, 0.0, increment=False)
    for s in range(law.ns):
        assert rel_err(dqg.numpy()[:, s], ref[:, s]) <= 5e-5, s


@pytest.mark.parametrize("law_kind", ["euler", "advection"])
def test_rlsrk54_entropy_conservation_1d(rb, cuda_ok, law_kind):
    """The reference's 1-D tests: a density square wave on [-1, 1], N = 4, K = 5, to
    t = 5 with RLSRK54 and entropy-conservative fluxes: entropy drift within 40 eps."""
    nq, K = 5, 5
    cell = rb.LobattoCell(nq)
    grid = rb.generate(rb.GridManager(cell, rb.brick((rb.jl_range(-1.0, 1.0, K + 1),), (True,))))
    x = grid.points[:, 0, :]
    rho = np.where(np.abs(x) < 0.5, 2.0, 1.0)
    if law_kind == "euler":
        law, flux = rb.EulerLaw(1), rb.EntropyConservativeFlux()
        q = np.zeros((nq, 3, K), order="F")
        q[:, 0], q[:, 1], q[:, 2] = rho, rho, 1.0 / 0.4 + rho * rho / (2 * rho)
        dt = 0.5 * (2.0 / K) / nq / np.sqrt(1.4)
    else:
        law, flux = rb.AdvectionLaw(1, (1.0,)), rb.CentralFlux()
        q = np.asfortranarray(rho[:, None, :].copy())
        dt = 0.25 * (2.0 / K) / nq
    dg = rb.DGSEM(law=law, grid=grid, volume_form=rb.FluxDifferencingForm(flux), surface_numericalflux=flux)
    qg = rb.GridArray.from_numpy(q)
    eta0 = rb.entropyintegral(dg, qg)
    solver = rb.RLSRK54(dg, qg, dt)
    steps = rb.solve(qg, 5.0, solver)
    eta1 = rb.entropyintegral(dg, qg)
    assert steps > 100 and abs(solver.gamma - 1) < 1e-2
    assert abs(eta1 - eta0) / abs(eta0) <= 40 * EPS
