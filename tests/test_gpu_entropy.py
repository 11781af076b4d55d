"""GPU parity for the entropy-family surface fluxes, the entropy measures and RLSRK(5,4).

Tolerances:
  * tendency with the Roe, matrix, EC and KG surface fluxes (FP64): max |gpu - oracle| <=
    1e-12 * max |oracle| per field, conforming and mortar grids;
  * entropyintegral / entropyproduct: 1e-13 relative;
  * RLSRK54 steps: state 1e-12 relative per field, relaxation parameter 1e-9 absolute;
  * entropy conservation of RLSRK54 with EC fluxes on the 1-D reference problem extruded
    to 2-D (one periodic element across): |eta_f - eta_0| / |eta_0| <= 40 eps, the bound
    of test/balancelaws/{euler,advection}/entropy_conservation_1d.jl.
"""

import numpy as np
import pytest

import oracle as O
from gpu_util import initial_state, oracle_law, product_scheme, rel_err, wrap_oracle_grid

pytestmark = pytest.mark.gpu

EPS = np.finfo(float).eps
FLUXES = ["roe", "matrix", "ec", "kg"]
OFLUX = {"roe": O.FLUX_ROE, "matrix": O.FLUX_MATRIX, "ec": O.FLUX_EC, "kg": O.FLUX_KG, "rusanov": O.FLUX_RUSANOV,
         "central": O.FLUX_CENTRAL}


def _pflux(rb, name):
    return {"roe": rb.RoeFlux, "matrix": rb.MatrixFlux, "ec": rb.EntropyConservativeFlux,
            "kg": rb.KennedyGruberFlux, "rusanov": rb.RusanovFlux, "central": rb.CentralFlux}[name]()


CASES = [
    # dim, nq, K, periodic, scheme, warp
    (2, 5, (3, 4), (1, 1), "eul_weak", O.WARP_NONE),
    (2, 6, (3, 3), (1, 0), "eul_kg", O.WARP_SINE),
    (3, 4, (2, 2, 3), (1, 1, 1), "eul_ec", O.WARP_NONE),
    (3, 5, (2, 2, 2), (1, 1, 0), "eul_fdc", O.WARP_SINE),
    (3, 8, (2, 2, 2), (1, 1, 1), "eul_kg", O.WARP_NONE),
]


def _build(rb, dim, nq, K, per, scheme, warp, sflux, precision="fp64"):
    og = O.Grid(dim, nq, K, [0.0] * dim, [10.0] * dim, per, warp, 0.1 if warp == O.WARP_SINE else 0.0)
    g = wrap_oracle_grid(og)
    law, form = product_scheme(rb, scheme, dim)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=_pflux(rb, sflux), precision=precision)
    olaw = oracle_law(scheme, dim)
    olaw.c.surface_flux = OFLUX[sflux]
    return og, dg, olaw, law


def _id(c):
    return f"{c[0]}d-nq{c[1]}-{c[4]}-warp{c[5]}"


@pytest.mark.parametrize("sflux", FLUXES)
@pytest.mark.parametrize("case", CASES, ids=[_id(c) for c in CASES])
def test_surface_flux_tendency(rb, cuda_ok, case, sflux):
    og, dg, olaw, law = _build(rb, *case, sflux)
    q = initial_state(og, olaw, case[4], seed=11)
    ref = og.tendency(olaw, q)
    qg = rb.GridArray.from_numpy(q)
    dqg = qg.similar()
    dg(dqg, qg, 0.0, increment=False)
    dg.sync_status()
    got = dqg.numpy()
    for s in range(law.ns):
        assert rel_err(got[:, s], ref[:, s]) <= 1e-12, f"field {s}"


@pytest.mark.parametrize("sflux", ["roe", "matrix"])
@pytest.mark.parametrize("dim", [2, 3])
def test_surface_flux_mortars(rb, cuda_ok, dim, sflux):
    from test_forest_host import _adapted, _oracle, _state

    from raven_b200 import forest

    K = (3, 2) if dim == 2 else (2, 2, 2)
    grid, _ = _adapted(rb, forest, dim, 4, K, (True,) * dim, 2)
    dg = rb.DGSEM(law=rb.EulerLaw(dim), grid=grid, volume_form=rb.FluxDifferencingForm(rb.KennedyGruberFlux()),
                  surface_numericalflux=_pflux(rb, sflux))
    olaw = O.Law(O.LAW_EULER, dim, form=O.FORM_FLUXDIFF, volume_flux=O.FLUX_KG, surface_flux=OFLUX[sflux])
    q = _state(grid, olaw, 12)
    ref = _oracle(grid).tendency(olaw, q)
    qg = rb.GridArray.from_numpy(q)
    dqg = qg.similar()
    dg(dqg, qg, 0.0, increment=False)
    got = dqg.numpy()
    for s in range(olaw.ns):
        assert rel_err(got[:, s], ref[:, s]) <= 1e-12, s
    MJ = grid.volume_weights()
    for s in range(olaw.ns):  # the mortar coupling stays conservative with these fluxes
        assert abs((MJ * got[:, s]).sum()) <= 1e-13 * np.abs(MJ * got[:, s]).sum()


@pytest.mark.parametrize("scheme,dim,warp", [("eul_kg", 2, O.WARP_NONE), ("eul_kg", 3, O.WARP_SINE),
                                             ("adv_weak", 2, O.WARP_SINE), ("adv_weak", 3, O.WARP_NONE)])
def test_entropy_measures(rb, cuda_ok, scheme, dim, warp):
    K = (3, 4) if dim == 2 else (2, 3, 2)
    sflux = "rusanov"
    og, dg, olaw, law = _build(rb, dim, 5, K, (1,) * dim, scheme, warp, sflux)
    q = initial_state(og, olaw, scheme, seed=13)
    k = initial_state(og, olaw, scheme, seed=14)
    ref = og.entropy_sums(olaw, q, None, 0.0, k)
    qg, kg = rb.GridArray.from_numpy(q), rb.GridArray.from_numpy(k)
    assert rb.entropyintegral(dg, qg) == pytest.approx(ref[0], rel=1e-13)
    assert rb.entropyproduct(dg, qg, kg) == pytest.approx(ref[1], rel=1e-13)


@pytest.mark.parametrize("case,sflux", [((2, 5, (3, 3), (1, 1), "eul_ec", O.WARP_NONE), "ec"),
                                        ((3, 4, (2, 2, 2), (1, 1, 1), "eul_ec", O.WARP_NONE), "matrix"),
                                        ((2, 4, (3, 2), (1, 1), "eul_kg", O.WARP_SINE), "roe"),
                                        ((3, 4, (2, 2, 2), (1, 1, 1), "adv_fdc", O.WARP_NONE), "central")],
                         ids=["2d-ec", "3d-matrix", "2d-curved-roe", "3d-adv"])
def test_rlsrk54_steps(rb, cuda_ok, case, sflux):
    og, dg, olaw, law = _build(rb, *case, sflux)
    q = initial_state(og, olaw, case[4], seed=15, amp=0.01)
    dt, steps = 2e-2, 4
    qo, dqo, go = q.copy(order="F"), og.state(olaw), np.ones(1)
    for i in range(steps):
        og.rlsrk54_step(olaw, qo, dqo, go, i * dt, dt)
    qg = rb.GridArray.from_numpy(q)
    solver = rb.RLSRK54(dg, qg, dt)
    solver.dostep(qg, 2)
    solver.dostep(qg, 2)
    got = qg.numpy()
    for s in range(law.ns):
        assert rel_err(got[:, s], qo[:, s]) <= 1e-12, s
    assert abs(solver.gamma - go[0]) <= 1e-9
    assert solver.gamma != 1.0


@pytest.mark.parametrize("law_kind", ["euler", "advection"])
def test_rlsrk54_entropy_conservation_extruded(rb, cuda_ok, law_kind):
    """The reference's 1-D entropy-conservation tests (N = 4, K = 5, t = 5) on a 2-D grid
    one periodic element across, with the fluxes the tests use."""
    nq, K = 5, 5
    og = O.Grid(2, nq, [K, 1], [-1.0, 0.0], [1.0, 1.0], [True, True])
    g = wrap_oracle_grid(og)
    x = og.points()
    rho = np.where(np.abs(x[:, 0, :]) < 0.5, 2.0, 1.0)
    if law_kind == "euler":
        law, flux = rb.EulerLaw(2), rb.EntropyConservativeFlux()
        q = np.zeros((og.np, 4, og.E), order="F")
        q[:, 0], q[:, 1], q[:, 3] = rho, rho, 1.0 / 0.4 + rho * rho / (2 * rho)
        dt = 0.5 * 0.4 / nq / np.sqrt(1.4)
    else:
        law, flux = rb.AdvectionLaw(2, (1.0, 0.0)), rb.CentralFlux()
        q = np.asfortranarray(rho[:, None, :].copy())
        dt = 0.25 * 0.4 / nq
    dg = rb.DGSEM(law=law, grid=g, volume_form=rb.FluxDifferencingForm(flux), surface_numericalflux=flux)
    qg = rb.GridArray.from_numpy(q)
    eta0 = rb.entropyintegral(dg, qg)
    solver = rb.RLSRK54(dg, qg, dt)
    steps = rb.solve(qg, 5.0, solver)
    eta1 = rb.entropyintegral(dg, qg)
    assert steps > 100
    assert abs(eta1 - eta0) / abs(eta0) <= 40 * EPS


def test_unsupported_combinations(rb, cuda_ok):
    case = (2, 4, (3, 3), (1, 1), "eul_kg", O.WARP_NONE)
    with pytest.raises(rb.RB200Error) as ei:
        _build(rb, *case, "roe", precision="fp32_bulk")
    assert ei.value.status == 6
    with pytest.raises(rb.RB200Error) as ei:
        _build(rb, 2, 4, (3, 3), (1, 1), "adv_weak", O.WARP_NONE, "matrix")
    assert ei.value.status == 6
    og, dg, olaw, law = _build(rb, *case, "rusanov", precision="fp32_bulk")
    qg = rb.GridArray.from_numpy(initial_state(og, olaw, "eul_kg", seed=1))
    with pytest.raises(rb.RB200Error) as ei:
        rb.RLSRK54(dg, qg, 1e-3).dostep(qg, 1)
    assert ei.value.status == 6


@pytest.mark.parametrize("precision,stepper", [("fp64", "lsrk"), ("fp32_bulk", "lsrk"), ("fp64", "rlsrk")])
def test_snapshot_resume(rb, cuda_ok, precision, stepper):
    """Resuming from a snapshot reproduces the uninterrupted run bit for bit."""
    import struct

    case = (3, 5, (2, 2, 2), (1, 1, 1), "eul_kg", O.WARP_NONE)
    og, dg, olaw, law = _build(rb, *case, "ec" if stepper == "rlsrk" else "rusanov", precision=precision)
    q0 = initial_state(og, olaw, "eul_kg", seed=16, amp=0.01)
    qg = rb.GridArray.from_numpy(q0)
    mk = rb.RLSRK54 if stepper == "rlsrk" else rb.LSRK54
    solver = mk(dg, qg, 1e-2)
    solver.dostep(qg, 3)
    snap = rb.snapshot(dg, qg, solver)
    magic, version, hbytes = struct.unpack_from("<8sII", snap, 0)
    assert magic == b"RB200SNP" and version == 1 and hbytes == 128
    solver.dostep(qg, 3)
    want, want_t = qg.numpy(), solver.time
    q2 = rb.GridArray.from_numpy(np.zeros_like(q0))
    s2 = mk(dg, q2, 5.0)
    rb.restore(dg, snap, q2, s2)
    assert s2.dt == 1e-2 and s2.time == pytest.approx(3e-2, abs=0)
    s2.dostep(q2, 3)
    assert np.array_equal(q2.numpy(), want) and s2.time == want_t
    bad = bytearray(snap)
    bad[-3] ^= 0x10
    with pytest.raises(rb.RB200Error) as ei:
        rb.restore(dg, bytes(bad), q2, s2)
    assert ei.value.status == 1
    other = _build(rb, 3, 5, (2, 2, 3), (1, 1, 1), "eul_kg", O.WARP_NONE, "rusanov", precision=precision)[1]
    with pytest.raises(rb.RB200Error) as ei:
        rb.restore(other, snap, q2, s2)
    assert ei.value.status == 2
