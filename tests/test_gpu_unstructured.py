"""Grids of unstructured coarse grids on the GPU: faces that meet rotated or on another
face of the neighbour, read through the vmapP table by the generic stage kernel,
against the oracle (which reads vmapP node by node, dgsem.jl:733-784).

Grids: the reference's two-cell meshes in all 2 + 8 orientations of the shared face
(refined once), and the cube shell (cubeshellgrid, warped onto the sphere; its sixth
tree is left-handed, as in the reference).

Tolerances: FP64 tendency and LSRK steps 1e-12 relative per field (max norm), FP32 bulk
tendency 5e-5; free stream on the GPU 1e-12 of the flux scale; rb200_face_vmapP equal
to the grid's vmapP.
"""

import json
import os

import numpy as np
import pytest

import oracle as O
from gpu_util import rel_err

pytestmark = pytest.mark.gpu

FIX = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "coarse_grid_fixtures.json")))["records"]
ROTATED = [i for i, r in enumerate(FIX) if r["source"] == "test/gridnumbering.jl"]

SCHEMES = {
    # name: (oracle law, form, volume flux), product factory
    "eul_kg": (O.LAW_EULER, O.FORM_FLUXDIFF, O.FLUX_KG),
    "eul_weak": (O.LAW_EULER, O.FORM_WEAK, O.FLUX_CENTRAL),
    "adv_weak": (O.LAW_ADVECTION, O.FORM_WEAK, O.FLUX_CENTRAL),
}


def _coarse(rb, k, level, nq=None):
    rec = FIX[k]
    dim = len(rec["vertices"][0])
    n = nq or rec["N"]
    return rb.generate(rb.GridManager(rb.LobattoCell(*(n,) * dim), rb.coarsegrid(rec["vertices"], rec["cells"]),
                                      min_level=level))


def _shell(rb, nq, level):
    return rb.generate(rb.GridManager(rb.LobattoCell(nq, nq, nq), rb.cubeshellgrid(2.0, 1.0), min_level=level))


def _dg(rb, g, scheme, precision="fp64"):
    lo, form, vf = SCHEMES[scheme]
    dim = g.dim
    adv = [1.0, 0.5, 0.25][:dim]
    if lo == O.LAW_ADVECTION:
        law = rb.AdvectionLaw(dim, adv)
    else:
        law = rb.EulerLaw(dim)
    pform = rb.WeakForm() if form == O.FORM_WEAK else rb.FluxDifferencingForm(rb.KennedyGruberFlux())
    dg = rb.DGSEM(law=law, grid=g, volume_form=pform, surface_numericalflux=rb.RusanovFlux(), precision=precision)
    og = O.Grid.from_arrays(dim, g.nq, g.points, g.volume_metrics, g.surface_metrics, g.vmapM, g.vmapP,
                            g.boundarycodes)
    return dg, law, og, O.Law(lo, dim, form=form, volume_flux=vf, adv=adv)


def _state(g, ns, seed):
    x = g.points
    rng = np.random.default_rng(seed)
    q = np.zeros((g.np, ns, g.E), order="F")
    if ns == 1:
        q[:, 0, :] = 1 + 0.3 * np.sin(2.1 * x[:, 0, :]) * np.cos(1.3 * x[:, 1, :])
    else:
        rho = 1 + 0.2 * np.exp(-((x - 0.3) ** 2).sum(1))
        q[:, 0, :] = rho
        for d in range(g.dim):
            q[:, 1 + d, :] = rho * 0.1 * np.sin(1.7 * x[:, (d + 1) % g.dim, :] + d)
        q[:, g.dim + 1, :] = 2.5 + 0.1 * np.cos(x[:, 0, :])
    return np.asfortranarray(q * (1 + 0.01 * rng.standard_normal(q.shape)))


def _check_tendency(rb, g, scheme, tol=1e-12, precision="fp64"):
    dg, law, og, olaw = _dg(rb, g, scheme, precision)
    q = _state(g, law.ns, 3)
    ref = og.tendency(olaw, q)
    qg = rb.GridArray.from_numpy(q)
    dqg = rb.GridArray.from_numpy(np.zeros_like(q))
    dg(dqg, qg, 0.0, increment=False)
    dg.sync_status()
    got = dqg.numpy()
    for s in range(law.ns):
        assert rel_err(got[:, s], ref[:, s]) <= tol, (scheme, s)
    return dg


@pytest.mark.parametrize("scheme", list(SCHEMES))
@pytest.mark.parametrize("k", ROTATED, ids=[f"mesh{k}" for k in ROTATED])
def test_rotated_faces_tendency(rb, cuda_ok, k, scheme):
    g = _coarse(rb, k, 1)
    dg = _check_tendency(rb, g, scheme)
    assert np.array_equal(dg.face_vmapP(), g.vmapP)


@pytest.mark.parametrize("nq", [4, 8])
@pytest.mark.parametrize("scheme", ["eul_kg", "adv_weak"])
def test_cubeshell_tendency(rb, cuda_ok, nq, scheme):
    g = _shell(rb, nq, 1)
    dg = _check_tendency(rb, g, scheme)
    assert dg.pipelined_ctas == 0  # general connectivity runs the generic kernel
    assert np.array_equal(dg.face_vmapP(), g.vmapP)


def test_cubeshell_tendency_fp32_bulk(rb, cuda_ok):
    _check_tendency(rb, _shell(rb, 5, 1), "eul_kg", tol=5e-5, precision="fp32_bulk")


@pytest.mark.parametrize("stepper", ["lsrk54", "lsrk144"])
def test_cubeshell_steps(rb, cuda_ok, stepper):
    g = _shell(rb, 5, 1)
    dg, law, og, olaw = _dg(rb, g, "eul_kg")
    q = _state(g, law.ns, 4)
    dt = 1e-3
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(5):
        getattr(og, f"{stepper}_step")(olaw, qo, dqo, i * dt, dt)
    qg = rb.GridArray.from_numpy(q)
    solver = (rb.LSRK54 if stepper == "lsrk54" else rb.LSRK144)(dg, qg, dt)
    solver.dostep(qg, 5)
    dg.sync_status()
    got = qg.numpy()
    for s in range(law.ns):
        assert rel_err(got[:, s], qo[:, s]) <= 1e-12, s


def test_cubeshell_free_stream(rb, cuda_ok):
    g = _shell(rb, 6, 1)
    dg, law, og, olaw = _dg(rb, g, "eul_kg")
    q = np.zeros((g.np, 5, g.E), order="F")
    q[:, 0, :], q[:, 1, :], q[:, 2, :], q[:, 3, :], q[:, 4, :] = 1.2, 0.3, -0.2, 0.1, 3.0
    qg = rb.GridArray.from_numpy(q)
    dqg = rb.GridArray.from_numpy(np.zeros_like(q))
    dg(dqg, qg, 0.0, increment=False)
    dg.sync_status()
    scale = np.abs(q).max() ** 2 / g.min_node_distance()
    assert np.abs(dqg.numpy()).max() <= 1e-12 * scale
