"""The oracle against the reference's own known-answer values.

Every ``expected_error`` of ``test/balancelaws/{advection,euler}/*.jl`` (all refinement
levels) is reproduced by the oracle's brick grid + DGSEM tendency + LSRK(5,4) to the
tolerance the reference test itself applies (``≈``: rtol sqrt(eps); ``10sqrt(eps)`` for
the 1-D files), and both golden ``vmapP`` vectors of ``test/gridnumbering.jl:369-386``
are reproduced bit for bit.
"""

import json
import math
import os

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_goldens.json")))

FORMS = {
    "weak": (O.FORM_WEAK, O.FLUX_CENTRAL),
    "fd_central": (O.FORM_FLUXDIFF, O.FLUX_CENTRAL),
    "fd_ec": (O.FORM_FLUXDIFF, O.FLUX_EC),
}


def run_reference_case(entry):
    """Restates the `run` function of the reference test file named in `entry`."""
    test, law, form, lev = entry["test"], entry["law"], entry["form"], entry["level"]
    N = 4
    K = 5 * 2 ** (lev - 1)
    fm, vf = FORMS[form]
    if test == "isentropicvortex":  # test/balancelaws/euler/isentropicvortex.jl:36-85
        L = O.Law(O.LAW_EULER, 2, form=fm, volume_flux=vf)
        g = O.Grid(2, N + 1, [K, K], [0.0, -5.0], [20.0, 5.0], [True, True])
        dt = 0.25 * (10.0 / K) / N
        T, kind = 5.0, 2
    else:
        dim = int(test[-2])
        g = O.Grid(dim, N + 1, [K] * dim, [-1.0] * dim, [1.0] * dim, [True] * dim)
        cfl = 0.5 if dim == 1 else 0.25
        if law == "advection":  # test/balancelaws/advection/wave_*d.jl:23-71
            L = O.Law(O.LAW_ADVECTION, dim, form=fm, volume_flux=vf)
            dt = cfl * (2.0 / K) / N / math.sqrt(dim)
            T, kind = 0.7, 0
        else:  # test/balancelaws/euler/wave_*d.jl
            L = O.Law(O.LAW_EULER, dim, form=fm, volume_flux=vf)
            dt = cfl * (2.0 / K) / N / math.sqrt(1.4)
            T = dt if dim == 3 else 0.7  # wave_3d.jl:61 runs a single step
            kind = 1
    q = g.initial_condition(L, kind)
    g.solve(L, q, dt, T)
    qe = g.initial_condition(L, kind, t=T)
    err, _ = g.weightednorm(q - qe, L.ns)
    return err


@pytest.mark.parametrize(
    "entry", GOLD["errors"], ids=[f"{e['law']}-{e['test']}-{e['form']}-L{e['level']}" for e in GOLD["errors"]]
)
def test_golden_l2_error(entry):
    err = run_reference_case(entry)
    assert err == pytest.approx(entry["expected"], rel=entry["rtol"]), entry["source"]


@pytest.mark.parametrize("entry", GOLD["vmapP"], ids=[f"{v['dim']}d" for v in GOLD["vmapP"]])
def test_golden_vmapP(entry):
    d = entry["dim"]
    g = O.Grid(d, entry["nq"], entry["elements_per_side"], [0.0] * d, [1.0] * d, entry["periodic"])
    assert g.vmapP().ravel(order="F").tolist() == entry["vmapP"], entry["source"]


def test_face_maps_match_points():
    """pts[vmapM] == pts[vmapP] on periodic-interior faces (test/gridnumbering.jl:342-343)."""
    for dim, K in ((2, (3, 4)), (3, (3, 2, 5))):
        g = O.Grid(dim, 4, K, [0.0] * dim, [1.0] * dim, [False] * dim)
        pts = g.points()
        flat = np.moveaxis(pts, 1, 2).reshape(-1, dim, order="F")
        vm, vp = g.vmapM().ravel(order="F") - 1, g.vmapP().ravel(order="F") - 1
        assert np.allclose(flat[vm], flat[vp])
        # boundary faces map to themselves and are flagged
        bc = g.boundary()
        assert (bc.sum() > 0) and np.all((vm == vp)[np.repeat(bc.ravel(order="F") > 0, g.nfp)])


def test_lgl_operators():
    r, w, D = O.lgl(5)
    assert np.allclose(r, [-1.0, -math.sqrt(3 / 7), 0.0, math.sqrt(3 / 7), 1.0], rtol=2e-16, atol=0)
    assert r[0] == -1.0 and r[2] == 0.0 and r[4] == 1.0 and r[1] == -r[3]
    assert np.allclose(w, [0.1, 49 / 90, 32 / 45, 49 / 90, 0.1], rtol=0, atol=1e-16)
    # D differentiates polynomials of degree <= N exactly
    for k in range(5):
        assert np.allclose(D @ r**k, k * r ** max(k - 1, 0) if k else 0 * r, atol=1e-13)


def test_brick_morton_order():
    """p4est brick trees follow a Morton curve (x lowest bit) for power-of-two bricks."""
    g = O.Grid(3, 2, [4, 4, 4], [0.0] * 3, [1.0] * 3, [True] * 3)
    t = g.tree_coords()
    for e in range(g.E):
        x = y = z = 0
        for b in range(2):
            x |= ((e >> (3 * b)) & 1) << b
            y |= ((e >> (3 * b + 1)) & 1) << b
            z |= ((e >> (3 * b + 2)) & 1) << b
        assert tuple(t[:, e]) == (x, y, z)


@pytest.mark.parametrize("p", [1, 2, 3, 2.5, math.inf])
def test_oracle_weightednorm_p(p):
    """The oracle's weightednorm(dg, q, p) against numpy, formula by formula
    (measures.jl:6-21: weighted p-sums per field, unweighted maximum for p = Inf, then
    LinearAlgebra.norm over the fields)."""
    g = O.Grid(2, 4, [3, 2], [0.0, 0.0], [1.0, 2.0], [True, True])
    L = O.Law(O.LAW_EULER, 2)
    rng = np.random.default_rng(7)
    q = np.asfortranarray(rng.standard_normal((g.np, L.ns, g.E)))
    mj = g.volume_metrics()[:, -1, :]
    tot, comp = g.weightednorm_p(q, L.ns, p)
    if math.isinf(p):
        want = [float(np.abs(q[:, s]).max()) for s in range(L.ns)]
        assert list(comp) == want and tot == max(want)
    else:
        want = [float((mj * np.abs(q[:, s]) ** p).sum() ** (1 / p)) for s in range(L.ns)]
        assert np.allclose(comp, want, rtol=1e-14, atol=0)
        assert tot == pytest.approx(np.linalg.norm(want, p), rel=1e-14)
    if p == 2:
        t2, c2 = g.weightednorm(q, L.ns)
        assert tot == pytest.approx(t2, rel=1e-15) and np.allclose(comp, c2, rtol=1e-15, atol=0)


def test_oracle_lsrk144_matches_lsrk54_golden():
    """LSRK144 (odesolvers.jl:191-239) in the setting of the reference's 2-D advection wave
    test (K = 5, N = 4, weak form, t = 0.7, the test's dt): the 14-stage fourth-order
    scheme gives the L2 error of the LSRK54 golden value to 1e-3 relative (the spatial
    error dominates; the two schemes' time errors differ by ~2e-4 of it), and its state
    differs from LSRK54's by time-discretisation error only."""
    entry = next(e for e in GOLD["errors"] if e["test"] == "wave_2d" and e["law"] == "advection"
                 and e["form"] == "weak" and e["level"] == 1)
    K, N = 5, 4
    L = O.Law(O.LAW_ADVECTION, 2, form=O.FORM_WEAK)
    g = O.Grid(2, N + 1, [K, K], [-1.0, -1.0], [1.0, 1.0], [True, True])
    dt = 0.25 * (2.0 / K) / N / math.sqrt(2)
    T = 0.7
    q54, q144 = g.initial_condition(L, 0), g.initial_condition(L, 0)
    dq54, dq144 = g.state(L), g.state(L)
    t, n = 0.0, 0
    while True:
        final = t + dt >= T
        h = T - t if final else dt
        g.lsrk54_step(L, q54, dq54, t, h)
        g.lsrk144_step(L, q144, dq144, t, h)
        t += h
        n += 1
        if final:
            break
    qe = g.initial_condition(L, 0, t=T)
    e54, _ = g.weightednorm(q54 - qe, L.ns)
    e144, _ = g.weightednorm(q144 - qe, L.ns)
    assert e54 == pytest.approx(entry["expected"], rel=entry["rtol"])
    assert e144 == pytest.approx(entry["expected"], rel=1e-3)
    assert np.abs(q144 - q54).max() < 1e-5  # time error; the spatial error is ~1e-3 in max norm


@pytest.mark.parametrize("form,vf", [(O.FORM_WEAK, O.FLUX_CENTRAL), (O.FORM_FLUXDIFF, O.FLUX_KG),
                                     (O.FORM_FLUXDIFF, O.FLUX_EC)], ids=["weak", "kg", "ec"])
@pytest.mark.parametrize("dim,warp", [(2, O.WARP_NONE), (3, O.WARP_NONE), (3, O.WARP_SINE)])
def test_oracle_directions_split_the_tendency(dim, warp, form, vf):
    """DGSEM(; directions) (dgsem.jl:46-81): the volume and surface terms are sums over
    directions, so the tendencies of the single directions add up to the full one
    (1e-13 of its scale), and a subset that holds every direction is the full tendency
    bit for bit."""
    nq, K = 4, (3, 2, 2)[:dim]
    og = O.Grid(dim, nq, K, [0.0] * dim, [10.0] * dim, [True] * dim, warp, 0.1 if warp == O.WARP_SINE else 0.0)
    law = O.Law(O.LAW_EULER, dim, form=form, volume_flux=vf)
    q = og.initial_condition(law, 1)
    q = np.asfortranarray(q * (1 + 0.01 * np.random.default_rng(5).standard_normal(q.shape)))
    full = og.tendency(law, q)
    parts = np.zeros_like(full)
    for d in range(1, dim + 1):
        og.set_directions([d])
        parts += og.tendency(law, q)
    assert np.abs(parts - full).max() <= 1e-13 * np.abs(full).max()
    og.set_directions(range(1, dim + 1))
    assert np.array_equal(og.tendency(law, q), full)
