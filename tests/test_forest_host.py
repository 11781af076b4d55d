"""Adapted grids on the host (no GPU): the forest, its 2:1 balance and face geometry,
the mortar operators, and the oracle's mortar coupling.

Tolerances: geometry exact (the small faces' node points lie on the large face);
mortar operators 1e-15; oracle free-stream preservation 1e-12 of the flux scale and
conservation (sum of MJ * dq per field) 1e-14 of sum |MJ * dq|.
"""

import numpy as np
import pytest

import oracle as O


@pytest.fixture(scope="module")
def F(rb):
    from raven_b200 import forest

    return forest


def periodic_warp(K, amp):
    """A smooth warp that fixes the brick's boundary planes (so periodic faces still
    meet): x_d += amp sin(2 pi x_d / K_d) sin(2 pi x_{d+1} / K_{d+1})."""

    def warp(*xs):
        dim = len(xs)
        return [xs[d] + amp * np.sin(2 * np.pi * xs[d] / K[d]) * np.sin(2 * np.pi * xs[(d + 1) % dim] / K[(d + 1) % dim])
                for d in range(dim)]

    return warp


def _adapted(rb, F, dim, nq, K, per, levels, seed=1, center=None, warp=None):
    coords = tuple(rb.jl_range(0.0, float(k), k + 1) for k in K)
    gm = rb.GridManager(rb.LobattoCell(*(nq,) * dim), rb.brick(coords, per), min_level=0)
    rng = np.random.default_rng(seed)
    for _ in range(levels):
        if center is None:
            flags = rng.choice([rb.AdaptNone, rb.AdaptRefine], len(gm))
        else:
            flags = F.sphere_refinement_flags(gm.forest, coords, center, 0.6)
        rb.adapt(gm, flags)
    return (rb.generate(gm) if warp is None else rb.generate(warp, gm)), gm


CASES = [(2, 4, (3, 2), (True, True), 2), (2, 5, (2, 2), (False, True), 3), (3, 3, (2, 2, 2), (True, True, True), 2),
         (3, 4, (2, 1, 2), (True, False, True), 2)]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}d-nq{c[1]}-L{c[4]}")
def test_forest_balanced_and_covering(rb, F, case):
    dim, nq, K, per, levels = case
    grid, gm = _adapted(rb, F, dim, nq, K, per, levels)
    fo = gm.forest
    kinds = set()
    for i in range(len(fo)):
        for f in range(2 * dim):
            kind, _ = fo.face_neighbours(i, f)
            kinds.add(kind)
            assert kind in ("same", "coarser", "finer", "boundary")
    assert "finer" in kinds and "coarser" in kinds
    # the leaves tile the brick: volumes add up, no two leaves share an anchor
    vol = sum(2.0 ** (-dim * lev) for _, lev, _ in fo.leaves)
    assert vol == pytest.approx(np.prod(K), rel=1e-15)
    assert len({fo.global_anchor(L) for L in fo.leaves}) == len(fo)
    # Morton order inside each tree, trees in brick order
    keys = [(L[0], F._morton(L[2], dim)) for L in fo.leaves]
    assert keys == sorted(keys)


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}d-nq{c[1]}-L{c[4]}")
def test_face_geometry(rb, F, case):
    """Conforming faces pair nodes at equal points (the reference's pts[vmapM] ≈
    pts[vmapP] check); small faces lie on the large face of their mortar."""
    dim, nq, K, per, levels = case
    grid, _ = _adapted(rb, F, dim, nq, K, per, levels)
    pts = grid.points
    n = grid.np * grid.E
    X = np.stack([pts[:, d, :].ravel(order="F") for d in range(dim)], axis=1)
    M, P = grid.vmapM.ravel(order="F") - 1, grid.vmapP.ravel(order="F") - 1
    conn = M != P
    diff = np.abs(X[M[conn]] - X[P[conn]])
    for d in range(dim):  # periodic wraps differ by a domain length
        L = float(K[d])
        diff[:, d] = np.minimum(diff[:, d], np.abs(diff[:, d] - L))
    assert diff.max() <= 1e-14 * max(K)
    assert grid.mortars.shape[0] == 2 + 2 ** (dim - 1)
    for col in grid.mortars.T:
        eC, fC = col[0], col[1]
        d = fC // 2
        face = [F.face_node(dim, nq, fC, j) for j in range(grid.nfp)]
        xC = pts[face, :, eC]
        lo, hi = xC.min(0), xC.max(0)
        for k, eF in enumerate(col[2:]):
            xF = pts[[F.face_node(dim, nq, fC ^ 1, j) for j in range(grid.nfp)], :, eF]
            plane = np.abs(xF[:, d] - xC[0, d])
            plane = np.minimum(plane, np.abs(plane - float(K[d])))
            assert plane.max() <= 1e-14 * max(K)
            inface = [e for e in range(dim) if e != d]
            for b, e2 in enumerate(inface):  # small face k covers the half (k >> b) & 1
                mid = (lo[e2] + hi[e2]) / 2
                half = (k >> b) & 1
                assert (xF[:, e2] >= mid - 1e-14).all() if half else (xF[:, e2] <= mid + 1e-14).all()


def test_mortar_operators(rb):
    from raven_b200.grids import lobatto_operators, tohalves_operators

    for nq in range(2, 9):
        r, w, _ = lobatto_operators(nq)
        IL, IU, PL, PU = tohalves_operators(nq)
        assert np.allclose(IL.sum(1), 1, atol=1e-15) and np.allclose(IU.sum(1), 1, atol=1e-15)
        assert np.abs(IL @ r - (r - 1) / 2).max() <= 1e-15
        assert np.abs(IU @ r - (r + 1) / 2).max() <= 1e-15
        f = np.cos(np.arange(nq) + 0.3)
        for Pm in (PL, PU):  # the projection keeps the integral: w . (P f) = (w / 2) . f
            assert abs(w @ (Pm @ f) - (w / 2) @ f) <= 1e-15
        # constants survive interpolation to the halves and the (lumped) projection back
        back = PL @ (IL @ np.ones(nq)) + PU @ (IU @ np.ones(nq))
        assert np.abs(back - 1).max() <= 1e-14


def _oracle(grid, mortars=True):
    return O.Grid.from_arrays(grid.dim, grid.nq, grid.points, grid.volume_metrics, grid.surface_metrics,
                              grid.vmapM, grid.vmapP, grid.boundarycodes,
                              grid.mortars if mortars else None, grid.tohalves if mortars else None,
                              curved=not grid.isunwarpedbrick)


def _state(grid, law, seed):
    x = grid.points
    rng = np.random.default_rng(seed)
    q = np.zeros((grid.np, law.ns, grid.E), order="F")
    if law.ns == 1:
        q[:, 0, :] = 1 + 0.3 * np.sin(2.1 * x[:, 0, :]) * np.cos(1.3 * x[:, 1, :])
    else:
        rho = 1 + 0.2 * np.exp(-((x - 0.7) ** 2).sum(1))
        q[:, 0, :] = rho
        for d in range(grid.dim):
            q[:, 1 + d, :] = rho * 0.1 * np.sin(1.7 * x[:, (d + 1) % grid.dim, :] + d)
        q[:, grid.dim + 1, :] = 2.5 + 0.1 * np.cos(x[:, 0, :])
    return np.asfortranarray(q * (1 + 0.01 * rng.standard_normal(q.shape)))


LAWS = [("eul_kg", O.LAW_EULER, O.FORM_FLUXDIFF, O.FLUX_KG), ("eul_weak", O.LAW_EULER, O.FORM_WEAK, O.FLUX_CENTRAL),
        ("adv_weak", O.LAW_ADVECTION, O.FORM_WEAK, O.FLUX_CENTRAL)]


@pytest.mark.parametrize("lw", LAWS, ids=lambda l: l[0])
@pytest.mark.parametrize("case", [CASES[0], CASES[2]], ids=lambda c: f"{c[0]}d")
def test_oracle_mortars_conserve_and_preserve_free_stream(rb, F, case, lw):
    dim, nq, K, per, levels = case
    grid, _ = _adapted(rb, F, dim, nq, K, (True,) * dim, levels)
    og = _oracle(grid)
    law = O.Law(lw[1], dim, form=lw[2], volume_flux=lw[3], adv=[1.0, 0.5, 0.25][:dim])
    # free stream
    q = np.zeros((grid.np, law.ns, grid.E), order="F")
    const = [1.2, 0.3, -0.1, 0.2, 3.0][: dim + 1] + [3.0] if law.ns > 1 else [1.7]
    for s in range(law.ns):
        q[:, s, :] = const[s]
    assert np.abs(og.tendency(law, q)).max() <= 1e-12
    # conservation on a periodic grid
    q = _state(grid, law, 3)
    dq = og.tendency(law, q)
    MJ = grid.volume_weights()
    for s in range(law.ns):
        tot = (MJ * dq[:, s, :]).sum()
        scale = np.abs(MJ * dq[:, s, :]).sum()
        assert abs(tot) <= 1e-14 * scale, (s, tot, scale)
    # the reference's uncoupled hanging faces do not conserve
    dq0 = _oracle(grid, mortars=False).tendency(law, q)
    lost = max(abs((MJ * dq0[:, s, :]).sum()) / np.abs(MJ * dq0[:, s, :]).sum() for s in range(law.ns))
    assert lost > 1e-8


@pytest.mark.parametrize("lw", LAWS, ids=lambda l: l[0])
@pytest.mark.parametrize("case", [CASES[0], CASES[2]], ids=lambda c: f"{c[0]}d")
def test_oracle_curved_mortars_conserve(rb, F, case, lw):
    """Warped adapted grids: the mortars take the small faces' own normals and surface
    measures, so the coupling conserves to round-off; the affine formula would not.
    Free stream holds up to the mismatch between the large face's polynomial geometry
    and its small faces' (the warp is evaluated at every element's own nodes), which
    falls spectrally with the order."""
    dim, nq, K, per, levels = case
    warp = periodic_warp(K, 0.05)
    grid, _ = _adapted(rb, F, dim, nq, K, (True,) * dim, levels, warp=warp)
    assert not grid.isunwarpedbrick and grid.mortars.size > 0
    law = O.Law(lw[1], dim, form=lw[2], volume_flux=lw[3], adv=[1.0, 0.5, 0.25][:dim])
    q = _state(grid, law, 3)
    MJ = grid.volume_weights()
    dq = _oracle(grid).tendency(law, q)
    for s in range(law.ns):
        assert abs((MJ * dq[:, s, :]).sum()) <= 1e-14 * np.abs(MJ * dq[:, s, :]).sum(), s
    aff = O.Grid.from_arrays(grid.dim, grid.nq, grid.points, grid.volume_metrics, grid.surface_metrics, grid.vmapM,
                             grid.vmapP, grid.boundarycodes, grid.mortars, grid.tohalves, curved=False)
    dq0 = aff.tendency(law, q)
    assert max(abs((MJ * dq0[:, s, :]).sum()) / np.abs(MJ * dq0[:, s, :]).sum() for s in range(law.ns)) > 1e-9
    # free stream: geometric mismatch only, falling with the order
    errs = []
    for n in (4, 8):
        g2, _ = _adapted(rb, F, dim, n, K, (True,) * dim, levels, warp=warp)
        qc = np.zeros((g2.np, law.ns, g2.E), order="F")
        const = [1.2, 0.3, -0.1, 0.2, 3.0][: dim + 1] + [3.0] if law.ns > 1 else [1.7]
        for s in range(law.ns):
            qc[:, s, :] = const[s]
        errs.append(np.abs(_oracle(g2).tendency(law, qc)).max())
    assert errs[1] <= 1e-2 * errs[0]


def test_config5_forest(rb, F):
    """The adapted grid of the benchmark: 4^3 trees on the periodic unit cube, two rounds
    of refinement within radius 0.25 of the centre, 2:1 balanced."""
    coords = tuple(rb.jl_range(0.0, 1.0, 5) for _ in range(3))
    gm = rb.GridManager(rb.LobattoCell(6, 6, 6), rb.brick(coords, (True,) * 3))
    for _ in range(2):
        rb.adapt(gm, F.sphere_refinement_flags(gm.forest, coords, (0.5, 0.5, 0.5), 0.25))
    levels = np.bincount([L[1] for L in gm.forest.leaves])
    assert list(levels) == [32, 192, 512]
    grid = rb.generate(gm)
    assert grid.mortars.shape == (6, 144)
