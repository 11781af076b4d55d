"""Unstructured coarse grids on the host (no GPU): face maps through rotated and
re-labelled tree faces, boundary codes, the cube shell, and the oracle on such grids.

The meshes are the reference's own (tests/golden/coarse_grid_fixtures.json, extracted
from test/gridnumbering.jl and test/grids.jl by make_coarse_goldens.py): two cells
whose shared face meets in each of the 2 (quadrilateral) and 8 (hexahedral) relative
orientations.  The checks are the reference's (test/gridnumbering.jl:340-360,
546-566): points(vmapM) = points(vmapP), and the faces with boundary code 1 are the
faces on the outer boundary max|x| = 1.

Tolerances: node coincidence 1e-14 (exact up to the trilinear interpolation's
round-off); cube shell radii 1e-14; oracle free-stream residual 1e-12 of the flux
scale.
"""

import json
import os

import numpy as np
import pytest

import oracle as O

FIX = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "coarse_grid_fixtures.json")))["records"]


def _grid(rb, rec, level, nq=None):
    dim = len(rec["vertices"][0])
    n = nq or rec["N"]
    gm = rb.GridManager(rb.LobattoCell(*(n,) * dim), rb.coarsegrid(rec["vertices"], rec["cells"]), min_level=level)
    return rb.generate(gm)


def _flat_points(g):
    return np.stack([g.points[:, d, :].reshape(-1, order="F") for d in range(g.dim)], 1)


@pytest.mark.parametrize("level", [0, 1, 2])
@pytest.mark.parametrize("k", range(len(FIX)), ids=[f"{r['source'][5:-3]}{i}" for i, r in enumerate(FIX)])
def test_face_maps_pair_coincident_nodes(rb, k, level):
    rec = FIX[k]
    g = _grid(rb, rec, level)
    pts = _flat_points(g)
    vM = g.vmapM.reshape(-1, order="F") - 1
    vP = g.vmapP.reshape(-1, order="F") - 1
    assert np.abs(pts[vM] - pts[vP]).max() <= 1e-14 * max(1.0, np.abs(pts).max())
    # every connected face node is paired back: vmapP is an involution on face nodes
    # (a corner node lies on several faces: some face slot holding p must point back at m)
    pairs = set(zip(vM.tolist(), vP.tolist()))
    bnd = np.repeat(g.boundarycodes.reshape(-1, order="F") == 1, g.nfp)
    for m, p in zip(vM[~bnd].tolist(), vP[~bnd].tolist()):
        assert (p, m) in pairs
    assert np.array_equal(vP[bnd], vM[bnd])
    assert len(g.boundarycodes.reshape(-1)) == 2 * g.dim * g.E


@pytest.mark.parametrize("k", [i for i, r in enumerate(FIX) if r["source"] == "test/gridnumbering.jl"])
def test_boundary_codes_on_the_outer_boundary(rb, k):
    rec = FIX[k]
    g = _grid(rb, rec, 1)
    pts = _flat_points(g)
    vM = (g.vmapM - 1).reshape(g.nfp, 2 * g.dim, g.E, order="F")
    for e in range(g.E):
        for f in range(2 * g.dim):
            on_box = np.isclose(np.abs(pts[vM[:, f, e]]).max(1), 1.0, rtol=0, atol=1e-14)
            if g.boundarycodes[f, e] == 1:
                assert on_box.all()
            else:
                assert not on_box.all()


def test_shared_face_meets_rotated(rb):
    """The hexahedral fixtures do exercise orientations other than the aligned one: the
    shared face's node order differs from the implied (brick) order."""
    nontrivial = 0
    for rec in FIX:
        if rec["source"] != "test/gridnumbering.jl" or len(rec["vertices"][0]) != 3:
            continue
        g = _grid(rb, rec, 0)
        f0 = [f for f in range(6) if g.boundarycodes[f, 0] == 0][0]
        rows = slice(f0 * g.nfp, (f0 + 1) * g.nfp)
        p = g.vmapP[rows, 0] - 1 - g.np
        from raven_b200.grids import face_node

        fB = [f for f in range(6) if g.boundarycodes[f, 1] == 0][0]
        implied = np.array([face_node(3, g.nq, fB, j) for j in range(g.nfp)])
        nontrivial += int(not np.array_equal(p, implied))
    assert nontrivial >= 7


@pytest.mark.parametrize("level", [0, 1, 2])
def test_cubeshell(rb, level):
    R, r = 2.0, 1.0
    g = rb.generate(rb.GridManager(rb.LobattoCell(5, 5, 5), rb.cubeshellgrid(R, r), min_level=level))
    assert g.E == 6 * 8**level
    pts = _flat_points(g)
    vM = g.vmapM.reshape(-1, order="F") - 1
    vP = g.vmapP.reshape(-1, order="F") - 1
    assert np.abs(pts[vM] - pts[vP]).max() <= 1e-14 * R
    rad = np.sqrt((pts**2).sum(1))
    assert rad.min() >= r * (1 - 1e-14) and rad.max() <= R * (1 + 1e-14)
    bnd = np.repeat(g.boundarycodes.reshape(-1, order="F") == 1, g.nfp)
    rb_ = rad[vM[bnd]]
    assert np.all(np.isclose(rb_, r, rtol=1e-14) | np.isclose(rb_, R, rtol=1e-14))
    assert bnd.sum() == 2 * 6 * 4**level * g.nfp
    # |wJ| integrates the shell's volume (spectrally accurate)
    vol = np.abs(g.volume_weights()).sum()
    assert vol == pytest.approx(4 / 3 * np.pi * (R**3 - r**3), rel=1e-3 / 4**level)
    # the reference's sixth tree (1, 2, 5, 6, 9, 10, 13, 14) is left-handed: its J < 0
    J = g.volume_metrics[:, 9, :]
    nqt = 8**level
    assert (J[:, :5 * nqt] > 0).all() and (J[:, 5 * nqt:] < 0).all()


def _oracle(g):
    return O.Grid.from_arrays(g.dim, g.nq, g.points, g.volume_metrics, g.surface_metrics, g.vmapM, g.vmapP,
                              g.boundarycodes)


@pytest.mark.parametrize("which", ["hex-rotated", "quad-rotated", "cubeshell"])
def test_oracle_free_stream(rb, which):
    """A constant state has zero tendency on these grids (discrete metric identities and
    consistent face pairing), for flux differencing and the weak form."""
    if which == "cubeshell":
        g = rb.generate(rb.GridManager(rb.LobattoCell(4, 4, 4), rb.cubeshellgrid(2.0, 1.0), min_level=1))
    else:
        rec = [r for r in FIX if r["source"] == "test/gridnumbering.jl" and
               len(r["vertices"][0]) == (3 if which == "hex-rotated" else 2)][-1]
        g = _grid(rb, rec, 1)
    og = _oracle(g)
    dim = g.dim
    for form, vf in ((O.FORM_FLUXDIFF, O.FLUX_KG), (O.FORM_WEAK, O.FLUX_CENTRAL)):
        law = O.Law(O.LAW_EULER, dim, form=form, volume_flux=vf)
        q = np.zeros((g.np, dim + 2, g.E), order="F")
        q[:, 0, :] = 1.2
        for d in range(dim):
            q[:, 1 + d, :] = 0.3 * (d + 1)
        q[:, dim + 1, :] = 3.0
        dq = og.tendency(law, q)
        scale = np.abs(q).max() ** 2 / g.min_node_distance()
        assert np.abs(dq).max() <= 1e-12 * scale
