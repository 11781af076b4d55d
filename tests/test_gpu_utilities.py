"""The utilities' CUDA kernels (rb200_kron_apply, rb200_gather, rb200_scatter,
rb200_decode_facecodes) against the oracle: bit-exact for every case (integer codes,
index maps, and floating-point results computed in the reference's order)."""

import json
import os

import numpy as np
import pytest

import oracle as O
from test_utilities_host import _brick, _mats, kron_cases

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def U(rb, cuda_ok):
    from raven_b200 import utilities

    return utilities


def test_decode_all_codes(U):
    import torch

    c8 = np.arange(256, dtype=np.uint8)
    got8 = U.decode(torch.from_numpy(c8).cuda()).cpu().numpy()
    assert np.array_equal(got8, O.decode(c8))
    c16 = np.arange(65536, dtype=np.uint16)
    got16 = U.decode(torch.from_numpy(c16.view(np.int16)).cuda()).cpu().numpy()
    assert np.array_equal(got16, O.decode(c16))
    with open(os.path.join(HERE, "golden", "facecode_goldens.json")) as f:
        d = json.load(f)
    for code, hf, he in d["uint16"]:
        assert got16[code].tolist() == hf + he
    for code, hf in d["uint8"]:
        assert got8[code].tolist() == hf


def _uargs(U, args):
    return tuple(U.Eye(a[1]) if isinstance(a, tuple) else a for a in args)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_kron_columns_bit_exact(U, dt):
    import torch

    rng = np.random.default_rng(37)
    for args in kron_cases(rng):
        mats, sizes, K = _mats(args, dt)
        ncol, C = 12, 2
        f = rng.random((ncol, K.shape[1], C)).astype(dt)
        ref = O.kron_apply(mats, sizes, f.ravel(), ncomp=C, in_strides=(C, 1, C * K.shape[1]),
                           out_strides=(C, 1, C * K.shape[0]), ncol=ncol).reshape(ncol, K.shape[0], C)
        kr = U.Kron(tuple(a.astype(dt) if not isinstance(a, U.Eye) else a for a in _uargs(U, args)))
        got = (kr * torch.from_numpy(f).cuda()).cpu().numpy()
        assert np.array_equal(got, ref), args
        v = rng.random(K.shape[1]).astype(dt)  # a plain vector
        refv = O.kron_apply(mats, sizes, v, ncomp=1, ncol=1)
        gotv = (kr * torch.from_numpy(v).cuda()).cpu().numpy()
        assert np.array_equal(gotv, refv), args


def test_kron_gridarray_bit_exact(rb, U):
    """Kron * GridArray on a 3-D grid of LobattoCell(2, 3, 5) (kron3dgridarray_testsuite)."""
    rng = np.random.default_rng(37)
    A, B, C = rng.random((5, 2)), rng.random((2, 3)), rng.random((3, 5))
    E, ns, nin = 8, 2, 2 * 3 * 5
    q = np.asfortranarray(rng.random((nin, ns, E)))
    for args in [(U.Eye(5), U.Eye(3), A), (U.Eye(5), B, U.Eye(2)), (C, U.Eye(3), U.Eye(2)), (U.Eye(5), B, A),
                 (C, U.Eye(3), A), (C, B, U.Eye(2)), (C, B, A)]:
        facs = list(reversed(args))
        mats = [None if isinstance(a, U.Eye) else a for a in facs]
        sizes = [a.shape[0] for a in facs]
        kr = U.Kron(args)
        nout = kr.size(1)
        ref = O.kron_apply(mats, sizes, q.ravel(order="F"), ncomp=ns, in_strides=(1, nin, nin * ns),
                           out_strides=(1, nout, nout * ns), ncol=E).reshape((nout, ns, E), order="F")
        got = (kr * rb.GridArray.from_numpy(q)).numpy()
        assert np.array_equal(got, ref)
        dense = np.einsum("ij,jse->ise", kr.collect(), q)
        assert np.abs(got - dense).max() <= 1e-14 * np.abs(dense).max()


@pytest.mark.parametrize("dim,nq,K,per", [(2, 4, (3, 2), (False, False)), (3, 3, (2, 2, 3), (True, False, True))])
def test_gather_scatter_bit_exact(rb, U, dim, nq, K, per):
    import torch

    grid = _brick(rb, dim, nq, K, per)
    dtoc, colptr, rowval = U.continuous_maps(grid)
    nc, n, ns = colptr.size - 1, grid.np * grid.E, 3
    rng = np.random.default_rng(5)
    q = np.asfortranarray(rng.standard_normal((grid.np, ns, grid.E)))
    dl = (grid.np, 1, grid.np * ns, grid.np)
    cl = (nc, ns, 0, 1)
    for op, opname, init in [(0, "+", 0.0), (1, "min", np.inf), (2, "max", -np.inf)]:
        ref = O.gather(np.zeros(nc * ns), cl, q.ravel(order="F"), dl, colptr, rowval, ns, op=op, init=init)
        dest = torch.zeros((nc, ns), dtype=torch.float64, device="cuda")
        U.gather(dest, rb.GridArray.from_numpy(q), colptr, rowval, op=opname, init=init)
        assert np.array_equal(dest.cpu().numpy().ravel(), ref), opname
    c = rng.standard_normal((nc, ns))
    ref = O.scatter(np.zeros(n * ns), dl, c.ravel(), cl, dtoc.ravel(order="F"), ns)
    out = rb.GridArray(torch.zeros((grid.E, ns, grid.np), dtype=torch.float64, device="cuda"), ns, grid.np, grid.E)
    U.scatter(out, torch.from_numpy(c).cuda(), dtoc)
    assert np.array_equal(out.numpy().ravel(order="F"), ref)
    # integer degree count: gather of ones (GridArray{Int})
    ones = rb.GridArray(torch.ones((grid.E, 1, grid.np), dtype=torch.int64, device="cuda"), 1, grid.np, grid.E)
    deg = torch.zeros((nc, 1), dtype=torch.int64, device="cuda")
    U.gather(deg, ones, colptr, rowval)
    assert np.array_equal(deg.cpu().numpy().ravel(), np.diff(colptr))


def test_gather_scatter_points_round_trip(rb, U):
    """gatherscatterpoints (test/mpitest_n3_gatherscatter.jl): points -> gather / degree
    -> scatter reproduces the points to 10 eps."""
    import torch

    grid = _brick(rb, 2, 4, (3, 2), (False, False))
    dtoc, colptr, rowval = U.continuous_maps(grid)
    nc = colptr.size - 1
    x = rb.GridArray.from_numpy(np.asfortranarray(grid.points))
    ca = torch.zeros((nc, grid.dim), dtype=torch.float64, device="cuda")
    U.gather(ca, x, colptr, rowval)
    ones = rb.GridArray(torch.ones((grid.E, 1, grid.np), dtype=torch.float64, device="cuda"), 1, grid.np, grid.E)
    deg = torch.zeros((nc, 1), dtype=torch.float64, device="cuda")
    U.gather(deg, ones, colptr, rowval)
    ca /= deg
    back = x.similar()
    U.scatter(back, ca, dtoc)
    err = (back.data - x.data).abs().max().item()
    assert err < 10 * np.finfo(float).eps * x.data.abs().max().item()


def test_gridarray_operations(rb, cuda_ok):
    """components, fill!, sum and norm of GridArray (gridarrays.jl:367-377, 573-615,
    663-673) on the device, against numpy on the same array."""
    rng = np.random.default_rng(7)
    a = np.asfortranarray(rng.standard_normal((27, 5, 11)))
    q = rb.GridArray.from_numpy(a)
    assert q.shape == a.shape
    comps = q.components()
    assert len(comps) == 5
    for s in range(5):
        assert np.array_equal(comps[s].cpu().numpy().T, a[:, s, :])
    comps[2].mul_(2.0)  # a view: writes go to q
    b = a.copy()
    b[:, 2, :] *= 2.0
    assert np.array_equal(q.numpy(), b)
    assert np.allclose(q.sum(), b.sum(axis=(0, 2)), rtol=1e-13, atol=1e-13)
    assert q.norm() == pytest.approx(np.linalg.norm(b.ravel()), rel=1e-13)
    q.fill_([1.0, 2.0, 3.0, 4.0, 5.0])
    assert np.array_equal(q.numpy()[0, :, 0], [1.0, 2.0, 3.0, 4.0, 5.0])
    q.fill_(0.5)
    assert np.all(q.numpy() == 0.5)
