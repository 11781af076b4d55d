"""Raven utilities beside the DGSEM path, on the device: ``Kron`` (src/kron.jl),
``gather!``/``scatter!`` (src/gatherscatter.jl) and ``decode`` (src/facecode.jl).

Arrays are torch CUDA tensors laid out byte for byte like Raven's (column-major):
  * a GridArray is ``raven_b200.GridArray`` (parent (Np, Ns, E));
  * a continuous array (Raven's ``GridArray(undef, grid, Val(true))``, parent (Ns, Nc))
    is a tensor of shape (Nc, Ns);
  * a Julia matrix of SVector{C} columns, (n, ncols), is a tensor of shape
    (ncols, n, C); a plain vector (n,) is a tensor of shape (n,).
The kernels are in libravenb200.so (``rb200_kron_apply``, ``rb200_gather``,
``rb200_scatter``, ``rb200_decode_facecodes``); their results are bit-identical to the
reference's arithmetic.
"""

import ctypes

import numpy as np

from . import _lib


def _torch():
    import torch

    return torch


def _dtype_code(t):
    torch = _torch()
    codes = {torch.float64: 0, torch.float32: 1, torch.int64: 2, torch.int32: 3}
    if t.dtype not in codes:
        raise TypeError(f"unsupported dtype {t.dtype}")
    return codes[t.dtype]


def _stream():
    return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)


def _check_cuda(*ts):
    for t in ts:
        if not (t.is_cuda and t.is_contiguous()):
            raise ValueError("arrays must be contiguous CUDA tensors (there is no CPU fallback)")


# ------------------------------------------------------------------------------- Kron


class Eye:
    """Raven.Eye{T}(N): the N x N identity, stored as nothing."""

    def __init__(self, n):
        self.n = int(n)
        self.shape = (self.n, self.n)


class Kron:
    """Raven.Kron(args): the Kronecker product of ``args = (X_n, ..., X_1)`` (Julia
    order, X_1 acting on the fastest index), applied without forming it."""

    def __init__(self, args):
        args = tuple(args)
        if not 1 <= len(args) <= 3:
            raise ValueError("Kron takes 1 to 3 factors")
        self.args = args

    def components(self):
        return self.args

    def size(self, j):
        return int(np.prod([a.shape[j - 1] for a in self.args]))

    def collect(self):
        """The dense matrix kron(args...) (host numpy; for checks)."""
        out = np.ones((1, 1))
        for a in self.args:
            m = np.eye(a.n) if isinstance(a, Eye) else np.asarray(a)
            out = np.kron(out, m)
        return out

    def _apply(self, f, in_strides, out_shape, out_strides, ncols, ncomp):
        torch = _torch()
        _check_cuda(f)
        dt = _dtype_code(f)
        if dt > 1:
            raise TypeError("Kron applies to float64 or float32 data")
        npdt = np.float64 if dt == 0 else np.float32
        facs = list(reversed(self.args))  # X_1 first
        keep = [None if isinstance(a, Eye) else np.asfortranarray(np.asarray(a, dtype=npdt)) for a in facs]
        mats = (ctypes.c_void_p * len(facs))(*[None if k is None else k.ctypes.data for k in keep])
        rows = (ctypes.c_int32 * len(facs))(*[a.shape[0] for a in facs])
        cols = (ctypes.c_int32 * len(facs))(*[a.shape[1] for a in facs])
        out = torch.empty(out_shape, dtype=f.dtype, device=f.device)
        si = (ctypes.c_int64 * 3)(*in_strides)
        so = (ctypes.c_int64 * 3)(*out_strides)
        _lib.check(_lib.lib().rb200_kron_apply(len(facs), mats, rows, cols, dt, ctypes.c_void_p(f.data_ptr()), si,
                                               ctypes.c_void_p(out.data_ptr()), so, int(ncols), int(ncomp),
                                               _stream()))
        return out

    def __mul__(self, f):
        from . import GridArray

        nin, nout = self.size(2), self.size(1)
        if isinstance(f, GridArray):
            if f.np != nin:
                raise ValueError(f"GridArray has {f.np} nodes per cell, Kron expects {nin}")
            data = self._apply(f.data, (1, nin, nin * f.ns), (f.E, f.ns, nout), (1, nout, nout * f.ns), f.E, f.ns)
            return GridArray(data, f.ns, nout, f.E)
        if f.dim() == 1:  # plain vector
            if f.shape[0] != nin:
                raise ValueError("dimension mismatch")
            return self._apply(f, (1, 0, 0), (nout,), (1, 0, 0), 1, 1)
        if f.dim() == 2:  # (ncols, n): a matrix of plain columns
            if f.shape[1] != nin:
                raise ValueError("dimension mismatch")
            return self._apply(f, (1, 0, nin), (f.shape[0], nout), (1, 0, nout), f.shape[0], 1)
        if f.dim() == 3:  # (ncols, n, C): a matrix of SVector{C} columns
            if f.shape[1] != nin:
                raise ValueError("dimension mismatch")
            C = f.shape[2]
            return self._apply(f, (C, 1, C * nin), (f.shape[0], nout, C), (C, 1, C * nout), f.shape[0], C)
        raise TypeError("Kron * f needs a GridArray or a 1- to 3-dimensional tensor")


# ------------------------------------------------------------------- gather / scatter


def _layout(a):
    """rb200_layout of a GridArray or a continuous (Nc, Ns) tensor, and its Ns."""
    from . import GridArray

    if isinstance(a, GridArray):
        return _lib.Layout(a.np, 1, a.np * a.ns, a.np), a.ns, a.data
    if a.dim() != 2:
        raise ValueError("a continuous array is a (Nc, Ns) tensor")
    return _lib.Layout(a.shape[0], a.shape[1], 0, 1), a.shape[1], a


def continuous_maps(grid):
    """(dtoc, colptr, rowval): Raven's discontinuoustocontinuous / continuoustodiscontinuous
    maps for a conforming grid, built from its face maps.

    The nodes joined through vmapM/vmapP form the continuous nodes.  They are numbered
    in the order of their first discontinuous node.  The numbering of a p4est forest
    (the reference's lnodes ids) is not reproduced: p4est is not available, and
    gather!/scatter! only need a consistent pair of maps.  dtoc: (Np, E) int64
    1-based; CSC arrays 1-based, the rows of each column ascending (sparse(1:n, dtoc,
    true))."""
    n = grid.np * grid.E
    parent = np.arange(n, dtype=np.int64)

    def find(x):
        root = x
        while parent[root] != root:
            root = parent[root]
        while parent[x] != root:
            parent[x], x = root, parent[x]
        return root

    a = np.asarray(grid.vmapM, dtype=np.int64).ravel(order="F") - 1
    b = np.asarray(grid.vmapP, dtype=np.int64).ravel(order="F") - 1
    for x, y in zip(a.tolist(), b.tolist()):
        rx, ry = find(x), find(y)
        if rx != ry:
            if rx < ry:
                parent[ry] = rx
            else:
                parent[rx] = ry
    roots = np.array([find(i) for i in range(n)], dtype=np.int64)
    uniq, first = np.unique(roots, return_index=True)
    order = np.argsort(first)  # number classes by their first node
    rank = np.empty(len(uniq), dtype=np.int64)
    rank[order] = np.arange(len(uniq))
    cid = rank[np.searchsorted(uniq, roots)]
    dtoc = (cid + 1).reshape((grid.np, grid.E), order="F")
    rows = np.argsort(cid, kind="stable")  # ascending rows within each column
    counts = np.bincount(cid, minlength=len(uniq))
    colptr = np.concatenate([[0], np.cumsum(counts)]) + 1
    return dtoc, colptr.astype(np.int64), (rows + 1).astype(np.int64)


def scatter(dest, src, dtoc):
    """scatter!(dest, src, dtoc): dest (GridArray) <- src (continuous) through dtoc."""
    torch = _torch()
    dl, ns_d, dd = _layout(dest)
    sl, ns_s, sd = _layout(src)
    if ns_d != ns_s or dd.dtype != sd.dtype:
        raise ValueError("dest and src differ in components or dtype")
    d = torch.as_tensor(np.asarray(dtoc, dtype=np.int64).ravel(order="F"), device=dd.device)
    n = d.numel()
    _check_cuda(dd, sd, d)
    _lib.check(_lib.lib().rb200_scatter(ctypes.c_void_p(dd.data_ptr()), ctypes.byref(dl),
                                        ctypes.c_void_p(sd.data_ptr()), ctypes.byref(sl),
                                        ctypes.c_void_p(d.data_ptr()), n, ns_d, _dtype_code(dd), _stream()))
    return dest


_OPS = {"+": 0, "min": 1, "max": 2}


def gather(dest, src, colptr, rowval, op="+", init=0):
    """gather!(dest, src, ctod; op, init): dest (continuous) <- src (GridArray)."""
    torch = _torch()
    dl, ns_d, dd = _layout(dest)
    sl, ns_s, sd = _layout(src)
    if ns_d != ns_s or dd.dtype != sd.dtype:
        raise ValueError("dest and src differ in components or dtype")
    cp = torch.as_tensor(np.asarray(colptr, dtype=np.int64), device=dd.device)
    rv = torch.as_tensor(np.asarray(rowval, dtype=np.int64), device=dd.device)
    ncols = cp.numel() - 1
    # gatherfinish! (gatherscatter.jl:87-89): length(dest) > n || m > length(src) throws
    if dd.numel() // ns_d > ncols or rv.numel() > sd.numel() // ns_s:
        raise ValueError("dest and/or src are incompatible with ctod")  # DimensionMismatch
    _check_cuda(dd, sd, cp, rv)
    _lib.check(_lib.lib().rb200_gather(ctypes.c_void_p(dd.data_ptr()), ctypes.byref(dl),
                                       ctypes.c_void_p(sd.data_ptr()), ctypes.byref(sl),
                                       ctypes.c_void_p(cp.data_ptr()), ctypes.c_void_p(rv.data_ptr()), ncols, ns_d,
                                       _dtype_code(dd), _OPS[op], float(init), _stream()))
    return dest


# ------------------------------------------------------------------------------ decode


def decode(codes):
    """decode(facecode) of every entry of a CUDA tensor of uint8 (2-D quadrant codes) or
    16-bit (3-D octant codes, torch.uint16 or int16 holding the same bits) codes.
    Returns a uint8 tensor (n, 4) of hanging faces, or (n, 18): 6 hanging faces then
    12 hanging edges."""
    torch = _torch()
    _check_cuda(codes)
    if codes.dtype == torch.uint8:
        bits, width = 8, 4
    elif codes.element_size() == 2 and not codes.is_floating_point():
        bits, width = 16, 18
    else:
        raise TypeError("facecodes are uint8 (2-D) or 16-bit (3-D)")
    n = codes.numel()
    out = torch.empty((n, width), dtype=torch.uint8, device=codes.device)
    _lib.check(_lib.lib().rb200_decode_facecodes(ctypes.c_void_p(codes.data_ptr()), bits, n,
                                                 ctypes.c_void_p(out.data_ptr()), _stream()))
    return out
