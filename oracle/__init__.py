"""TEST INFRASTRUCTURE ONLY -- the CPU FP64 oracle for the DGSEM tendency + LSRK(5,4) path.

This package wraps ``oracle/oracle.cpp`` (a C++ restatement of Raven.jl's brick grid,
DGSEM tendency and LSRK(5,4) stepper, citations in that file) and
``oracle/utilities.cpp`` (Kron, gather!/scatter! and decode).  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import it; the
product package (``raven.jl_b200``) never does.

The oracle is pinned against the reference's own golden values
(``tests/golden/reference_goldens.json``, produced by ``tests/golden/make_goldens.py``,
and ``tests/golden/facecode_goldens.json``, produced by
``tests/golden/make_facecode_goldens.py``).
"""

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

LAW_ADVECTION, LAW_EULER = 0, 1
FORM_WEAK, FORM_FLUXDIFF = 0, 1
FLUX_CENTRAL, FLUX_KG, FLUX_EC, FLUX_RUSANOV, FLUX_ROE, FLUX_MATRIX = 0, 1, 2, 3, 4, 5
WARP_NONE, WARP_SINE, WARP_IDENTITY_CURVED = 0, 1, 2


def build(force=False):
    """Compile oracle.cpp into oracle/_build/liboracle.so (g++, -ffp-contract=off, OpenMP)."""
    srcs = [os.path.join(HERE, "oracle.cpp"), os.path.join(HERE, "utilities.cpp")]
    hdr = os.path.join(HERE, "oracle.h")
    os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
    if (
        not force
        and os.path.exists(LIB_PATH)
        and os.path.getmtime(LIB_PATH) >= max([os.path.getmtime(f) for f in srcs] + [os.path.getmtime(hdr)])
    ):
        return LIB_PATH
    cmd = [
        "g++", "-O2", "-std=gnu++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
        "-fno-fast-math", "-o", LIB_PATH, *srcs, "-lquadmath",
    ]
    subprocess.check_call(cmd)
    return LIB_PATH


class _Law(ctypes.Structure):
    _fields_ = [
        ("law", ctypes.c_int),
        ("form", ctypes.c_int),
        ("volume_flux", ctypes.c_int),
        ("surface_flux", ctypes.c_int),
        ("gamma", ctypes.c_double),
        ("adv", ctypes.c_double * 3),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        L.og_grid_create.restype = P
        L.og_grid_create.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P, P, ctypes.c_int, ctypes.c_double]
        L.og_grid_destroy.argtypes = [P]
        L.og_grid_from_arrays.restype = P
        L.og_grid_from_arrays.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int64, P, P, P, P, P, P]
        L.og_grid_set_mortars.argtypes = [P, P, ctypes.c_int64, P, P, P, P]
        L.og_grid_set_curved_mortars.argtypes = [P, ctypes.c_int]
        L.og_grid_set_directions.argtypes = [P, ctypes.c_int]
        L.og_grid_set_boundary_condition.argtypes = [P, ctypes.c_int, ctypes.c_int, P]
        L.og_lsrk_step_coeffs.argtypes = [P, P, P, P, P, P, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.og_rlsrk_step_coeffs.argtypes = [P, P, P, P, P, P, P, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.og_rlsrk_step_coeffs.restype = ctypes.c_int
        for name in ("og_grid_sizes", "og_grid_points", "og_grid_vmet", "og_grid_smet", "og_grid_vmapM",
                     "og_grid_vmapP", "og_grid_boundary", "og_grid_tree_coords"):
            getattr(L, name).argtypes = [P, P]
        L.og_grid_lgl.argtypes = [P, P, P, P]
        L.og_lgl.argtypes = [ctypes.c_int, P, P, P]
        L.og_initial_condition.argtypes = [P, P, ctypes.c_int, P, ctypes.c_double, P]
        L.og_tendency.argtypes = [P, P, P, P, ctypes.c_double, ctypes.c_int, ctypes.c_int64, ctypes.c_int64]
        L.og_lsrk54_step.argtypes = [P, P, P, P, ctypes.c_double, ctypes.c_double]
        L.og_lsrk144_step.argtypes = [P, P, P, P, ctypes.c_double, ctypes.c_double]
        L.og_solve.restype = ctypes.c_int64
        L.og_solve.argtypes = [P, P, P, ctypes.c_double, ctypes.c_double]
        L.og_entropy_sums.argtypes = [P, P, P, P, ctypes.c_double, P, P]
        L.og_rlsrk54_step.restype = ctypes.c_int
        L.og_rlsrk54_step.argtypes = [P, P, P, P, P, ctypes.c_double, ctypes.c_double]
        L.og_rlsrk144_step.restype = ctypes.c_int
        L.og_rlsrk144_step.argtypes = [P, P, P, P, P, ctypes.c_double, ctypes.c_double]
        L.og_solve_rlsrk.restype = ctypes.c_int64
        L.og_solve_rlsrk.argtypes = [P, P, P, ctypes.c_double, ctypes.c_double, P]
        L.og_weightednorm.restype = ctypes.c_double
        L.og_weightednorm.argtypes = [P, P, ctypes.c_int, P]
        L.og_weightednorm_p.restype = ctypes.c_double
        L.og_weightednorm_p.argtypes = [P, P, ctypes.c_int, ctypes.c_double, P]
        L.og_integrals.argtypes = [P, P, ctypes.c_int, P]
        L.og_decode8.argtypes = [P, ctypes.c_int64, P]
        L.og_decode16.argtypes = [P, ctypes.c_int64, P]
        L.og_kron_apply_f64.argtypes = [ctypes.c_int, P, P, P, P, P, P, P, ctypes.c_int64, ctypes.c_int]
        L.og_kron_apply_f32.argtypes = [ctypes.c_int, P, P, P, P, P, P, P, ctypes.c_int64, ctypes.c_int]
        L.og_scatter_f64.argtypes = [P, P, P, P, P, ctypes.c_int64, ctypes.c_int]
        L.og_gather_f64.argtypes = [P, P, P, P, P, P, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.og_num_threads.restype = ctypes.c_int
        L.og_set_num_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def lgl(nq):
    r = np.zeros(nq)
    w = np.zeros(nq)
    D = np.zeros((nq, nq), order="F")
    lib().og_lgl(nq, _ptr(r), _ptr(w), _ptr(D))
    return r, w, D


class Law:
    """Law/scheme selection for the oracle (mirrors Raven's DGSEM keyword arguments)."""

    def __init__(self, law, dim, form=FORM_WEAK, volume_flux=FLUX_CENTRAL, surface_flux=FLUX_RUSANOV,
                 gamma=1.4, adv=None):
        self.dim = dim
        self.c = _Law()
        self.c.law = law
        self.c.form = form
        self.c.volume_flux = volume_flux
        self.c.surface_flux = surface_flux
        self.c.gamma = gamma
        a = adv if adv is not None else [1.0] * dim
        for i in range(3):
            self.c.adv[i] = a[i] if i < len(a) else 0.0
        self.ns = 1 if law == LAW_ADVECTION else dim + 2


class Grid:
    """A brick grid built by the oracle (element order, points, metrics, face maps)."""

    def __init__(self, dim, nq, K, lo, hi, periodic, warp=WARP_NONE, warp_amp=0.0):
        K3 = np.array(list(K) + [1] * (3 - len(K)), dtype=np.int32)
        lo3 = np.array(list(lo) + [0.0] * (3 - len(lo)), dtype=np.float64)
        hi3 = np.array(list(hi) + [1.0] * (3 - len(hi)), dtype=np.float64)
        p3 = np.array([int(bool(p)) for p in periodic] + [0] * (3 - len(periodic)), dtype=np.int32)
        self._keep = (K3, lo3, hi3, p3)
        self.h = lib().og_grid_create(dim, nq, _ptr(K3), _ptr(lo3), _ptr(hi3), _ptr(p3), warp, warp_amp)
        s = np.zeros(8, dtype=np.int64)
        lib().og_grid_sizes(self.h, _ptr(s))
        self.dim, self.nq, self.np, self.nfp, self.nfaces, self.E, self.nvmet, self.nsmet = (int(v) for v in s)

    @classmethod
    def from_arrays(cls, dim, nq, points, volume_metrics, surface_metrics, vmapM, vmapP, boundarycodes,
                    mortars=None, tohalves=None, curved=False):
        """A grid from the arrays of a generated grid (adapted grids); with mortars
        ((2 + 2^(dim-1), M) int64 0-based) and tohalves (I_lower, I_upper, P_lower,
        P_upper) the hanging faces are coupled through mortars, with the small faces'
        own geometry when `curved` (a warped adapted grid)."""
        self = cls.__new__(cls)
        keep = [np.asfortranarray(a, dtype=np.float64) for a in (points, volume_metrics, surface_metrics)]
        keep += [np.asfortranarray(a, dtype=np.int64) for a in (vmapM, vmapP, boundarycodes)]
        E = keep[0].shape[2]
        self.h = lib().og_grid_from_arrays(dim, nq, E, *[_ptr(a) for a in keep])
        self._keep = keep
        s = np.zeros(8, dtype=np.int64)
        lib().og_grid_sizes(self.h, _ptr(s))
        self.dim, self.nq, self.np, self.nfp, self.nfaces, self.E, self.nvmet, self.nsmet = (int(v) for v in s)
        if mortars is not None and mortars.size:
            m = np.asfortranarray(mortars, dtype=np.int64)
            ops = [np.ascontiguousarray(a, dtype=np.float64) for a in tohalves]
            lib().og_grid_set_mortars(self.h, _ptr(m), m.shape[1], *[_ptr(a) for a in ops])
            lib().og_grid_set_curved_mortars(self.h, int(bool(curved)))
            self._keep += [m] + ops
        return self

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.og_grid_destroy(self.h)
            self.h = None

    def _get(self, name, shape, dtype):
        a = np.zeros(shape, dtype=dtype, order="F")
        getattr(lib(), name)(self.h, _ptr(a))
        return a

    def lgl(self):
        r = np.zeros(self.nq)
        w = np.zeros(self.nq)
        D = np.zeros((self.nq, self.nq), order="F")
        lib().og_grid_lgl(self.h, _ptr(r), _ptr(w), _ptr(D))
        return r, w, D

    def points(self):
        return self._get("og_grid_points", (self.np, self.dim, self.E), np.float64)

    def volume_metrics(self):
        return self._get("og_grid_vmet", (self.np, self.nvmet, self.E), np.float64)

    def surface_metrics(self):
        return self._get("og_grid_smet", (self.nsmet, self.nfaces * self.nfp, self.E), np.float64)

    def vmapM(self):
        return self._get("og_grid_vmapM", (self.nfaces * self.nfp, self.E), np.int64)

    def vmapP(self):
        return self._get("og_grid_vmapP", (self.nfaces * self.nfp, self.E), np.int64)

    def boundary(self):
        return self._get("og_grid_boundary", (self.nfaces, self.E), np.int64)

    def tree_coords(self):
        return self._get("og_grid_tree_coords", (3, self.E), np.int32)

    # ---- state ----
    def state(self, law):
        return np.zeros((self.np, law.ns, self.E), order="F")

    def initial_condition(self, law, kind, params=(), t=0.0):
        q = self.state(law)
        prm = np.array(list(params) + [0.0] * 8, dtype=np.float64)
        lib().og_initial_condition(self.h, ctypes.byref(law.c), kind, _ptr(prm), t, _ptr(q))
        return q

    def tendency(self, law, q, dq=None, t=0.0, increment=False, e0=0, e1=None):
        q = np.asfortranarray(q, dtype=np.float64)
        if dq is None:
            dq = self.state(law)
        lib().og_tendency(self.h, ctypes.byref(law.c), _ptr(dq), _ptr(q), t, int(increment), e0,
                          self.E if e1 is None else e1)
        return dq

    def set_boundary_condition(self, tag, kind, state=None):
        """boundarystate of the faces with code `tag`: 0 q+ = q-, 1 q+ = state, 2 a wall."""
        st = None if state is None else np.ascontiguousarray(state, dtype=np.float64)
        self._bc_keep = getattr(self, "_bc_keep", []) + [st]
        lib().og_grid_set_boundary_condition(self.h, int(tag), int(kind), None if st is None else _ptr(st))

    def set_directions(self, directions):
        """DGSEM(; directions): 1-based directions whose terms are computed."""
        lib().og_grid_set_directions(self.h, sum(1 << (int(d) - 1) for d in directions))

    def lsrk54_step(self, law, q, dq, time, dt):
        lib().og_lsrk54_step(self.h, ctypes.byref(law.c), _ptr(q), _ptr(dq), time, dt)

    def lsrk144_step(self, law, q, dq, time, dt):
        lib().og_lsrk144_step(self.h, ctypes.byref(law.c), _ptr(q), _ptr(dq), time, dt)

    def solve(self, law, q, dt, timeend):
        return lib().og_solve(self.h, ctypes.byref(law.c), _ptr(q), dt, timeend)

    def entropy_sums(self, law, base, direction=None, c=0.0, k=None):
        """(sum MJ eta(p), sum MJ v(p).k) for p = base + c * direction."""
        out = np.zeros(2)
        base = np.asfortranarray(base, dtype=np.float64)
        d = None if direction is None else np.asfortranarray(direction, dtype=np.float64)
        kk = None if k is None else np.asfortranarray(k, dtype=np.float64)
        lib().og_entropy_sums(self.h, ctypes.byref(law.c), _ptr(base), None if d is None else _ptr(d), c,
                              None if kk is None else _ptr(kk), _ptr(out))
        return out

    def rlsrk54_step(self, law, q, dq, gamma, time, dt):
        """One RLSRK(5,4) step in place; gamma is a 1-element float64 array carried
        between steps.  Returns the Newton iterations."""
        return lib().og_rlsrk54_step(self.h, ctypes.byref(law.c), _ptr(q), _ptr(dq), _ptr(gamma), time, dt)

    def lsrk_step(self, law, q, dq, rka, rkb, time, dt):
        """One LSRK step with the table (rka, rkb)."""
        a, b = np.ascontiguousarray(rka, dtype=np.float64), np.ascontiguousarray(rkb, dtype=np.float64)
        lib().og_lsrk_step_coeffs(self.h, ctypes.byref(law.c), _ptr(q), _ptr(dq), _ptr(a), _ptr(b), a.size, time, dt)

    def rlsrk_step(self, law, q, dq, gamma, rka, rkb, time, dt):
        """One RLSRK step with the table (rka, rkb) (see rlsrk54_step)."""
        a, b = np.ascontiguousarray(rka, dtype=np.float64), np.ascontiguousarray(rkb, dtype=np.float64)
        return lib().og_rlsrk_step_coeffs(self.h, ctypes.byref(law.c), _ptr(q), _ptr(dq), _ptr(gamma), _ptr(a),
                                          _ptr(b), a.size, time, dt)

    def rlsrk144_step(self, law, q, dq, gamma, time, dt):
        """One RLSRK(14,4) step in place (see rlsrk54_step)."""
        return lib().og_rlsrk144_step(self.h, ctypes.byref(law.c), _ptr(q), _ptr(dq), _ptr(gamma), time, dt)

    def solve_rlsrk(self, law, q, dt, timeend):
        gamma = np.ones(1)
        steps = lib().og_solve_rlsrk(self.h, ctypes.byref(law.c), _ptr(q), dt, timeend, _ptr(gamma))
        return steps, gamma[0]

    def weightednorm(self, q, ns):
        comp = np.zeros(ns)
        v = lib().og_weightednorm(self.h, _ptr(np.asfortranarray(q)), ns, _ptr(comp))
        return v, comp

    def weightednorm_p(self, q, ns, p):
        """weightednorm for any p >= 1 or p = inf: (total, per-field)."""
        comp = np.zeros(ns)
        v = lib().og_weightednorm_p(self.h, _ptr(np.asfortranarray(q)), ns, float(p), _ptr(comp))
        return v, comp

    def integrals(self, q, ns):
        out = np.zeros(ns)
        lib().og_integrals(self.h, _ptr(np.asfortranarray(q)), ns, _ptr(out))
        return out


def num_threads():
    return lib().og_num_threads()


def set_num_threads(n):
    lib().og_set_num_threads(int(n))


# ------------------------------------------------------------------------- utilities


def decode(codes):
    """decode(facecode) for an array of UInt8 (-> (n, 4) hangingface) or UInt16 codes
    (-> (n, 18): 6 hangingface then 12 hangingedge values)."""
    codes = np.ascontiguousarray(codes)
    n = codes.size
    if codes.dtype == np.uint8:
        out = np.zeros((n, 4), dtype=np.uint8)
        lib().og_decode8(_ptr(codes), n, _ptr(out))
    elif codes.dtype == np.uint16:
        out = np.zeros((n, 18), dtype=np.uint8)
        lib().og_decode16(_ptr(codes), n, _ptr(out))
    else:
        raise TypeError("facecodes are uint8 (2-D) or uint16 (3-D)")
    return out


def kron_apply(mats, sizes, f, ncomp=1, in_strides=None, out_strides=None, ncol=None):
    """Kron(args) * f: mats[d] = X_{d+1} (acts on index d, fastest first) or None for
    Eye(sizes[d]).  f: flat array addressed f[node*sn + comp*sc + col*scol]."""
    nf = len(mats)
    dt = f.dtype
    rows = np.array([m.shape[0] if m is not None else sizes[d] for d, m in enumerate(mats)], dtype=np.int32)
    cols = np.array([m.shape[1] if m is not None else sizes[d] for d, m in enumerate(mats)], dtype=np.int32)
    keep = [None if m is None else np.asfortranarray(m, dtype=dt) for m in mats]
    ptrs = (ctypes.c_void_p * nf)(*[None if m is None else m.ctypes.data for m in keep])
    nin, nout = int(np.prod(cols)), int(np.prod(rows))
    if in_strides is None:
        in_strides = (1, nin, nin * ncomp)
    if out_strides is None:
        out_strides = (1, nout, nout * ncomp)
    if ncol is None:
        ncol = f.size // (nin * ncomp)
    out = np.zeros(max(1, out_strides[0] * (nout - 1) + out_strides[1] * (ncomp - 1)
                       + out_strides[2] * (ncol - 1) + 1), dtype=dt)
    si = np.array(in_strides, dtype=np.int64)
    so = np.array(out_strides, dtype=np.int64)
    fc = np.ascontiguousarray(f)
    fn = lib().og_kron_apply_f64 if dt == np.float64 else lib().og_kron_apply_f32
    fn(nf, ptrs, _ptr(rows), _ptr(cols), _ptr(fc), _ptr(si), _ptr(out), _ptr(so), int(ncol), int(ncomp))
    return out


def scatter(dest, dest_layout, src, src_layout, dtoc, ncomp):
    dl = np.array(dest_layout, dtype=np.int64)
    sl = np.array(src_layout, dtype=np.int64)
    d = np.ascontiguousarray(dtoc, dtype=np.int64)
    lib().og_scatter_f64(_ptr(dest), _ptr(dl), _ptr(src), _ptr(sl), _ptr(d), d.size, int(ncomp))
    return dest


def gather(dest, dest_layout, src, src_layout, colptr, rowval, ncomp, op=0, init=0.0):
    dl = np.array(dest_layout, dtype=np.int64)
    sl = np.array(src_layout, dtype=np.int64)
    cp = np.ascontiguousarray(colptr, dtype=np.int64)
    rv = np.ascontiguousarray(rowval, dtype=np.int64)
    lib().og_gather_f64(_ptr(dest), _ptr(dl), _ptr(src), _ptr(sl), _ptr(cp), _ptr(rv), cp.size - 1, int(ncomp),
                        int(op), float(init))
    return dest
