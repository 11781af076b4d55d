"""Serving loop: many independent brick solves batched on one GPU.

Raven's drivers run one ``solve!(q, timeend, LSRK54(dg, q, dt))`` per process
(src/balancelaws/odesolvers.jl:9-30).  A service that answers many small requests
(parameter sweeps, ensembles, interactive what-ifs) would leave a B200 mostly idle
that way.  The server of libravenb200 (``rb200_server_*`` in include/raven_b200.h)
keeps every running solve resident in one device arena.  It advances all running
solves of a class with one batched launch per LSRK stage.  A class is a set of solves
with the same dimension, Nq, law, form, precision and constants.  Results are bit for
bit those of each solve run alone.

This module is the Python side:
* ``brick_arrays`` builds a request's per-element geometry and connectivity straight
  from the brick's vertex coordinates, without per-node arrays;
* ``Server`` wraps the C ABI;
* ``poisson_mix`` and ``run_load`` generate and replay a seeded request stream.
"""

import ctypes
import math
import threading
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from .grids import brick_tree_order, jl_range, lobatto_operators

# ------------------------------------------------------------------------ brick arrays


def brick_arrays(dim, nq, coordinates, periodic):
    """Per-element data of an unwarped brick, in the order of Raven's generated grid.

    Returns (elem_geo (4, E), neighbors (2*dim, E) int32, corners (2, dim, E)), all
    Fortran-ordered, equal to what the DGSEM handle extracts from the full ``Grid``.
    * elem_geo is dr/dx, ds/dy, dt/dz (0 in 2-D) and J.  It comes from the brick
      metrics (lobattocells.jl:3190-3232), including the 3-D quirk that element e reads
      the corner points of element ``e mod max(512 / Nq^2, 1)``.
    * neighbors is the element across each face (-1 on a non-periodic boundary).
    * corners holds each element's lower corner and width per direction.
    """
    K = [len(c) - 1 for c in coordinates]
    if len(K) != dim:
        raise ValueError("need one vertex array per dimension")
    tree = brick_tree_order(K)
    E = tree.shape[1]
    corners = np.zeros((2, dim, E), order="F")
    dX = np.zeros((dim, E))
    for d in range(dim):
        c = np.asarray(coordinates[d], dtype=np.float64)
        width = c[1:] - c[:-1]
        t = tree[d]
        corners[0, d, :] = c[t]
        corners[1, d, :] = width[t]
        # last node fma(width, (1+1)/2, c) minus first node fma(width, 0, c)
        dX[d] = (c[:-1] + width)[t] - c[t]
    Qw = max(512 // (nq * nq), 1)
    src = np.arange(E) % Qw if dim == 3 else np.arange(E)
    dXs = dX[:, src]
    geo = np.zeros((4, E), order="F")
    for d in range(dim):
        geo[d] = 2.0 / dXs[d]
    J = dXs[0] / 2.0
    for d in range(1, dim):
        J = J * (dXs[d] / 2.0)
    geo[3] = J
    lookup = -np.ones(tuple(K), dtype=np.int64)
    lookup[tuple(tree[d] for d in range(dim))] = np.arange(E)
    nbr = np.full((2 * dim, E), -1, dtype=np.int32, order="F")
    for f in range(2 * dim):
        d, side = f // 2, f % 2
        nb = [tree[k].copy() for k in range(dim)]
        nb[d] = nb[d] + (1 if side else -1)
        inside = (nb[d] >= 0) & (nb[d] < K[d])
        if periodic[d]:
            nb[d] = nb[d] % K[d]
            inside[:] = True
        else:
            nb[d] = np.clip(nb[d], 0, K[d] - 1)
        nbr[f] = np.where(inside, lookup[tuple(nb)], -1)
    return geo, nbr, corners


# ------------------------------------------------------------------------------ requests

INIT_VORTEX, INIT_SINE_GAUSSIAN = 1, 2


@dataclass
class SolveSpec:
    """One solve: a brick [lo, hi]^dim with K elements per direction (periodic),
    ``nsteps`` LSRK54 steps of size dt from device-evaluated (or given) initial data."""

    dim: int
    nq: int
    law: int  # _lib.LAW_*
    K: tuple
    lo: tuple
    hi: tuple
    nsteps: int
    dt: float
    precision: int = _lib.PRECISION_FP64
    surface_flux: int = _lib.FLUX_RUSANOV
    gamma: float = 1.4
    advection_velocity: tuple = (1.0, 1.0, 1.0)
    init_params: tuple = ()
    q0: np.ndarray = None  # (Np, Ns, E) Fortran; None = device initial data
    periodic: tuple = None

    @property
    def ns(self):
        return 1 if self.law == _lib.LAW_ADVECTION else self.dim + 2

    @property
    def num_elements(self):
        return int(np.prod(self.K))

    @property
    def np(self):
        return self.nq**self.dim

    def coordinates(self):
        return tuple(jl_range(self.lo[d], self.hi[d], self.K[d] + 1) for d in range(self.dim))

    def dof_updates(self):
        """Node-field updates, one per LSRK stage (5 right-hand sides per step)."""
        return self.np * self.ns * self.num_elements * self.nsteps * 5


def vortex_spec(dim, nq, K, nsteps, precision=_lib.PRECISION_FP64, cfl=0.4, strength=3.0):
    """Euler isentropic vortex (background Mach 0.5, u0 = 0.5 sqrt(1.4)) centred in the
    periodic box [0, 10]^dim, with dt = cfl * min node distance / 2.8.

    The default strength 3 keeps the coarsest solves of the stream (4 elements per side
    at N = 3) stable for 500 steps.  Strength 5, as in the 32^3 benchmark, blows up
    there within 6 steps under Kennedy-Gruber + Rusanov.  2.8 bounds max(|u| + c) for
    strengths up to 5: |u| <= u0 + 5 e^(1/2) / (2 pi sqrt 2) < 1.53 and
    c <= sqrt(1.4) < 1.19."""
    if not 0 < strength <= 5:
        raise ValueError("the time-step bound assumes a vortex strength in (0, 5]")
    r, _, _ = lobatto_operators(nq)
    h = 10.0 / max(K)
    dmin = h * (r[1] - r[0]) / 2
    return SolveSpec(dim=dim, nq=nq, law=_lib.LAW_EULER, K=tuple(K), lo=(0.0,) * dim, hi=(10.0,) * dim,
                     nsteps=nsteps, dt=cfl * dmin / 2.8, precision=precision,
                     init_params=(float(strength), 0.5 * math.sqrt(1.4), 5.0, 5.0))


def wave_spec(dim, nq, K, nsteps, precision=_lib.PRECISION_FP64, cfl=0.4):
    """Advection with velocity (1, 0.5[, 0.25]) of sin(2 pi x) sin(2 pi y) [sin(2 pi z)]
    plus a Gaussian of width 0.05 at the centre, on the periodic unit box."""
    r, _, _ = lobatto_operators(nq)
    h = 1.0 / max(K)
    dmin = h * (r[1] - r[0]) / 2
    a = (1.0, 0.5, 0.25)[:dim]
    return SolveSpec(dim=dim, nq=nq, law=_lib.LAW_ADVECTION, K=tuple(K), lo=(0.0,) * dim, hi=(1.0,) * dim,
                     nsteps=nsteps, dt=cfl * dmin / math.hypot(*a), precision=precision,
                     advection_velocity=a, init_params=(0.05, 0.5, 0.5, 0.5))


_OPS = {}


def _operators(nq):
    if nq not in _OPS:
        r, w, D = lobatto_operators(nq)
        _OPS[nq] = (np.ascontiguousarray(r), np.ascontiguousarray(w), np.asfortranarray(D))
    return _OPS[nq]


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


# -------------------------------------------------------------------------------- server


class Server:
    """A serving loop on one GPU (``rb200_server_create``).

    ``submit(spec)`` queues a solve and returns a ticket; ``wait(ticket)`` blocks until
    it finished and returns (final state (Np, Ns, E) Fortran array, latency in s)."""

    def __init__(self, arena_bytes=8 << 30, device=0):
        L = _lib.lib()
        h = ctypes.c_void_p()
        _lib.check(L.rb200_server_create(int(device), int(arena_bytes), ctypes.byref(h)))
        self._h = h
        self._out = {}
        self._lock = threading.Lock()

    def submit(self, spec, keep_result=True):
        L = _lib.lib()
        r, w, D = _operators(spec.nq)
        geo, nbr, corners = brick_arrays(spec.dim, spec.nq, spec.coordinates(),
                                         spec.periodic or (True,) * spec.dim)
        q_out = np.empty((spec.np, spec.ns, spec.num_elements), order="F") if keep_result else None
        q0 = None if spec.q0 is None else np.asfortranarray(spec.q0, dtype=np.float64)
        if q0 is not None and q0.shape != (spec.np, spec.ns, spec.num_elements):
            raise ValueError("q0 must have shape (Np, Ns, E)")
        req = _lib.Request()
        req.abi_version = _lib.RB200_ABI_VERSION
        req.dim, req.nq, req.law = spec.dim, spec.nq, spec.law
        req.num_elements = spec.num_elements
        if spec.law == _lib.LAW_ADVECTION:
            req.volume_form, req.volume_flux = _lib.FORM_WEAK, _lib.FLUX_CENTRAL
        else:
            req.volume_form, req.volume_flux = _lib.FORM_FLUXDIFF, _lib.FLUX_KENNEDY_GRUBER
        req.surface_flux = spec.surface_flux
        req.precision = spec.precision
        req.gamma = spec.gamma
        req.advection_velocity[:] = list(spec.advection_velocity[: spec.dim]) + [0.0] * (3 - spec.dim)
        req.D, req.w, req.r = _p(D), _p(w), _p(r)
        req.elem_geo, req.neighbors, req.corners = _p(geo), _p(nbr), _p(corners)
        req.q0 = _p(q0)
        req.init_kind = 0 if q0 is not None else (INIT_VORTEX if spec.law == _lib.LAW_EULER else INIT_SINE_GAUSSIAN)
        req.init_params[:] = list(spec.init_params) + [0.0] * (8 - len(spec.init_params))
        req.dt = spec.dt
        req.nsteps = spec.nsteps
        req.q_out = _p(q_out)
        ticket = ctypes.c_uint64()
        with self._lock:
            st = L.rb200_server_submit(self._h, ctypes.byref(req), ctypes.byref(ticket))
            if st != 0:
                raise _lib.RB200Error(st, self.last_error() or "submit rejected")
            self._out[ticket.value] = q_out
        return ticket.value

    def wait(self, ticket, timeout=600.0):
        L = _lib.lib()
        lat = ctypes.c_double()
        st = L.rb200_server_wait(self._h, ctypes.c_uint64(ticket), float(timeout), ctypes.byref(lat))
        if st != 0:
            raise _lib.RB200Error(st, self.last_error() or "wait failed")
        with self._lock:
            q = self._out.pop(ticket)
        return q, lat.value

    def stats(self):
        out = (ctypes.c_double * 9)()
        st = _lib.lib().rb200_server_stats(self._h, out, 9)
        keys = ("completed", "submitted", "running", "queued", "dof_updates", "arena_used", "arena_peak",
                "ticks", "busy_seconds")
        d = dict(zip(keys, list(out)))
        d["status"] = st
        return d

    def class_tiles(self):
        """[(dim, nq, kernel combination, chosen elements per CTA or 0)] per class."""
        buf = (ctypes.c_int32 * 256)()
        _lib.check(_lib.lib().rb200_server_class_tiles(self._h, buf, 256))
        vals = list(buf)
        return [tuple(vals[i:i + 4]) for i in range(0, 256, 4) if vals[i] != 0]

    def class_stats(self):
        """Per class: dim, nq, kernel combination, completed ticks, device milliseconds of
        those ticks (classes overlap on the device) and their DOF updates."""
        buf = (ctypes.c_double * 384)()
        _lib.check(_lib.lib().rb200_server_class_stats(self._h, buf, 384))
        vals = list(buf)
        keys = ("dim", "nq", "combo", "ticks", "device_ms", "dof_updates")
        rows = []
        for i in range(0, 384, 6):
            if vals[i] == 0:
                continue
            r = dict(zip(keys, vals[i:i + 6]))
            for k in ("dim", "nq", "combo", "ticks"):
                r[k] = int(r[k])
            rows.append(r)
        return rows

    def last_error(self):
        return _lib.lib().rb200_server_last_error(self._h).decode()

    def close(self):
        if self._h:
            _lib.check(_lib.lib().rb200_server_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------- load model


@dataclass
class Arrival:
    t: float
    spec: SolveSpec


def poisson_mix(seed, n, rate=200.0, dims=(2, 3), nqs=(4, 6, 8), laws=(_lib.LAW_ADVECTION, _lib.LAW_EULER),
                steps=(50, 500), k2d=(8, 64), k3d=(4, 32), precision=_lib.PRECISION_FP32_BULK):
    """A seeded request stream: Poisson arrivals at ``rate`` per second.

    Each solve draws, uniformly, a dimension, a polynomial order (Nq in ``nqs``), a law
    (advection: sine + Gaussian; Euler: isentropic vortex) and a step count in
    ``steps``.  The elements per direction are log-uniform in ``k2d`` or ``k3d``."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(n):
        t += rng.exponential(1.0 / rate)
        dim = int(rng.choice(dims))
        nq = int(rng.choice(nqs))
        law = int(rng.choice(laws))
        lo, hi = k2d if dim == 2 else k3d
        k = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        ns = int(rng.integers(steps[0], steps[1] + 1))
        spec = (vortex_spec if law == _lib.LAW_EULER else wave_spec)(dim, nq, (k,) * dim, ns, precision=precision)
        out.append(Arrival(t, spec))
    return out


def run_load(server, arrivals, keep_results=False, timeout=600.0):
    """Replays ``arrivals`` against ``server`` in real time and waits for all of them.

    Returns a dict: latencies (s, per solve), wall (s), busy_seconds (first submit to
    last completion), solves_per_s, dof_updates_per_s, results (if keep_results)."""
    tickets = [None] * len(arrivals)
    errors = []

    def submitter():
        t0 = time.perf_counter()
        try:
            for i, a in enumerate(arrivals):
                delay = a.t - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                tickets[i] = server.submit(a.spec, keep_result=keep_results)
        except Exception as e:  # surfaced below
            errors.append(e)

    th = threading.Thread(target=submitter)
    t_start = time.perf_counter()
    th.start()
    lat = []
    results = []
    for i in range(len(arrivals)):
        while tickets[i] is None and not errors:
            time.sleep(0.0005)
        if errors:
            break
        q, l = server.wait(tickets[i], timeout=timeout)
        lat.append(l)
        results.append(q)
    th.join()
    if errors:
        raise errors[0]
    wall = time.perf_counter() - t_start
    dof = sum(a.spec.dof_updates() for a in arrivals)
    busy = server.stats()["busy_seconds"] or wall
    return {
        "latencies": np.array(lat),
        "wall": wall,
        "busy_seconds": busy,
        "solves_per_s": len(arrivals) / busy,
        "dof_updates_per_s": dof / busy,
        "results": results if keep_results else None,
    }
