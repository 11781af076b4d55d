"""raven.jl_b200 -- Raven.jl's DGSEM tendency + LSRK(5,4) path on one B200 (sm_100a).

The names, argument meanings and error behaviour follow Raven.jl's balance-law API
(src/balancelaws/{dgsem,odesolvers,measures}.jl, src/lobattocells.jl,
src/coarsegrids.jl, src/gridmanager.jl) so that a Raven driver script maps line by
line:

    Raven.jl                                        raven_b200
    cell = LobattoCell{FT,A}(Nq, Nq, Nq)            cell = LobattoCell(Nq, Nq, Nq)
    cg = brick((vx, vy, vz), (true, true, true))    cg = brick((vx, vy, vz), (True, True, True))
    grid = generate(GridManager(cell, cg))          grid = generate(GridManager(cell, cg))
    dg = DGSEM(; law, grid, volume_form,            dg = DGSEM(law=law, grid=grid, volume_form=...,
               surface_numericalflux)                          surface_numericalflux=RusanovFlux())
    q = GridArray(undef, law, grid)                 q = GridArray.zeros(law, grid)
    dg(dq, q, t; increment = true)                  dg(dq, q, t, increment=True)
    solve!(q, timeend, LSRK54(dg, q, dt))           solve(q, timeend, LSRK54(dg, q, dt))
    weightednorm(dg, q)                             weightednorm(dg, q)

Every operation on a GridArray runs the CUDA kernels of libravenb200.so through its C
ABI (include/raven_b200.h).  There is no CPU fallback: without a CUDA device or
without the built library the calls raise.

Layout: a GridArray's data is a torch CUDA tensor of shape (E, Ns, Np), row-major,
which is byte for byte Raven's GridArray parent array (Np, Ns, E) in column-major
order.
"""

import ctypes
import math

import numpy as np

from . import _lib
from ._lib import RB200Error
from .coarse import CoarseGrid, UnstructuredGrid, coarsegrid, cubeshellgrid
from .forest import AdaptCoarsen, AdaptNone, AdaptRefine, Forest, ForestGrid
from .grids import Grid, brick_tree_order, jl_range, lobatto_operators

__all__ = [
    "LobattoCell", "brick", "BrickGrid", "GridManager", "generate", "Grid", "AdvectionLaw", "EulerLaw",
    "RusanovFlux", "CentralFlux", "KennedyGruberFlux", "EntropyConservativeFlux", "RoeFlux", "MatrixFlux", "WeakForm",
    "FluxDifferencingForm", "GridArray", "DGSEM", "LSRK", "LSRK54", "LSRK144", "RLSRK", "RLSRK54", "RLSRK144", "solve",
    "weightednorm", "integrals",
    "entropyintegral", "entropyproduct", "snapshot", "restore",
    "jl_range", "RB200Error", "brick_tree_order", "adapt", "AdaptRefine", "AdaptNone", "AdaptCoarsen",
    "ForestGrid", "CoarseGrid", "coarsegrid", "cubeshellgrid", "UnstructuredGrid",
]

# --------------------------------------------------------------------------- cells and grids


class LobattoCell:
    """LobattoCell{Float64}(Nq...) (src/lobattocells.jl:89-250); all directions equal."""

    def __init__(self, *sizes):
        if len(sizes) not in (1, 2, 3) or len(set(sizes)) != 1:
            raise ValueError("LobattoCell needs 1, 2 or 3 equal sizes (cubic cells, dgsem.jl:92)")
        self.dim = len(sizes)
        self.nq = int(sizes[0])
        if not 2 <= self.nq <= 8:
            raise ValueError("Nq must be in 2..8")
        self.r, self.w, self.D = lobatto_operators(self.nq)

    def size(self):
        return (self.nq,) * self.dim

    def derivatives_1d(self):
        return (self.D,) * self.dim

    def weights_1d(self):
        return (self.w,) * self.dim

    def points_1d(self):
        return (self.r,) * self.dim


class BrickGrid:
    def __init__(self, coordinates, periodic):
        self.coordinates = tuple(np.asarray(c, dtype=np.float64) for c in coordinates)
        self.periodic = tuple(bool(p) for p in periodic)


def brick(coordinates, periodic=None):
    """brick(coordinates, periodic) (src/coarsegrids.jl:306-405).  `coordinates` is a
    tuple of vertex arrays (use jl_range for Julia's `range(a, stop=b, length=n)`) or a
    tuple of element counts (vertices 0:n)."""
    coords = []
    for c in coordinates:
        if np.isscalar(c):
            coords.append(np.arange(int(c) + 1, dtype=np.float64))
        else:
            coords.append(np.asarray(c, dtype=np.float64))
    if periodic is None:
        periodic = (False,) * len(coords)
    if len(periodic) != len(coords):
        raise ValueError("periodic must have one flag per dimension")
    return BrickGrid(coords, periodic)


class GridManager:
    """GridManager(cell, coarsegrid; min_level) (src/gridmanager.jl:53-94): a forest of
    trees on the brick, each refined uniformly to min_level, adaptable with adapt.  On
    an unstructured coarse grid (CoarseGrid, cubeshellgrid) every cell is a tree,
    refined uniformly to min_level; adapting such a forest is not implemented."""

    def __init__(self, cell, coarsegrid, min_level=0):
        self.cell = cell
        self.coarsegrid = coarsegrid
        self.min_level = int(min_level)
        if isinstance(coarsegrid, CoarseGrid):
            if coarsegrid.dim != cell.dim:
                raise ValueError("cell and coarse grid dimensions differ")
            self.forest = None
            return
        if cell.dim == 1:  # a line: uniform refinement only, as the reference's 1-D forest
            if len(coarsegrid.coordinates) != 1:
                raise ValueError("cell and coarse grid dimensions differ")
            self.forest = None
            return
        if len(coarsegrid.coordinates) != cell.dim:
            raise ValueError("cell and coarse grid dimensions differ")
        K = [len(c) - 1 for c in coarsegrid.coordinates]
        self.forest = Forest(cell.dim, K, coarsegrid.periodic, min_level=min_level)

    def __len__(self):
        if self.forest is None and self.cell.dim == 1:
            return (len(self.coarsegrid.coordinates[0]) - 1) << self.min_level
        if self.forest is None:
            return len(self.coarsegrid) << (self.cell.dim * self.min_level)
        return len(self.forest)


def adapt(gm, flags):
    """adapt!(gm, flags) (src/gridmanager.jl:160-173): refine (AdaptRefine), keep
    (AdaptNone) or coarsen (AdaptCoarsen, whole families) each leaf, then balance 2:1
    across faces."""
    if gm.forest is None:
        raise NotImplementedError("adapting a 1-D forest or a forest on an unstructured coarse grid is not "
                                  "implemented (gridmanager.jl:158)")
    gm.forest.adapt(flags)


def generate(arg, gm=None):
    """generate(gm) or generate(warp, gm) (src/gridmanager.jl:1084-1208).  `warp` maps
    the coordinate arrays (x, y[, z]) to new ones; a warped grid gets curved metrics.
    A forest that is not one level-0 leaf per tree gives an adapted grid (ForestGrid)
    whose hanging faces are coupled by mortars, warped or not."""
    if gm is None:
        gm, warp = arg, None
    else:
        warp = arg
    if gm.forest is None and gm.cell.dim == 1:
        return Grid(gm.cell, gm.coarsegrid, warp=warp, level=gm.min_level)
    if gm.forest is None:
        return UnstructuredGrid(gm.cell, gm.coarsegrid, gm.min_level, warp=warp)
    if all(L[1] == 0 for L in gm.forest.leaves):
        return Grid(gm.cell, gm.coarsegrid, warp=warp)
    return ForestGrid(gm.cell, gm.forest, gm.coarsegrid.coordinates, warp=warp)


# ------------------------------------------------------------------------ laws and fluxes


class AdvectionLaw:
    """AdvectionLaw{Float64,D}(u) (balancelaws/advection.jl:8-16)."""

    code = _lib.LAW_ADVECTION

    def __init__(self, dim, u=None):
        self.dim = dim
        self.u = tuple(float(x) for x in (u if u is not None else (1.0,) * dim))
        if len(self.u) != dim:
            raise ValueError("advection velocity must have `dim` components")
        self.ns = 1
        self.gamma = 1.4


class EulerLaw:
    """EulerLaw{Float64,D}(; gamma = 7//5) (balancelaws/euler.jl:9-19)."""

    code = _lib.LAW_EULER

    def __init__(self, dim, gamma=1.4):
        self.dim = dim
        self.gamma = float(gamma)
        self.u = (0.0,) * dim
        self.ns = dim + 2

    def pressure(self, rho, rhou, rhoe):
        return (self.gamma - 1) * (rhoe - sum(m * m for m in rhou) / (2 * rho))

    def energy(self, rho, rhou, p):
        return p / (self.gamma - 1) + sum(m * m for m in rhou) / (2 * rho)

    def soundspeed(self, rho, p):
        return np.sqrt(self.gamma * p / rho)


class RusanovFlux:
    code = _lib.FLUX_RUSANOV


class CentralFlux:
    code = _lib.FLUX_CENTRAL


class KennedyGruberFlux:
    code = _lib.FLUX_KENNEDY_GRUBER


class EntropyConservativeFlux:
    code = _lib.FLUX_ENTROPY_CONSERVATIVE


class RoeFlux:
    """Roe's approximate Riemann solver for the Euler law (balancelaws/euler.jl:93-149)."""

    code = _lib.FLUX_ROE


class MatrixFlux:
    """Entropy-stable matrix-dissipation flux for the Euler law (balancelaws/euler.jl:218-300)."""

    code = _lib.FLUX_MATRIX


class WeakForm:
    code = _lib.FORM_WEAK
    volume_numericalflux = CentralFlux()


class FluxDifferencingForm:
    code = _lib.FORM_FLUXDIFF

    # The reference's three loop organisations of the same flux-differencing sum
    # (dgsem.jl:163-255: :naive, :per_dir, :per_dir_symmetric).  They differ only in the
    # order of the floating-point sums; one device kernel family serves all three.
    KERNEL_TYPES = ("naive", "per_dir", "per_dir_symmetric")

    def __init__(self, volume_numericalflux, kernel_type="per_dir"):
        kt = str(kernel_type).lstrip(":")
        if kt not in self.KERNEL_TYPES:
            raise ValueError(f"Unknown kernel type {kernel_type}")  # dgsem.jl:253
        self.volume_numericalflux = volume_numericalflux
        self.kernel_type = kt


# ------------------------------------------------------------------------------ GridArray


def _torch():
    import torch

    return torch


class GridArray:
    """State array in Raven's GridArray parent layout, resident on a CUDA device."""

    def __init__(self, data, ns, np_, E):
        self.data = data
        self.ns, self.np, self.E = ns, np_, E

    @classmethod
    def zeros(cls, law, grid, device="cuda", dtype=None):
        torch = _torch()
        t = torch.zeros((grid.E, law.ns, grid.np), dtype=dtype or torch.float64, device=device)
        return cls(t, law.ns, grid.np, grid.E)

    @classmethod
    def from_numpy(cls, arr, device="cuda"):
        """arr: (Np, Ns, E) column-major (Raven parent layout)."""
        torch = _torch()
        a = np.asarray(arr, dtype=np.float64)
        np_, ns, E = a.shape
        t = torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0))).to(device)
        return cls(t, ns, np_, E)

    def numpy(self):
        """(Np, Ns, E) column-major copy on the host."""
        return np.asfortranarray(self.data.detach().cpu().numpy().transpose(2, 1, 0))

    def similar(self):
        return GridArray(_torch().zeros_like(self.data), self.ns, self.np, self.E)

    def copy(self):
        return GridArray(self.data.clone(), self.ns, self.np, self.E)

    def ptr(self):
        if not self.data.is_cuda or not self.data.is_contiguous() or self.data.dtype != _torch().float64:
            raise ValueError("GridArray data must be a contiguous float64 CUDA tensor")
        return ctypes.c_void_p(self.data.data_ptr())

    # GridArray operations of gridarrays.jl used around the tendency (device tensors, no copies)
    def components(self):
        """components(q) (gridarrays.jl:573-615): one view per field, (E, Np) each, writes
        go to q."""
        return tuple(self.data[:, s, :] for s in range(self.ns))

    def fill_(self, x):
        """fill!(q, x) (gridarrays.jl:369-377): every node set to the state x (Ns values,
        or one value for every field)."""
        v = np.broadcast_to(np.asarray(x, dtype=np.float64), (self.ns,))
        for s in range(self.ns):
            self.data[:, s, :].fill_(float(v[s]))
        return self

    def sum(self):
        """sum(q) (gridarrays.jl:663-673): the per-field sums over all nodes (not weighted
        by MJ; integrals(dg, q) gives the weighted ones)."""
        return self.data.sum(dim=(0, 2)).cpu().numpy()

    def norm(self):
        """norm(q) (gridarrays.jl:367): the 2-norm of all entries."""
        return float(_torch().linalg.vector_norm(self.data).item())

    @property
    def shape(self):
        """Raven's parent size (Np, Ns, E)."""
        return (self.np, self.ns, self.E)


def _stream_ptr():
    torch = _torch()
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


# ----------------------------------------------------------------------------------- DGSEM


class DGSEM:
    """DGSEM(; law, grid, surface_numericalflux, volume_form, directions) (src/balancelaws/dgsem.jl:46-81).

    directions: the 1-based directions whose volume and surface terms are computed, as
    Raven's `directions = 1:ndims(law)` (default: all), e.g. (1, 2) or (3,) for a split
    into horizontal and vertical operators.
    boundary_conditions: {tag: condition} for the faces with that boundary code, the
    exterior state Raven's `boundarystate(law, problem, n, q-, aux-, tag)` returns
    (balancelaw.jl:22 and its overloads in the reference's examples): a sequence of Ns
    values (a prescribed state), "wall" (reflecting wall, Euler), or None (q+ = q-, the
    default).
    precision: "fp64" (plain FP64) or "fp32_bulk" (FP32 volume/surface arithmetic, FP64
    geometry, state accumulation and reductions)."""

    def __init__(self, *, law, grid, surface_numericalflux, volume_form=None, directions=None,
                 boundary_conditions=None, precision="fp64", device=None):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("raven_b200.DGSEM needs a CUDA device (no CPU fallback)")
        volume_form = volume_form or WeakForm()
        if law.dim != grid.dim:
            raise ValueError("law and grid dimensions differ")
        if precision not in ("fp64", "fp32_bulk"):
            raise ValueError("precision must be 'fp64' or 'fp32_bulk'")
        if directions is None:
            directions = tuple(range(1, grid.dim + 1))
        directions = tuple(int(d) for d in directions)
        if not directions or any(d < 1 or d > grid.dim for d in directions) or len(set(directions)) != len(directions):
            raise ValueError(f"directions must be distinct values in 1:{grid.dim}")
        self.directions = directions
        self.law, self.grid, self.volume_form = law, grid, volume_form
        self.surface_numericalflux = surface_numericalflux
        self.precision = precision
        self.device = torch.cuda.current_device() if device is None else int(device)
        L = _lib.lib()
        d = _lib.Desc()
        d.abi_version = _lib.RB200_ABI_VERSION
        d.dim, d.nq, d.law = grid.dim, grid.nq, law.code
        d.num_elements = grid.E
        d.volume_form = volume_form.code
        d.volume_flux = getattr(volume_form, "volume_numericalflux", CentralFlux()).code
        d.surface_flux = surface_numericalflux.code
        d.precision = _lib.PRECISION_FP64 if precision == "fp64" else _lib.PRECISION_FP32_BULK
        d.gamma = law.gamma
        for i in range(3):
            d.advection_velocity[i] = law.u[i] if i < len(law.u) else 0.0
        keep = [
            np.asfortranarray(grid.cell.D, dtype=np.float64),
            np.ascontiguousarray(grid.cell.w, dtype=np.float64),
            np.asfortranarray(grid.volume_metrics, dtype=np.float64),
            np.asfortranarray(grid.surface_metrics, dtype=np.float64),
            np.asfortranarray(grid.vmapM, dtype=np.int64),
            np.asfortranarray(grid.vmapP, dtype=np.int64),
            np.asfortranarray(grid.boundarycodes, dtype=np.int64),
        ]
        (d.D, d.w, d.volume_metrics, d.surface_metrics, d.vmapM, d.vmapP, d.boundary_codes) = [
            k.ctypes.data_as(ctypes.c_void_p) for k in keep
        ]
        d.device = self.device
        h = ctypes.c_void_p()
        st = L.rb200_create(ctypes.byref(d), ctypes.byref(h))
        self._h = h
        if st != 0:
            msg = L.rb200_last_error(h).decode() if h else ""
            if h:
                L.rb200_destroy(h)
            self._h = None
            raise RB200Error(st, msg)
        mortars = getattr(grid, "mortars", None)
        if mortars is not None and mortars.size:
            m = np.asfortranarray(mortars, dtype=np.int64)
            ops = [np.ascontiguousarray(a, dtype=np.float64) for a in grid.tohalves]
            st = L.rb200_set_mortars(h, m.ctypes.data_as(ctypes.c_void_p), m.shape[1],
                                     *[a.ctypes.data_as(ctypes.c_void_p) for a in ops])
            if st != 0:
                msg = L.rb200_last_error(h).decode()
                L.rb200_destroy(h)
                self._h = None
                raise RB200Error(st, msg)
        if len(directions) < grid.dim:
            mask = sum(1 << (d - 1) for d in directions)
            st = L.rb200_set_directions(h, mask)
            if st != 0:
                msg = L.rb200_last_error(h).decode()
                L.rb200_destroy(h)
                self._h = None
                raise RB200Error(st, msg)
        for tag, cond in (boundary_conditions or {}).items():
            try:
                self.set_boundary_condition(tag, cond)
            except Exception:
                L.rb200_destroy(h)
                self._h = None
                raise
        self._read_info()

    def _read_info(self):
        """rb200_get_info: `info` (10 values), `geometry`, `pipelined_ctas` and
        `cluster_ctas` (CTAs of the one-launch cluster step kernel of small weak-form
        advection bricks; 0 when the steps run as stage launches)."""
        info = (ctypes.c_int64 * 10)()
        _lib.check(_lib.lib().rb200_get_info(self._h, info, 10), self._h)
        self.info = list(info)
        self.geometry = "affine" if info[4] == 0 else "curved"
        self.pipelined_ctas = int(info[8])
        self.cluster_ctas = int(info[9])

    def set_boundary_condition(self, tag, condition):
        """The exterior state of the faces with boundary code `tag` (1..8): a sequence of
        Ns values, "wall", or None (see the class docstring)."""
        if condition is None:
            kind, st = 0, None
        elif isinstance(condition, str):
            if condition != "wall":
                raise ValueError("a boundary condition is a state, 'wall' or None")
            kind, st = 2, None
        else:
            st = np.ascontiguousarray(condition, dtype=np.float64).ravel()
            if st.size != self.law.ns:
                raise ValueError(f"a prescribed boundary state has {self.law.ns} values")
            kind = 1
        _lib.check(_lib.lib().rb200_set_boundary_condition(self._h, int(tag), kind,
                                                           None if st is None else st.ctypes.data_as(ctypes.c_void_p)),
                   self._h)
        self._read_info()  # the kernel choice may have changed

    def set_kernel_path(self, path):
        """'auto' (pipelined kernel where eligible) or 'generic' (generic stage kernel only)."""
        _lib.check(_lib.lib().rb200_set_kernel_path(self._h, {"auto": 0, "generic": 1}[path]), self._h)
        self._read_info()

    def sync_status(self):
        """Synchronizes and raises RB200Error(TIMEOUT) if a kernel gave up a bounded wait."""
        _lib.check(_lib.lib().rb200_sync_status(self._h, _stream_ptr()), self._h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _lib.lib().rb200_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def MJ(self):
        return self.grid.volume_weights()

    def __call__(self, dq, q, time=0.0, increment=True):
        """(dg::DGSEM)(dq, q, time; increment) (dgsem.jl:84-126)."""
        _lib.check(_lib.lib().rb200_tendency(self._h, dq.ptr(), q.ptr(), float(time), int(bool(increment)),
                                             _stream_ptr()), self._h)
        return dq

    def set_active_elements(self, num_active):
        """Elements 0..num_active-1 are computed; the rest are ghost elements filled by an
        exchange (Raven's GridArray ghost cells, gridarrays.jl:26-40)."""
        _lib.check(_lib.lib().rb200_set_active_elements(self._h, int(num_active)), self._h)

    def lsrk54_stage(self, q_in, q_out, dq, stage, time, dt):
        """One LSRK(5,4) stage from q_in to q_out (odesolvers.jl:163-189)."""
        _lib.check(_lib.lib().rb200_lsrk54_stage(self._h, q_in.ptr(), q_out.ptr(), dq.ptr() if dq is not None else None,
                                                 int(stage), float(time), float(dt), _stream_ptr()), self._h)

    def lsrk54_stage_range(self, q_in, q_out, dq, stage, e_begin, e_end, time, dt):
        """One LSRK(5,4) stage on the active elements e_begin..e_end-1."""
        _lib.check(_lib.lib().rb200_lsrk54_stage_range(self._h, q_in.ptr(), q_out.ptr(),
                                                       dq.ptr() if dq is not None else None, int(stage),
                                                       int(e_begin), int(e_end), float(time), float(dt),
                                                       _stream_ptr()), self._h)

    def lsrk_stage_range(self, q_in, q_out, dq, rka, rkb, e_begin, e_end, time, dt):
        """One stage of any low-storage table (coefficients rka, rkb) on the active
        elements e_begin..e_end-1."""
        _lib.check(_lib.lib().rb200_lsrk_stage_range(self._h, q_in.ptr(), q_out.ptr(),
                                                     dq.ptr() if dq is not None else None, float(rka), float(rkb),
                                                     int(e_begin), int(e_end), float(time), float(dt),
                                                     _stream_ptr()), self._h)

    def lsrk54_steps(self, q, dq, time, dt, nsteps):
        _lib.check(_lib.lib().rb200_lsrk54_step(self._h, q.ptr(), dq.ptr() if dq is not None else None,
                                                float(time), float(dt), int(nsteps), _stream_ptr()), self._h)

    def lsrk144_steps(self, q, dq, time, dt, nsteps):
        """nsteps LSRK(14,4) steps (odesolvers.jl:191-239), fused stages."""
        _lib.check(_lib.lib().rb200_lsrk144_step(self._h, q.ptr(), dq.ptr() if dq is not None else None,
                                                 float(time), float(dt), int(nsteps), _stream_ptr()), self._h)

    def lsrk54_steps_host(self, q_host, time, dt, nsteps):
        """nsteps LSRK(5,4) steps on a host array (Np, Ns, E) column-major, in place."""
        if not (q_host.flags["F_CONTIGUOUS"] and q_host.dtype == np.float64):
            raise ValueError("q_host must be a column-major float64 array")
        _lib.check(_lib.lib().rb200_lsrk54_step_host(self._h, q_host.ctypes.data_as(ctypes.c_void_p), float(time),
                                                     float(dt), int(nsteps), _stream_ptr()), self._h)

    def face_vmapP(self):
        torch = _torch()
        out = torch.empty((self.grid.E, 2 * self.grid.dim * self.grid.nfp), dtype=torch.int64, device="cuda")
        _lib.check(_lib.lib().rb200_face_vmapP(self._h, ctypes.c_void_p(out.data_ptr()), _stream_ptr()), self._h)
        return np.asfortranarray(out.cpu().numpy().T)


# ------------------------------------------------------------------------------- LSRK(5,4)


# LSRK(5,4) stage times c_i (odesolvers.jl:181-187), rationals rounded once to Float64
LSRK54_RKC = (0.0, 1432997174477 / 9575080441755, 2526269341429 / 6820363962896,
              2006345519317 / 3224310063776, 2802321613138 / 2924317926251)


class LSRK54:
    """LSRK54(rhs!, q, dt; t0 = 0) (src/balancelaws/odesolvers.jl:63-66, 32-49)."""

    def __init__(self, dg, q, dt, t0=0.0):
        self.dg = dg
        self.dt = float(dt)
        self.time = float(t0)
        self.dq = q.similar()  # fill!(dq, 0)
        self._stage_out = None

    def dostep(self, q, nsteps=1, after_stage=None):
        """dostep!(q, lsrk, after_stage) (odesolvers.jl:51-61), `nsteps` times with the
        same dt.  Without `after_stage` the steps run as fused, graph-replayed stage
        kernels.  With it, every stage is its own kernel (rb200_lsrk54_stage) whose
        result is written back into `q` before `after_stage(stagetime, q)` is called
        with stagetime = time + c_i dt, so the callback may read or change q in place,
        as in the reference."""
        if after_stage is None:
            self.dg.lsrk54_steps(q, self.dq, self.time, self.dt, nsteps)
            for _ in range(nsteps):
                self.time += self.dt
            return
        if self._stage_out is None or self._stage_out.data.shape != q.data.shape:
            self._stage_out = q.similar()
        out = self._stage_out
        for _ in range(nsteps):
            for stage in range(5):
                stagetime = self.time + LSRK54_RKC[stage] * self.dt
                self.dg.lsrk54_stage(q, out, self.dq, stage, stagetime, self.dt)
                q.data.copy_(out.data)
                after_stage(stagetime, q)
            self.time += self.dt


class LSRK:
    """LSRK(rhs!, rka, rkb, rkc, q, dt, t0) (src/balancelaws/odesolvers.jl:32-61): any
    low-storage (2N) Runge-Kutta table of 1..32 stages on the fused stage kernels.
    dostep(q, n) runs n fused steps (rb200_lsrk_step); with `after_stage` every stage is
    its own kernel (rb200_lsrk_stage), written back into q before
    after_stage(time + rkc_i dt, q) is called, as LSRK54.dostep does."""

    def __init__(self, dg, rka, rkb, rkc, q, dt, t0=0.0):
        self.dg = dg
        self.rka = np.ascontiguousarray(rka, dtype=np.float64)
        self.rkb = np.ascontiguousarray(rkb, dtype=np.float64)
        self.rkc = np.ascontiguousarray(rkc, dtype=np.float64)
        if not (self.rka.size == self.rkb.size == self.rkc.size) or not 1 <= self.rka.size <= 32:
            raise ValueError("rka, rkb and rkc must have the same length, 1..32")
        self.dt = float(dt)
        self.time = float(t0)
        self.dq = q.similar()  # fill!(dq, 0)
        self._stage_out = None

    def dostep(self, q, nsteps=1, after_stage=None):
        """dostep!(q, lsrk, after_stage) (odesolvers.jl:51-61), `nsteps` times."""
        L, h = _lib.lib(), self.dg._h
        if after_stage is None:
            dq = self.dq.ptr() if self.dg.precision == "fp64" else None
            _lib.check(L.rb200_lsrk_step(h, q.ptr(), dq, self.rka.ctypes.data_as(ctypes.c_void_p),
                                         self.rkb.ctypes.data_as(ctypes.c_void_p), int(self.rka.size), self.time,
                                         self.dt, int(nsteps), _stream_ptr()), h)
            for _ in range(nsteps):
                self.time += self.dt
            return
        if self._stage_out is None or self._stage_out.data.shape != q.data.shape:
            self._stage_out = q.similar()
        out = self._stage_out
        for _ in range(nsteps):
            for i in range(self.rka.size):
                stagetime = self.time + self.rkc[i] * self.dt
                _lib.check(L.rb200_lsrk_stage(h, q.ptr(), out.ptr(), self.dq.ptr(), float(self.rka[i]),
                                              float(self.rkb[i]), stagetime, self.dt, _stream_ptr()), h)
                q.data.copy_(out.data)
                after_stage(stagetime, q)
            self.time += self.dt


# LSRK(14,4) (odesolvers.jl:191-239, coefficients_lsrk144): the reference's Float64 literals
LSRK144_RKA = (0.0, -0.7188012108672410, -0.7785331173421570, -0.0053282796654044, -0.8552979934029281,
               -3.9564138245774565, -1.5780575380587385, -2.0837094552574054, -0.7483334182761610,
               -0.7032861106563359, 0.0013917096117681, -0.0932075369637460, -0.9514200470875948,
               -7.1151571693922548)
LSRK144_RKB = (0.0367762454319673, 0.3136296607553959, 0.1531848691869027, 0.0030097086818182, 0.3326293790646110,
               0.2440251405350864, 0.3718879239592277, 0.6204126221582444, 0.1524043173028741, 0.0760894927419266,
               0.0077604214040978, 0.0024647284755382, 0.0780348340049386, 5.5059777270269628)
LSRK144_RKC = (0.0, 0.0367762454319673, 0.1249685262725025, 0.2446177702277698, 0.2476149531070420,
               0.2969311120382472, 0.3978149645802642, 0.5270854589440328, 0.6981269994175695, 0.8190890835352128,
               0.8527059887098624, 0.8604711817462826, 0.8627060376969976, 0.8734213127600976)


class LSRK144(LSRK):
    """LSRK144(rhs!, q, dt; t0 = 0) (src/balancelaws/odesolvers.jl:68-71, 191-239): the
    14-stage fourth-order low-storage scheme.  The fused steps use rb200_lsrk144_step;
    stage callbacks run the stages one by one as LSRK does."""

    def __init__(self, dg, q, dt, t0=0.0):
        super().__init__(dg, LSRK144_RKA, LSRK144_RKB, LSRK144_RKC, q, dt, t0)

    def dostep(self, q, nsteps=1, after_stage=None):
        """dostep!(q, lsrk, after_stage) (odesolvers.jl:51-61), `nsteps` times."""
        if after_stage is not None:
            return super().dostep(q, nsteps, after_stage)
        self.dg.lsrk144_steps(q, self.dq, self.time, self.dt, nsteps)
        for _ in range(nsteps):
            self.time += self.dt


class RLSRK54:
    """RLSRK54(rhs!, q, dt; t0 = 0) (src/balancelaws/odesolvers.jl:73-161): LSRK(5,4) with
    relaxation, so that the entropy integral changes by exactly the stages' entropy
    production (entropy-conservative fluxes then conserve it to round-off).  `gamma` is
    the relaxation parameter, carried between steps.  FP64 operators only."""

    def __init__(self, dg, q, dt, t0=0.0):
        self.dg = dg
        self.dt = float(dt)
        self.time = float(t0)
        self.gamma = 1.0
        self.dq = q.similar()  # fill!(dq, 0)

    def dostep(self, q, nsteps=1, after_stage=None):
        """dostep!(q, rlsrk) (odesolvers.jl:118-151), `nsteps` times with the same dt.
        The stages and the relaxation run fused on the device, so a stage callback cannot
        be honoured: `after_stage` raises instead of being ignored."""
        if after_stage is not None:
            raise NotImplementedError(f"{type(self).__name__} runs its stages fused on the device; "
                                      "after_stage is not supported")
        g = ctypes.c_double(self.gamma)
        _lib.check(self._entry()(self.dg._h, q.ptr(), self.dq.ptr(), ctypes.byref(g), self.time, self.dt,
                                 int(nsteps), _stream_ptr()), self.dg._h)
        self.gamma = g.value
        for _ in range(nsteps):
            self.time += self.dt

    def _entry(self):
        return _lib.lib().rb200_rlsrk54_step


class RLSRK(RLSRK54):
    """RLSRK(rhs!, rka, rkb, rkc, q, dt, t0) (src/balancelaws/odesolvers.jl:73-151): the
    relaxation step over any low-storage table of 1..32 stages.  FP64 operators only."""

    def __init__(self, dg, rka, rkb, rkc, q, dt, t0=0.0):
        super().__init__(dg, q, dt, t0)
        self.rka = np.ascontiguousarray(rka, dtype=np.float64)
        self.rkb = np.ascontiguousarray(rkb, dtype=np.float64)
        self.rkc = np.ascontiguousarray(rkc, dtype=np.float64)
        if not (self.rka.size == self.rkb.size == self.rkc.size) or not 1 <= self.rka.size <= 32:
            raise ValueError("rka, rkb and rkc must have the same length, 1..32")

    def _entry(self):
        L = _lib.lib()
        rka, rkb, n = self.rka.ctypes.data_as(ctypes.c_void_p), self.rkb.ctypes.data_as(ctypes.c_void_p), self.rka.size

        def call(h, q, dq, g, time, dt, nsteps, stream):
            return L.rb200_rlsrk_step(h, q, dq, g, rka, rkb, int(n), time, dt, nsteps, stream)

        return call


class RLSRK144(RLSRK54):
    """RLSRK144(rhs!, q, dt; t0 = 0) (src/balancelaws/odesolvers.jl:158-161): relaxation
    over the 14 stages of LSRK(14,4).  FP64 operators only."""

    def _entry(self):
        return _lib.lib().rb200_rlsrk144_step


def solve(q, timeend, solver, after_step=None, after_stage=None, adjust_final=True):
    """solve!(q, timeend, solver; after_step, after_stage, adjust_final) (odesolvers.jl:9-30).

    The reference loop is `time = solver.time; if time + dt >= timeend (dt = timeend -
    time; final); dostep!(q, solver, after_stage); after_step(step, time, q)`.  Here the
    number of non-final steps is found by replaying the same floating-point time
    accumulation on the host, and (without callbacks) those steps go to the device in
    one call.  With `after_stage`, every stage is a separate kernel followed by the
    callback (LSRK54.dostep)."""
    step = 0
    while True:
        if after_step is None and after_stage is None:
            n, t = 0, solver.time
            while not (t + solver.dt >= timeend):
                t += solver.dt
                n += 1
            if n:
                solver.dostep(q, n)
                step += n
        time = solver.time
        final = time + solver.dt >= timeend
        if final and adjust_final:
            solver.dt = timeend - time
        if after_stage is None:
            solver.dostep(q, 1)
        else:
            solver.dostep(q, 1, after_stage=after_stage)
        step += 1
        if after_step is not None:
            after_step(step, time, q)
        if final:
            return step


# ------------------------------------------------------------------------- snapshot / resume


def snapshot(dg, q, solver):
    """The time-stepper state (q, dq, time, dt and, for RLSRK54, gamma) as bytes: a
    checksummed header, then q and the LSRK register (see rb200_snapshot)."""
    n = ctypes.c_size_t()
    _lib.check(_lib.lib().rb200_snapshot_bytes(dg._h, ctypes.byref(n)), dg._h)
    buf = ctypes.create_string_buffer(n.value)
    _lib.check(_lib.lib().rb200_snapshot(dg._h, q.ptr(), solver.dq.ptr(), solver.time, solver.dt,
                                         getattr(solver, "gamma", 1.0), buf, n.value, _stream_ptr()), dg._h)
    return buf.raw


def restore(dg, data, q, solver):
    """Loads a snapshot taken with the same discretization into q and the solver."""
    t, dt, g = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    _lib.check(_lib.lib().rb200_restore(dg._h, data, len(data), q.ptr(), solver.dq.ptr(), ctypes.byref(t),
                                        ctypes.byref(dt), ctypes.byref(g), _stream_ptr()), dg._h)
    solver.time, solver.dt = t.value, dt.value
    if hasattr(solver, "gamma"):
        solver.gamma = g.value


# ------------------------------------------------------------------------------- measures


def weightednorm(dg, q, p=2, componentwise=False):
    """weightednorm(dg, q, p=2; componentwise) (src/balancelaws/measures.jl:6-21).

    p = 2 (default), any p > 0, or p = math.inf (Julia's `Inf`): the per-field
    (sum MJ |q_s|^p)^(1/p), or max |q_s| for p = Inf, then their p-norm."""
    out = (ctypes.c_double * (q.ns + 1))()
    if p == 2:
        _lib.check(_lib.lib().rb200_weightednorm(dg._h, q.ptr(), out, _stream_ptr()), dg._h)
    else:
        _lib.check(_lib.lib().rb200_weightednorm_p(dg._h, q.ptr(), float(p), out, _stream_ptr()), dg._h)
    vals = list(out)
    return vals[: q.ns] if componentwise else vals[q.ns]


def entropyintegral(dg, q):
    """entropyintegral(dg, q) = sum(MJ .* entropy(q)) (src/balancelaws/measures.jl:23-27)."""
    out = ctypes.c_double()
    _lib.check(_lib.lib().rb200_entropy_integral(dg._h, q.ptr(), ctypes.byref(out), _stream_ptr()), dg._h)
    return out.value


def entropyproduct(dg, p, q):
    """entropyproduct(dg, p, q) = sum(MJ .* entropyvariables(p) . q) (measures.jl:28-33)."""
    out = ctypes.c_double()
    _lib.check(_lib.lib().rb200_entropy_product(dg._h, p.ptr(), q.ptr(), ctypes.byref(out), _stream_ptr()), dg._h)
    return out.value


def integrals(dg, q):
    """sum(MJ .* q_s) for every field (FP64): the conservation monitor."""
    out = (ctypes.c_double * q.ns)()
    _lib.check(_lib.lib().rb200_integrals(dg._h, q.ptr(), out, _stream_ptr()), dg._h)
    return list(out)
