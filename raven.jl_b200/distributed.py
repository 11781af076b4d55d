"""Element-partitioned DGSEM across ranks: one process per GPU, face traces exchanged
between stages over torch.distributed (NCCL on GPUs, gloo on CPU).

Raven's distributed design (src/balancelaws/dgsem.jl:95-100, src/communication.jl) keeps
ghost cells behind the local cells of every GridArray (gridarrays.jl:26-40) and
exchanges them with a CommPattern around each right-hand side:
``start!(q, comm_manager)``, volume term, ``finish!(q, comm_manager)``, surface term.
Here:

* ``partition`` gives rank r the contiguous element range [E r / P, E (r + 1) / P) of the
  grid's element order (the brick's tree order, so each range is a compact block).
* ``LocalGrid`` holds the rank's elements followed by its ghost elements: the remote
  face neighbours of its elements, in global order.  Faces between local elements and
  ghosts are remapped into the local numbering; every face of a ghost maps to itself.
* ``node_comm_pattern`` builds the CommPattern (communication.jl:3-40) fields with
  0-based indices into the (Np, Ns, E + ghosts) state: only the face nodes a rank's
  kernels read from each neighbour rank, for every field (``Nfp * Ns`` values per
  partition-boundary face), not Raven's whole shared-node set.
* ``HaloExchange`` packs the send buffer, posts one grouped send/receive per neighbour
  rank and scatters the received buffer into the ghost elements.  On CUDA tensors the
  buffer fills are the rb200_pack_values / rb200_unpack_values kernels; on CPU tensors
  (gloo, host-logic tests) they are torch index operations.
* ``DistributedDGSEM`` runs LSRK(5,4) stage by stage: it posts the exchange of the
  stage's input, runs the interior elements (rb200_lsrk54_stage_range) while the face
  traces travel, waits, scatters them into the ghosts and runs the partition-boundary
  elements.  The DGSEM handle computes only the rank's own elements
  (rb200_set_active_elements).
"""

import types

import numpy as np

from . import _lib


def partition(num_elements, nranks):
    """Contiguous element ranges [(start, stop)] of the ranks (stop exclusive)."""
    if nranks < 1:
        raise ValueError("nranks must be positive")
    return [(num_elements * r // nranks, num_elements * (r + 1) // nranks) for r in range(nranks)]


def owner_of(parts, elements):
    """Rank owning each global element index."""
    stops = np.array([p[1] for p in parts], dtype=np.int64)
    return np.searchsorted(stops, np.asarray(elements, dtype=np.int64), side="right")


def _local_order(grid, parts, rank):
    """The rank's own elements in local order (interior ones, those without a face
    neighbour on another rank, first; each group in global order), the inverse map
    (global - start -> local index), the number of interior elements and the ghost
    elements (ascending global indices)."""
    e0, e1 = parts[rank]
    np_ = grid.np
    vP = np.asarray(grid.vmapP, dtype=np.int64)[:, e0:e1]
    nbr = (vP - 1) // np_
    remote = (nbr < e0) | (nbr >= e1)
    ghosts = np.unique(nbr[remote])
    own = np.arange(e0, e1, dtype=np.int64)
    boundary = remote.any(axis=0)
    order = np.concatenate([own[~boundary], own[boundary]])
    inv = np.empty(e1 - e0, dtype=np.int64)
    inv[order - e0] = np.arange(e1 - e0, dtype=np.int64)
    return order, inv, int((~boundary).sum()), ghosts


class LocalGrid:
    """The rank's elements followed by its ghost elements, as a Raven-style grid object
    the DGSEM constructor accepts (``.grid``).  The own elements come interior first
    (``num_interior`` of them), then those with a face on another rank."""

    def __init__(self, grid, parts, rank):
        e0, e1 = parts[rank]
        np_ = grid.np
        order, inv, n_int, ghosts = _local_order(grid, parts, rank)
        vP = np.asarray(grid.vmapP, dtype=np.int64)[:, order]
        nbr = (vP - 1) // np_  # global element of every face node's neighbour node
        remote = (nbr < e0) | (nbr >= e1)
        El, G = e1 - e0, len(ghosts)
        glob = np.concatenate([order, ghosts])
        local_el = np.where(remote, El + np.searchsorted(ghosts, nbr), inv[np.clip(nbr - e0, 0, El - 1)])
        vP_loc = np.empty((vP.shape[0], El + G), dtype=np.int64)
        vP_loc[:, :El] = local_el * np_ + (vP - 1) % np_ + 1
        vM = np.asarray(grid.vmapM, dtype=np.int64)[:, glob]
        vM_loc = (vM - 1) % np_ + np_ * np.arange(El + G, dtype=np.int64)[None, :] + 1
        vP_loc[:, El:] = vM_loc[:, El:]  # ghost faces map to themselves
        bc = np.zeros((grid.nfaces, El + G), dtype=np.int64)
        if getattr(grid, "boundarycodes", None) is not None:
            bc[:, :El] = np.asarray(grid.boundarycodes, dtype=np.int64)[:, order]
        self.rank, self.parts = rank, parts
        self.start, self.stop = e0, e1
        self.num_local, self.num_ghosts, self.num_interior = El, G, n_int
        self.ghosts = ghosts  # global indices of the ghost elements, ascending
        self.global_elements = glob  # global index of every local element (own, then ghosts)
        vm = np.asfortranarray(np.asarray(grid.volume_metrics)[:, :, glob])
        g = types.SimpleNamespace(
            cell=grid.cell, dim=grid.dim, nq=grid.nq, np=np_, nfp=grid.nfp, nfaces=grid.nfaces, E=El + G,
            points=np.asfortranarray(np.asarray(grid.points)[:, :, glob]),
            volume_metrics=vm,
            surface_metrics=np.asfortranarray(np.asarray(grid.surface_metrics)[:, :, glob]),
            vmapM=np.asfortranarray(vM_loc), vmapP=np.asfortranarray(vP_loc), boundarycodes=np.asfortranarray(bc),
        )
        g.volume_weights = lambda: vm[:, grid.dim * grid.dim + 1, :]
        self.grid = g

    def local_state(self, q_global):
        """The rank's (Np, Ns, E_local + ghosts) block of a global state (ghosts filled)."""
        return np.asfortranarray(np.asarray(q_global)[:, :, self.global_elements])


class CommPattern:
    """Raven's CommPattern fields (communication.jl:3-27) with 0-based flat indices into
    the rank's (Np, Ns, E_local + ghosts) state and (start, stop) slices per rank."""

    def __init__(self, recvindices, recvranks, recvrankindices, sendindices, sendranks, sendrankindices):
        self.recvindices = np.asarray(recvindices, dtype=np.int64)
        self.recvranks = list(recvranks)
        self.recvrankindices = list(recvrankindices)
        self.sendindices = np.asarray(sendindices, dtype=np.int64)
        self.sendranks = list(sendranks)
        self.sendrankindices = list(sendrankindices)


def _needed_nodes(grid, parts, reader, owner):
    """Global (element, node) pairs of rank `owner` that rank `reader`'s faces read,
    sorted by (element, node)."""
    np_ = grid.np
    r0, r1 = parts[reader]
    o0, o1 = parts[owner]
    vP = np.asarray(grid.vmapP, dtype=np.int64)[:, r0:r1].ravel() - 1
    el = vP // np_
    sel = np.unique(vP[(el >= o0) & (el < o1)])  # global node indices, sorted = (element, node) order
    return sel // np_, sel % np_


def _flat(elements_global, elements_local, nodes, np_, ns):
    """Flat indices n + Np (s + Ns e_local) of the given (element, node) pairs for every
    field, in (global element, field, node) order: the order both the sender and the
    receiver list the values in, whatever their local numbering."""
    g = np.repeat(np.asarray(elements_global, dtype=np.int64), ns)
    e = np.repeat(np.asarray(elements_local, dtype=np.int64), ns)
    n = np.repeat(np.asarray(nodes, dtype=np.int64), ns)
    s = np.tile(np.arange(ns, dtype=np.int64), len(nodes))
    return (n + np_ * (s + ns * e))[np.lexsort((n, s, g))]


def node_comm_pattern(grid, parts, rank, ns):
    """The rank's CommPattern for a law with `ns` fields (local numbering of LocalGrid)."""
    np_ = grid.np
    nranks = len(parts)
    e0, e1 = parts[rank]
    _, inv, _, ghosts = _local_order(grid, parts, rank)
    El = e1 - e0
    recv, recvranks, recvslices = [], [], []
    send, sendranks, sendslices = [], [], []
    for other in range(nranks):
        if other == rank:
            continue
        ge, gn = _needed_nodes(grid, parts, rank, other)  # what this rank reads from `other`
        if len(ge):
            idx = _flat(ge, El + np.searchsorted(ghosts, ge), gn, np_, ns)
            recvslices.append((sum(len(x) for x in recv), sum(len(x) for x in recv) + len(idx)))
            recv.append(idx)
            recvranks.append(other)
        se, sn = _needed_nodes(grid, parts, other, rank)  # what `other` reads from this rank
        if len(se):
            idx = _flat(se, inv[se - e0], sn, np_, ns)
            sendslices.append((sum(len(x) for x in send), sum(len(x) for x in send) + len(idx)))
            send.append(idx)
            sendranks.append(other)
    cat = lambda xs: np.concatenate(xs) if xs else np.zeros(0, dtype=np.int64)  # noqa: E731
    pat = CommPattern(cat(recv), recvranks, recvslices, cat(send), sendranks, sendslices)
    total = np_ * ns * (El + len(ghosts))
    if pat.sendindices.size and (pat.sendindices.min() < 0 or pat.sendindices.max() >= np_ * ns * El):
        raise AssertionError("send indices outside the rank's own elements")
    if pat.recvindices.size and (pat.recvindices.min() < np_ * ns * El or pat.recvindices.max() >= total):
        raise AssertionError("receive indices outside the rank's ghost elements")
    return pat


class HaloExchange:
    """start!/finish! of a buffered comm manager (communication.jl:296-334) over
    torch.distributed point-to-point operations."""

    def __init__(self, pattern, device=None, group=None, tag=0):
        import torch

        if not 0 <= tag <= 32767:  # the tag range of commmanager (communication.jl:167-169)
            raise ValueError(f"The tag={tag} is not in the valid range 0:32767")
        self.pattern = pattern
        self.group = group
        self.tag = tag
        self.device = torch.device("cpu") if device is None else torch.device(device)
        self.send_idx = torch.as_tensor(pattern.sendindices, dtype=torch.int64, device=self.device)
        self.recv_idx = torch.as_tensor(pattern.recvindices, dtype=torch.int64, device=self.device)
        self.sendbuf = torch.zeros(len(pattern.sendindices), dtype=torch.float64, device=self.device)
        self.recvbuf = torch.zeros(len(pattern.recvindices), dtype=torch.float64, device=self.device)
        self._reqs = []

    def pack(self, q):
        """Send buffer <- the values of the flat state q the other ranks read."""
        import torch

        if q.is_cuda:
            from . import _stream_ptr

            _lib.check(_lib.lib().rb200_pack_values(q.data_ptr(), q.numel(), self.send_idx.data_ptr(),
                                                    self.send_idx.numel(), self.sendbuf.data_ptr(), _stream_ptr()))
        else:
            torch.index_select(q, 0, self.send_idx, out=self.sendbuf)

    def unpack(self, q):
        """Ghost values of the flat state q <- receive buffer."""
        if q.is_cuda:
            from . import _stream_ptr

            _lib.check(_lib.lib().rb200_unpack_values(self.recvbuf.data_ptr(), self.recv_idx.data_ptr(),
                                                      self.recv_idx.numel(), q.data_ptr(), q.numel(), _stream_ptr()))
        else:
            q.index_copy_(0, self.recv_idx, self.recvbuf)

    def start(self, q):
        import torch.distributed as dist

        self.pack(q)
        p = self.pattern
        ops = [dist.P2POp(dist.irecv, self.recvbuf[a:b], r, self.group, self.tag)
               for r, (a, b) in zip(p.recvranks, p.recvrankindices)]
        ops += [dist.P2POp(dist.isend, self.sendbuf[a:b], r, self.group, self.tag)
                for r, (a, b) in zip(p.sendranks, p.sendrankindices)]
        self._reqs = dist.batch_isend_irecv(ops) if ops else []

    def finish(self, q):
        for r in self._reqs:
            r.wait()
        self._reqs = []
        if self.recv_idx.numel():
            self.unpack(q)

    def share(self, q):
        self.start(q)
        self.finish(q)


class DistributedDGSEM:
    """DGSEM over the ranks of a process group: this rank's elements plus ghosts on its
    GPU, LSRK(5,4) stage by stage with a ghost exchange before every stage."""

    def __init__(self, *, law, grid, surface_numericalflux, volume_form=None, directions=None,
                 boundary_conditions=None, precision="fp64", group=None, device=None):
        import torch.distributed as dist

        from . import DGSEM

        self.rank = dist.get_rank(group)
        self.nranks = dist.get_world_size(group)
        self.parts = partition(grid.E, self.nranks)
        self.local = LocalGrid(grid, self.parts, self.rank)
        self.law = law
        self.dg = DGSEM(law=law, grid=self.local.grid, surface_numericalflux=surface_numericalflux,
                        volume_form=volume_form, directions=directions, boundary_conditions=boundary_conditions,
                        precision=precision, device=device)
        self.dg.set_active_elements(self.local.num_local)
        self.pattern = node_comm_pattern(grid, self.parts, self.rank, law.ns)
        # NCCL addresses peers by global rank
        ranks = dist.get_process_group_ranks(group) if group is not None else None
        if ranks is not None:
            self.pattern.recvranks = [ranks[r] for r in self.pattern.recvranks]
            self.pattern.sendranks = [ranks[r] for r in self.pattern.sendranks]
        self.halo = HaloExchange(self.pattern, device=f"cuda:{self.dg.device}", group=group)
        self._qtmp = None
        # a grouped point-to-point call must not be a group's first collective unless
        # every rank takes part in it; a rank without neighbour ranks posts none
        dist.barrier(group=group)

    def state(self, q_global):
        """This rank's GridArray (elements and ghosts) of a global host state."""
        from . import GridArray

        return GridArray.from_numpy(self.local.local_state(q_global))

    def lsrk54_steps(self, q, dq, time, dt, nsteps):
        """nsteps of LSRK(5,4) on this rank's elements (dostep!, odesolvers.jl:51-66)."""
        if self._qtmp is None or self._qtmp.data.shape != q.data.shape:
            self._qtmp = q.similar()
        cur, oth = q, self._qtmp
        n_int, n_loc = self.local.num_interior, self.local.num_local
        for step in range(nsteps):
            t = time + step * dt
            for s in range(5):
                # start!: pack and post the exchange; the interior elements read no ghost
                # and run while it is in flight; finish!, then the partition-boundary ones
                self.halo.start(cur.data.view(-1))
                self.dg.lsrk54_stage_range(cur, oth, dq, s, 0, n_int, t, dt)
                self.halo.finish(cur.data.view(-1))
                self.dg.lsrk54_stage_range(cur, oth, dq, s, n_int, n_loc, t, dt)
                cur, oth = oth, cur
        if cur is not q:
            q.data.copy_(cur.data)

    def lsrk_steps(self, q, dq, rka, rkb, rkc, time, dt, nsteps):
        """nsteps of LSRK(rhs!, rka, rkb, rkc, ...) on this rank's elements, any table."""
        if self._qtmp is None or self._qtmp.data.shape != q.data.shape:
            self._qtmp = q.similar()
        cur, oth = q, self._qtmp
        n_int, n_loc = self.local.num_interior, self.local.num_local
        for step in range(nsteps):
            t = time + step * dt
            for a, b, c in zip(rka, rkb, rkc):
                self.halo.start(cur.data.view(-1))
                self.dg.lsrk_stage_range(cur, oth, dq, a, b, 0, n_int, t + c * dt, dt)
                self.halo.finish(cur.data.view(-1))
                self.dg.lsrk_stage_range(cur, oth, dq, a, b, n_int, n_loc, t + c * dt, dt)
                cur, oth = oth, cur
        if cur is not q:
            q.data.copy_(cur.data)

    def weightednorm(self, q, p=2, componentwise=False):
        """weightednorm over all ranks (measures.jl:6-21): each field's sum of MJ |q|^p is
        added over the ranks with one all-reduce (MPI.SUM), or its maximum |q| taken with
        one all-reduce (MPI.MAX) for p = Inf; then the p-norm over the fields."""
        import math

        import torch
        import torch.distributed as dist

        from . import weightednorm

        per = weightednorm(self.dg, q, p, componentwise=True)
        dev = f"cuda:{self.dg.device}"
        if math.isinf(p):
            t = torch.tensor(per, dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.halo.group)
            comp = [float(v) for v in t.tolist()]
            return comp if componentwise else max(comp)
        t = torch.tensor([v ** p for v in per], dtype=torch.float64, device=dev)
        dist.all_reduce(t, group=self.halo.group)
        comp = [float(v) ** (1.0 / p) for v in t.tolist()]
        if componentwise:
            return comp
        return sum(c ** p for c in comp) ** (1.0 / p)
