"""The element-partitioned path on one GPU.

The ranks of a partition are emulated in one process: each rank has its own DGSEM
handle on its local grid (elements plus ghosts), and between stages the ranks' send
buffers, packed by rb200_pack_values, are copied into the receivers' buffers and
scattered by rb200_unpack_values.  No kernel waits on another rank.  Bar: the
partitioned LSRK steps equal the single-handle steps bit for bit on every rank's
elements (the per-element arithmetic is the same; only the element walk differs).
A one-rank process group (NCCL) runs DistributedDGSEM itself.
"""

import os
import socket

import numpy as np
import pytest

import oracle as O
from gpu_util import initial_state, oracle_law, product_scheme, wrap_oracle_grid

pytestmark = pytest.mark.gpu

CASES = [
    # scheme, nq, K, periodic, precision: pipelined Euler, pipelined advection, generic kernel
    ("eul_kg", 8, (6, 5, 4), (1, 1, 0), "fp64"),
    ("eul_kg", 6, (6, 5, 4), (1, 1, 1), "fp32_bulk"),
    ("adv_weak", 8, (6, 5, 4), (1, 0, 1), "fp64"),
    ("eul_kg", 5, (5, 4, 4), (1, 1, 1), "fp64"),
]


def _setup(rb, scheme, nq, K, per, precision):
    L = 1.0 if scheme.startswith("adv") else 10.0  # the Euler initial state lives on [0, 10]^3
    og = O.Grid(3, nq, K, [0.0] * 3, [L] * 3, per)
    g = wrap_oracle_grid(og)
    adv = [1.0, 0.5, -0.25] if scheme.startswith("adv") else None
    law, form = product_scheme(rb, scheme, 3, adv=adv)
    olaw = oracle_law(scheme, 3, adv=adv)
    q0 = initial_state(og, olaw, scheme, seed=31, amp=0.01)
    return og, g, law, form, q0


@pytest.mark.parametrize("nranks", [2, 3])
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-nq{c[1]}-{c[4]}")
def test_partitioned_steps_equal_single_handle(rb, cuda_ok, case, nranks):
    import torch

    from raven_b200 import distributed as D

    scheme, nq, K, per, precision = case
    og, g, law, form, q0 = _setup(rb, scheme, nq, K, per, precision)
    dt, nsteps = 1e-3, 2
    ref_dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux(), precision=precision)
    ref = rb.GridArray.from_numpy(q0)
    ref_dg.lsrk54_steps(ref, ref.similar(), 0.0, dt, nsteps)
    ref_dg.sync_status()
    q_ref = ref.numpy()

    parts = D.partition(g.E, nranks)
    locs = [D.LocalGrid(g, parts, r) for r in range(nranks)]
    dgs, halos, qs, tmps, dqs = [], [], [], [], []
    for r, L in enumerate(locs):
        dg = rb.DGSEM(law=law, grid=L.grid, volume_form=form, surface_numericalflux=rb.RusanovFlux(),
                      precision=precision)
        dg.set_active_elements(L.num_local)
        assert (dg.pipelined_ctas > 0) == (ref_dg.pipelined_ctas > 0)
        s = L.local_state(q0)
        s[:, :, L.num_local:] = 0.0
        q = rb.GridArray.from_numpy(s)
        dgs.append(dg)
        halos.append(D.HaloExchange(D.node_comm_pattern(g, parts, r, law.ns), device="cuda"))
        qs.append(q)
        tmps.append(q.similar())
        dqs.append(q.similar())
    cur, oth = qs, tmps
    for step in range(nsteps):
        for st in range(5):
            # the order of DistributedDGSEM: pack, interior elements, exchange, the rest
            for r in range(nranks):
                halos[r].pack(cur[r].data.view(-1))
                dgs[r].lsrk54_stage_range(cur[r], oth[r], dqs[r], st, 0, locs[r].num_interior, step * dt, dt)
            for r in range(nranks):
                p = halos[r].pattern
                for peer, (a, b) in zip(p.recvranks, p.recvrankindices):
                    pp = halos[peer].pattern
                    sa, sb = pp.sendrankindices[pp.sendranks.index(r)]
                    halos[r].recvbuf[a:b].copy_(halos[peer].sendbuf[sa:sb])
                halos[r].unpack(cur[r].data.view(-1))
            for r in range(nranks):
                L = locs[r]
                dgs[r].lsrk54_stage_range(cur[r], oth[r], dqs[r], st, L.num_interior, L.num_local, step * dt, dt)
            cur, oth = oth, cur
    torch.cuda.synchronize()
    for r, L in enumerate(locs):
        dgs[r].sync_status()
        got = cur[r].numpy()[:, :, : L.num_local]
        want = q_ref[:, :, L.global_elements[: L.num_local]]
        assert np.array_equal(got, want), (r, np.abs(got - want).max())


def test_pack_unpack_kernels(rb, cuda_ok):
    """rb200_pack_values / rb200_unpack_values against torch indexing, and the skipped
    out-of-range indices."""
    import torch

    from raven_b200 import _lib, _stream_ptr

    src = torch.randn(1000, dtype=torch.float64, device="cuda")
    idx = torch.tensor([5, 999, 0, 17, 2000, -3, 400], dtype=torch.int64, device="cuda")
    buf = torch.full((7,), -1.0, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().rb200_pack_values(src.data_ptr(), src.numel(), idx.data_ptr(), 7, buf.data_ptr(),
                                            _stream_ptr()))
    want = torch.where((idx >= 0) & (idx < 1000), src[idx.clamp(0, 999)], torch.full_like(buf, -1.0))
    assert torch.equal(buf, want)
    dest = torch.zeros(1000, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().rb200_unpack_values(buf.data_ptr(), idx.data_ptr(), 7, dest.data_ptr(), dest.numel(),
                                              _stream_ptr()))
    ok = (idx >= 0) & (idx < 1000)
    assert torch.equal(dest[idx[ok]], buf[ok])
    assert int((dest != 0).sum()) == int(ok.sum())


def test_reference_patterns_on_device(rb, cuda_ok):
    """The reference's three-rank patterns (test/mpitest_n3_communication.jl) through the
    device pack/unpack kernels, the ranks emulated in one process."""
    import torch

    import commpattern_cases as C
    from raven_b200 import distributed as D

    halos, data = [], []
    for r in range(3):
        halos.append(D.HaloExchange(C.pattern(D, r), device="cuda"))
        data.append(torch.arange(1, C.CASES[r]["datalength"] + 1, dtype=torch.float64, device="cuda") + 100 * r)
    for r in range(3):
        halos[r].pack(data[r])
    for r in range(3):
        p = halos[r].pattern
        for peer, (a, b) in zip(p.recvranks, p.recvrankindices):
            pp = halos[peer].pattern
            sa, sb = pp.sendrankindices[pp.sendranks.index(r)]
            halos[r].recvbuf[a:b].copy_(halos[peer].sendbuf[sa:sb])
        halos[r].unpack(data[r])
    for r in range(3):
        assert data[r].cpu().tolist() == [float(v) for v in C.CASES[r]["datacomm"]]


def test_stage_api_checks(rb, cuda_ok):
    og, g, law, form, q0 = _setup(rb, "eul_kg", 4, (3, 3, 3), (1, 1, 1), "fp64")
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux())
    q = rb.GridArray.from_numpy(q0)
    with pytest.raises(rb.RB200Error):
        dg.lsrk54_stage(q, q, q.similar(), 0, 0.0, 1e-3)  # in place
    with pytest.raises(rb.RB200Error):
        dg.lsrk54_stage(q, q.similar(), q.similar(), 5, 0.0, 1e-3)
    with pytest.raises(rb.RB200Error):
        dg.set_active_elements(g.E + 1)
    with pytest.raises(rb.RB200Error):
        dg.lsrk54_stage_range(q, q.similar(), q.similar(), 0, 3, 2, 0.0, 1e-3)
    with pytest.raises(rb.RB200Error):
        dg.lsrk54_stage_range(q, q.similar(), q.similar(), 0, 0, g.E + 1, 0.0, 1e-3)
    # five stages by hand, whole or in two element ranges, equal one step
    b = rb.GridArray.from_numpy(q0)
    dg.lsrk54_steps(b, b.similar(), 0.0, 1e-3, 1)
    for split in (None, 0, 11, g.E):
        a, dq = rb.GridArray.from_numpy(q0), q.similar()
        cur, oth = a, a.similar()
        for st in range(5):
            if split is None:
                dg.lsrk54_stage(cur, oth, dq, st, 0.0, 1e-3)
            else:
                dg.lsrk54_stage_range(cur, oth, dq, st, 0, split, 0.0, 1e-3)
                dg.lsrk54_stage_range(cur, oth, dq, st, split, g.E, 0.0, 1e-3)
            cur, oth = oth, cur
        assert np.array_equal(cur.numpy(), b.numpy()), split


@pytest.mark.parametrize("precision", ["fp32_bulk", "fp64"])
def test_stage_ranges_curved(rb, cuda_ok, precision):
    """Stages split into element ranges on a warped grid (the curved pipelined kernels in
    FP32 bulk and in FP64) equal whole stages bit for bit."""
    og = O.Grid(3, 8, (5, 4, 4), [0.0] * 3, [10.0] * 3, (1, 1, 1), O.WARP_SINE, 0.1)
    g = wrap_oracle_grid(og)
    law, form = product_scheme(rb, "eul_kg", 3)
    q0 = initial_state(og, oracle_law("eul_kg", 3), "eul_kg", seed=33, amp=0.01)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux(), precision=precision)
    assert dg.geometry == "curved" and dg.pipelined_ctas > 0
    res = []
    for split in (None, 37):
        a, dq = rb.GridArray.from_numpy(q0), rb.GridArray.from_numpy(q0).similar()
        cur, oth = a, a.similar()
        for st in range(5):
            if split is None:
                dg.lsrk54_stage(cur, oth, dq, st, 0.0, 1e-3)
            else:
                dg.lsrk54_stage_range(cur, oth, dq, st, 0, split, 0.0, 1e-3)
                dg.lsrk54_stage_range(cur, oth, dq, st, split, g.E, 0.0, 1e-3)
            cur, oth = oth, cur
        dg.sync_status()
        res.append(cur.numpy())
    assert np.array_equal(res[0], res[1])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_distributed_dgsem_one_rank(rb, cuda_ok):
    """DistributedDGSEM on a one-rank NCCL group equals the plain handle (no ghosts)."""
    import datetime

    import torch.distributed as dist

    from raven_b200 import distributed as D

    og, g, law, form, q0 = _setup(rb, "eul_kg", 8, (4, 4, 3), (1, 1, 1), "fp64")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    import torch

    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", torch.cuda.current_device()))
    try:
        ddg = D.DistributedDGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux())
        assert ddg.local.num_ghosts == 0 and ddg.pattern.recvindices.size == 0
        q = ddg.state(q0)
        ddg.lsrk54_steps(q, q.similar(), 0.0, 1e-3, 3)
        dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux())
        r = rb.GridArray.from_numpy(q0)
        dg.lsrk54_steps(r, r.similar(), 0.0, 1e-3, 3)
        assert np.array_equal(q.numpy(), r.numpy())
        n = ddg.weightednorm(q)
        assert abs(n - rb.weightednorm(dg, r)) <= 1e-14 * n
    finally:
        dist.destroy_process_group()


def test_bench_sharded_one_rank(rb, cuda_ok):
    """bench.py --sharded on one rank prints its line (no ghosts, no exchange)."""
    import json
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("MASTER_PORT", "RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--sharded", "--steps", "3", "--warmup", "3",
                        "--elements-per-side", "6"], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["n_gpus"] == 1 and line["scaling"] == "strong" and line["value"] > 0
    assert line["exchange"]["bytes_received_per_stage_all_ranks"] == 0
    assert line["exchange"]["ghost_elements_all_ranks"] == 0


@pytest.mark.parametrize("nranks", [2, 3])
def test_partitioned_any_table_walls_directions(rb, cuda_ok, nranks):
    """The partitioned stages with the generic entry (rb200_lsrk_stage_range, the LSRK144
    table), reflecting walls and a direction subset on every rank equal a single handle
    with the same settings, bit for bit."""
    import torch

    from raven_b200 import distributed as D

    og, g, law, form, q0 = _setup(rb, "eul_kg", 5, (5, 4, 3), (1, 0, 0), "fp64")
    kw = dict(law=law, volume_form=form, surface_numericalflux=rb.RusanovFlux(), directions=(1, 3),
              boundary_conditions={1: "wall"})
    dt, nsteps = 1e-3, 2
    ref_dg = rb.DGSEM(grid=g, **kw)
    ref = rb.GridArray.from_numpy(q0)
    rb.LSRK144(ref_dg, ref, dt).dostep(ref, nsteps)
    ref_dg.sync_status()
    q_ref = ref.numpy()
    parts = D.partition(g.E, nranks)
    locs = [D.LocalGrid(g, parts, r) for r in range(nranks)]
    dgs, halos, cur, oth, dqs = [], [], [], [], []
    for r, L in enumerate(locs):
        dg = rb.DGSEM(grid=L.grid, **kw)
        dg.set_active_elements(L.num_local)
        s = L.local_state(q0)
        s[:, :, L.num_local:] = 0.0
        q = rb.GridArray.from_numpy(s)
        dgs.append(dg)
        halos.append(D.HaloExchange(D.node_comm_pattern(g, parts, r, law.ns), device="cuda"))
        cur.append(q)
        oth.append(q.similar())
        dqs.append(q.similar())
    for step in range(nsteps):
        for a, b in zip(rb.LSRK144_RKA, rb.LSRK144_RKB):
            for r in range(nranks):
                halos[r].pack(cur[r].data.view(-1))
                dgs[r].lsrk_stage_range(cur[r], oth[r], dqs[r], a, b, 0, locs[r].num_interior, step * dt, dt)
            for r in range(nranks):
                p = halos[r].pattern
                for peer, (lo, hi) in zip(p.recvranks, p.recvrankindices):
                    pp = halos[peer].pattern
                    sa, sb = pp.sendrankindices[pp.sendranks.index(r)]
                    halos[r].recvbuf[lo:hi].copy_(halos[peer].sendbuf[sa:sb])
                halos[r].unpack(cur[r].data.view(-1))
            for r in range(nranks):
                L = locs[r]
                dgs[r].lsrk_stage_range(cur[r], oth[r], dqs[r], a, b, L.num_interior, L.num_local, step * dt, dt)
            cur, oth = oth, cur
    torch.cuda.synchronize()
    for r, L in enumerate(locs):
        got = cur[r].numpy()[:, :, : L.num_local]
        want = q_ref[:, :, L.global_elements[: L.num_local]]
        assert np.array_equal(got, want), (r, np.abs(got - want).max())
