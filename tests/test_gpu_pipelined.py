"""The persistent TMA-pipelined kernels (3-D, Nq = 4, 6 and 8, unwarped brick: Kennedy-Gruber /
entropy-conservative flux differencing, and weak-form advection) against the oracle and
against the generic stage kernel.  The grids have more elements than the kernel has CTAs, so every CTA
walks several elements through both halves of its shared-memory double buffer.

Tolerances: FP64 1e-12 relative (max norm per field); FP32 bulk 5e-5 for a tendency
and 1e-6 relative on the state after two steps of dt = 1e-3 (the flux-differencing sum
cancels terms ~100x larger than the tendency, so FP32 rounding shows at ~1e-8 of the
state); kernel paths agree to 1e-13.
"""

import numpy as np
import pytest

import oracle as O
from gpu_util import initial_state, oracle_law, product_scheme, rel_err, wrap_oracle_grid

pytestmark = pytest.mark.gpu

SCHEMES = ["eul_kg", "eul_ec"]


# Nq and a grid with more elements than the kernel has CTAs at that Nq
NQS = [(8, (9, 8, 7)), (6, (12, 12, 10)), (4, (20, 20, 16))]


def _build(rb, scheme, K=(8, 8, 7), per=(1, 1, 0), precision="fp64", nq=8):
    og = O.Grid(3, nq, K, [0.0] * 3, [10.0] * 3, per)
    g = wrap_oracle_grid(og)
    law, form = product_scheme(rb, scheme, 3)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux(), precision=precision)
    return og, dg, oracle_law(scheme, 3), law


@pytest.mark.parametrize("nqk", NQS, ids=lambda c: f"nq{c[0]}")
@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("increment", [False, True])
def test_pipelined_tendency_fp64(rb, cuda_ok, scheme, increment, nqk):
    og, dg, olaw, law = _build(rb, scheme, K=nqk[1], nq=nqk[0])
    assert dg.pipelined_ctas > 0 and og.E > dg.pipelined_ctas
    q = initial_state(og, olaw, scheme, seed=11, amp=0.01)
    dq0 = initial_state(og, olaw, scheme, seed=12, amp=0.01) if increment else og.state(olaw)
    ref = og.tendency(olaw, q, dq=np.asfortranarray(dq0.copy()), increment=increment)
    qg, dqg = rb.GridArray.from_numpy(q), rb.GridArray.from_numpy(dq0)
    dg(dqg, qg, 0.0, increment=increment)
    dg.sync_status()
    got = dqg.numpy()
    for s in range(law.ns):
        assert rel_err(got[:, s], ref[:, s]) <= 1e-12


@pytest.mark.parametrize("nqk", NQS, ids=lambda c: f"nq{c[0]}")
@pytest.mark.parametrize("scheme", SCHEMES)
def test_pipelined_steps_fp64_and_paths_agree(rb, cuda_ok, scheme, nqk):
    og, dg, olaw, law = _build(rb, scheme, K=nqk[1], nq=nqk[0])
    q = initial_state(og, olaw, scheme, seed=13, amp=0.01)
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(2):
        og.lsrk54_step(olaw, qo, dqo, i * 1e-3, 1e-3)
    qa = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, qa, 1e-3).dostep(qa, 2)
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(qa.numpy()[:, s], qo[:, s]) <= 1e-12
    dg.set_kernel_path("generic")
    qb = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, qb, 1e-3).dostep(qb, 2)
    dg.set_kernel_path("auto")
    assert rel_err(qa.numpy(), qb.numpy()) <= 1e-13


@pytest.mark.parametrize("nqk", NQS, ids=lambda c: f"nq{c[0]}")
@pytest.mark.parametrize("scheme", SCHEMES)
def test_pipelined_fp32_bulk_steps(rb, cuda_ok, scheme, nqk):
    og, dg, olaw, law = _build(rb, scheme, precision="fp32_bulk", K=nqk[1], nq=nqk[0])
    q = initial_state(og, olaw, scheme, seed=14, amp=0.01)
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(2):
        og.lsrk54_step(olaw, qo, dqo, i * 1e-3, 1e-3)
    qg = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, qg, 1e-3).dostep(qg, 2)
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(qg.numpy()[:, s], qo[:, s]) <= 1e-6
    # the tendency in FP32-bulk mode goes through the generic kernel (FP64 dq output)
    ref = og.tendency(olaw, q)
    dqg = qg.similar()
    dg(dqg, rb.GridArray.from_numpy(q), 0.0, increment=False)
    for s in range(law.ns):
        assert rel_err(dqg.numpy()[:, s], ref[:, s]) <= 5e-5


ADV = [1.0, 0.5, -0.25]
# the advection kernel runs more CTAs per SM, so its grids are larger
ADV_NQS = [(8, (12, 12, 10)), (6, (12, 12, 10)), (4, (20, 20, 16))]


def _build_adv(rb, nq, K, per=(1, 1, 0), precision="fp64", surface="rusanov"):
    og = O.Grid(3, nq, K, [0.0] * 3, [1.0] * 3, per)
    g = wrap_oracle_grid(og)
    law, form = product_scheme(rb, "adv_weak", 3, adv=ADV)
    sflux = rb.RusanovFlux() if surface == "rusanov" else rb.CentralFlux()
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=sflux, precision=precision)
    olaw = O.Law(O.LAW_ADVECTION, 3, form=O.FORM_WEAK, volume_flux=O.FLUX_CENTRAL, adv=ADV,
                 surface_flux=O.FLUX_RUSANOV if surface == "rusanov" else O.FLUX_CENTRAL)
    return og, dg, olaw


@pytest.mark.parametrize("nqk", ADV_NQS, ids=lambda c: f"nq{c[0]}")
@pytest.mark.parametrize("surface", ["rusanov", "central"])
@pytest.mark.parametrize("increment", [False, True])
def test_pipelined_advection_tendency_fp64(rb, cuda_ok, surface, increment, nqk):
    """The pipelined weak-form advection kernel (one field) against the oracle, with open
    faces along z (default boundary state), 1e-12 relative."""
    og, dg, olaw = _build_adv(rb, nqk[0], nqk[1], surface=surface)
    assert dg.pipelined_ctas > 0 and og.E > dg.pipelined_ctas
    q = initial_state(og, olaw, "adv_weak", seed=21)
    dq0 = initial_state(og, olaw, "adv_weak", seed=22) if increment else og.state(olaw)
    ref = og.tendency(olaw, q, dq=np.asfortranarray(dq0.copy()), increment=increment)
    qg, dqg = rb.GridArray.from_numpy(q), rb.GridArray.from_numpy(dq0)
    dg(dqg, qg, 0.0, increment=increment)
    dg.sync_status()
    assert rel_err(dqg.numpy(), ref) <= 1e-12


@pytest.mark.parametrize("nqk", ADV_NQS, ids=lambda c: f"nq{c[0]}")
def test_pipelined_advection_steps(rb, cuda_ok, nqk):
    """Three LSRK steps against the oracle (FP64 1e-12; FP32 bulk 1e-6) and the FP64 run
    against the generic kernel (1e-13)."""
    og, dg, olaw = _build_adv(rb, nqk[0], nqk[1])
    q = initial_state(og, olaw, "adv_weak", seed=23)
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(3):
        og.lsrk54_step(olaw, qo, dqo, i * 1e-3, 1e-3)
    qa = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, qa, 1e-3).dostep(qa, 3)
    dg.sync_status()
    assert rel_err(qa.numpy(), qo) <= 1e-12
    dg.set_kernel_path("generic")
    qb = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, qb, 1e-3).dostep(qb, 3)
    dg.set_kernel_path("auto")
    assert rel_err(qa.numpy(), qb.numpy()) <= 1e-13
    og32, dg32, _ = _build_adv(rb, nqk[0], nqk[1], precision="fp32_bulk")
    assert dg32.pipelined_ctas > 0 and og.E > dg32.pipelined_ctas
    qc = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg32, qc, 1e-3).dostep(qc, 3)
    dg32.sync_status()
    assert rel_err(qc.numpy(), qo) <= 1e-6


def test_misaligned_state_falls_back_to_generic_kernel(rb, cuda_ok):
    import torch

    og, dg, olaw, law = _build(rb, "eul_kg", K=(3, 2, 2), per=(1, 1, 1))
    q = initial_state(og, olaw, "eul_kg", seed=15)
    ref = og.tendency(olaw, q)
    n = q.size
    buf = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
    qv = rb.GridArray(buf[1:].view(og.E, law.ns, og.np), law.ns, og.np, og.E)  # 8-byte aligned only
    qv.data.copy_(rb.GridArray.from_numpy(q).data)
    dqg = rb.GridArray.zeros(law, og)
    dg(dqg, qv, 0.0, increment=False)
    assert rel_err(dqg.numpy(), ref) <= 1e-12


@pytest.mark.parametrize("warp,per", [(O.WARP_SINE, (1, 1, 1)), (O.WARP_SINE, (1, 0, 1)),
                                      (O.WARP_IDENTITY_CURVED, (1, 1, 0))], ids=["sine", "sine-open-y", "identity"])
def test_curved_pipelined_fp32_bulk_steps(rb, cuda_ok, warp, per):
    """The curved-grid pipelined kernel (FP32 bulk, Kennedy-Gruber) against the oracle
    after two steps (1e-6 relative, as for the brick kernel) and against the generic
    kernel after five steps, the last three replayed from a CUDA graph (1e-6)."""
    og = O.Grid(3, 8, (8, 8, 7), [0.0] * 3, [10.0] * 3, per, warp, 0.1 if warp == O.WARP_SINE else 0.0)
    g = wrap_oracle_grid(og)
    law, form = product_scheme(rb, "eul_kg", 3)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux(), precision="fp32_bulk")
    olaw = oracle_law("eul_kg", 3)
    assert dg.geometry == "curved" and dg.pipelined_ctas > 0 and og.E > dg.pipelined_ctas
    q = initial_state(og, olaw, "eul_kg", seed=16, amp=0.01)
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(2):
        og.lsrk54_step(olaw, qo, dqo, i * 1e-3, 1e-3)
    qg = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, qg, 1e-3).dostep(qg, 2)
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(qg.numpy()[:, s], qo[:, s]) <= 1e-6, s
    qa = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, qa, 1e-3).dostep(qa, 5)
    dg.sync_status()
    dg.set_kernel_path("generic")
    qb = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, qb, 1e-3).dostep(qb, 5)
    dg.set_kernel_path("auto")
    for s in range(law.ns):
        assert rel_err(qa.numpy()[:, s], qb.numpy()[:, s]) <= 1e-6, s


@pytest.mark.parametrize("warp,per", [(O.WARP_SINE, (1, 1, 1)), (O.WARP_SINE, (1, 0, 1)),
                                      (O.WARP_IDENTITY_CURVED, (1, 1, 0))], ids=["sine", "sine-open-y", "identity"])
def test_curved_pipelined_fp64_steps(rb, cuda_ok, warp, per):
    """The curved-grid pipelined kernel in FP64 (Kennedy-Gruber) against the oracle after
    three steps (1e-12 relative per field, the register 1e-11) on a grid with more
    elements than CTAs, and against the generic curved kernel after five steps, the last
    three replayed from a CUDA graph (1e-12)."""
    og = O.Grid(3, 8, (8, 8, 7), [0.0] * 3, [10.0] * 3, per, warp, 0.1 if warp == O.WARP_SINE else 0.0)
    g = wrap_oracle_grid(og)
    law, form = product_scheme(rb, "eul_kg", 3)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux(), precision="fp64")
    olaw = oracle_law("eul_kg", 3)
    assert dg.geometry == "curved" and dg.pipelined_ctas > 0 and og.E > dg.pipelined_ctas
    q = initial_state(og, olaw, "eul_kg", seed=17, amp=0.01)
    qo, dqo = q.copy(order="F"), og.state(olaw)
    for i in range(3):
        og.lsrk54_step(olaw, qo, dqo, i * 1e-3, 1e-3)
    qg = rb.GridArray.from_numpy(q)
    solver = rb.LSRK54(dg, qg, 1e-3)
    solver.dostep(qg, 3)
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(qg.numpy()[:, s], qo[:, s]) <= 1e-12, s
    assert rel_err(solver.dq.numpy(), dqo) <= 1e-11
    qa = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, qa, 1e-3).dostep(qa, 5)
    dg.sync_status()
    dg.set_kernel_path("generic")
    qb = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, qb, 1e-3).dostep(qb, 5)
    dg.set_kernel_path("auto")
    for s in range(law.ns):
        assert rel_err(qa.numpy()[:, s], qb.numpy()[:, s]) <= 1e-12, s


def test_curved_pipelined_fp64_central_surface_flux(rb, cuda_ok):
    """The FP64 curved pipelined kernel with the central surface flux, one step against
    the oracle (1e-12)."""
    og = O.Grid(3, 8, (3, 3, 2), [0.0] * 3, [10.0] * 3, (1, 1, 1), O.WARP_SINE, 0.1)
    g = wrap_oracle_grid(og)
    law, form = product_scheme(rb, "eul_kg", 3)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.CentralFlux(), precision="fp64")
    assert dg.pipelined_ctas > 0
    olaw = O.Law(O.LAW_EULER, 3, form=O.FORM_FLUXDIFF, volume_flux=O.FLUX_KG, surface_flux=O.FLUX_CENTRAL)
    q = initial_state(og, olaw, "eul_kg", seed=18, amp=0.02)
    qo, dqo = q.copy(order="F"), og.state(olaw)
    og.lsrk54_step(olaw, qo, dqo, 0.0, 1e-3)
    qg = rb.GridArray.from_numpy(q)
    rb.LSRK54(dg, qg, 1e-3).dostep(qg, 1)
    dg.sync_status()
    for s in range(law.ns):
        assert rel_err(qg.numpy()[:, s], qo[:, s]) <= 1e-12, s
