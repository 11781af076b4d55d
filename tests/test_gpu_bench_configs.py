"""GPU parity at the benchmark workloads themselves.

Each test sets up the product path exactly as ``bench.py`` does for one of its workloads
(``bench.problem`` / ``bench.setup``: the same grid generator, initial data, time step,
precision and kernel selection) and compares it with the oracle on the same grid and the
same initial state.  At 32^3 elements each CTA of the persistent stage kernels walks
70-110 elements, so the element cursor, the one-element-ahead bulk copies, the mbarrier
phase flips and the double-buffered geometry/neighbour slots are exercised the way the
bench exercises them, not just on the first element of each CTA.

Tolerances (max |gpu - oracle| over max |oracle| per field; the three momentum fields
are one vector and share the scale max over |rho u|, |rho v|, |rho w|, because the
z-invariant vortex has rho w = 0 up to round-off):
  * FP64 plain form: 1e-12 for the state after one LSRK(5,4) step (Raven's own full-grid
    check takes one step too: test/balancelaws/euler/wave_3d.jl:18-61);
  * the FP64 LSRK register: 1e-12 of the size of the terms it sums.  On these smooth
    32^3 fields the register is a small difference of much larger flux-differencing
    terms (Nq partners x |S| x |flux|), so its round-off is bounded by that size, not by
    |dq|.  The kernels order the sums differently from the oracle (factored two-point
    fluxes), which moved the 32^3 register by 3e-11 of max |dq| while the state after
    the step stayed within 1e-12; a wrong neighbour or face would move it by O(|dq|);
  * FP32 bulk: 1e-6 after one step;
  * config 1 (2-D advection 16x16, N = 4, 100 steps): 1e-12.

The oracle takes a few seconds per 32^3 step on the host cores.
"""

import math

import numpy as np
import pytest

import bench
import oracle as O

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP64_DQ_TOL = 1e-12  # of the summed terms' size (term_scale)
FP32_TOL = 1e-6


def field_errors(got, ref, law):
    """Per-field max |got - ref| / scale (momentum fields share one scale)."""
    ns = ref.shape[1]
    scale = [float(np.abs(ref[:, s]).max()) for s in range(ns)]
    if ns > 1:  # Euler: fields 1..dim are the momentum vector
        dim = ns - 2
        m = max(scale[1:1 + dim])
        for s in range(1, 1 + dim):
            scale[s] = m
    return [float(np.abs(got[:, s] - ref[:, s]).max()) / max(scale[s], 1e-300) for s in range(ns)]


def term_scale(grid, law, q):
    """Size of the terms one right-hand side sums per node: Nq partners per direction x
    max |S| (S[a,i] = D[a,i] w_a / w_i - D[i,a] of esvolumeterm_dir!, dgsem.jl:576-600)
    x the largest metric factor |drdx| x the largest flux component."""
    D, w = grid.cell.D, grid.cell.w
    S = D * (w[:, None] / w[None, :]) - D.T
    dim = grid.dim
    X = grid.points
    nq = grid.nq
    h = min(float(np.abs(X[nq - 1, 0, :] - X[0, 0, :]).min()), float(np.abs(X[nq * (nq - 1), 1, :] - X[0, 1, :]).min()))
    drdx = 2.0 / h
    if law.ns == 1:
        fmax = max(abs(a) for a in law.u) * float(np.abs(q).max())
    else:
        rho, E = q[:, 0, :], q[:, dim + 1, :]
        u = [q[:, 1 + d, :] / rho for d in range(dim)]
        p = (law.gamma - 1) * (E - 0.5 * rho * sum(ui * ui for ui in u))
        fmax = max(float(np.abs(rho * u[d] * u[k] + (p if d == k else 0)).max()) for d in range(dim) for k in range(dim))
        fmax = max(fmax, max(float(np.abs(u[d] * (E + p)).max()) for d in range(dim)))
    return nq * float(np.abs(S).max()) * drdx * fmax


def register_error(got, ref, scale):
    return float(np.abs(got - ref).max()) / scale


def oracle_scheme(w):
    dim = w["dim"]
    if w["law"] == "euler":
        return O.Law(O.LAW_EULER, dim, form=O.FORM_FLUXDIFF, volume_flux=O.FLUX_KG)
    return O.Law(O.LAW_ADVECTION, dim, form=O.FORM_WEAK, adv=list(bench.ADV_VELOCITY[:dim]))


def oracle_grid(w, grid):
    """The oracle's own brick for an unwarped workload (checked against the product grid,
    node for node); for a warped one the oracle steps on the product's arrays, so that
    the comparison isolates the kernels from the grid generator (which is tested
    separately against the oracle's warped metrics at 1e-13)."""
    dim, N, K, L = w["dim"], w["N"], w["K"], w["L"]
    if not w["warp"]:
        og = O.Grid(dim, N + 1, [K] * dim, [0.0] * dim, [L] * dim, [True] * dim)
        assert og.E == grid.E
        assert np.array_equal(og.vmapP(), grid.vmapP), "oracle and product face maps differ"
        assert np.array_equal(og.points(), grid.points), "oracle and product node points differ"
        return og
    return O.Grid.from_arrays(dim, N + 1, grid.points, grid.volume_metrics, grid.surface_metrics, grid.vmapM,
                              grid.vmapP, grid.boundarycodes)


class Case:
    """One workload: product handle, oracle grid, initial state and the oracle's state and
    register after `steps` LSRK(5,4) steps."""

    def __init__(self, rb, name, steps=1, **override):
        w = dict(bench.WORKLOADS[name])
        w.update(override)
        self.w = w
        self.grid, self.law, self.dg, self.q0, self.dt = bench.setup(rb, w, 0)
        self.og = oracle_grid(w, self.grid)
        self.olaw = oracle_scheme(w)
        self.steps = steps
        qo = np.asfortranarray(self.q0.copy())
        dqo = self.og.state(self.olaw)
        for i in range(steps):
            self.og.lsrk54_step(self.olaw, qo, dqo, i * self.dt, self.dt)
        self.q_ref, self.dq_ref = qo, dqo

    def run_product(self, rb, dg=None):
        dg = dg or self.dg
        q = rb.GridArray.from_numpy(self.q0)
        dq = q.similar()
        dg.lsrk54_steps(q, dq, 0.0, self.dt, self.steps)
        dg.sync_status()
        return q.numpy(), dq.numpy()


@pytest.fixture(scope="module")
def config2(rb, cuda_ok):
    """3-D Euler, periodic 32^3 brick on [0,10]^3, N = 7, Kennedy-Gruber + Rusanov,
    isentropic vortex (strength 5, Mach 0.5), FP64: the bench's default workload."""
    return Case(rb, "euler3d_kg_n7_32_fp64")


def test_config2_fp64_one_step(rb, config2):
    c = config2
    assert c.grid.E == 32 ** 3
    assert c.dg.pipelined_ctas > 0, "the bench workload runs the pipelined brick kernel"
    assert c.grid.E / c.dg.pipelined_ctas > 50, "each CTA walks many elements"
    q, dq = c.run_product(rb)
    err_q = field_errors(q, c.q_ref, c.law)
    err_dq = register_error(dq, c.dq_ref, term_scale(c.grid, c.law, c.q0))
    assert max(err_q) <= FP64_TOL, f"state after one step beyond {FP64_TOL}: {err_q}"
    assert err_dq <= FP64_DQ_TOL, f"LSRK register beyond {FP64_DQ_TOL} of the term size: {err_dq}"


def test_config2_fp32_bulk_one_step(rb, config2):
    c = config2
    dg32 = rb.DGSEM(law=c.law, grid=c.grid, volume_form=rb.FluxDifferencingForm(rb.KennedyGruberFlux()),
                    surface_numericalflux=rb.RusanovFlux(), precision="fp32_bulk", device=0)
    assert dg32.pipelined_ctas > 0
    q, _ = c.run_product(rb, dg32)
    err = field_errors(q, c.q_ref, c.law)
    assert max(err) <= FP32_TOL, f"FP32-bulk state after one step beyond {FP32_TOL}: {err}"


def test_config2_e2e_host_path(rb, config2):
    """The end-to-end entry point (state in host memory, copied in and out by the call)
    gives the device path's result bit for bit."""
    c = config2
    qd, _ = c.run_product(rb)
    qh = np.asfortranarray(c.q0.copy())
    c.dg.lsrk54_steps_host(qh, 0.0, c.dt, 1)
    assert np.array_equal(qh, qd)


def test_config3_warped_fp32_bulk_one_step(rb, cuda_ok):
    """Config 3: the same vortex on the sine-warped 32^3 grid, FP32 bulk on the curved
    pipelined kernel."""
    c = Case(rb, "euler3d_kg_n7_32_fp32bulk_warped")
    assert c.dg.geometry == "curved" and c.dg.pipelined_ctas > 0
    q, _ = c.run_product(rb)
    err = field_errors(q, c.q_ref, c.law)
    assert max(err) <= FP32_TOL, f"FP32-bulk warped state after one step beyond {FP32_TOL}: {err}"


def test_config3_warped_fp64_one_step(rb, cuda_ok):
    """Config 3's FP64 comparison run (the warped grid in FP64)."""
    c = Case(rb, "euler3d_kg_n7_32_fp64_warped")
    assert c.dg.geometry == "curved"
    q, dq = c.run_product(rb)
    err_q = field_errors(q, c.q_ref, c.law)
    err_dq = register_error(dq, c.dq_ref, term_scale(c.grid, c.law, c.q0))
    assert max(err_q) <= FP64_TOL, f"warped FP64 state after one step beyond {FP64_TOL}: {err_q}"
    assert err_dq <= FP64_DQ_TOL, f"warped FP64 register beyond {FP64_DQ_TOL} of the term size: {err_dq}"


def test_config1_exact_100_steps(rb, cuda_ok):
    """Config 1 as stated: 2-D advection, a = (1, 0.5), periodic 16x16 brick on [0,1]^2,
    N = 4, weak form, upwind (= Rusanov) flux, u = sin(2 pi x) sin(2 pi y) + Gaussian
    (sigma = 0.05 at (0.5, 0.5)), LSRK(5,4) at CFL 0.5, 100 steps, FP64."""
    c = Case(rb, "adv2d_weak_n4_16_fp64", steps=100)
    assert c.grid.E == 256 and c.grid.np == 25
    assert c.law.u == (1.0, 0.5)
    x = c.grid.points
    expect = (np.sin(2 * np.pi * x[:, 0, :]) * np.sin(2 * np.pi * x[:, 1, :])
              + np.exp(-((x[:, 0, :] - 0.5) ** 2 + (x[:, 1, :] - 0.5) ** 2) / (2 * 0.05 ** 2)))
    assert np.allclose(c.q0[:, 0, :], expect, rtol=1e-14, atol=1e-14)
    assert c.dt == pytest.approx(0.5 * c.grid.min_node_distance() / math.hypot(1.0, 0.5), rel=1e-15)
    q, dq = c.run_product(rb)
    err_q = field_errors(q, c.q_ref, c.law)
    assert max(err_q) <= FP64_TOL, f"state after 100 steps beyond {FP64_TOL}: {err_q}"
    assert register_error(dq, c.dq_ref, term_scale(c.grid, c.law, c.q0)) <= FP64_DQ_TOL


def test_config5_adapted_one_step(rb, cuda_ok):
    """Config 5 as the bench sets it up: a 4^3 forest refined twice within radius 0.25 of
    the centre (2:1 balanced, hanging faces coupled by mortars), N = 5, density pulse,
    FP32 bulk (1e-6 after one step), and the same grid in FP64 (1e-12), against the
    oracle's mortar restatement on the product's own grid arrays."""
    w = dict(bench.WORKLOADS["euler3d_kg_n5_adapted_fp32bulk"])
    grid, law, dg32, q0, dt = bench.setup(rb, w, 0)
    assert grid.mortars.shape[1] > 0 and dg32.pipelined_ctas > 0
    og = O.Grid.from_arrays(3, w["N"] + 1, grid.points, grid.volume_metrics, grid.surface_metrics, grid.vmapM,
                            grid.vmapP, grid.boundarycodes, grid.mortars, grid.tohalves)
    olaw = oracle_scheme(w)
    qo, dqo = np.asfortranarray(q0.copy()), og.state(olaw)
    og.lsrk54_step(olaw, qo, dqo, 0.0, dt)
    dg64 = rb.DGSEM(law=law, grid=grid, volume_form=rb.FluxDifferencingForm(rb.KennedyGruberFlux()),
                    surface_numericalflux=rb.RusanovFlux(), precision="fp64", device=0)
    # the pulse starts at rest under uniform pressure, so the momenta after one step are
    # round-off-sized in FP64 (the pressure gradient cancels): all fields are measured
    # against the magnitude of the state, not against their own (near-zero) size
    scale = float(np.abs(qo).max())
    errs = {}
    for dg, tol in ((dg32, FP32_TOL), (dg64, FP64_TOL)):
        q = rb.GridArray.from_numpy(q0)
        dq = q.similar()
        dg.lsrk54_steps(q, dq, 0.0, dt, 1)
        dg.sync_status()
        got = q.numpy()
        errs[dg.precision] = ([float(np.abs(got[:, s] - qo[:, s]).max()) / scale for s in range(law.ns)], tol)
    for prec, (err, tol) in errs.items():
        assert max(err) <= tol, f"{prec} adapted state after one step beyond {tol}: {err}"
