"""The serving loop on the GPU (rb200_server_* through raven_b200.serving).

What is checked, and to which tolerance:
  * a served solve equals the same solve through the DGSEM handle bit for bit (FP64 and
    FP32 bulk), on the same kernel: the pipelined kernel for 3-D Nq=8 Euler classes, the
    generic stage kernel otherwise; and the oracle's FP64 LSRK(5,4) steps to 1e-12
    relative (max norm over the state array);
  * a solve's result in a mixed stream of other classes and other solves of its own class
    equals its result alone, bit for bit, whichever tile the autotuner picked;
  * admission by footprint: solves that do not fit wait, run when memory frees up, and
    give the same results; a solve larger than the arena is refused at submit;
  * initial data evaluated on the device agrees with the host's to 1e-13 relative after
    one step (exp, pow and sin may differ from the host's libm in the last bit);
  * error statuses: unsupported Nq, unknown tickets, timeouts of rb200_server_wait.
"""

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def S(rb, cuda_ok):
    from raven_b200 import serving

    return serving


@pytest.fixture(scope="module")
def server(S):
    s = S.Server(arena_bytes=1 << 30)
    yield s
    s.close()


def _grid(rb, spec):
    return rb.generate(rb.GridManager(rb.LobattoCell(*(spec.nq,) * spec.dim),
                                      rb.brick(spec.coordinates(), (True,) * spec.dim)))


def _host_q0(rb, spec):
    """Initial data on the host at the product grid's nodes (same formulas as the device)."""
    from raven_b200 import initial_conditions as ic

    grid = _grid(rb, spec)
    p = spec.init_params
    if spec.law == rb._lib.LAW_EULER:
        return ic.isentropic_vortex(grid, rb.EulerLaw(spec.dim), beta=p[0], u0=p[1], center=(p[2], p[3]))
    law = rb.AdvectionLaw(spec.dim, spec.advection_velocity[: spec.dim])
    return ic.sine_plus_gaussian(grid, law, sigma=p[0], center=p[1:4])


def _spec(S, dim, nq, law, K, nsteps, prec=0):
    f = S.vortex_spec if law == 1 else S.wave_spec
    return f(dim, nq, K, nsteps, precision=prec)


def _dgsem_same_kernel(rb, spec, q0):
    grid = _grid(rb, spec)
    if spec.law == rb._lib.LAW_EULER:
        law, form = rb.EulerLaw(spec.dim), rb.FluxDifferencingForm(rb.KennedyGruberFlux())
    else:
        law, form = rb.AdvectionLaw(spec.dim, spec.advection_velocity[: spec.dim]), rb.WeakForm()
    dg = rb.DGSEM(law=law, grid=grid, volume_form=form, surface_numericalflux=rb.RusanovFlux(),
                  precision="fp64" if spec.precision == 0 else "fp32_bulk")
    pipelined = spec.dim == 3 and spec.nq in (4, 6, 8)  # Euler KG and advection classes
    dg.set_kernel_path("auto" if pipelined else "generic")
    if pipelined:
        assert dg.pipelined_ctas > 0
    q = rb.GridArray.from_numpy(q0)
    dq = q.similar()
    dg.lsrk54_steps(q, dq, 0.0, spec.dt, spec.nsteps)
    dg.sync_status()
    return q.numpy()


PARITY = [
    # dim, nq, law (0 advection, 1 Euler KG), K, steps, precision
    (2, 4, 0, (6, 5), 7, 0),
    (2, 6, 1, (4, 4), 5, 0),
    (2, 8, 1, (3, 5), 4, 1),
    (3, 4, 1, (3, 4, 3), 5, 0),
    (3, 6, 0, (3, 3, 2), 6, 1),
    (3, 6, 1, (3, 3, 3), 4, 0),
    (3, 8, 1, (3, 3, 3), 3, 0),
    (3, 8, 1, (2, 3, 2), 3, 1),
    (3, 4, 0, (4, 4, 4), 6, 0),
    (3, 8, 0, (3, 4, 3), 5, 0),
    (3, 8, 0, (4, 3, 3), 4, 1),
]


def _pid(c):
    return f"{c[0]}d-nq{c[1]}-{'euler' if c[2] else 'adv'}-{'fp32' if c[5] else 'fp64'}"


@pytest.mark.parametrize("case", PARITY, ids=_pid)
def test_served_equals_dgsem(rb, S, server, case):
    dim, nq, law, K, steps, prec = case
    spec = _spec(S, dim, nq, law, K, steps, prec)
    spec.q0 = _host_q0(rb, spec)
    q_srv, lat = server.wait(server.submit(spec))
    assert lat > 0
    q_ref = _dgsem_same_kernel(rb, spec, spec.q0)
    assert q_srv.shape == q_ref.shape
    assert np.array_equal(q_srv, q_ref), f"max diff {np.abs(q_srv - q_ref).max()}"


@pytest.mark.parametrize("case", [c for c in PARITY if c[5] == 0], ids=_pid)
def test_served_fp64_against_oracle(rb, S, server, case):
    dim, nq, law, K, steps, _ = case
    spec = _spec(S, dim, nq, law, K, steps, 0)
    spec.q0 = _host_q0(rb, spec)
    q_srv, _ = server.wait(server.submit(spec))
    og = O.Grid(dim, nq, K, list(spec.lo), list(spec.hi), [1] * dim)
    if law == 1:
        olaw = O.Law(O.LAW_EULER, dim, form=O.FORM_FLUXDIFF, volume_flux=O.FLUX_KG)
    else:
        olaw = O.Law(O.LAW_ADVECTION, dim, form=O.FORM_WEAK, volume_flux=O.FLUX_CENTRAL,
                     adv=list(spec.advection_velocity[:dim]))
    q = np.asfortranarray(spec.q0.copy())
    dq = og.state(olaw)
    for i in range(steps):
        og.lsrk54_step(olaw, q, dq, i * spec.dt, spec.dt)
    # max norm over the whole state (the vortex's z momentum stays at rounding level, so
    # a per-field scale would divide by ~1e-16)
    err = np.abs(q_srv - q).max() / np.abs(q).max()
    assert err <= 1e-12, err


def _mix_specs(S):
    return [
        _spec(S, 3, 8, 1, (3, 3, 3), 6, 1),
        _spec(S, 2, 4, 0, (8, 8), 9, 1),
        _spec(S, 3, 4, 1, (4, 3, 4), 5, 1),
        _spec(S, 3, 8, 1, (2, 2, 4), 4, 1),  # same class as the first
        _spec(S, 2, 6, 1, (6, 6), 7, 1),
        _spec(S, 3, 6, 0, (3, 3, 3), 8, 1),
        _spec(S, 2, 8, 0, (5, 4), 3, 1),
        _spec(S, 3, 8, 1, (3, 3, 3), 6, 1),  # identical to the first
        _spec(S, 2, 4, 1, (10, 10), 12, 0),
        _spec(S, 3, 4, 0, (5, 5, 5), 10, 0),
        _spec(S, 2, 4, 0, (9, 7), 2, 1),  # same class as the second
        _spec(S, 3, 6, 1, (3, 3, 3), 11, 1),
    ]


def test_mix_equals_alone(rb, S):
    """Each solve of a mixed batch (nine classes, shared launches, staggered completion)
    gives exactly its result alone."""
    specs = _mix_specs(S)
    with S.Server(arena_bytes=1 << 30) as alone:
        ref = [alone.wait(alone.submit(s))[0] for s in specs]
    with S.Server(arena_bytes=1 << 30) as mixed:
        tickets = [mixed.submit(s) for s in specs]
        got = [mixed.wait(t)[0] for t in tickets]
        st = mixed.stats()
        tiles = mixed.class_tiles()
    for i, (a, b) in enumerate(zip(got, ref)):
        assert np.all(np.isfinite(b)), f"solve {i} is not finite"
        assert np.array_equal(a, b), f"solve {i}: max diff {np.abs(a - b).max()}"
    assert np.array_equal(got[0], got[7])
    assert st["completed"] == len(specs) and st["running"] == 0 and st["queued"] == 0
    assert st["arena_used"] == 0 and st["arena_peak"] > 0
    assert st["dof_updates"] == sum(s.dof_updates() for s in specs)
    assert len(tiles) == 9  # (dim, nq, law/form, precision) classes of the mix


def _footprint(spec):
    a = lambda n: (n + 255) // 256 * 256
    n = spec.np * spec.ns * spec.num_elements
    return (2 * a(8 * n) + a((4 if spec.precision else 8) * n) + a(32 * spec.num_elements)
            + a(8 * spec.dim * spec.num_elements))


def test_admission_by_footprint(rb, S):
    """With room for one solve at a time, queued solves run one after another and their
    results are unchanged; a solve larger than the whole arena is refused."""
    spec = _spec(S, 3, 8, 1, (4, 4, 4), 3, 0)
    fp = _footprint(spec)
    arena = max(int(fp * 1.5), 1 << 20)
    with S.Server(arena_bytes=1 << 30) as big:
        ref = big.wait(big.submit(spec))[0]
    with S.Server(arena_bytes=arena) as small:
        tickets = [small.submit(spec) for _ in range(3)]
        outs = [small.wait(t)[0] for t in tickets]
        st = small.stats()
        with pytest.raises(rb.RB200Error) as ei:
            small.submit(_spec(S, 3, 8, 1, (8, 8, 8), 1, 0))
        assert ei.value.status == 3  # RB200_ERR_OOM
    for o in outs:
        assert np.array_equal(o, ref)
    assert fp <= st["arena_peak"] <= arena
    assert st["completed"] == 3


@pytest.mark.parametrize("law", [0, 1])
@pytest.mark.parametrize("dim", [2, 3])
def test_device_initial_data(rb, S, server, law, dim):
    spec = _spec(S, dim, 6, law, (5,) * dim, 1, 0)
    q_dev, _ = server.wait(server.submit(spec))
    spec.q0 = _host_q0(rb, spec)
    q_host, _ = server.wait(server.submit(spec))
    scale = np.abs(q_host).max()
    assert np.abs(q_dev - q_host).max() <= 1e-13 * scale


def test_errors_and_timeouts(rb, S, server):
    with pytest.raises(rb.RB200Error) as ei:
        server.submit(_spec(S, 3, 5, 1, (3, 3, 3), 1, 0))
    assert ei.value.status == 6  # RB200_ERR_UNSUPPORTED: served orders are Nq 4, 6, 8
    with pytest.raises(rb.RB200Error) as ei:
        server.wait(123456789)
    assert ei.value.status == 1  # RB200_ERR_BAD_ARG
    t = server.submit(_spec(S, 3, 8, 1, (4, 4, 4), 400, 0), keep_result=False)
    with pytest.raises(rb.RB200Error) as ei:
        server.wait(t, timeout=0.0)
    assert ei.value.status == 5  # RB200_ERR_TIMEOUT; the ticket stays valid
    _, lat = server.wait(t, timeout=300.0)
    assert lat > 0


def test_small_poisson_stream(rb, S):
    arrivals = S.poisson_mix(3, 40, rate=400.0, k2d=(4, 12), k3d=(3, 5), steps=(5, 30))
    with S.Server(arena_bytes=2 << 30) as srv:
        res = S.run_load(srv, arrivals, keep_results=True)
        st = srv.stats()
    assert len(res["latencies"]) == 40 and np.all(res["latencies"] > 0)
    assert st["completed"] == 40 and st["arena_used"] == 0
    assert all(np.all(np.isfinite(q)) for q in res["results"])
    assert res["solves_per_s"] > 0 and res["dof_updates_per_s"] > 0
