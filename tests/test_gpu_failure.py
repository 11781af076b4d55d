"""Failure detection on the GPU without a fault: a bounded mbarrier wait that nothing
completes gives up after its poll limit, the kernel records RB200_ERR_TIMEOUT in a
device status word and returns, and the context stays usable (a tendency computed right
after still matches the oracle to 1e-12)."""

import time

import numpy as np
import pytest

import oracle as O
from gpu_util import initial_state, oracle_law, product_scheme, rel_err, wrap_oracle_grid

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_the_context_survives(rb, cuda_ok):
    L = rb._lib.lib()
    t0 = time.time()
    assert L.rb200_probe_bounded_wait(1000, None) == 5  # RB200_ERR_TIMEOUT
    assert time.time() - t0 < 60
    og = O.Grid(3, 4, (2, 2, 2), [0.0] * 3, [1.0] * 3, (1, 1, 1))
    g = wrap_oracle_grid(og)
    law, form = product_scheme(rb, "eul_kg", 3)
    dg = rb.DGSEM(law=law, grid=g, volume_form=form, surface_numericalflux=rb.RusanovFlux())
    olaw = oracle_law("eul_kg", 3)
    q = initial_state(og, olaw, "eul_kg", seed=31)
    ref = og.tendency(olaw, q)
    qg = rb.GridArray.from_numpy(q)
    dqg = qg.similar()
    dg(dqg, qg, 0.0, increment=False)
    dg.sync_status()  # the handle's own status word saw no timeout
    assert rel_err(dqg.numpy(), ref) <= 1e-12


def test_fp64_rate_probe(rb, cuda_ok):
    """The FP64 throughput probe behind the bench's arithmetic roofline: a plausible
    B200 figure (nominal 37-40 TFLOP/s), and argument checks before any device call."""
    import ctypes

    L = rb._lib.lib()
    out = ctypes.c_double(0.0)
    assert L.rb200_probe_fp64_rate(3, ctypes.byref(out), None) == 1
    assert L.rb200_probe_fp64_rate(1 << 12, None, None) == 1
    assert L.rb200_probe_fp64_rate(1 << 14, ctypes.byref(out), None) == 0
    assert 10.0 < out.value < 100.0
