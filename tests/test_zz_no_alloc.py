"""rb200_weighted_sums_noalloc: weighted sums for callers that cannot allocate.

Some callers cannot call cudaMalloc: code whose device memory belongs to a pooling
allocator (CUDA.jl, PyTorch) and code running where allocation is not allowed, such as a
monitoring hook between solver steps.  The entry point takes the state and the nodal
weights MJ as inputs, writes 2*Ns sums to a caller-owned device buffer and keeps its
partial sums in a fixed device array of the library instead of allocating.

The test calls it through the C ABI twice in a row, on two different states, and checks
each result against the handle-based entry points rb200_weightednorm and
rb200_integrals (relative tolerance 1e-13: the two reductions add in different orders).
It creates all of its data itself, so it passes alone in a fresh process and after the
other tests.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_weighted_sums_without_allocation_match_handle_api(rb, cuda_ok):
    import torch

    cell = rb.LobattoCell(5, 5, 5)
    grid = rb.generate(rb.GridManager(cell, rb.brick(tuple(rb.jl_range(0.0, 1.0, 4) for _ in range(3)),
                                                     (True, True, True))))
    law = rb.EulerLaw(3)
    dg = rb.DGSEM(law=law, grid=grid, volume_form=rb.FluxDifferencingForm(rb.KennedyGruberFlux()),
                  surface_numericalflux=rb.RusanovFlux())
    L = rb._lib.lib()
    mj = torch.from_numpy(np.ascontiguousarray(grid.volume_weights().T)).cuda()  # (E, Np) = (Np, E) col-major
    out = torch.full((2 * law.ns,), float("nan"), dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(7)
    for call in range(2):  # two calls in a row share the library's scratch array
        q0 = 1.0 + rng.random((grid.np, law.ns, grid.E)) * (call + 1)
        q = rb.GridArray.from_numpy(q0)
        st = L.rb200_weighted_sums_noalloc(q.ptr(), ctypes.c_void_p(mj.data_ptr()), grid.np, law.ns, grid.E,
                                           ctypes.c_void_p(out.data_ptr()), stream)
        assert st == 0
        got = out.cpu().numpy()
        norms = rb.weightednorm(dg, q, componentwise=True)
        ints = rb.integrals(dg, q)
        assert np.allclose(np.sqrt(got[: law.ns]), norms, rtol=1e-13, atol=0)
        assert np.allclose(got[law.ns:], ints, rtol=1e-13, atol=0)
    # sizes beyond the fixed scratch array are rejected, not truncated
    st = L.rb200_weighted_sums_noalloc(q.ptr(), ctypes.c_void_p(mj.data_ptr()), grid.np, 6, grid.E,
                                       ctypes.c_void_p(out.data_ptr()), stream)
    assert st == 6  # RB200_ERR_UNSUPPORTED
    # arrays that are not device memory of the current device are rejected before any
    # launch (a host buffer here), instead of failing later as a launch error
    host_out = np.zeros(2 * law.ns)
    st = L.rb200_weighted_sums_noalloc(q.ptr(), ctypes.c_void_p(mj.data_ptr()), grid.np, law.ns, grid.E,
                                       host_out.ctypes.data_as(ctypes.c_void_p), stream)
    assert st == 1  # RB200_ERR_BAD_ARG
