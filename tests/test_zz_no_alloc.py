"""sphg_sum_density_noalloc: the allocation-free summation density.

Hosts whose GPU memory belongs to another runtime's pool allocator, or solver
loops with a fixed memory budget, cannot let the library call cudaMalloc.
This entry point gives them the water-only step's summation density with all
working memory in one static device array.  The test calls it through the C
ABI on device buffers and checks it against the density the ordinary entry
point (sphg_single_step on a water-only scene) computes, within the FP64
tolerance of the other parity tests, on two calls in a row with different
inputs, so stale contents of the shared array would show.
"""
import ctypes as C

import numpy as np
import pytest

from sources_b200 import Solver, scenes
from sources_b200.abi import SPHG_ERR_BAD_ARG, SPHG_FP64

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 32768   # SPHG_NOALLOC_MAX_PARTICLES in include/sphg.h


def reference_density(scene):
    with Solver(scene) as g:
        g.single_step(1)
        return g.download(1).rho


def test_noalloc_density_matches_single_step(cuda_ok, lib):
    import torch

    cases = [scenes.jitter(scenes.small("dam_break", precision=SPHG_FP64), 0.0004, seed=1),
             scenes.jitter(scenes.dam_break(precision=SPHG_FP64), 0.0008, seed=2)]
    stream = torch.cuda.current_stream()
    for call, s in enumerate(cases):
        ref = reference_density(s)
        P = s.phases[0]
        dev = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
        x, h, m, r = dev(P.x), dev(P.hsml), dev(P.mass), dev(P.rho)
        out = torch.full((P.n,), -1.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        rc = lib.sphg_sum_density_noalloc(C.byref(s.params), P.n, x.data_ptr(), h.data_ptr(), m.data_ptr(),
                                          r.data_ptr(), out.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert rc == 0, (call, rc)
        # The first call on a device loads the library's device module, and
        # with it the static array (CUDA loads modules lazily); from then on a
        # call leaves free device memory unchanged.
        if call > 0:
            assert free1 == free0, ("device memory changed", call, free0 - free1)
        got = out.cpu().numpy()
        err = float(np.abs(got - ref).max() / np.abs(ref).max())
        assert err <= 1e-9, (call, err)


def test_noalloc_rejects_sizes_beyond_the_limit(cuda_ok, lib):
    import torch

    s = scenes.small("dam_break", precision=SPHG_FP64)
    n = MAX_PARTICLES + 1
    buf = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    assert lib.sphg_sum_density_noalloc(C.byref(s.params), n, p, p, p, p, p, None) == SPHG_ERR_BAD_ARG
    # a grid with more cells than the static cell arrays hold
    big = scenes.small("dam_break", precision=SPHG_FP64)
    big.params.x_max = 1.0e3
    P = big.phases[0]
    dev = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    x, h, m, r = dev(P.x), dev(P.hsml), dev(P.mass), dev(P.rho)
    out = torch.zeros(P.n, dtype=torch.float64, device="cuda")
    rc = lib.sphg_sum_density_noalloc(C.byref(big.params), P.n, x.data_ptr(), h.data_ptr(), m.data_ptr(),
                                      r.data_ptr(), out.data_ptr(), None)
    assert rc == SPHG_ERR_BAD_ARG
