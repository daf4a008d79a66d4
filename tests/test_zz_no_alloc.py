"""sphg_sum_density_noalloc: the allocation-free summation density.

Hosts whose GPU memory belongs to another runtime's pool allocator, or solver
loops with a fixed memory budget, cannot let the library call cudaMalloc.
This entry point gives them the water-only step's summation density with all
working memory in one static device array.  The test calls it through the C
ABI on device buffers, on two calls in a row with different inputs (so stale
contents of the shared array would show), and checks each result against the
CPU oracle's sum_density (m_particles.f90:2243-2298) and against the density
the ordinary entry point (sphg_single_step on the same water-only scene)
computes, within the FP64 tolerance of the other parity tests.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import Oracle
from sources_b200 import Solver, scenes
from sources_b200.abi import SPHG_ERR_BAD_ARG, SPHG_ERR_NONFINITE, SPHG_FP64

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 32768   # SPHG_NOALLOC_MAX_PARTICLES in include/sphg.h
SCRATCH_BYTES = 4 << 20  # the static array is about 4.3 MB


def entry_point_density(scene):
    with Solver(scene) as g:
        g.single_step(1)
        return g.download(1).rho


def oracle_density(scene):
    o = Oracle(scene)
    assert o.single_step(1) == 0   # the water-only step starts with sum_density
    return o.download(1).rho


def device_inputs(P):
    import torch
    dev = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    return dev(P.x), dev(P.hsml), dev(P.mass), dev(P.rho)


def call(lib, s, x, h, m, r, out, stream=None):
    return lib.sphg_sum_density_noalloc(C.byref(s.params), s.phases[0].n, x.data_ptr(), h.data_ptr(), m.data_ptr(),
                                        r.data_ptr(), out.data_ptr(), stream)


def test_noalloc_density_matches_oracle_and_single_step(cuda_ok, lib):
    import torch

    cases = [scenes.jitter(scenes.small("dam_break", precision=SPHG_FP64), 0.0004, seed=1),
             scenes.jitter(scenes.dam_break(precision=SPHG_FP64), 0.0008, seed=2)]
    stream = torch.cuda.current_stream()
    for k, s in enumerate(cases):
        ref = oracle_density(s)
        ep = entry_point_density(s)
        P = s.phases[0]
        x, h, m, r = device_inputs(P)
        out = torch.full((P.n,), -1.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        reserved0 = torch.cuda.memory_reserved()
        rc = call(lib, s, x, h, m, r, out, stream.cuda_stream)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert rc == 0, (k, rc)
        assert torch.cuda.memory_reserved() == reserved0
        # The first call on a device loads the library's device module, and
        # with it the static array (CUDA loads modules lazily).  From then on
        # a call allocates nothing: free device memory moves by less than the
        # array it would otherwise have needed.
        if k > 0:
            assert abs(free1 - free0) < SCRATCH_BYTES, ("device memory changed", k, free0 - free1)
        got = out.cpu().numpy()
        scale = np.abs(ref).max()
        assert float(np.abs(got - ref).max() / scale) <= 1e-9, (k, "oracle")
        assert float(np.abs(got - ep).max() / scale) <= 1e-9, (k, "sphg_single_step")


def test_noalloc_reports_nonfinite_positions(cuda_ok, lib):
    import torch

    s = scenes.small("dam_break", precision=SPHG_FP64)
    s.phases[0].x[7, 1] = np.nan
    x, h, m, r = device_inputs(s.phases[0])
    out = torch.zeros(s.phases[0].n, dtype=torch.float64, device="cuda")
    assert call(lib, s, x, h, m, r, out) == SPHG_ERR_NONFINITE
    torch.cuda.synchronize()
    # the shared array is usable again at once
    s2 = scenes.small("dam_break", precision=SPHG_FP64)
    x, h, m, r = device_inputs(s2.phases[0])
    assert call(lib, s2, x, h, m, r, out) == 0
    torch.cuda.synchronize()
    ref = oracle_density(s2)
    assert float(np.abs(out.cpu().numpy() - ref).max() / np.abs(ref).max()) <= 1e-9


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
    x, h, m, r = device_inputs(big.phases[0])
    out = torch.zeros(big.phases[0].n, dtype=torch.float64, device="cuda")
    assert call(lib, big, x, h, m, r, out) == SPHG_ERR_BAD_ARG
