"""GPU test of gr_reconstruct_pair_noalloc, the entry point for callers that
must not allocate device memory when they reconstruct (stream capture into a
CUDA graph, or a memory manager that already owns the GPU's memory).

It reconstructs with the library's static device scratch array instead of the
plan's workspaces.  The test calls it through the C ABI twice in a row with
different inputs -- the array keeps the previous call's contents, so the
second call also shows that nothing stale leaks into a result -- and compares
each result with gr_reconstruct_pair on the same plan.  It also checks that a
plan too large for the array is refused with a clear error.  This file is
collected last so a failure here comes after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from projects_b200 import gridrec as G
from projects_b200 import phantom as ph

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-3  # the relative-L2 bound of the other GPU parity tests


def _stream():
    return int(torch.cuda.current_stream().cuda_stream)


def test_noalloc_matches_reconstruct_pair_two_calls():
    n, a = 512, 360
    th = ph.angles_deg(a)
    lib = G.lib()
    with G.Plan(n, a, th, center=256.3, filter=G.FILTER_SHEPP_LOGAN) as plan:
        for seed in (1, 2):  # two calls in a row, different data
            s1 = torch.from_numpy(ph.shepp_logan_sinogram(n, a, center=256.3, noise_seed=seed)).cuda()
            s2 = torch.from_numpy(
                ph.random_ellipse_sinogram(seed, n, a, center=256.3)[0]).cuda()
            ref = torch.zeros((2, plan.M0, n), device="cuda")
            got = torch.full((2, plan.M0, n), float("nan"), device="cuda")
            rc = lib.gr_reconstruct_pair(plan.handle, s1.data_ptr(), s2.data_ptr(),
                                         ref[0].data_ptr(), ref[1].data_ptr(), n, _stream())
            assert rc == 0, G.last_error()
            rc = lib.gr_reconstruct_pair_noalloc(plan.handle, s1.data_ptr(), s2.data_ptr(),
                                                 got[0].data_ptr(), got[1].data_ptr(), n,
                                                 _stream())
            assert rc == 0, G.last_error()
            torch.cuda.synchronize()
            r = ref[:, :, :plan.M0].cpu().numpy()
            g = got[:, :, :plan.M0].cpu().numpy()
            assert np.isfinite(g).all()
            assert ph.rel_l2(g[0], r[0]) < TOL and ph.rel_l2(g[1], r[1]) < TOL
            # same kernels and a fixed summation order: identical bits
            np.testing.assert_array_equal(g, r)


def test_noalloc_refuses_sizes_beyond_the_static_array():
    n, a = 2048, 1500
    lib = G.lib()
    with G.Plan(n, a, ph.angles_deg(a)) as plan:
        x = torch.zeros((a, n), device="cuda")
        o = torch.zeros((plan.M0, n), device="cuda")
        rc = lib.gr_reconstruct_pair_noalloc(plan.handle, x.data_ptr(), x.data_ptr(),
                                             o.data_ptr(), o.data_ptr(), n, _stream())
        assert rc == -5  # GR_ERR_UNSUPPORTED
        assert "static" in G.last_error()
