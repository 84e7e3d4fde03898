"""GPU test of gr_reconstruct_pair_noalloc, the entry point for callers that
cannot call cudaMalloc while they reconstruct: an application whose own memory
pool has already reserved the GPU's memory (a further cudaMalloc would fail),
or a loop that cannot accept the device-wide synchronisation cudaMalloc may
imply.

It reconstructs with the library's static device scratch array instead of the
plan's workspaces.  The test calls it through the C ABI twice in a row with
different inputs -- the array keeps the previous call's contents, so the
second call also shows that nothing stale leaks into a result -- and compares
each result with gr_reconstruct_pair on the same plan (identical bits: same
kernels, same summation order) and with the float64 oracle.  It also checks
that plans too large for the array are refused with a clear error.  This file
is collected last so a failure here comes after every other test has run.
"""
import numpy as np
import pytest

from oracle import oracle as O
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
            h1 = ph.shepp_logan_sinogram(n, a, center=256.3, noise_seed=seed)
            h2 = ph.random_ellipse_sinogram(seed, n, a, center=256.3)[0]
            s1 = torch.from_numpy(h1).cuda()
            s2 = torch.from_numpy(h2).cuda()
            ref = torch.zeros((2, plan.M0, n), device="cuda")
            got = torch.full((2, plan.M0, n), float("nan"), device="cuda")
            rc = lib.gr_reconstruct_pair(plan.handle, s1.data_ptr(), s2.data_ptr(),
                                         ref[0].data_ptr(), ref[1].data_ptr(), n, _stream())
            assert rc == 0, G.last_error()
            l0 = plan.launches()
            rc = lib.gr_reconstruct_pair_noalloc(plan.handle, s1.data_ptr(), s2.data_ptr(),
                                                 got[0].data_ptr(), got[1].data_ptr(), n,
                                                 _stream())
            assert rc == 0, G.last_error()
            assert plan.launches() - l0 in (5, 6)  # + split reduction when tiles are split
            torch.cuda.synchronize()
            plan.device_status()  # no bounded wait of the call ran out
            r = ref[:, :, :plan.M0].cpu().numpy()
            g = got[:, :, :plan.M0].cpu().numpy()
            assert np.isfinite(g).all()
            # same kernels and a fixed summation order: identical bits
            np.testing.assert_array_equal(g, r)
            o1, o2 = O.port_gridrec_pair(h1, h2, th, center1=256.3, filter=G.FILTER_SHEPP_LOGAN)
            assert ph.rel_l2(g[0], o1[:, :plan.M0]) < TOL
            assert ph.rel_l2(g[1], o2[:, :plan.M0]) < TOL


@pytest.mark.parametrize("n,a,sampl", [(2048, 1500, 1.0), (1024, 1024, 1.2)])
def test_noalloc_refuses_sizes_beyond_the_static_array(n, a, sampl):
    lib = G.lib()
    with G.Plan(n, a, ph.angles_deg(a), sampl=sampl) as plan:
        x = torch.zeros((a, n), device="cuda")
        o = torch.zeros((plan.M0, max(plan.M0, n)), device="cuda")
        rc = lib.gr_reconstruct_pair_noalloc(plan.handle, x.data_ptr(), x.data_ptr(),
                                             o.data_ptr(), o.data_ptr(), o.shape[1], _stream())
        assert rc == -5  # GR_ERR_UNSUPPORTED
        assert "static" in G.last_error()
