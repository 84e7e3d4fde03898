"""GPU tests of the reference-shaped call surfaces: the header-only C++ GridRec
class (include/gridrec_b200.hpp), used as tomo_recon and find_shift use theirs, the
GridrecCPP 5.2 C sequence (include/gridrec_cpp_b200.h) and the one-pair host entry
point gr_reconstruct_pair_host."""
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from projects_b200 import gridrec as G
from projects_b200 import phantom as ph
from tests.test_host import _build_demo, _build_shim

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
TOL = 1e-3


def test_cxx_gridrec_class_matches_oracle(tmp_path):
    n, a = 256, 180
    s1 = ph.shepp_logan_sinogram(n, a, center=128.0, noise_seed=7)
    s2 = ph.shepp_logan_sinogram(n, a, center=128.0, noise_seed=8)
    np.stack([s1, s2]).astype(np.float32).tofile(tmp_path / "in.bin")
    exe = _build_shim(tmp_path)
    subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), str(n), str(a), "2"],
                   check=True)
    out = np.fromfile(tmp_path / "out.bin", np.float32).reshape(2, n, n)
    o1, o2 = O.port_gridrec_pair(s1, s2, ph.angles_deg(a), filter=2)
    m = o1.shape[0]
    assert ph.rel_l2(out[0, :m, :m], o1[:, :m]) < 1e-3
    assert ph.rel_l2(out[1, :m, :m], o2[:, :m]) < 1e-3
    assert np.all(out[:, m:, :] == 0) and np.all(out[:, :, m:] == 0)


def test_find_shift_style_caller_with_centre_shift(tmp_path):
    """find_shift's sequence with setCenterShift(-1.7) before init: the centre is
    n_det / 2 - 1.7; images against float64 gridrec at that centre."""
    n, a, shift = 256, 180, -1.7
    c = n // 2 + shift
    s1 = ph.random_ellipse_sinogram(3, n, a, center=c)[0]
    s2 = ph.random_ellipse_sinogram(4, n, a, center=c)[0]
    np.stack([s1, s2]).astype(np.float32).tofile(tmp_path / "in.bin")
    exe = _build_demo(tmp_path, "find_shift_demo.cpp")
    subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), str(n), str(a), "2",
                    str(shift)], check=True)
    out = np.fromfile(tmp_path / "out.bin", np.float32).reshape(2, n, n)
    o1, o2 = O.port_gridrec_pair(s1, s2, ph.angles_deg(a), center1=c, filter=2)
    m = o1.shape[0]
    assert ph.rel_l2(out[0, :m, :m], o1[:, :m]) < TOL
    assert ph.rel_l2(out[1, :m, :m], o2[:, :m]) < TOL


@pytest.mark.parametrize("layout", ["flat", "rows"])
def test_gridrec_cpp_sequence_against_oracle_and_reference(tmp_path, layout):
    """GridrecCPP's recon_init / do_recon / recon_free through the row-pointer globals,
    with contiguous rows and with every row its own allocation: images against
    float64 gridrec and against the reference's own GridrecCPP 5.2 build (centre
    127.6, Hann, sampl 1.2 -> a 512 grid and 425 x 425 images); recon_init sets
    sampl to M / M0."""
    n, a, c = 256, 180, 127.6
    s1 = ph.random_ellipse_sinogram(5, n, a, center=c)[0]
    s2 = ph.random_ellipse_sinogram(6, n, a, center=c)[0]
    np.stack([s1, s2]).astype(np.float32).tofile(tmp_path / "in.bin")
    exe = _build_demo(tmp_path, "gridrec_cpp_demo.c")
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), str(n), str(a),
                        str(c), "hann", "6.0", "1.2", layout], check=True, capture_output=True,
                       text=True)
    raw = np.fromfile(tmp_path / "out.bin", np.float32)
    m = int(raw[0])
    out = raw[1:].reshape(2, m, m)
    assert f"sampl {512 / m:.6f}" in r.stdout
    th = ph.angles_deg(a)
    o1, o2 = O.port_gridrec_pair(s1, s2, th, center1=c, filter=2, sampl=1.2)
    assert o1.shape[0] == m
    assert ph.rel_l2(out[0], o1[:, :m]) < TOL and ph.rel_l2(out[1], o2[:, :m]) < TOL
    if O.ref_available():
        r1, r2, m0 = O.refb_gridrec_pair(s1, s2, th, c, "hann", 6.0, 1.2)
        assert m0 == m
        assert ph.rel_l2(out[0], r1[:, :m]) < 2 * TOL and ph.rel_l2(out[1], r2[:, :m]) < 2 * TOL


def test_gridrec_cpp_caller_filter_function(tmp_path):
    """A caller's own filter function (not one of get_filter's) is sampled at j / pdim
    as filphase_su does: a float Hann written by the caller gives the images of the
    built-in Hann to float rounding of the filter values."""
    n, a, c = 128, 90, 64.2
    s = np.stack([ph.random_ellipse_sinogram(k, n, a, center=c)[0] for k in (7, 8)])
    s.astype(np.float32).tofile(tmp_path / "in.bin")
    exe = _build_demo(tmp_path, "gridrec_cpp_demo.c")
    outs = {}
    for name in ("hann", "custom"):
        subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / f"{name}.bin"), str(n), str(a),
                        str(c), name, "6.0", "1.0", "flat"], check=True, capture_output=True)
        raw = np.fromfile(tmp_path / f"{name}.bin", np.float32)
        outs[name] = raw[1:].reshape(2, int(raw[0]), int(raw[0]))
    assert ph.rel_l2(outs["custom"], outs["hann"]) < 1e-5


def test_reconstruct_pair_host_equals_device_pair():
    """gr_reconstruct_pair_host (pageable host buffers in, strided host images out)
    equals gr_reconstruct_pair on device buffers bit for bit, and leaves the image
    rows' extra columns untouched."""
    n, a = 256, 180
    th = ph.angles_deg(a)
    s1 = ph.random_ellipse_sinogram(9, n, a, center=128.0)[0].astype(np.float32)
    s2 = ph.random_ellipse_sinogram(10, n, a, center=128.0)[0].astype(np.float32)
    lib = G.lib()
    with G.Plan(n, a, th, filter=G.FILTER_HANN) as plan:
        m = plan.M0
        o = torch.zeros((2, m, 300), device="cuda")
        plan.reconstruct_pair(torch.from_numpy(s1).cuda(), torch.from_numpy(s2).cuda(), o[0], o[1])
        torch.cuda.synchronize()
        h = np.full((2, m, 300), -7.0, np.float32)
        rc = lib.gr_reconstruct_pair_host(plan.handle, s1.ctypes.data, s2.ctypes.data,
                                          h[0].ctypes.data, h[1].ctypes.data, 300, None)
        assert rc == 0, G.last_error()
    np.testing.assert_array_equal(h[:, :, :m], o.cpu().numpy()[:, :, :m])
    assert np.all(h[:, :, m:] == -7.0)


def test_reconstruct_pair_host_pinned_and_pageable_agree():
    """Pinned caller buffers (direct copies) and pageable ones (staged through the plan's
    pinned memory by host threads, in chunks) give the device call's images bit for bit,
    with one slice only (sino2 / out2 NULL) too, and leave the rows' extra columns alone."""
    n, a = 512, 360
    th = ph.angles_deg(a)
    s1 = ph.random_ellipse_sinogram(11, n, a, center=256.0)[0].astype(np.float32)
    s2 = ph.random_ellipse_sinogram(12, n, a, center=256.0)[0].astype(np.float32)
    lib = G.lib()
    with G.Plan(n, a, th, filter=G.FILTER_HANN) as plan:
        m = plan.M0
        o = torch.zeros((2, m, m), device="cuda")
        plan.reconstruct_pair(torch.from_numpy(s1).cuda(), torch.from_numpy(s2).cuda(), o[0], o[1])
        torch.cuda.synchronize()
        ref = o.cpu().numpy()
        ps1, ps2 = torch.from_numpy(s1).pin_memory(), torch.from_numpy(s2).pin_memory()
        pout = torch.full((2, m, m + 5), -3.0).pin_memory()
        rc = lib.gr_reconstruct_pair_host(plan.handle, ps1.data_ptr(), ps2.data_ptr(),
                                          pout[0].data_ptr(), pout[1].data_ptr(), m + 5, None)
        assert rc == 0, G.last_error()
        np.testing.assert_array_equal(pout[:, :, :m].numpy(), ref)
        assert np.all(pout[:, :, m:].numpy() == -3.0)
        one = np.full((m, m + 3), -1.0, np.float32)
        rc = lib.gr_reconstruct_pair_host(plan.handle, s1.ctypes.data, None, one.ctypes.data, None,
                                          m + 3, None)
        assert rc == 0, G.last_error()
        o1 = torch.zeros((m, m), device="cuda")
        plan.reconstruct_pair(torch.from_numpy(s1).cuda(), None, o1, None)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(one[:, :m], o1.cpu().numpy())
        assert np.all(one[:, m:] == -1.0)

