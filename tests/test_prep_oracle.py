"""CPU tests of the slice-pipeline oracle (ring suppression, shift + half
padding, crop, entropy) against the reference's own code: the committed
prep_*.npz fixtures, and the live reference build when it is present."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from projects_b200 import gridrec as G

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(pattern):
    return [dict(np.load(f)) for f in sorted(glob.glob(os.path.join(GOLDEN, pattern)))]


def test_prep_fixtures_present():
    assert len(_load("prep_shift_pad_*.npz")) == 2
    assert len(_load("prep_ring_*.npz")) == 1
    assert len(_load("prep_entropy_*.npz")) == 1
    assert len(_load("prep_xcorr_*.npz")) == 1
    assert len(_load("prep_fbp_*.npz")) == 1


def test_fbp_oracle_matches_reference_fixture():
    """OptimizedFBP restated in float64: within the reference's float FFT noise."""
    z = _load("prep_fbp_*.npz")[0]
    got = O.port_optimized_fbp(z["sino"], z["theta"])
    ref = z["recon"].astype(np.float64)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-5


def test_xcorr_oracle_matches_reference_fixture():
    z = _load("prep_xcorr_*.npz")[0]
    roi = tuple(int(v) for v in z["roi"])
    for (tx, ty), ref in zip(z["trans"], z["scores"]):
        got = O.port_xcorr_score(z["templ"], z["match"], roi, tx, ty)
        assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)), (tx, ty, got, ref)
    assert abs(z["scores"][0] - 1.0) < 1e-12  # the template's own translation


@pytest.mark.parametrize("z", _load("prep_shift_pad_*.npz"))
def test_shift_pad_oracle_bit_exact(z):
    for x, ref in zip(z["shifts"], z["outs"]):
        assert np.array_equal(O.port_shift_pad(z["sino1"], x), ref[0])
        assert np.array_equal(O.port_shift_pad(z["sino2"], x), ref[1])


def test_shift_pad_odd_width_leaves_last_column_zero():
    z = _load("prep_shift_pad_63x20.npz")[0]
    out = O.port_shift_pad(z["sino1"], 1.5)
    assert out.shape == (20, 126)
    # pad 31 left, 63 data, 31 right: column 125 is never written (tomo_recon.cpp:3797-3805)
    assert np.all(out[:, 125] == 0) and np.all(out[:, :31] == out[:, 31:32])


def test_ring_oracle_matches_reference_fixture():
    z = _load("prep_ring_*.npz")[0]
    out = O.port_ring_removal(z["sino"], float(z["ring_coeff"]), 20)
    ref = z["out"].astype(np.float64)
    assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < 1e-5
    assert np.abs(out - ref).max() < 1e-4
    # the clamp keeps values >= 0 (the zero row is never rescaled); stripes are reduced
    assert out.min() >= 0.0
    src = z["sino"].astype(np.float64)
    prof = lambda s: s.mean(0)[10:90]  # noqa: E731
    assert np.abs(np.diff(prof(out), 2)).max() < np.abs(np.diff(prof(src), 2)).max()


def test_entropy_oracle_matches_reference_fixture():
    z = _load("prep_entropy_*.npz")[0]
    for (lo, hi, nb), ref in zip(z["cfg"], z["entropy"]):
        e = O.port_entropy(z["image"], lo, hi, int(nb))
        # the reference sums the per-bin terms in float
        assert abs(e - ref) < 2e-5 * max(1.0, abs(ref)), (nb, e, ref)


def test_entropy_oracle_edge_cases():
    assert O.port_entropy(np.zeros((4, 4), np.float32), 0.0, 1.0, 10) == 0.0
    x = np.array([[-0.5, 0.05, 0.15, np.nan, 2.0]], np.float32)  # -0.5 truncates to bin -5
    # bins: 0.05 -> 0, 0.15 -> 1; n counts every pixel (p = count / 5)
    e = O.port_entropy(x, 0.0, 1.0, 10)
    assert abs(e - 2 * (-(0.2) * np.log2(0.2))) < 1e-12
    y = np.array([[-0.05, 0.05]], np.float32)  # truncation toward zero: both in bin 0
    assert abs(O.port_entropy(y, 0.0, 1.0, 10)) < 1e-12


def test_crop_oracle():
    rng = np.random.default_rng(3)
    rec = rng.standard_normal((40, 44)).astype(np.float32)
    out = O.port_crop(rec, 20, 10)
    assert np.array_equal(out, rec[10:30, 10:30])
    m = O.port_crop(rec, 20, 10, radius=7)
    jj, kk = np.mgrid[0:20, 0:20]
    inside = (kk - 10) ** 2 + (jj - 10) ** 2 < 49
    assert np.array_equal(m[inside], rec[10:30, 10:30][inside]) and np.all(m[~inside] == 0)


@pytest.mark.skipif(not O.prep_ref_available(), reason="reference build absent")
def test_live_reference_shift_pad_and_ring():
    rng = np.random.default_rng(9)
    for n, a in ((33, 7), (128, 50)):
        s1 = rng.standard_normal((a, n)).astype(np.float32)
        s2 = rng.standard_normal((a, n)).astype(np.float32)
        for x in rng.uniform(-n, n, 6).astype(np.float32):
            r = O.ref_shift_pad(s1, s2, x)
            assert np.array_equal(O.port_shift_pad(s1, x), r[0])
            assert np.array_equal(O.port_shift_pad(s2, x), r[1])
        p = (rng.random((a, n)) + 0.2).astype(np.float32)
        out = O.port_ring_removal(p, 0.7, 20)
        ref = O.ref_ring_removal(p, 0.7)
        assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < 1e-5


@pytest.mark.skipif(not O.prep_ref_available(), reason="reference build absent")
def test_live_reference_xcorr():
    rng = np.random.default_rng(10)
    m = rng.standard_normal((30, 50))
    roi = (5, 40, 3, 25)
    t = rng.standard_normal((23, 36))
    for tx, ty in rng.uniform(-8, 8, (8, 2)):
        assert O.port_xcorr_score(t, m, roi, tx, ty) == pytest.approx(
            O.ref_xcorr_score(t, m, roi, tx, ty), rel=1e-12, abs=1e-14)


@pytest.mark.skipif(not O.fbp_ref_available(), reason="reference build absent")
def test_live_reference_fbp():
    rng = np.random.default_rng(14)
    th = np.sort(rng.uniform(0, 180, 37)).astype(np.float32)
    sino = rng.uniform(-6, 6, (37, 32)).astype(np.float32)  # some values outside the gate
    got = O.port_optimized_fbp(sino, th)
    ref = O.ref_optimized_fbp(sino, th).astype(np.float64)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-5


# ---- C ABI argument checks (no GPU needed: they fail before any CUDA call)

def test_prep_abi_rejects_bad_arguments():
    L = G.lib()
    dummy = 16  # any non-null address; the calls must fail before touching it
    assert L.gr_ring_removal(None, 1, 64, 10, 1.0, 20, dummy, None) == -1
    assert L.gr_ring_removal(dummy, 1, 2, 10, 1.0, 20, dummy, None) == -1
    assert L.gr_shift_pad(dummy, dummy, 1, 64, 10, dummy, 63, None) == -1  # out_width < n_det
    assert L.gr_crop_center(dummy, 10, 100, dummy, 8, 64, 1, 8, 4, 0, None) == -1
    assert L.gr_entropy(dummy, 1, 1, 4, 4, 4, 16, 16, 1.0, 0.0, 10, dummy, dummy, None) == -1
    assert L.gr_entropy(dummy, 1, 1, 4, 4, 4, 16, 16, 0.0, 1.0, 50001, dummy, dummy, None) == -1
    assert "entropy" in G.last_error()
    assert L.gr_center_search(None, dummy, dummy, 64, 10, None, 3, 0.0, 1.0, 10, None, None,
                              None, None) == -1
    import ctypes as C
    out = (C.c_double * 4)()
    assert L.gr_xcorr_scores(dummy, dummy, 64, 32, 0, 64, 0, 10, 0.0, 0.0, 1.0, 1.0, 2, 2,
                             out, None) == -1  # roi_x1 beyond the image
    assert L.gr_xcorr_scores(dummy, dummy, 64, 32, 0, 10, 0, 10, 0.0, 0.0, 1.0, 1.0, 300, 300,
                             out, None) == -1  # more than 65535 translations
    h = C.c_void_p()
    th = (C.c_float * 10)()
    assert L.gr_fbp_create(100, 10, th, 1, 0, C.byref(h)) == -1  # width not a power of two
    assert L.gr_ring_workspace_bytes(2, 64, 10) >= 4 * 2 * (64 + 10)
    assert L.gr_entropy_workspace_bytes(3, 100) == 3 * 101 * 4
    assert L.gr_entropy_workspace_bytes(0, 100) == 0
