"""GPU parity tests of the slice-pipeline kernels (ring suppression, shift + half
padding, crop, entropy, padded reconstruction, centre search) through the C ABI,
against the reference fixtures (prep_*.npz) and the oracle.

Tolerances: shift/pad and crop are bit-exact (the kernels repeat the
reference's float operations); entropy histograms are exact, entropies within
1e-5 of the oracle's double sum; ring suppression sums in a different order
than the reference, relative L2 <= 2e-5; padded reconstructions relative
L2 <= 1e-3 against float64 gridrec.
"""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from projects_b200 import gridrec as G
from projects_b200 import phantom as ph

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(pattern):
    return [dict(np.load(f)) for f in sorted(glob.glob(os.path.join(GOLDEN, pattern)))]


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("z", _load("prep_shift_pad_*.npz"))
def test_shift_pad_bit_exact_against_reference(z):
    k = len(z["shifts"])
    sinos = _dev(np.stack([z["sino1"], z["sino2"]] * k))  # slice 2c+t, shift c
    offs = np.repeat(z["shifts"], 2)
    out = G.shift_pad(sinos, offs).cpu().numpy()
    ref = z["outs"].reshape(2 * k, *z["outs"].shape[2:])
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("n_ang,n_det,width", [(50, 300, 700), (50, 301, 603), (3, 12290, 24581)],
                         ids=["aligned-rows", "unaligned-rows", "rows-longer-than-staging"])
def test_shift_pad_wide_rows_and_port(n_ang, n_det, width):
    """Rows staged in shared memory by 16-byte loads (aligned rows), by 4-byte loads
    (odd n_det), and rows too long to stage (taps read from global memory)."""
    rng = np.random.default_rng(5)
    s = rng.standard_normal((3, n_ang, n_det)).astype(np.float32)
    offs = np.array([-7.25, 0.5, 151.0], np.float32)
    out = G.shift_pad(_dev(s), offs, out_width=width).cpu().numpy()
    for i in range(3):
        assert np.array_equal(out[i], O.port_shift_pad(s[i], offs[i], width))


def test_ring_removal_against_reference():
    z = _load("prep_ring_*.npz")[0]
    x = _dev(z["sino"][None])
    G.ring_removal(x, float(z["ring_coeff"]), 20)
    out = x.cpu().numpy()[0]
    ref = z["out"]
    assert ph.rel_l2(out, ref) < 2e-5
    assert np.abs(out - ref).max() < 2e-4


def test_ring_removal_batch_against_oracle():
    rng = np.random.default_rng(6)
    S, a, n = 3, 180, 256
    s = (rng.random((S, a, n)) + 0.3).astype(np.float32)
    s[:, :, 40] *= 1.3
    s[1, 7, :] = 0.0
    x = _dev(s)
    G.ring_removal(x, 0.8, 20)
    out = x.cpu().numpy()
    for i in range(S):
        assert ph.rel_l2(out[i], O.port_ring_removal(s[i], 0.8, 20)) < 2e-5
    y = _dev(s)
    G.ring_removal(y, 0.8, 0)  # zero rounds leave the data untouched
    assert np.array_equal(y.cpu().numpy(), s)


@pytest.mark.parametrize("n_det,offset", [(256, 0), (256, 1), (258, 0), (3000, 0)],
                         ids=["aligned", "unaligned-base", "odd-width", "wider-than-2048"])
def test_ring_removal_round_kernel_forms(n_det, offset):
    """The fused round kernel at 1, 2 and 16 columns per thread, on a sinogram that
    starts 4 bytes past an allocation and with rows of zeros, against the oracle."""
    rng = np.random.default_rng(8)
    S, a = 2, 70
    s = (rng.random((S, a, n_det)) + 0.3).astype(np.float32)
    s[:, :, 17] *= 1.2
    s[0, 5, :] = 0.0
    base = torch.zeros(S * a * n_det + offset, dtype=torch.float32, device="cuda")
    x = base[offset:].view(S, a, n_det)
    x.copy_(torch.as_tensor(s))
    G.ring_removal(x, 0.9, 20)
    out = x.cpu().numpy()
    for i in range(S):
        assert ph.rel_l2(out[i], O.port_ring_removal(s[i], 0.9, 20)) < 2e-5


def test_ring_removal_full_size_and_wide_rows():
    """A batch of 2048 x 1500 slices, and rows wider than the fused round kernel
    takes (separate update and column passes)."""
    g = torch.Generator(device="cuda").manual_seed(11)
    x = torch.rand((6, 1500, 2048), device="cuda", generator=g) + 0.5
    x[:, :, 700] *= 1.1
    src = x.cpu().numpy()
    G.ring_removal(x, 1.0, 20)
    out = x.cpu().numpy()
    for i in (0, 5):
        assert ph.rel_l2(out[i], O.port_ring_removal(src[i], 1.0, 20)) < 2e-5
    rng = np.random.default_rng(12)
    w = (rng.random((1, 20, 9000)) + 0.2).astype(np.float32)
    y = _dev(w)
    G.ring_removal(y, 1.0, 20)
    assert ph.rel_l2(y.cpu().numpy()[0], O.port_ring_removal(w[0], 1.0, 20)) < 2e-5


def test_crop_and_circle_mask():
    rng = np.random.default_rng(7)
    rec = rng.standard_normal((2, 70, 75)).astype(np.float32)
    d = _dev(rec)
    for radius in (0, 15):
        out = G.crop_center(d, 40, 12, radius).cpu().numpy()
        for i in range(2):
            assert np.array_equal(out[i], O.port_crop(rec[i], 40, 12, radius))


def test_entropy_against_reference_and_port():
    z = _load("prep_entropy_*.npz")[0]
    img = z["image"]
    for (lo, hi, nb), ref in zip(z["cfg"], z["entropy"]):
        e = float(G.entropy(_dev(img[None]), lo, hi, int(nb)).cpu()[0])
        assert abs(e - O.port_entropy(img, lo, hi, int(nb))) < 1e-5
        assert abs(e - ref) < 3e-5 * max(1.0, abs(ref))
    # groups of two images score as one (find_shift scores the slice pair together)
    rng = np.random.default_rng(8)
    ims = rng.standard_normal((6, 64, 64)).astype(np.float32)
    got = G.entropy(_dev(ims), -2.0, 2.0, 1000, group=2).cpu().numpy()
    for g in range(3):
        assert abs(got[g] - O.port_entropy(ims[2 * g:2 * g + 2], -2.0, 2.0, 1000)) < 1e-5


def _padded_oracle(s, th, xoffset):
    n = s.shape[1]
    p = O.port_shift_pad(s, xoffset)
    o, _ = O.port_gridrec_pair(p, p, th, filter=2)
    return o[n // 2:n // 2 + n, n // 2:n // 2 + n]


def test_reconstruct_padded_against_oracle():
    n, a = 128, 90
    th = ph.angles_deg(a)
    s = np.stack([ph.shepp_logan_sinogram(n, a, center=63.0, noise_seed=k) for k in range(3)])
    with G.Plan(2 * n, a, th, filter=G.FILTER_HANN, max_pairs=1) as plan:
        out = G.reconstruct_padded(plan, _dev(s.astype(np.float32)), xoffset=1.0).cpu().numpy()
        plan.device_status()
    for i in range(3):
        assert ph.rel_l2(out[i], _padded_oracle(s[i].astype(np.float32), th, 1.0)) < 1e-3


def test_center_search_finds_axis_and_matches_oracle():
    n, a = 128, 120
    th = ph.angles_deg(a)
    c_true = 62.0  # best shift = n/2 - c_true = 2.0 (plan centre n of the 2n-wide rows)
    s1 = ph.shepp_logan_sinogram(n, a, center=c_true, noise_seed=3).astype(np.float32)
    s2 = ph.shepp_logan_sinogram(n, a, center=c_true, noise_seed=4).astype(np.float32)
    shifts = np.arange(-1.0, 5.01, 0.5).astype(np.float32)
    lo, hi, nb = -0.01, 0.03, 1000
    with G.Plan(2 * n, a, th, filter=G.FILTER_HANN, max_pairs=4) as plan:
        scores, best, imgs = G.center_search(plan, _dev(s1), _dev(s2), shifts, lo, hi, nb,
                                             want_images=True)
        plan.device_status()
    assert abs(shifts[best] - 2.0) <= 0.5
    assert best == int(np.argmin(scores))
    im = imgs.cpu().numpy()
    # the score of the returned images, recomputed on the CPU from the same pixels
    assert abs(scores[best] - O.port_entropy(im, lo, hi, nb)) < 1e-5
    # the images equal the oracle pipeline at that shift
    x = float(shifts[best])
    assert ph.rel_l2(im[0], _padded_oracle(s1, th, x)) < 1e-3
    assert ph.rel_l2(im[1], _padded_oracle(s2, th, x)) < 1e-3
    # scores follow the oracle pipeline's (pixels near bin edges may move one bin)
    ref = np.array([O.port_entropy(np.stack([_padded_oracle(s1, th, float(v)),
                                             _padded_oracle(s2, th, float(v))]).astype(np.float32),
                                   lo, hi, nb) for v in shifts])
    assert np.abs(scores - ref).max() < 2e-2
    assert int(np.argmin(ref)) == best


def test_xcorr_scores_against_reference_and_oracle():
    z = _load("prep_xcorr_*.npz")[0]
    roi = tuple(int(v) for v in z["roi"])
    t = _dev(z["templ"].astype(np.float32))
    m = _dev(z["match"].astype(np.float32))
    for (tx, ty), ref in zip(z["trans"], z["scores"]):
        got = G.xcorr_scores(t, m, roi, tx, ty, 1.0, 1.0, 1, 1)[0, 0]
        # inputs rounded to float32 on the device: compare with the oracle on those
        want = O.port_xcorr_score(z["templ"].astype(np.float32), z["match"].astype(np.float32),
                                  roi, tx, ty)
        assert abs(got - want) < 1e-12, (tx, ty, got, want)
        assert abs(got - ref) < 1e-6
    # a grid of translations in one call equals the per-translation oracle
    got = G.xcorr_scores(t, m, roi, -2.0, -1.5, 0.75, 0.5, 9, 7)
    for k in range(7):
        for i in range(9):
            want = O.port_xcorr_score(z["templ"].astype(np.float32),
                                      z["match"].astype(np.float32), roi, -2.0 + 0.75 * i,
                                      -1.5 + 0.5 * k)
            assert abs(got[k, i] - want) < 1e-12


def test_find_shift_xcorr_recovers_subpixel_translation():
    """A projection pair whose true translation is 6.4 px in x, 0 in y: the coarse
    grid finds 6, the sub-pixel pass 6.4 (step 0.2)."""
    rng = np.random.default_rng(13)
    h, w = 64, 256
    xs = np.arange(w + 16, dtype=np.float64)
    base = np.stack([np.interp(xs, np.sort(rng.uniform(0, w + 16, 40)),
                               rng.uniform(0.2, 2.0, 40)) for _ in range(h)])
    match = base[:, 8:8 + w]
    true_tx = 6.4
    xq = np.arange(w, dtype=np.float64) - true_tx + 8
    shifted = np.stack([np.interp(xq, xs, base[r]) for r in range(h)])
    roi = (40, 200, 8, 55)
    templ = shifted[roi[2]:roi[3] + 1, roi[0]:roi[1] + 1]
    tx, ty, coarse, sub = G.find_shift_xcorr(_dev(templ.astype(np.float32)),
                                             _dev(match.astype(np.float32)), roi,
                                             (-20.0, 20.0, 1.0), (-2.0, 2.0, 1.0), 5)
    assert coarse.shape == (5, 41) and sub.shape == (11,)
    assert ty == 0.0
    assert abs(tx - true_tx) <= 0.1 + 1e-9


def test_fbp_comparator_against_reference_and_oracle():
    z = _load("prep_fbp_*.npz")[0]
    f = G.FBP(64, 45, z["theta"], max_slices=2)
    out = f.reconstruct(_dev(z["sino"][None])).cpu().numpy()[0]
    assert ph.rel_l2(out, z["recon"]) < 1e-5
    assert ph.rel_l2(out, O.port_optimized_fbp(z["sino"], z["theta"])) < 1e-5
    f.close()
    # a batch of three 256 x 180 slices (two launches of max_slices = 2)
    n, a = 256, 180
    th = ph.angles_deg(a)
    sinos = np.stack([ph.shepp_logan_sinogram(n, a, center=n / 2, noise_seed=k) for k in range(3)])
    f = G.FBP(n, a, th, max_slices=2)
    out = f.reconstruct(_dev(sinos)).cpu().numpy()
    for k in range(3):
        assert ph.rel_l2(out[k], O.port_optimized_fbp(sinos[k], th)) < 1e-5
    f.close()


@pytest.mark.parametrize("clamps,radius", [((-1e30, 1e30), 0), ((-0.2, 0.9), 0), ((-0.5, 2.0), 37)])
def test_threshold_u8_bit_exact(clamps, radius):
    """8-bit slices of the reference's BMP/TIFF writer (thresholds from all slices,
    clamped; the cropped copy) against the oracle, byte for byte; NaN included."""
    rng = np.random.default_rng(5)
    imgs = rng.normal(0.3, 0.5, size=(3, 101, 96)).astype(np.float32)
    imgs[1, 5, 7] = np.nan
    imgs[2, 50, 50] = 7.0
    ref, (lo, hi) = O.port_to_u8(imgs, *clamps, radius=radius)
    d = torch.zeros((3, 101, 128), device="cuda")
    d[:, :, :96] = torch.as_tensor(imgs).cuda()
    view = d[:, :, :96]
    lohi = G.threshold_range(view, *clamps)
    got = G.to_u8(view, lohi, radius=radius).cpu().numpy()
    assert tuple(lohi.cpu().numpy().tolist()) == (lo, hi)
    assert np.array_equal(got, ref)


def test_wrappers_on_a_side_stream_match_the_current_stream():
    """Every wrapper that allocates its outputs or workspace, called with a side
    stream, queues that torch work on the same stream as its kernels and gives the
    current stream's results bit for bit."""
    rng = np.random.default_rng(11)
    s = rng.random((4, 60, 128), dtype=np.float32) + 0.5
    offs = [0.5, -1.25, 2.0, 0.0]

    def run(stream):
        x = _dev(s)
        torch.cuda.synchronize()
        r = {"ring": G.ring_removal(x, 1.0, 5, stream=stream)}
        r["shift"] = G.shift_pad(x, offs, stream=stream)
        r["shift1"] = G.shift_pad(x, 1.5, stream=stream)
        r["crop"] = G.crop_center(r["shift"], 50, 5, radius=20, stream=stream)
        r["lohi"] = G.threshold_range(r["crop"], stream=stream)
        r["u8"] = G.to_u8(r["crop"], r["lohi"], stream=stream)
        r["ent"] = G.entropy(r["crop"], 0.0, 2.0, 64, stream=stream)
        torch.cuda.synchronize()
        return {k: v.cpu().numpy() for k, v in r.items()}

    a = run(None)
    b = run(torch.cuda.Stream())
    for k in a:
        assert np.array_equal(a[k], b[k]), k
