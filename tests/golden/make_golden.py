"""Generates the golden fixtures in this directory from the reference itself.

Run from the repository root after ``oracle/build_ref.sh`` (needs the
reference tree, so it runs in the build container, not on the GPU box):

    python tests/golden/make_golden.py

Each case_*.npz holds the inputs (two float32 sinograms, float32 angles,
parameters) and the reference's outputs for them:
  * ``ref32`` -- the reference GridRec class (FP32, NR FFT), gridrec/GPU/gridrec.cu
  * ``ref64`` -- the same sources built with float -> double
  * ``refb``  -- GridrecCPP 5.2 (explicit centre / sampl / C / filter name)
Each prep_*.npz holds inputs and outputs of the reference's slice-pipeline
code (oracle/_ref/libprep_ref.so): ring suppression, shift + half padding,
and find_shift's histogram entropy.
Inputs are seeded synthetic sinograms (analytic ellipses + Poisson noise) or
uniform random rows, so the files are reproducible from this script.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from projects_b200 import phantom as ph  # noqa: E402


def _pair_phantom(n, a, center, seed, theta=None):
    th = ph.angles_deg(a) if theta is None else theta
    p = ph.line_integrals(ph.shepp_logan_ellipses(), n, th, center)
    p *= 2.0 / p.max()
    s1 = ph.poisson_log(p, 1e4, seed)
    q = ph.line_integrals(ph.random_ellipses(seed), n, th, center) / (n / 2.0)
    s2 = ph.poisson_log(q, 1e4, seed + 1)
    return s1, s2, th.astype(np.float32)


def case_gridrec_class(name, n, a, filt, seed, theta=None):
    """Reference GridRec class (centre n/2, sampl 1, C 6)."""
    s1, s2, th = _pair_phantom(n, a, n // 2, seed, theta)
    r1, r2, m0, _ = O.ref_gridrec_pair(s1, s2, th, filter=filt)
    q1, q2, _, _ = O.ref_gridrec_pair(s1, s2, th, filter=filt, fp64=True)
    np.savez_compressed(os.path.join(HERE, f"case_{name}.npz"), kind="gridrec", sino1=s1,
                        sino2=s2, theta=th, n_det=n, n_ang=a, filter=filt, center=n // 2,
                        sampl=1.0, C=6.0, M0=m0, ref32_1=r1[:m0, :m0], ref32_2=r2[:m0, :m0],
                        ref64_1=q1[:m0, :m0], ref64_2=q2[:m0, :m0])


def case_gridrec_cpp(name, n, a, center, fname, C_, sampl, seed, geom=0, roi=(1.0, 1.0, 0.0, 0.0)):
    """GridrecCPP 5.2 with explicit centre, oversampling, PSWF C and filter name; geom 1
    generates its angles (uniform on [0, pi)) by its FP32 recurrence; roi = (R, MaxPixSiz,
    X0, Y0) of its grid_struct."""
    s1, s2, th = _pair_phantom(n, a, center, seed)
    b1, b2, m0 = O.refb_gridrec_pair(s1, s2, th, center=center, filter_name=fname, C_=C_,
                                     sampl=sampl, geom=geom, roi_size=roi[0], pixel_size=roi[1],
                                     x0=roi[2], y0=roi[3])
    np.savez_compressed(os.path.join(HERE, f"case_{name}.npz"), kind="gridrec_cpp", sino1=s1,
                        sino2=s2, theta=th, n_det=n, n_ang=a, filter_name=fname, center=center,
                        sampl=sampl, C=C_, M0=m0, refb_1=b1[:m0, :m0], refb_2=b2[:m0, :m0],
                        geom=geom, roi=np.array(roi))


def prep_cases(rng):
    """Reference ring suppression, shift/half-padding and entropy."""
    # shift + half padding: odd and even widths, shifts of both signs and beyond the row
    for n, a in ((63, 20), (64, 24)):
        s1 = rng.standard_normal((a, n)).astype(np.float32)
        s2 = (rng.random((a, n)) * 3).astype(np.float32)
        shifts = np.array([-3.7, 0.0, 0.25, 12.5, -70.2], np.float32)
        outs = np.stack([O.ref_shift_pad(s1, s2, x) for x in shifts])
        np.savez_compressed(os.path.join(HERE, f"prep_shift_pad_{n}x{a}.npz"), sino1=s1,
                            sino2=s2, shifts=shifts, outs=outs)
    # ring suppression: positive sinogram with detector stripes and a zero-mean row
    n, a = 96, 40
    th = ph.angles_deg(a)
    p = ph.line_integrals(ph.shepp_logan_ellipses(), n, th, n // 2).astype(np.float32)
    p = p / p.max() + 0.05
    p[:, 17] *= 1.2
    p[:, 60] += 0.1
    p[:, 61] -= 0.05
    p[5, :] = 0.0
    ring = O.ref_ring_removal(p, 1.0)
    np.savez_compressed(os.path.join(HERE, "prep_ring_96x40.npz"), sino=p, ring_coeff=1.0,
                        out=ring)
    # entropy: two images side by side as find_shift scores them (xm = 2 um, ym = um)
    img = (rng.standard_normal((48, 96)) * 0.01).astype(np.float32)
    img[10:20, 30:50] += 0.02
    cfg = np.array([[-0.05, 0.05, 100], [-0.02, 0.03, 1000], [-0.1, 0.1, 10000]], np.float64)
    ent = np.array([O.ref_entropy(img, lo, hi, int(nb)) for lo, hi, nb in cfg], np.float64)
    np.savez_compressed(os.path.join(HERE, "prep_entropy_48x96.npz"), image=img, cfg=cfg,
                        entropy=ent)
    # brute-force cross-correlation scores: a match image and the template cut from a
    # shifted copy of it, several translations (integer, fractional, out of the image)
    h, w = 40, 72
    match = (rng.standard_normal((h, w)) * 0.3 + 1.0)
    roi = (12, 55, 6, 31)
    shifted = np.roll(match, (1, 3), axis=(0, 1))
    templ = shifted[roi[2]:roi[3] + 1, roi[0]:roi[1] + 1].copy()
    trans = np.array([[3.0, 1.0], [0.0, 0.0], [2.5, 1.0], [3.25, 0.75], [-4.5, 2.0],
                      [30.0, -10.0], [70.0, 0.0]])
    scores = np.array([O.ref_xcorr_score(templ, match, roi, tx, ty) for tx, ty in trans])
    np.savez_compressed(os.path.join(HERE, "prep_xcorr_40x72.npz"), match=match, templ=templ,
                        roi=np.array(roi), trans=trans, scores=scores)
    # the reference's CPU OptimizedFBP (FBP comparator) on a Shepp-Logan sinogram
    if O.fbp_ref_available():
        n, a = 64, 45
        th = ph.angles_deg(a)
        sino = ph.shepp_logan_sinogram(n, a, center=n / 2, noise_seed=5)
        np.savez_compressed(os.path.join(HERE, "prep_fbp_64x45.npz"), sino=sino, theta=th,
                            recon=O.ref_optimized_fbp(sino, th))


def main():
    if not O.ref_available():
        raise SystemExit("build the reference first: oracle/build_ref.sh")
    rng = np.random.default_rng(7)
    case_gridrec_class("a64x48_shlo", 64, 48, 1, 11)
    case_gridrec_cpp("b100x37_c50_hann", 100, 37, 50.0, "hann", 6.0, 1.0, 12)
    uneven = np.sort(rng.uniform(0.0, 180.0, 90)).astype(np.float32)
    case_gridrec_class("a128x90_hamm_uneven", 128, 90, 3, 13, theta=uneven)
    case_gridrec_class("a128x64_ramp", 128, 64, 4, 14)
    case_gridrec_class("a32x50_none", 32, 50, 0, 15)
    case_gridrec_cpp("b96x60_c47.3_s1.2_ramlak", 96, 60, 47.3, "ramlak", 6.0, 1.2, 21)
    case_gridrec_cpp("b64x40_c31.7_C4_hann", 64, 40, 31.7, "hann", 4.0, 1.0, 22)
    case_gridrec_cpp("b120x72_c61.2_C7_s1.2_shepp", 120, 72, 61.2, "shepp", 7.0, 1.2, 23)
    case_gridrec_cpp("b72x45_c36.5_C5_hamming", 72, 45, 36.5, "hamming", 5.0, 1.0, 24)
    case_gridrec_cpp("b96x90_c47.5_geom1_hann", 96, 90, 47.5, "hann", 6.0, 1.0, 25, geom=1)
    case_gridrec_cpp("b96x80_c48_R0.75_X0.04_Y-0.03_hann", 96, 80, 48.0, "hann", 6.0, 1.0, 26,
                     roi=(0.75, 1.0, 0.04, -0.03))
    case_gridrec_cpp("b96x80_c48_R0.8_pix1.5_X0.05_Y0.02_shlo", 96, 80, 48.0, "shlo", 6.0, 1.0,
                     27, roi=(0.8, 1.5, 0.05, 0.02))
    if O.prep_ref_available():
        prep_cases(np.random.default_rng(8))
    print("\n".join(sorted(f for f in os.listdir(HERE) if f.endswith(".npz"))))


if __name__ == "__main__":
    main()
