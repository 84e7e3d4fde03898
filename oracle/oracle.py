"""ctypes access to the gridrec oracles -- TEST INFRASTRUCTURE ONLY.

* ``port_*``  -- the float64 C restatement in gridrec_oracle.c (always built).
* ``ref_*``   -- the reference's own CPU GridRec compiled from its sources into
  ``_ref/`` by build_ref.sh: FP32 (``libgridrec_ref.so``), the FP64 sed build
  (``libgridrec_ref64.so``) and GridrecCPP 5.2 (``libgridrec_refb.so``).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_REF = os.path.join(_HERE, "_ref")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


class OrcParams(C.Structure):
    _fields_ = [("n_det", C.c_int), ("n_ang", C.c_int), ("center1", C.c_double),
                ("center2", C.c_double), ("filter", C.c_int), ("C", C.c_double),
                ("sampl", C.c_double), ("ltbl", C.c_int), ("roi_size", C.c_double),
                ("pixel_size", C.c_double), ("x0", C.c_double), ("y0", C.c_double)]


class OrcSizes(C.Structure):
    _fields_ = [("pdim", C.c_long), ("M", C.c_long), ("M02", C.c_long), ("M0", C.c_long),
                ("sampl", C.c_double), ("L", C.c_double), ("scale", C.c_double),
                ("C", C.c_double), ("lmbda", C.c_double)]


_port = None


def port_lib():
    global _port
    if _port is None:
        path = os.path.join(_HERE, "libgridrec_oracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle not built: {path} (run make -C oracle)")
        lib = C.CDLL(path)
        P = C.POINTER(OrcParams)
        lib.orc_sizes.argtypes = [P, C.POINTER(OrcSizes)]
        lib.orc_tables.argtypes = [P, _dp, C.c_void_p]
        lib.orc_spectra.argtypes = [P, _dp, _dp, _dp]
        lib.orc_grid.argtypes = [P, _dp, _dp, _dp]
        lib.orc_fft1d.argtypes = [_dp, C.c_long, C.c_int]
        lib.orc_fft2d.argtypes = [_dp, C.c_long]
        lib.orc_fft2d.restype = None
        lib.orc_fft1d.restype = None
        lib.orc_deapod.argtypes = [P, _dp, _dp, _dp, C.c_long]
        lib.orc_gridrec_pair.argtypes = [P, _dp, _dp, _dp, _dp, _dp, C.c_long]
        lib.orc_ring_removal.argtypes = [_dp, C.c_int, C.c_int, C.c_double, C.c_int]
        lib.orc_ring_removal.restype = None
        lib.orc_shift_pad.argtypes = [_fp, _fp, C.c_int, C.c_int, C.c_float, C.c_int]
        lib.orc_shift_pad.restype = None
        lib.orc_crop.argtypes = [_fp, C.c_long, _fp, C.c_int, C.c_int, C.c_int]
        lib.orc_crop.restype = None
        lib.orc_minmax.argtypes = [_fp, C.c_long, C.c_float, C.c_float, C.POINTER(C.c_float),
                                   C.POINTER(C.c_float)]
        lib.orc_minmax.restype = None
        lib.orc_to_u8.argtypes = [_fp, C.c_int, C.c_int, C.c_long, C.c_float, C.c_float, C.c_int,
                                  C.c_void_p]
        lib.orc_to_u8.restype = None
        lib.orc_entropy.argtypes = [_fp, C.c_long, C.c_float, C.c_float, C.c_int]
        lib.orc_xcorr_score.argtypes = [_dp, _dp] + [C.c_int] * 6 + [C.c_double, C.c_double]
        lib.orc_xcorr_score.restype = C.c_double
        lib.orc_optimized_fbp.argtypes = [C.c_int, C.c_int, _fp, _fp, _dp]
        lib.orc_optimized_fbp.restype = C.c_int
        lib.orc_entropy.restype = C.c_double
        _port = lib
    return _port


def params(n_det, n_ang, center1=None, center2=None, filter=1, C_=6.0, sampl=1.0, ltbl=512,
           roi_size=1.0, pixel_size=1.0, x0=0.0, y0=0.0):
    # GridRec::init: center = sinogram_x_dim / 2 in integer arithmetic (gridrec.cu:227)
    c1 = float(n_det // 2) if center1 is None else float(center1)
    c2 = c1 if center2 is None else float(center2)
    return OrcParams(int(n_det), int(n_ang), c1, c2, int(filter), float(C_), float(sampl),
                     int(ltbl), float(roi_size), float(pixel_size), float(x0), float(y0))


def port_sizes(p: OrcParams) -> OrcSizes:
    s = OrcSizes()
    rc = port_lib().orc_sizes(C.byref(p), C.byref(s))
    if rc:
        raise ValueError(f"orc_sizes failed ({rc})")
    return s


def port_tables(p: OrcParams):
    s = port_sizes(p)
    wtbl = np.zeros(p.ltbl + 1)
    winv = np.zeros(s.M0)
    port_lib().orc_tables(C.byref(p), wtbl, winv.ctypes.data)
    return wtbl, winv


def port_spectra(p, sino1, sino2):
    s = port_sizes(p)
    J = s.pdim // 2
    spec = np.zeros((p.n_ang, 2, J, 2))
    rc = port_lib().orc_spectra(C.byref(p), np.ascontiguousarray(sino1, np.float64),
                                np.ascontiguousarray(sino2, np.float64), spec)
    if rc:
        raise ValueError(rc)
    return spec[..., 0] + 1j * spec[..., 1]


def port_grid(p, theta_deg, spec):
    s = port_sizes(p)
    sp = np.ascontiguousarray(np.stack([spec.real, spec.imag], -1), np.float64)
    H = np.zeros((s.M, s.M, 2))
    rc = port_lib().orc_grid(C.byref(p), np.ascontiguousarray(theta_deg, np.float64), sp, H)
    if rc:
        raise ValueError(rc)
    return H[..., 0] + 1j * H[..., 1]


def port_fft2d(H):
    M = H.shape[0]
    h = np.ascontiguousarray(np.stack([H.real, H.imag], -1), np.float64)
    port_lib().orc_fft2d(h, M)
    return h[..., 0] + 1j * h[..., 1]


def port_gridrec_pair(sino1, sino2, theta_deg, center1=None, center2=None, filter=1,
                      C_=6.0, sampl=1.0, ltbl=512, out_stride=None, roi_size=1.0,
                      pixel_size=1.0, x0=0.0, y0=0.0):
    """float64 gridrec of one pair; returns (out1, out2) of shape (M0, stride)."""
    n_ang, n_det = sino1.shape
    p = params(n_det, n_ang, center1, center2, filter, C_, sampl, ltbl, roi_size, pixel_size,
               x0, y0)
    s = port_sizes(p)
    stride = max(n_det, s.M0) if out_stride is None else out_stride
    o1 = np.zeros((s.M0, stride))
    o2 = np.zeros((s.M0, stride))
    rc = port_lib().orc_gridrec_pair(C.byref(p), np.ascontiguousarray(theta_deg, np.float64),
                                     np.ascontiguousarray(sino1, np.float64),
                                     np.ascontiguousarray(sino2, np.float64), o1, o2, stride)
    if rc:
        raise ValueError(f"orc_gridrec_pair failed ({rc})")
    return o1, o2


def port_ring_removal(sino, ring_coeff=1.0, iterations=20):
    x = np.ascontiguousarray(sino, np.float64).copy()
    port_lib().orc_ring_removal(x, x.shape[1], x.shape[0], float(ring_coeff), int(iterations))
    return x


def port_shift_pad(sino, xoffset, out_width=None):
    """float32 sinogram (n_ang, n_det) -> (n_ang, out_width) shifted, half-padded rows."""
    n_ang, n_det = sino.shape
    w = 2 * n_det if out_width is None else int(out_width)
    out = np.zeros((n_ang, w), np.float32)
    port_lib().orc_shift_pad(np.ascontiguousarray(sino, np.float32), out, n_det, n_ang,
                             float(xoffset), w)
    return out


def port_to_u8(images, lower_clamp=-1e30, upper_clamp=1e30, radius=0):
    """8-bit slices of the reference's BMP/TIFF writer: thresholds from all the
    given slices (S, rows, cols), then the conversion (and crop) per slice."""
    imgs = np.ascontiguousarray(images, np.float32)
    lo, hi = C.c_float(), C.c_float()
    port_lib().orc_minmax(imgs, imgs.size, float(lower_clamp), float(upper_clamp), C.byref(lo),
                          C.byref(hi))
    S, rows, cols = imgs.shape
    out = np.zeros((S, rows, cols), np.uint8)
    for s in range(S):
        port_lib().orc_to_u8(imgs[s], rows, cols, cols, lo.value, hi.value, int(radius),
                             out[s].ctypes.data)
    return out, (lo.value, hi.value)


def port_crop(rec, n, offset, radius=0):
    """Centre crop rec[offset:offset+n, offset:offset+n] with optional circular mask."""
    r = np.ascontiguousarray(rec, np.float32)
    out = np.zeros((n, n), np.float32)
    port_lib().orc_crop(r, r.shape[1], out, int(n), int(offset), int(radius))
    return out


def port_entropy(img, vmin, vmax, nbins):
    x = np.ascontiguousarray(img, np.float32).ravel()
    return port_lib().orc_entropy(x, x.size, float(vmin), float(vmax), int(nbins))


def port_optimized_fbp(sino, theta_deg):
    """OptimizedFBP of one (n_ang, n_det) sinogram -> (n_det, n_det) float64 image."""
    n_ang, n = sino.shape
    out = np.zeros((n, n))
    rc = port_lib().orc_optimized_fbp(n, n_ang, np.ascontiguousarray(theta_deg, np.float32),
                                      np.ascontiguousarray(sino, np.float32), out)
    if rc:
        raise ValueError("orc_optimized_fbp: n_det must be a power of two")
    return out


def port_xcorr_score(templ_roi, match, roi, tx, ty):
    """find_shift's brute-force score for one translation; roi = (x0, x1, y0, y1)."""
    h, w = match.shape
    return port_lib().orc_xcorr_score(np.ascontiguousarray(templ_roi, np.float64),
                                      np.ascontiguousarray(match, np.float64), w, h, *roi,
                                      float(tx), float(ty))


# ---------------------------------------------------------------- reference builds

def ref_available() -> bool:
    return os.path.exists(os.path.join(_REF, "libgridrec_ref.so"))


_refs: dict = {}


def _ref_lib(name, real):
    if name not in _refs:
        path = os.path.join(_REF, name)
        if not os.path.exists(path):
            raise RuntimeError(f"reference oracle not built: {path}")
        lib = C.CDLL(path)
        rp = np.ctypeslib.ndpointer(dtype=real, flags="C_CONTIGUOUS")
        if name == "libprep_ref.so":
            lib.ref_ring_removal.argtypes = [rp, C.c_int, C.c_int, C.c_float]
            lib.ref_ring_removal.restype = None
            lib.ref_entropy.argtypes = [rp, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int]
            lib.ref_entropy.restype = C.c_float
            lib.ref_shift_pad.argtypes = [rp, rp, C.c_int, C.c_int, C.c_float, rp]
            lib.ref_shift_pad.restype = None
            dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
            lib.ref_xcorr_score.argtypes = [dp, dp] + [C.c_int] * 6 + [C.c_double, C.c_double]
            lib.ref_xcorr_score.restype = C.c_double
        elif name == "libgridrec_refb.so":
            lib.refb_gridrec_pair.argtypes = [C.c_int, C.c_int, rp, C.c_float, C.c_char_p,
                                              C.c_float, C.c_float, C.c_int, rp, rp, rp, rp,
                                              C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                              C.c_float]
            lib.refb_gridrec_pair.restype = C.c_int
        else:
            lib.ref_gridrec_pair.argtypes = [C.c_int, C.c_int, rp, C.c_int, rp, rp, rp, rp,
                                             C.POINTER(C.c_double), C.POINTER(C.c_double)]
            lib.ref_gridrec_pair.restype = C.c_int
            lib.ref_gridrec_pairs.argtypes = [C.c_int, C.c_int, rp, C.c_int, C.c_int, rp, rp]
            lib.ref_gridrec_pairs.restype = C.c_double
        _refs[name] = lib
    return _refs[name]


def ref_gridrec_pair(sino1, sino2, theta_deg, filter=1, fp64=False):
    """The reference GridRec class (centre n_det/2).  Returns (out1, out2, M0, t_recon)."""
    real = np.float64 if fp64 else np.float32
    lib = _ref_lib("libgridrec_ref64.so" if fp64 else "libgridrec_ref.so", real)
    n_ang, n_det = sino1.shape
    m0 = port_sizes(params(n_det, n_ang)).M0
    if m0 > n_det:
        # GridRec writes M0 columns with row stride n_det (gridrec.cu:196-197,
        # 691-719): rows overlap and the caller's n_det x n_det buffer overflows.
        raise ValueError(f"reference GridRec needs M0 <= n_det (M0={m0}, n_det={n_det})")
    o1 = np.zeros((n_det, n_det), real)
    o2 = np.zeros((n_det, n_det), real)
    tr, tt = C.c_double(), C.c_double()
    m0 = lib.ref_gridrec_pair(n_det, n_ang, np.ascontiguousarray(theta_deg, real), int(filter),
                              np.ascontiguousarray(sino1, real),
                              np.ascontiguousarray(sino2, real), o1, o2, C.byref(tr),
                              C.byref(tt))
    return o1, o2, m0, tr.value


def ref_gridrec_pairs(sinos, theta_deg, filter=1):
    """Reference GridRec over consecutive pairs of an (2P, n_ang, n_det) float32 stack.

    Returns (outs[2P, n_det, n_det], seconds spent in reconstruct())."""
    lib = _ref_lib("libgridrec_ref.so", np.float32)
    n2, n_ang, n_det = sinos.shape
    if port_sizes(params(n_det, n_ang)).M0 > n_det:
        raise ValueError("reference GridRec needs M0 <= n_det")
    outs = np.zeros((n2, n_det, n_det), np.float32)
    t = lib.ref_gridrec_pairs(n_det, n_ang, np.ascontiguousarray(theta_deg, np.float32),
                              int(filter), n2 // 2, np.ascontiguousarray(sinos, np.float32),
                              outs)
    return outs, t


def refb_gridrec_pair(sino1, sino2, theta_deg, center, filter_name="shlo", C_=6.0, sampl=1.2,
                      ltbl=512, geom=0, roi_size=1.0, pixel_size=1.0, x0=0.0, y0=0.0):
    """GridrecCPP 5.2 (explicit centre/sampl/filter name).  Returns (out1, out2, M0)."""
    lib = _ref_lib("libgridrec_refb.so", np.float32)
    n_ang, n_det = sino1.shape
    th = np.ascontiguousarray(theta_deg, np.float32)
    s1 = np.ascontiguousarray(sino1, np.float32)
    s2 = np.ascontiguousarray(sino2, np.float32)
    dummy = np.zeros(1, np.float32)
    m0 = lib.refb_gridrec_pair(n_det, n_ang, th, center, filter_name.encode(), C_, sampl, ltbl,
                               s1, s2, dummy, dummy, 0, int(geom), roi_size, pixel_size, x0, y0)
    stride = max(m0, n_det)
    o1 = np.zeros((m0, stride), np.float32)
    o2 = np.zeros((m0, stride), np.float32)
    lib.refb_gridrec_pair(n_det, n_ang, th, center, filter_name.encode(), C_, sampl, ltbl,
                          s1, s2, o1, o2, stride, int(geom), roi_size, pixel_size, x0, y0)
    return o1, o2, m0


def prep_ref_available() -> bool:
    return os.path.exists(os.path.join(_REF, "libprep_ref.so"))


def ref_ring_removal(sino, ring_coeff=1.0):
    """RingCorrectionSinogram of the reference (20 rounds, float32, in place on a copy)."""
    lib = _ref_lib("libprep_ref.so", np.float32)
    x = np.ascontiguousarray(sino, np.float32).copy()
    lib.ref_ring_removal(x, x.shape[1], x.shape[0], float(ring_coeff))
    return x


def ref_entropy(img, vmin, vmax, nbins):
    """find_shift's entropy() over a (ym, xm) float32 image."""
    lib = _ref_lib("libprep_ref.so", np.float32)
    x = np.ascontiguousarray(img, np.float32)
    ym, xm = x.shape
    return float(lib.ref_entropy(x, float(vmin), float(vmax), int(nbins), xm, ym))


def ref_shift_pad(sino1, sino2, xoffset):
    """GridRecSlices' shift and half padding of a slice pair -> (2, n_ang, 2 n_det)."""
    lib = _ref_lib("libprep_ref.so", np.float32)
    n_ang, n_det = sino1.shape
    out = np.zeros((2, n_ang, 2 * n_det), np.float32)
    lib.ref_shift_pad(np.ascontiguousarray(sino1, np.float32),
                      np.ascontiguousarray(sino2, np.float32), n_det, n_ang, float(xoffset), out)
    return out


def ref_xcorr_score(templ_roi, match, roi, tx, ty):
    """The reference's own data_interp + cross_correlation for one translation."""
    lib = _ref_lib("libprep_ref.so", np.float32)
    h, w = match.shape
    return float(lib.ref_xcorr_score(np.ascontiguousarray(templ_roi, np.float64),
                                     np.ascontiguousarray(match, np.float64), w, h, *roi,
                                     float(tx), float(ty)))


def ref_optimized_fbp(sino, theta_deg):
    """The reference's own CPU OptimizedFBP -> (n_det, n_det) float32 image."""
    path = os.path.join(_REF, "libfbp_ref.so")
    if "fbp" not in _refs:
        if not os.path.exists(path):
            raise RuntimeError(f"reference oracle not built: {path}")
        lib = C.CDLL(path)
        fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
        lib.ref_optimized_fbp.argtypes = [C.c_int, C.c_int, fp, fp, fp]
        lib.ref_optimized_fbp.restype = None
        _refs["fbp"] = lib
    n_ang, n = sino.shape
    out = np.zeros((n, n), np.float32)
    _refs["fbp"].ref_optimized_fbp(n, n_ang, np.ascontiguousarray(theta_deg, np.float32),
                                   np.ascontiguousarray(sino, np.float32).copy(), out)
    return out


def fbp_ref_available() -> bool:
    return os.path.exists(os.path.join(_REF, "libfbp_ref.so"))
