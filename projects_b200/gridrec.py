"""Python host side of the B200 gridrec: ctypes bindings of the C ABI
(include/gridrec_b200.h) plus a ``GridRec`` class with the reference's
setter API (gridrec/GPU/gridrec.h:72-143, recon_algorithm.h:56-95).

The library ``libgridrec_b200.so`` is built in-tree (projects_b200/build.py).
There is no CPU fallback: every compute call goes to the sm_100a kernels and
raises if the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgridrec_b200.so")

GR_OK = 0
STATUS = {0: "GR_OK", -1: "GR_ERR_ARG", -2: "GR_ERR_PSWF", -3: "GR_ERR_CUDA",
          -4: "GR_ERR_NOMEM", -5: "GR_ERR_UNSUPPORTED", -6: "GR_ERR_TIMEOUT"}

FILTER_NONE, FILTER_SHEPP_LOGAN, FILTER_HANN, FILTER_HAMMING, FILTER_RAMP, FILTER_FBP = range(6)
DTYPE_F32, DTYPE_F16, DTYPE_BF16, DTYPE_U16_RAW, DTYPE_U16_LINEAR = range(5)

# Functions declared in include/gridrec_b200.h (checked by the CPU tests).
EXPORTS = ("gr_params_default", "gr_filter_code", "gr_plan_create", "gr_plan_destroy",
           "gr_plan_sizes", "gr_plan_device_bytes", "gr_reconstruct_pair",
           "gr_reconstruct_batch", "gr_reconstruct_host", "gr_last_error",
           "gr_plan_launch_count", "gr_plan_work_stats", "gr_worklist_export",
           "gr_worklist_export_wide", "gr_plan_grid_kernel",
           "gr_plan_set_timing", "gr_plan_stage_times", "gr_reconstruct_pair_noalloc",
           "gr_reconstruct_pair_host",
           "gr_plan_device_status", "gr_selftest_wait_timeout", "gr_ring_workspace_bytes",
           "gr_ring_removal", "gr_shift_pad", "gr_crop_center", "gr_entropy_workspace_bytes",
           "gr_entropy", "gr_reconstruct_padded", "gr_center_search", "gr_graph_create",
           "gr_graph_launch", "gr_graph_launch_count", "gr_graph_destroy", "gr_plan_autotune",
           "gr_plan_tuning", "gr_plan_set_tuning", "gr_plan_tuning_ex", "gr_xcorr_scores", "gr_fbp_create", "gr_fbp_reconstruct",
           "gr_threshold_workspace_bytes", "gr_threshold_range", "gr_to_u8",
           "gr_fbp_destroy", "gr_cnn_param_count", "gr_cnn_workspace_bytes",
           "gr_cnn_forward_workspace_bytes", "gr_cnn_forward",
           "gr_cnn_backward", "gr_cnn_adam", "gr_cnn_infer_workspace_bytes", "gr_cnn_infer",
           "gr_cnn_infer_status")
STAGES = ("phase", "spectra", "grid", "cols", "rows_deapod")


class GrError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__(f"{where}: {STATUS.get(code, code)}: {last_error()}")


class GrParams(C.Structure):
    _fields_ = [("n_det", C.c_int), ("n_ang", C.c_int), ("theta_deg", C.POINTER(C.c_float)),
                ("center", C.c_float), ("filter", C.c_int), ("pswf_c", C.c_float),
                ("sampl", C.c_float), ("ltbl", C.c_int), ("max_pairs", C.c_int),
                ("device", C.c_int), ("geom", C.c_int), ("roi_size", C.c_float),
                ("pixel_size", C.c_float), ("roi_x0", C.c_float), ("roi_y0", C.c_float),
                ("wide_grid", C.c_int)]


class GrBatch(C.Structure):
    _fields_ = [("n_slices", C.c_int), ("dtype", C.c_int), ("sinos", C.c_void_p),
                ("centers", C.c_void_p), ("flat", C.c_void_p), ("dark", C.c_void_p),
                ("outs", C.c_void_p), ("out_stride", C.c_long), ("flat_stride", C.c_long)]


class GrGraphItem(C.Structure):
    _fields_ = [("plan", C.c_void_p), ("batch", GrBatch)]


_lib = None


def lib():
    """Loads libgridrec_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run projects_b200/build.py (needs nvcc)")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER(GrParams)
        L.gr_params_default.argtypes = [P, C.c_int, C.c_int, C.POINTER(C.c_float)]
        L.gr_filter_code.argtypes = [C.c_char_p]
        L.gr_plan_create.argtypes = [P, C.POINTER(C.c_void_p)]
        L.gr_plan_destroy.argtypes = [C.c_void_p]
        L.gr_plan_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    C.POINTER(C.c_int), C.POINTER(C.c_float),
                                    C.POINTER(C.c_float)]
        L.gr_plan_device_bytes.argtypes = [C.c_void_p, C.POINTER(C.c_size_t)]
        L.gr_reconstruct_pair.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_long, C.c_void_p]
        L.gr_reconstruct_pair_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p,
                                                  C.c_void_p, C.c_void_p, C.c_long, C.c_void_p]
        L.gr_reconstruct_pair_host.argtypes = L.gr_reconstruct_pair.argtypes
        L.gr_reconstruct_batch.argtypes = [C.c_void_p, C.POINTER(GrBatch), C.c_void_p]
        L.gr_reconstruct_host.argtypes = [C.c_void_p, C.POINTER(GrBatch), C.c_void_p]
        L.gr_last_error.restype = C.c_char_p
        L.gr_plan_launch_count.argtypes = [C.c_void_p, C.POINTER(C.c_long)]
        L.gr_plan_work_stats.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int), C.POINTER(C.c_long)]
        L.gr_plan_set_timing.argtypes = [C.c_void_p, C.c_int]
        L.gr_plan_device_status.argtypes = [C.c_void_p, C.c_void_p]
        L.gr_selftest_wait_timeout.argtypes = [C.c_int]
        L.gr_plan_stage_times.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_long)]
        ip = C.POINTER(C.c_int)
        L.gr_worklist_export.argtypes = [P, ip, ip, ip, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_int, C.c_int]
        L.gr_worklist_export_wide.argtypes = L.gr_worklist_export.argtypes
        L.gr_plan_grid_kernel.argtypes = [C.c_void_p, C.c_int, ip]
        vp, i_, l_, f_ = C.c_void_p, C.c_int, C.c_long, C.c_float
        L.gr_ring_workspace_bytes.argtypes = [i_, i_, i_]
        L.gr_ring_workspace_bytes.restype = C.c_size_t
        L.gr_ring_removal.argtypes = [vp, i_, i_, i_, f_, i_, vp, vp]
        L.gr_shift_pad.argtypes = [vp, vp, i_, i_, i_, vp, i_, vp]
        L.gr_crop_center.argtypes = [vp, l_, l_, vp, l_, l_, i_, i_, i_, i_, vp]
        L.gr_threshold_workspace_bytes.restype = C.c_size_t
        L.gr_threshold_range.argtypes = [vp, i_, i_, i_, l_, l_, f_, f_, vp, vp, vp]
        L.gr_to_u8.argtypes = [vp, i_, i_, i_, l_, l_, vp, i_, vp, l_, l_, vp]
        L.gr_entropy_workspace_bytes.argtypes = [i_, i_]
        L.gr_entropy_workspace_bytes.restype = C.c_size_t
        L.gr_entropy.argtypes = [vp, i_, i_, i_, i_, l_, l_, l_, f_, f_, i_, vp, vp, vp]
        L.gr_reconstruct_padded.argtypes = [vp, vp, i_, i_, i_, f_, vp, l_, vp]
        L.gr_center_search.argtypes = [vp, vp, vp, i_, i_, C.POINTER(f_), i_, f_, f_, i_,
                                       C.POINTER(f_), C.POINTER(i_), vp, vp]
        L.gr_graph_create.argtypes = [C.c_void_p, i_, C.POINTER(C.c_void_p)]
        L.gr_graph_launch.argtypes = [vp, vp]
        L.gr_graph_launch_count.argtypes = [vp, C.POINTER(C.c_long)]
        L.gr_graph_destroy.argtypes = [vp]
        L.gr_plan_autotune.argtypes = [vp, vp]
        L.gr_fbp_create.argtypes = [i_, i_, C.POINTER(f_), i_, i_, C.POINTER(vp)]
        L.gr_fbp_reconstruct.argtypes = [vp, vp, i_, vp, vp]
        L.gr_fbp_destroy.argtypes = [vp]
        d_ = C.c_double
        L.gr_xcorr_scores.argtypes = [vp, vp] + [i_] * 6 + [d_] * 4 + [i_, i_,
                                                                         C.POINTER(d_), vp]
        L.gr_plan_tuning.argtypes = [vp, C.POINTER(i_), C.POINTER(i_)]
        L.gr_plan_set_tuning.argtypes = [vp, i_, i_, i_, i_]
        L.gr_plan_tuning_ex.argtypes = [vp] + [C.POINTER(i_)] * 4
        _lib = L
    return _lib


def last_error() -> str:
    return lib().gr_last_error().decode()


def _check(rc: int, where: str):
    if rc != GR_OK:
        raise GrError(rc, where)


def filter_code(name: str) -> int:
    """GridrecCPP filter name -> ReconAlgorithm code (filters.cpp:26-48)."""
    return int(lib().gr_filter_code(name.encode()))


def make_params(n_det: int, n_ang: int, theta_deg, center=None, filter=FILTER_SHEPP_LOGAN,
                pswf_c=6.0, sampl=1.0, ltbl=512, max_pairs=1, device=0, geom=0, roi_size=1.0,
                pixel_size=1.0, roi_x0=0.0, roi_y0=0.0, wide_grid=0):
    """GrParams plus the float32 theta array that must outlive plan creation."""
    th = np.ascontiguousarray(theta_deg, dtype=np.float32)
    if th.shape != (n_ang,):
        raise ValueError(f"theta_deg must have {n_ang} entries")
    if isinstance(filter, str):
        filter = filter_code(filter)
    p = GrParams()
    lib().gr_params_default(C.byref(p), n_det, n_ang, th.ctypes.data_as(C.POINTER(C.c_float)))
    p.center = -1.0 if center is None else float(center)
    p.filter = int(filter)
    p.pswf_c = float(pswf_c)
    p.sampl = float(sampl)
    p.ltbl = int(ltbl)
    p.max_pairs = int(max_pairs)
    p.device = int(device)
    p.geom = int(geom)
    p.roi_size, p.pixel_size = float(roi_size), float(pixel_size)
    p.roi_x0, p.roi_y0 = float(roi_x0), float(roi_y0)
    p.wide_grid = int(wide_grid)
    return p, th


def worklist(n_det, n_ang, theta_deg, sampl=1.0, pswf_c=6.0, wide=False):
    """Host-only gridding work list: (items[n,4], runs[n,4], splits[tiles,4], tiles_v).

    runs rows are (direction, jlo, jhi, P): direction = 2*angle + half, samples
    jlo..jhi, processed in steps of samples P apart.  wide=True: the 16-pair
    kernel's list (4 x 8 tiles, P = 1)."""
    p, th = make_params(n_det, n_ang, theta_deg, sampl=sampl, pswf_c=pswf_c)
    ni, nr, tv = C.c_int(), C.c_int(), C.c_int()
    fn = lib().gr_worklist_export_wide if wide else lib().gr_worklist_export
    _check(fn(C.byref(p), C.byref(ni), C.byref(nr), C.byref(tv), None,
              None, None, 0, 0), "gr_worklist_export")
    items = np.zeros((ni.value, 4), np.int32)
    runs = np.zeros((nr.value, 4), np.int32)
    # one split record per tile: tiles_v x tiles_v square tiles, or 2 tiles_v rows of
    # 4 x 8 tiles for the 16-pair list
    splits = np.zeros(((2 if wide else 1) * tv.value * tv.value, 4), np.int32)
    _check(fn(C.byref(p), C.byref(ni), C.byref(nr), C.byref(tv),
              items.ctypes.data, runs.ctypes.data, splits.ctypes.data,
              ni.value, nr.value), "gr_worklist_export")
    return items, runs, splits, tv.value


def _ptr(t) -> int:
    """Device address of a torch tensor (or an int address)."""
    if t is None:
        return 0
    if isinstance(t, int):
        return t
    return int(t.data_ptr())


def _stream_ptr(stream) -> int:
    if stream is None:
        import torch
        return int(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)


def _on_stream(stream):
    """Context in which a wrapper's own torch work (its outputs, workspaces and
    small uploads) is queued on the stream its kernels run on, so that the caching
    allocator hands that memory to later work only in stream order after the
    kernels.  A raw int handle or None leaves the current stream as it is (the
    caller then orders its streams itself)."""
    import contextlib
    import torch
    if stream is None or isinstance(stream, int):
        return contextlib.nullcontext()
    return torch.cuda.stream(stream)


class Plan:
    """A gridrec plan: sizes, tables, work list and workspaces on one GPU."""

    def __init__(self, n_det: int, n_ang: int, theta_deg, center=None,
                 filter=FILTER_SHEPP_LOGAN, pswf_c=6.0, sampl=1.0, ltbl=512, max_pairs=1,
                 device=0, geom=0, roi_size=1.0, pixel_size=1.0, roi_x0=0.0, roi_y0=0.0,
                 wide_grid=0):
        self._params, self._theta = make_params(n_det, n_ang, theta_deg, center, filter,
                                                pswf_c, sampl, ltbl, max_pairs, device, geom,
                                                roi_size, pixel_size, roi_x0, roi_y0, wide_grid)
        h = C.c_void_p()
        _check(lib().gr_plan_create(C.byref(self._params), C.byref(h)), "gr_plan_create")
        self._h = h
        self.n_det, self.n_ang, self.device = n_det, n_ang, device
        self.max_pairs = max_pairs
        pd, M, M0 = C.c_int(), C.c_int(), C.c_int()
        L, sc = C.c_float(), C.c_float()
        _check(lib().gr_plan_sizes(h, C.byref(pd), C.byref(M), C.byref(M0), C.byref(L),
                                   C.byref(sc)), "gr_plan_sizes")
        self.pdim, self.M, self.M0, self.L, self.scale = pd.value, M.value, M0.value, L.value, sc.value

    def close(self):
        if getattr(self, "_h", None):
            lib().gr_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def grid_kernel(self, pairs=None) -> str:
        """'wide32' (32 pairs per warp), 'wide' (16 pairs per warp), 'tensor'
        (tcgen05) or 'tiles' for a chunk of `pairs` pairs."""
        w = C.c_int()
        _check(lib().gr_plan_grid_kernel(self._h, int(pairs or self.max_pairs), C.byref(w)),
               "gr_plan_grid_kernel")
        return ("tiles", "wide", "tensor", "wide32")[w.value]

    def device_bytes(self) -> int:
        b = C.c_size_t()
        _check(lib().gr_plan_device_bytes(self._h, C.byref(b)), "gr_plan_device_bytes")
        return b.value

    def launches(self) -> int:
        n = C.c_long()
        _check(lib().gr_plan_launch_count(self._h, C.byref(n)), "gr_plan_launch_count")
        return n.value

    def device_status(self, stream=None):
        """Raises GrError(GR_ERR_TIMEOUT) if a bounded device wait ran out."""
        _check(lib().gr_plan_device_status(self._h, _stream_ptr(stream)), "gr_plan_device_status")

    def set_timing(self, enable: bool):
        _check(lib().gr_plan_set_timing(self._h, int(enable)), "gr_plan_set_timing")

    def stage_times(self):
        """({stage: summed ms}, chunks) since set_timing(True); synchronises."""
        ms = (C.c_double * 5)()
        n = C.c_long()
        _check(lib().gr_plan_stage_times(self._h, ms, C.byref(n)), "gr_plan_stage_times")
        return dict(zip(STAGES, list(ms))), n.value

    def autotune(self, stream=None):
        """Times the gridding kernel of a full chunk, its item cap and the column-FFT
        group width; returns the choice (tuning())."""
        _check(lib().gr_plan_autotune(self._h, _stream_ptr(stream)), "gr_plan_autotune")
        return self.tuning()

    GRID_KERNEL_CODES = {"tiles": 0, "wide": 1, "wide32": 3}

    def set_tuning(self, grid_kernel=None, item_cap=0, cols_group=0, cols_ring=None):
        """Pins a tuning: grid_kernel ('tiles', 'wide', 'wide32' or None for the
        choice by chunk size) for full chunks, its work list's item cap (0: keep),
        the column-FFT group width (0: keep) and cols_ring (True: persistent
        double-buffered column FFT, False: one strip per CTA, None: keep)."""
        k = -1 if grid_kernel is None else self.GRID_KERNEL_CODES[grid_kernel]
        ring = -1 if cols_ring is None else int(bool(cols_ring))
        _check(lib().gr_plan_set_tuning(self._h, k, int(item_cap), int(cols_group), ring),
               "gr_plan_set_tuning")
        return self.tuning()

    def tuning(self):
        k, cap, g, ring = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(lib().gr_plan_tuning_ex(self._h, C.byref(k), C.byref(cap), C.byref(g),
                                       C.byref(ring)), "gr_plan_tuning_ex")
        return {"grid_kernel": ("tiles", "wide", "tensor", "wide32")[k.value],
                "item_cap": cap.value, "cols_group": g.value, "cols_ring": bool(ring.value),
                "tile": "32 x 32 (tile kernel) / 4 x 8 (register sub-tile kernels): one "
                        "compiled instance each"}

    def work_stats(self):
        a, b, c, d = C.c_int(), C.c_int(), C.c_int(), C.c_long()
        _check(lib().gr_plan_work_stats(self._h, C.byref(a), C.byref(b), C.byref(c),
                                        C.byref(d)), "gr_plan_work_stats")
        return {"items": a.value, "runs": b.value, "slots": c.value, "samples": d.value}

    def reconstruct_pair(self, sino1, sino2, out1, out2, out_stride=None, stream=None):
        """Device tensors: sino (n_ang, n_det) float32, out (M0, >= M0) float32."""
        stride = out1.shape[-1] if out_stride is None else out_stride
        _check(lib().gr_reconstruct_pair(self._h, _ptr(sino1), _ptr(sino2), _ptr(out1),
                                         _ptr(out2), stride, _stream_ptr(stream)),
               "gr_reconstruct_pair")

    def _batch(self, n_slices, dtype, sinos, centers, flat, dark, outs, out_stride,
               flat_stride=0):
        b = GrBatch()
        b.n_slices, b.dtype = int(n_slices), int(dtype)
        b.sinos, b.centers, b.flat, b.dark, b.outs = sinos, centers, flat, dark, outs
        b.out_stride = int(out_stride)
        b.flat_stride = int(flat_stride)
        return b

    def reconstruct_batch(self, sinos, outs, centers=None, flat=None, dark=None, dtype=None,
                          stream=None):
        """Device tensors: sinos (S, n_ang, n_det) f32/f16/bf16/uint16, outs (S, M0, stride)."""
        b = self.batch_desc(sinos, outs, centers, flat, dark, dtype)
        _check(lib().gr_reconstruct_batch(self._h, C.byref(b), _stream_ptr(stream)),
               "gr_reconstruct_batch")

    def batch_desc(self, sinos, outs, centers=None, flat=None, dark=None, dtype=None):
        """GrBatch for device tensors (as reconstruct_batch takes them)."""
        import torch
        if dtype is None:
            dtype = {torch.float32: DTYPE_F32, torch.float16: DTYPE_F16,
                     torch.bfloat16: DTYPE_BF16, torch.uint16: DTYPE_U16_RAW,
                     torch.int16: DTYPE_U16_RAW}[sinos.dtype]
        fs = flat.shape[-1] if flat is not None and flat.dim() == 2 else 0  # per-slice rows
        return self._batch(sinos.shape[0], dtype, _ptr(sinos), _ptr(centers), _ptr(flat),
                           _ptr(dark), _ptr(outs), outs.shape[-1], fs)

    def capture_batch(self, sinos, outs, centers=None, flat=None, dark=None, dtype=None):
        """A Graph that replays reconstruct_batch on these buffers with one launch."""
        return Graph([(self, self.batch_desc(sinos, outs, centers, flat, dark, dtype))])

    def reconstruct_host(self, sinos: np.ndarray, outs: np.ndarray, centers=None, flat=None,
                         dark=None, dtype=None, stream=0):
        """Host arrays (numpy or pinned torch CPU tensors); blocks until done."""
        def addr(x):
            if x is None:
                return None
            if isinstance(x, np.ndarray):
                return x.ctypes.data
            return int(x.data_ptr())
        if dtype is None:
            dt = str(sinos.dtype)
            dtype = DTYPE_F32 if "float32" in dt else DTYPE_F16 if "float16" in dt and "b" not in dt \
                else DTYPE_BF16 if "bfloat16" in dt else DTYPE_U16_RAW
        keep = []
        if centers is not None and isinstance(centers, np.ndarray):
            centers = np.ascontiguousarray(centers, np.float32)
            keep.append(centers)
        fs = flat.shape[-1] if flat is not None and len(flat.shape) == 2 else 0
        b = self._batch(sinos.shape[0], dtype, addr(sinos), addr(centers), addr(flat), addr(dark),
                        addr(outs), outs.shape[-1], fs)
        _check(lib().gr_reconstruct_host(self._h, C.byref(b), stream), "gr_reconstruct_host")


class Graph:
    """Batches of one or more plans recorded into one CUDA graph (gr_graph_create).

    items: list of (Plan, GrBatch).  The tensors behind the batches must stay
    alive while the graph is used: their addresses are baked in."""

    def __init__(self, items):
        arr = (GrGraphItem * len(items))()
        for k, (plan, b) in enumerate(items):
            arr[k].plan = plan.handle
            arr[k].batch = b
        h = C.c_void_p()
        _check(lib().gr_graph_create(C.cast(arr, C.c_void_p), len(items), C.byref(h)),
               "gr_graph_create")
        self._h = h
        self._plans = [p for p, _ in items]

    def launch(self, stream=None):
        _check(lib().gr_graph_launch(self._h, _stream_ptr(stream)), "gr_graph_launch")

    def launches(self) -> int:
        n = C.c_long()
        _check(lib().gr_graph_launch_count(self._h, C.byref(n)), "gr_graph_launch_count")
        return n.value

    def close(self):
        if getattr(self, "_h", None):
            lib().gr_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GridRec:
    """The reference's GridRec call surface on the B200 library.

    Mirrors gridrec/GPU/gridrec.h:72-143 and recon_algorithm.h:56-95: set the
    sinogram dimensions, theta list (degrees), filter code and device, call
    init(), hand over the two slices' host buffers with setSinoAndReconBuffers
    (sinogram n_ang x n_det float32; reconstruction n_det x n_det float32, the
    leading M0 x M0 block written with row stride n_det as in gridrec.cu:196-197),
    then reconstruct().  setCenter() adds the rotation centre that GridRec::init
    fixes at n_det/2 (gridrec.cu:227); setCenterShift() is find_shift's form of it
    (centre = n_det // 2 + shift at init, find_shift/src/main/gridrec.cu:229, 809-813).
    """

    def __init__(self):
        self._dims = None
        self._theta = None
        self._filter = FILTER_NONE
        self._device = 0
        self._center = None
        self._shift = None
        self._bufs = {}
        self._plan = None

    def numberOfSinogramsNeeded(self) -> int:
        return 2

    def numberOfReconstructions(self) -> int:
        return 2

    def setSinogramDimensions(self, x_dim: int, y_dim: int):
        self._dims = (int(x_dim), int(y_dim))

    def getSinogramXDimension(self):
        return self._dims[0]

    def getSinogramYDimension(self):
        return self._dims[1]

    def setThetaList(self, theta_list, theta_list_size: int):
        self._theta = np.asarray(theta_list, np.float32)[:theta_list_size]

    def getThetaListSize(self):
        return len(self._theta)

    def setFilter(self, filter_name: int):
        self._filter = int(filter_name)

    def getFilter(self) -> int:
        return self._filter

    def setGPUDeviceID(self, device: int):
        self._device = int(device)

    def getGPUDeviceID(self) -> int:
        return self._device

    def setCenter(self, center: float):
        self._center = float(center)
        self._shift = None

    def setCenterShift(self, shift: float):
        self._shift = float(shift)

    def getThetaList(self):
        return self._theta

    def getCenter(self):
        if self._shift is not None:
            return float(np.float32(self._dims[0] // 2) + np.float32(self._shift))
        return self._center

    def init(self):
        n_det, n_ang = self._dims
        self._plan = Plan(n_det, n_ang, self._theta, center=self.getCenter(),
                          filter=self._filter, device=self._device, max_pairs=1)
        self.M0 = self._plan.M0

    def setSinoAndReconBuffers(self, number: int, sinogram, reconstruction):
        if number in (1, 2):
            self._bufs[number] = (sinogram, reconstruction)

    def reconstruct(self):
        n_det, n_ang = self._dims
        s1, r1 = self._bufs[1]
        s2, r2 = self._bufs.get(2, (None, None))
        m0 = self.M0

        def host_f32(x, shape):
            a = np.asarray(x)
            ok = a.dtype == np.float32 and a.flags.c_contiguous and a.size == shape[0] * shape[1]
            return a if ok else np.ascontiguousarray(a, np.float32).reshape(shape)
        in1 = host_f32(s1, (n_ang, n_det))
        in2 = host_f32(s2, (n_ang, n_det)) if s2 is not None else None
        direct = m0 <= n_det and all(
            r is None or (isinstance(r, np.ndarray) and r.dtype == np.float32 and
                          r.flags.c_contiguous and r.size >= m0 * n_det) for r in (r1, r2))
        if direct:  # the caller's host arrays in and out, rows of stride n_det
            _check(lib().gr_reconstruct_pair_host(
                self._plan.handle, in1.ctypes.data, in2.ctypes.data if in2 is not None else None,
                r1.ctypes.data, r2.ctypes.data if r2 is not None else None, n_det, None),
                "gr_reconstruct_pair_host")
            return
        stride = max(m0, n_det)
        outs = np.zeros((2, m0, stride), np.float32)
        _check(lib().gr_reconstruct_pair_host(
            self._plan.handle, in1.ctypes.data, in2.ctypes.data if in2 is not None else None,
            outs[0].ctypes.data, outs[1].ctypes.data, stride, None), "gr_reconstruct_pair_host")
        for r, o in ((r1, outs[0]), (r2, outs[1])):
            if r is None:
                continue
            rv = np.asarray(r).reshape(-1, n_det)
            k = min(m0, n_det)
            rows = min(m0, rv.shape[0])
            rv[:rows, :k] = o[:rows, :k]

    def destroy(self):
        if self._plan is not None:
            self._plan.close()
            self._plan = None


# ---------------------------------------------------------------- slice pipeline
# Steps of the reference's drivers around gridrec (gridrec/GPU/tomo_recon.cpp,
# find_shift/src/main/find_shift.cpp), on device tensors.

def ring_removal(sinos, ring_coeff=1.0, iterations=20, stream=None):
    """In place on a (S, n_ang, n_det) float32 CUDA tensor: RingCorrectionSinogram
    (tomo_recon.cpp:3905-3972; the reference runs 20 rounds, RING_COEFF 1.0)."""
    import torch
    S, a, n = sinos.shape
    with _on_stream(stream):
        ws = torch.empty(lib().gr_ring_workspace_bytes(S, n, a), dtype=torch.uint8,
                         device=sinos.device)
        _check(lib().gr_ring_removal(_ptr(sinos), S, n, a, float(ring_coeff), int(iterations),
                                     _ptr(ws), _stream_ptr(stream)), "gr_ring_removal")
    return sinos


def shift_pad(sinos, xoffsets, out_width=None, stream=None):
    """(S, n_ang, n_det) float32 -> (S, n_ang, out_width): sub-pixel shift by
    xoffsets[s] and half padding (tomo_recon.cpp:3708-3807)."""
    import torch
    S, a, n = sinos.shape
    w = 2 * n if out_width is None else int(out_width)
    with _on_stream(stream):
        xo = torch.as_tensor(xoffsets, dtype=torch.float32).reshape(-1)
        if xo.device != sinos.device:
            # staged from pageable memory by the call itself; non_blocking spares
            # the stream synchronisation of a blocking copy
            xo = xo.to(sinos.device, non_blocking=True)
        if xo.numel() == 1:
            xo = xo.expand(S).contiguous()
        out = torch.empty((S, a, w), dtype=torch.float32, device=sinos.device)
        _check(lib().gr_shift_pad(_ptr(sinos), _ptr(out), S, n, a, _ptr(xo), w,
                                  _stream_ptr(stream)), "gr_shift_pad")
    return out


def crop_center(recs, n, offset, radius=0, stream=None):
    """(S, rows, stride) float32 -> (S, n, n) window at (offset, offset); radius > 0
    zeroes pixels outside the circle of tomo_recon.cpp:2150-2165."""
    import torch
    S, rows, stride = recs.shape
    if offset + n > rows:
        raise ValueError("crop window exceeds the image rows")
    with _on_stream(stream):
        out = torch.empty((S, n, n), dtype=torch.float32, device=recs.device)
        _check(lib().gr_crop_center(_ptr(recs), stride, rows * stride, _ptr(out), n, n * n, S, n,
                                    offset, int(radius), _stream_ptr(stream)), "gr_crop_center")
    return out


def threshold_range(images, lower_clamp=-1e30, upper_clamp=1e30, stream=None):
    """(lo, hi) of the reference's 8-bit slice writer for images (S, rows, cols),
    a CUDA float32 tensor or a view with unit column stride, as a (2,) float32 CUDA
    tensor (tomo_recon.cpp:2282-2311)."""
    import torch
    S, rows, cols = images.shape
    if images.stride(2) != 1:
        raise ValueError("images need unit column stride")
    with _on_stream(stream):
        ws = torch.empty(lib().gr_threshold_workspace_bytes(), dtype=torch.uint8,
                         device=images.device)
        lohi = torch.empty(2, dtype=torch.float32, device=images.device)
        _check(lib().gr_threshold_range(_ptr(images), S, rows, cols, images.stride(1),
                                        images.stride(0), float(lower_clamp), float(upper_clamp),
                                        _ptr(lohi), _ptr(ws), _stream_ptr(stream)),
               "gr_threshold_range")
    return lohi


def to_u8(images, lohi, radius=0, out=None, stream=None):
    """8-bit slices (S, rows, cols) uint8 of the reference's BMP/TIFF writer
    (tomo_recon.cpp:2338-2361), optionally its cropped copy (radius > 0)."""
    import torch
    S, rows, cols = images.shape
    if images.stride(2) != 1:
        raise ValueError("images need unit column stride")
    with _on_stream(stream):
        if out is None:
            out = torch.empty((S, rows, cols), dtype=torch.uint8, device=images.device)
        _check(lib().gr_to_u8(_ptr(images), S, rows, cols, images.stride(1), images.stride(0),
                              _ptr(lohi), int(radius), _ptr(out), out.stride(1), out.stride(0),
                              _stream_ptr(stream)), "gr_to_u8")
    return out


def entropy(images, vmin, vmax, nbins, group=1, stream=None):
    """Histogram entropy (find_shift.cpp:2078-2115) of each group of `group`
    consecutive (rows, cols) images of a (G*group, rows, cols) float32 tensor."""
    import torch
    N, rows, cols = images.shape
    if N % group:
        raise ValueError("image count must be a multiple of group")
    G = N // group
    st = images.stride()
    with _on_stream(stream):
        ws = torch.empty(lib().gr_entropy_workspace_bytes(G, nbins), dtype=torch.uint8,
                         device=images.device)
        out = torch.empty(G, dtype=torch.float32, device=images.device)
        _check(lib().gr_entropy(_ptr(images), G, group, rows, cols, st[1], st[0], st[0] * group,
                                float(vmin), float(vmax), int(nbins), _ptr(out), _ptr(ws),
                                _stream_ptr(stream)), "gr_entropy")
    return out


def reconstruct_padded(plan: "Plan", sinos, xoffset=0.0, stream=None):
    """GridRecSlices (tomo_recon.cpp:3679-3862): shift by xoffset, half-pad to the
    plan's width (2 n_det), reconstruct, crop n_det x n_det.  sinos (S, n_ang, n_det)."""
    import torch
    S, a, n = sinos.shape
    with _on_stream(stream):
        out = torch.empty((S, n, n), dtype=torch.float32, device=sinos.device)
        _check(lib().gr_reconstruct_padded(plan.handle, _ptr(sinos), S, n, a, float(xoffset),
                                           _ptr(out), n, _stream_ptr(stream)),
               "gr_reconstruct_padded")
    return out


def center_search(plan: "Plan", sino1, sino2, shifts, hist_lo, hist_hi, nbins,
                  want_images=False, stream=None):
    """find_shift's entropy refinement (find_shift.cpp:1653-1900).

    Returns (scores[n_cand] numpy, best index, best pair images (2, n, n) or None)."""
    import torch
    a, n = sino1.shape
    sh = np.ascontiguousarray(shifts, np.float32)
    scores = np.zeros(sh.size, np.float32)
    best = C.c_int(-1)
    fp = C.POINTER(C.c_float)
    with _on_stream(stream):
        imgs = torch.empty((2, n, n), dtype=torch.float32, device=sino1.device) \
            if want_images else None
        _check(lib().gr_center_search(plan.handle, _ptr(sino1), _ptr(sino2), n, a,
                                      sh.ctypes.data_as(fp), sh.size, float(hist_lo),
                                      float(hist_hi), int(nbins), scores.ctypes.data_as(fp),
                                      C.byref(best), _ptr(imgs), _stream_ptr(stream)),
               "gr_center_search")
    return scores, best.value, imgs


def xcorr_scores(templ_roi, match, roi, tx0, ty0, dtx, dty, n_tx, n_ty, stream=None):
    """find_shift's brute-force cross-correlation scores (find_shift.cpp:1975-2076) on
    device tensors: templ_roi (roi_h, roi_w), match (height, width) float32; roi =
    (x0, x1, y0, y1) inclusive.  Returns (n_ty, n_tx) float64 numpy scores."""
    h, w = match.shape
    out = np.zeros((n_ty, n_tx), np.float64)
    _check(lib().gr_xcorr_scores(_ptr(templ_roi), _ptr(match), w, h, *[int(v) for v in roi],
                                 float(tx0), float(ty0), float(dtx), float(dty), int(n_tx),
                                 int(n_ty), out.ctypes.data_as(C.POINTER(C.c_double)),
                                 _stream_ptr(stream)), "gr_xcorr_scores")
    return out


def find_shift_xcorr(templ_roi, match, roi, tx_range, ty_range, n_subpixel, stream=None):
    """The translation search of find_shift (find_shift.cpp:1283-1480, GPU brute-force
    branch): scores over tx_range = (start, end, step) x ty_range, the first maximum,
    then 2 n_subpixel + 1 sub-pixel steps of step/n_subpixel in x from one coarse
    step below it.  Returns (tx_subpixel, ty, coarse scores, sub-pixel scores); the
    rotation axis offset the reference prints is tx_subpixel / 2."""
    sx, ex, ix = tx_range
    sy, ey, iy = ty_range
    n_tx = int((ex - sx) / ix) + 1
    n_ty = int((ey - sy) / iy) + 1
    coarse = xcorr_scores(templ_roi, match, roi, sx, sy, ix, iy, n_tx, n_ty, stream)
    best = int(np.argmax(coarse.reshape(-1)))  # first maximum, as the reference's scan
    by, bx = divmod(best, n_tx)
    ty = sy + by * iy
    sub_step = ix / n_subpixel
    start = sx + (bx - 1) * ix
    sub = xcorr_scores(templ_roi, match, roi, start, ty, sub_step, iy, 2 * n_subpixel + 1, 1,
                       stream)[0]
    # The reference keeps the coarse best score as the bar for the sub-pixel scan
    # (find_shift.cpp:1440-1455), so when no sub-pixel score beats it the result
    # falls back to index 0, one coarse step low; the maximum is taken here.
    bs = int(np.argmax(sub))
    return start + bs * sub_step, ty, coarse, sub


class FBP:
    """The FBP comparator (OptimizedFBP, gridrec/GPU/filteredbackprojection.cpp:190-330)."""

    def __init__(self, n_det, n_ang, theta_deg, max_slices=4, device=0):
        th = np.ascontiguousarray(theta_deg, np.float32)
        h = C.c_void_p()
        _check(lib().gr_fbp_create(int(n_det), int(n_ang), th.ctypes.data_as(C.POINTER(C.c_float)),
                                   int(max_slices), int(device), C.byref(h)), "gr_fbp_create")
        self._h = h
        self.n_det, self.n_ang = n_det, n_ang

    def reconstruct(self, sinos, recons=None, stream=None):
        """sinos (S, n_ang, n_det) float32 CUDA tensor -> (S, n_det, n_det)."""
        import torch
        S = sinos.shape[0]
        with _on_stream(stream):
            if recons is None:
                recons = torch.empty((S, self.n_det, self.n_det), dtype=torch.float32,
                                     device=sinos.device)
            _check(lib().gr_fbp_reconstruct(self._h, _ptr(sinos), S, _ptr(recons),
                                            _stream_ptr(stream)), "gr_fbp_reconstruct")
        return recons

    def close(self):
        if getattr(self, "_h", None):
            lib().gr_fbp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
