"""Learned narrow-kernel gridrec: gridding with the narrowest PSWF kernel of the
reference's table (C = 4, 3 x 3 taps instead of 4 x 4 at C = 6) followed by a
3-layer, 16-channel residual CNN that corrects the slice toward full-width
gridrec.  Plain gridrec stays the fallback and the judge: a batch whose held-out
error against the full kernel exceeds the tolerance is recomputed with it.

The network runs on this library's own kernels (projects_b200/csrc/gridrec_cnn.cu):
inference is one fused kernel per launch (tcgen05 BF16 MMAs for the 16 -> 16 layer
and conv3's 1x1 partials, FP32 accumulation in tensor memory, activations kept in
shared memory); training runs its own forward, backward and Adam kernels.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import gridrec as G

N_PARAMS = 2625
def params_file(pswf_c=4.0):
    """Trained parameters of the network for the narrow kernel of PSWF parameter C."""
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), f"correction_c{pswf_c:g}.npy")


PARAMS_FILE = params_file(4.0)


def _lib():
    L = G.lib()
    if not getattr(L, "_cnn_bound", False):
        vp, i_, f_ = C.c_void_p, C.c_int, C.c_float
        L.gr_cnn_param_count.restype = C.c_int
        L.gr_cnn_workspace_bytes.argtypes = [i_, i_, i_]
        L.gr_cnn_workspace_bytes.restype = C.c_size_t
        L.gr_cnn_forward_workspace_bytes.argtypes = [i_, i_, i_]
        L.gr_cnn_forward_workspace_bytes.restype = C.c_size_t
        L.gr_cnn_forward.argtypes = [vp, vp, vp, i_, i_, i_, vp, vp]
        L.gr_cnn_backward.argtypes = [vp, vp, vp, vp, i_, i_, i_, vp, C.POINTER(C.c_double), vp,
                                      vp]
        L.gr_cnn_adam.argtypes = [vp, vp, vp, vp, i_, f_, f_, f_, f_, vp]
        L.gr_cnn_infer_workspace_bytes.restype = C.c_size_t
        L.gr_cnn_infer.argtypes = [vp, vp, vp, vp, i_, i_, i_, vp, vp]
        L.gr_cnn_infer_status.argtypes = [vp, vp]
        L._cnn_bound = True
    return L


def init_params(seed=0):
    """He-scaled random first two layers; the last layer starts at zero, so the
    untrained network is the identity (y = x)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    p[0:144] = rng.normal(0, np.sqrt(2.0 / 9), 144)
    p[160:2464] = rng.normal(0, np.sqrt(2.0 / 144), 2304)
    return p


class CorrectionNet:
    """The residual CNN on a CUDA device (parameters, Adam state, workspace)."""

    def __init__(self, params=None, device="cuda"):
        import torch
        if G.lib().gr_cnn_param_count() != N_PARAMS:
            raise RuntimeError("library CNN parameter count mismatch")
        p = init_params() if params is None else np.asarray(params, np.float32)
        self.params = torch.tensor(p, device=device)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grads = torch.zeros_like(self.params)
        self.step = 0
        self._ws = None
        self._ws_shape = None
        # the fused inference kernel's error word (zeroed; gr_cnn_infer_status clears it)
        self._iws = torch.zeros(int(_lib().gr_cnn_infer_workspace_bytes()), dtype=torch.uint8,
                                device=self.params.device)
        # these buffers are filled on the current stream; later calls may run on
        # another one, so they are complete before the constructor returns
        torch.cuda.current_stream(self.params.device).synchronize()

    def _workspace(self, n, h, w, train=False):
        """Forward-only workspace (the activations) unless training needs the
        gradient buffers too; grows to the larger kind when asked for it."""
        import torch
        key = (n, h, w, train)
        have = self._ws_shape
        if have is None or have[:3] != (n, h, w) or (train and not have[3]):
            nbytes = (_lib().gr_cnn_workspace_bytes(n, h, w) if train
                      else _lib().gr_cnn_forward_workspace_bytes(n, h, w))
            self._ws = None
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=self.params.device)
            self._ws_shape = key
        return self._ws

    def forward(self, x, y=None, stream=None, train=False):
        """x: (N, H, W) float32 CUDA tensor -> y = x + correction."""
        import torch
        n, h, w = x.shape
        with G._on_stream(stream):
            if y is None:
                y = torch.empty_like(x)
            ws = self._workspace(n, h, w, train)
            G._check(_lib().gr_cnn_forward(G._ptr(self.params), G._ptr(x), G._ptr(y), n, h, w,
                                           G._ptr(ws), G._stream_ptr(stream)), "gr_cnn_forward")
        return y

    def infer(self, x, y=None, stream=None, scale=None):
        """x: (N, H, W) float32 CUDA tensor -> y = x + correction, by the fused
        tcgen05 inference kernel (weights and conv1's input in BF16, FP32
        accumulators; no activation workspace).  scale (N floats on the device):
        y_i = s_i * net(x_i / s_i), the scaling done inside the kernel."""
        import torch
        n, h, w = x.shape
        with G._on_stream(stream):
            if y is None:
                y = torch.empty_like(x)
            sp = None
            if scale is not None:
                scale = scale.reshape(-1).contiguous()
                if scale.numel() != n or scale.dtype != torch.float32 or scale.device != x.device:
                    raise ValueError("scale: one float32 per image, on the images' device")
                sp = G._ptr(scale)
            G._check(_lib().gr_cnn_infer(G._ptr(self.params), G._ptr(x), G._ptr(y), sp, n, h, w,
                                         G._ptr(self._iws), G._stream_ptr(stream)),
                     "gr_cnn_infer")
        return y

    def infer_status(self, stream=None):
        """Synchronises; raises if a bounded wait of the fused kernel ran out."""
        G._check(_lib().gr_cnn_infer_status(G._ptr(self._iws), G._stream_ptr(stream)),
                 "gr_cnn_infer_status")

    def loss_and_grads(self, x, target, stream=None):
        """Forward + backward; fills self.grads, returns the mean-squared loss."""
        y = self.forward(x, stream=stream, train=True)
        n, h, w = x.shape
        loss = C.c_double()
        G._check(_lib().gr_cnn_backward(G._ptr(self.params), G._ptr(x), G._ptr(y),
                                        G._ptr(target), n, h, w, G._ptr(self.grads),
                                        C.byref(loss), G._ptr(self._ws), G._stream_ptr(stream)),
                 "gr_cnn_backward")
        return loss.value

    def train_step(self, x, target, lr=1e-3, stream=None):
        loss = self.loss_and_grads(x, target, stream)
        self.step += 1
        G._check(_lib().gr_cnn_adam(G._ptr(self.params), G._ptr(self.grads), G._ptr(self.m),
                                    G._ptr(self.v), self.step, lr, 0.9, 0.999, 1e-8,
                                    G._stream_ptr(stream)), "gr_cnn_adam")
        return loss

    def numpy_params(self):
        return self.params.detach().cpu().numpy().copy()


class LearnedGridrec:
    """Narrow-kernel (C = 4 by default, or 5) gridrec + correction CNN, with
    full-width (C = 6) fallback.

    reconstruct_batch() reconstructs with the narrow plan, corrects with the
    network, then reconstructs the first pair with the full plan and compares:
    if its relative L2 error exceeds `tol`, the whole batch is recomputed with
    the full plan (the result is then plain gridrec)."""

    def __init__(self, n_det, n_ang, theta_deg, params=None, tol=1e-3, max_pairs=8,
                 filter=G.FILTER_HANN, device=0, pswf_c=4.0):
        self.narrow = G.Plan(n_det, n_ang, theta_deg, filter=filter, pswf_c=pswf_c,
                             max_pairs=max_pairs, device=device)
        self.full = G.Plan(n_det, n_ang, theta_deg, filter=filter, pswf_c=6.0,
                           max_pairs=max_pairs, device=device)
        if self.narrow.M0 != self.full.M0:
            raise ValueError("narrow and full plans disagree on the image size")
        if params is None and os.path.exists(params_file(pswf_c)):
            params = np.load(params_file(pswf_c))
        self.net = CorrectionNet(params, device=f"cuda:{device}")
        self.tol = tol
        self.M0 = self.full.M0

    @staticmethod
    def scales(images):
        """Per-slice RMS, (S, 1, 1): the network sees every slice at unit RMS, so
        its correction does not depend on the absolute scale of the values (which
        follows the pixel size, i.e. the detector width)."""
        import torch
        n = images.shape[1] * images.shape[2]
        rms = torch.linalg.vector_norm(images, dim=(1, 2), keepdim=True) / math.sqrt(n)
        return rms.clamp_min(1e-30)

    def correct(self, raw, stream=None):
        """s * net(raw / s) per slice (the fused inference kernel, which applies s).
        The scales are computed on `stream`, after the kernels that wrote raw."""
        with G._on_stream(stream):
            return self.net.infer(raw.contiguous(), stream=stream, scale=self.scales(raw))

    def corrected(self, sinos, centers=None, stream=None):
        """Narrow-kernel images corrected by the network, (S, M0, M0)."""
        import torch
        S = sinos.shape[0]
        with G._on_stream(stream):
            raw = torch.empty((S, self.M0, self.M0), dtype=torch.float32, device=sinos.device)
            self.narrow.reconstruct_batch(sinos, raw, centers=centers, stream=stream)
            return self.correct(raw, stream=stream)

    def reconstruct_batch(self, sinos, centers=None, stream=None):
        """Returns (images, info): info = {"held_out_rel_l2", "fallback"}.  The first
        pair is judged before the rest is reconstructed, so a batch that falls back
        runs the narrow kernel and the network on two slices only."""
        import torch
        k = min(2, sinos.shape[0])
        ck = None if centers is None else centers[:k]
        # the torch work here (norms, copies, allocations) runs on `stream`, in
        # order with the kernels
        with G._on_stream(stream):
            ref = torch.empty((k, self.M0, self.M0), dtype=torch.float32, device=sinos.device)
            self.full.reconstruct_batch(sinos[:k], ref, centers=ck, stream=stream)
            probe = self.corrected(sinos[:k], ck, stream)
            err = float(torch.linalg.vector_norm(probe - ref) / torch.linalg.vector_norm(ref))
            fallback = err > self.tol
            out = torch.empty((sinos.shape[0], self.M0, self.M0), dtype=torch.float32,
                              device=sinos.device)
            if fallback:
                self.full.reconstruct_batch(sinos, out, centers=centers, stream=stream)
            else:
                out.copy_(self.corrected(sinos, centers, stream))
        return out, {"held_out_rel_l2": err, "fallback": fallback}

    def close(self):
        self.narrow.close()
        self.full.close()
