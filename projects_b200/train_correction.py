"""Trains the correction network of the learned narrow-kernel path on the GPU and
writes projects_b200/correction_c<C>.npy (C = 4: correction_c4.npy).

Training data follow the learned-path configuration: random-ellipse slices from
1024-detector x 900-angle sinograms; input = narrow-kernel (PSWF C = 4 or 5)
gridrec, target = full-width (C = 6) FP32 gridrec of the same sinogram.
Evaluation: held-out 2048 x 1500 slices, relative L2 and PSNR against full-width
gridrec, for the narrow kernel alone and with the network.

    python -m projects_b200.train_correction [--pswf-c 4] [--slices 4096] [--batch 8]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main():
    import torch

    from projects_b200 import gridrec as G
    from projects_b200 import learned as Lrn
    from projects_b200 import phantom as ph
    ap = argparse.ArgumentParser()
    ap.add_argument("--slices", type=int, default=4096)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--eval-slices", type=int, default=8)
    ap.add_argument("--pswf-c", type=float, default=4.0, help="narrow kernel's PSWF C (4 or 5)")
    ap.add_argument("--out", default=None, help="default: projects_b200/correction_c<C>.npy")
    args = ap.parse_args()
    out = args.out or Lrn.params_file(args.pswf_c)
    dev = torch.device("cuda")
    n, a = 1024, 900
    th = ph.angles_deg(a)
    narrow = G.Plan(n, a, th, filter=G.FILTER_HANN, pswf_c=args.pswf_c, max_pairs=args.batch // 2)
    full = G.Plan(n, a, th, filter=G.FILTER_HANN, pswf_c=6.0, max_pairs=args.batch // 2)
    net = Lrn.CorrectionNet()
    t0 = time.time()
    losses = []
    for b0 in range(0, args.slices, args.batch):
        s = torch.stack([ph.random_ellipse_sinogram(b0 + i, n, a, device=dev)[0]
                         for i in range(args.batch)])
        x = torch.empty((args.batch, narrow.M0, narrow.M0), device=dev)
        t = torch.empty_like(x)
        narrow.reconstruct_batch(s, x)
        full.reconstruct_batch(s, t)
        sc = Lrn.LearnedGridrec.scales(x)
        lr = args.lr * (0.1 if b0 > 0.8 * args.slices else 1.0)
        losses.append(net.train_step((x / sc).contiguous(), (t / sc).contiguous(), lr=lr))
    train_s = time.time() - t0
    narrow.close()
    full.close()
    np.save(out, net.numpy_params())
    # held-out evaluation at 2048 x 1500
    n2, a2 = 2048, 1500
    th2 = ph.angles_deg(a2)
    lg = Lrn.LearnedGridrec(n2, a2, th2, params=net.numpy_params(), max_pairs=4,
                            pswf_c=args.pswf_c)
    e_raw, e_cnn, p_raw, p_cnn = [], [], [], []
    for k in range(args.eval_slices):
        s = ph.random_ellipse_sinogram(10_000_000 + k, n2, a2, device=dev)[0][None]
        s = torch.cat([s, s])
        x = torch.empty((2, lg.M0, lg.M0), device=dev)
        ref = torch.empty_like(x)
        lg.narrow.reconstruct_batch(s, x)
        lg.full.reconstruct_batch(s, ref)
        y = lg.correct(x)
        r = ref[0].cpu().numpy()
        for img, el, pl in ((x[0].cpu().numpy(), e_raw, p_raw), (y[0].cpu().numpy(), e_cnn, p_cnn)):
            el.append(ph.rel_l2(img, r))
            pl.append(ph.psnr(img, r))
    lg.close()
    print(json.dumps({"pswf_c": args.pswf_c, "train_slices": args.slices, "train_s": train_s,
                      "loss_first": losses[0], "loss_last": float(np.mean(losses[-10:])),
                      "heldout_2048x1500": {"rel_l2_narrow": float(np.mean(e_raw)),
                                            "rel_l2_narrow_cnn": float(np.mean(e_cnn)),
                                            "psnr_narrow": float(np.mean(p_raw)),
                                            "psnr_narrow_cnn": float(np.mean(p_cnn))},
                      "params": out}))


if __name__ == "__main__":
    main()
