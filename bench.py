#!/usr/bin/env python
"""Throughput benchmark of the B200 gridrec hot path.

Workload (one "step"): plain full-width gridrec of 256 slices, 2048 detector
pixels x 1500 angles on [0, pi), float32 sinograms of random-ellipse phantoms
(seed = slice index, 1e4-photon Poisson noise), per-slice rotation centres
1024 + U[-2, 2], Hann filter, PSWF C = 6 (L = 3.82), output 2047 x 2047 valid
in 2048-stride float32 images.  Inputs (3.1 GB per step) are larger than L2.

  value  slices/s with sinograms resident in HBM (gr_reconstruct_batch)
  e2e    slices/s through the host-buffer entry point (gr_reconstruct_host)
         with pinned host inputs/outputs, H2D and D2H inside the timed region
  roofline  dominant kernel's algorithmic bytes / its CUDA-event time vs the
         measured copy bandwidth
  cpu_baseline  the reference's own CPU GridRec (compiled from its sources into
         oracle/_ref) on the host cores, bounded sample
  parity relL2 / max-abs of two timed images against float64 gridrec (CPU leg)
  uneven the 512-slice uneven batch (1024x720, 2048x1500, 4096x3000 at 3:2:1), raw
         uint16 with flat/dark fused on load, one CUDA-graph launch per step, plus
         f32 and f16 storage; their error against float64 in the CPU leg
  stream 128 slices of 4096x3000 raw uint16 streamed from pinned host memory and back,
         end to end next to kernel-only

python bench.py [--gpus N --steps K --warmup W] [--impl reference]
Under torchrun each rank reconstructs its own 256 slices (weak scaling, no
collective on the data path); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("slices/s 2048²@1500 angles, learned vs plain gridrec, 1 B200, "
          "relL2≤1e-3; %HBM peak")
UNIT = "slices/s"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--slices", type=int, default=256)
    ap.add_argument("--n-det", type=int, default=2048)
    ap.add_argument("--n-ang", type=int, default=1500)
    ap.add_argument("--max-pairs", type=int, default=32)
    ap.add_argument("--dtype", default="f32", choices=["f32", "f16", "bf16"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--e2e-max-pairs", type=int, default=8,
                    help="pairs per streamed chunk of the end-to-end (host buffer) measurement")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-pipeline", action="store_true",
                    help="skip the slice-pipeline step timings (ring, shift/pad, padded "
                         "reconstruction, centre search)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default gridding item cap and column-FFT group width")
    ap.add_argument("--config", default="batch", choices=["batch", "uneven", "stream"],
                    help="batch: 256 slices of n_det x n_ang (default); uneven: 512 slices "
                         "mixing 1024x720, 2048x1500, 4096x3000 (3:2:1), raw uint16 with "
                         "per-slice flat/dark, all shapes in one CUDA-graph launch; stream: "
                         "4096 x 3000 raw uint16 slices streamed from pinned host memory "
                         "(--stream-slices, cycling a 64-slice host ring)")
    ap.add_argument("--stream-slices", type=int, default=2048)
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the uneven-batch and streaming keys of the default run")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers

def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


def bf16_sustained_tflops():
    """Sustained dense BF16 TFLOP/s of MEASURED_PEAKS.json, else the 1.4 PFLOP/s fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f).get("bf16_tflops_sustained", 1400.0))
    return 1400.0


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = str(device)
        try:  # nvidia-smi numbering can differ from CUDA's: select by UUID
            import torch
            u = str(torch.cuda.get_device_properties(device).uuid)
            self.device = u if u.startswith("GPU-") else "GPU-" + u
        except Exception:
            pass
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", self.device], stdout=self.f,
                stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return None
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        if not sm:
            return None
        loaded = [x for x in sm if x > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "samples": len(sm),
                "reasons": sorted(reasons)}


def max_over_ranks(seconds, device, world):
    """The job's time: the maximum of the ranks' elapsed times (all_reduce MAX)."""
    if world <= 1:
        return seconds
    import torch
    import torch.distributed as dist
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_first_seed(rank, slices_per_rank):
    """Each rank reconstructs its own slices (weak scaling): seeds rank*S .. rank*S+S-1."""
    return rank * slices_per_rank


def make_sinograms(n_slices, n_det, n_ang, first_seed, device):
    """Random-ellipse sinograms (seed = slice index) on the device + centres."""
    import torch

    from projects_b200 import phantom as ph
    th = ph.angles_deg(n_ang)
    sinos = torch.empty((n_slices, n_ang, n_det), dtype=torch.float32, device=device)
    centers = np.zeros(n_slices, np.float32)
    for i in range(n_slices):
        s, c = ph.random_ellipse_sinogram(first_seed + i, n_det, n_ang, device=device)
        sinos[i].copy_(s)
        centers[i] = c
    return th, sinos, centers


def algorithmic_bytes_per_pair(n_det, n_ang, pdim, M, M0, in_bytes=4):
    """Bytes each stage must move per slice pair (read + write), staged design."""
    J = pdim // 2
    spec = 2 * n_ang * J * 8
    return {
        "phase": J * 16,
        "spectra": 2 * n_ang * n_det * in_bytes + spec,
        "grid": spec + M * M * 8,
        "cols": 2 * M * M * 8,
        "rows_deapod": M * M * 8 + 2 * M0 * M0 * 4,
    }


class gpu_local_cpus:
    """Runs the enclosed allocations on the host CPUs local to the GPU (its PCI
    device's local_cpulist in sysfs), so that pinned host buffers, placed on first
    touch, sit on the GPU's NUMA node: host<->device copies then avoid the
    inter-socket link.  The previous affinity is restored on exit; where the
    information is missing nothing changes.  `self.cpus` records what was found:
    the local CPU list and whether the process was narrowed to it, was on it
    already, or has no CPU on it; or why the list could not be read."""

    def __init__(self, device):
        self.device, self.cpus, self._old = device, None, None

    def __enter__(self):
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.device)
            bdf = "%04x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            with open(f"/sys/bus/pci/devices/{bdf}/local_cpulist") as f:
                spec = f.read().strip()
            cpus = set()
            for part in spec.split(","):
                lo, _, hi = part.partition("-")
                cpus.update(range(int(lo), int(hi or lo) + 1))
            old = os.sched_getaffinity(0)
            use = cpus & old
            if use and use != old:
                os.sched_setaffinity(0, use)
                self._old, self.cpus = old, f"{spec} (process narrowed to them)"
            elif use:
                self.cpus = f"{spec} (process already on them)"
            else:
                self.cpus = f"{spec} (no process CPU among them: placement unchanged)"
        except (OSError, ValueError, AttributeError, RuntimeError) as e:
            self.cpus = f"GPU-local CPU list unavailable ({type(e).__name__})"
        return self

    def __exit__(self, *exc):
        if self._old:
            os.sched_setaffinity(0, self._old)
        return False


def traffic_from_profile(stage, pairs_per_launch, n_det, n_ang):
    """DRAM bytes per launch (ncu read + write per pair, scaled by the pairs of
    one launch) from the committed profile summary of this workload."""
    path = os.path.join(ROOT, "profiles", f"traffic_{n_det}x{n_ang}.txt")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) == 2 and parts[0] == stage:
                return float(parts[1]) * pairs_per_launch
    return None


def cpu_reference(n_det, n_ang, seconds, threads=None, steps=None):
    """The reference CPU GridRec on the host cores: returns (slices/s, info).

    Each thread reconstructs slice pairs with its own GridRec instance until
    `seconds` elapse (or `steps` rounds of one pair per thread)."""
    from oracle import oracle as O
    from projects_b200 import phantom as ph
    th = ph.angles_deg(n_ang)
    s = [ph.random_ellipse_sinogram(k, n_det, n_ang)[0] for k in range(2)]
    pair = np.stack(s)
    threads = threads or os.cpu_count() or 1
    if O.ref_available():
        kind = "reference"

        def one():
            return O.ref_gridrec_pairs(pair, th, filter=2)[1]
    else:
        kind = "port"

        def one():
            t0 = time.perf_counter()
            O.port_gridrec_pair(pair[0], pair[1], th, filter=2)
            return time.perf_counter() - t0

    def worker(deadline, rounds):
        done = 0
        while True:
            one()
            done += 1
            if rounds is not None and done >= rounds:
                return done
            if rounds is None and time.perf_counter() >= deadline:
                return done

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as ex:
        futs = [ex.submit(worker, t0 + seconds, steps) for _ in range(threads)]
        pairs = sum(f.result() for f in futs)
    wall = time.perf_counter() - t0
    return 2.0 * pairs / wall, {"kind": kind, "cores": threads, "pairs": pairs, "wall_s": wall}


def parity_check(sinos, outs, centers, th, M0):
    """relL2 and max-abs of the first slice pair of the timed step's images against
    float64 gridrec of the same sinograms (the oracle as the checker, after the
    timed region)."""
    from oracle import oracle as O
    from projects_b200 import phantom as ph
    s = sinos[:2].float().cpu().numpy()
    got = outs[:2, :, :M0].cpu().numpy().astype(np.float64)
    r1, r2 = O.port_gridrec_pair(s[0], s[1], th, center1=float(centers[0]),
                                 center2=float(centers[1]), filter=2)
    res = {"slices": [0, 1], "reference": "float64 gridrec (oracle/gridrec_oracle.c)",
           "tolerance_rel_l2": 1e-3}
    for k, r in ((0, r1[:, :M0]), (1, r2[:, :M0])):
        res[f"slice{k}"] = {"rel_l2": ph.rel_l2(got[k], r), "max_abs": float(np.abs(got[k] - r).max()),
                            "peak": float(np.abs(r).max())}
    return res


def measure_slice_pipeline(G, sinos, th, n, a, dev, stream, peak):
    """CUDA-event timings of the steps around gridrec on 16 resident slices:
    ring suppression (20 rounds), shift + half padding, the half-padded
    reconstruction (2n-wide plan) and the entropy centre search (21 shifts)."""
    import torch
    S = min(16, sinos.shape[0])
    src = sinos[:S].float().contiguous()
    sl_bytes = a * n * 4

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1000.0 / reps

    out = {"slices": S}
    x = src.clone()
    t = timed(lambda: G.ring_removal(x, 1.0, 20, stream=stream), 3)
    per_round = 2 * sl_bytes * S * 20
    out["ring_removal"] = {
        "ms_per_slice": 1000.0 * t / S, "rounds": 20,
        "round_bytes_gbs": per_round / t / 1e9,
        "round_bytes_frac_of_hbm": per_round / t / 1e9 / peak,
        "note": "round bytes = one read + write of the sinogram per round (each round "
                "depends on every row of the previous one)"}
    t = timed(lambda: G.shift_pad(src, 1.5, stream=stream), 10)
    b = S * (sl_bytes + 2 * sl_bytes)
    out["shift_pad"] = {"ms_per_slice": 1000.0 * t / S, "gbs": b / t / 1e9,
                        "frac_of_hbm": b / t / 1e9 / peak}
    with G.Plan(2 * n, a, th, filter=G.FILTER_HANN, max_pairs=8,
                device=dev.index or 0) as p2:
        t = timed(lambda: G.reconstruct_padded(p2, src, 1.5, stream=stream), 3)
        out["reconstruct_padded"] = {"slices_per_s": S / t, "plan_width": 2 * n,
                                     "image": f"{n}x{n} crop of {p2.M0}^2"}
        shifts = np.arange(-5.0, 5.01, 0.5)
        G.center_search(p2, src[0], src[1], shifts, 0.0, 1.0, 10000, stream=stream)
        t0 = time.perf_counter()
        G.center_search(p2, src[0], src[1], shifts, 0.0, 1.0, 10000, stream=stream)
        tc = time.perf_counter() - t0
        out["center_search"] = {"ms": 1000.0 * tc, "candidates": len(shifts),
                                "ms_per_candidate": 1000.0 * tc / len(shifts),
                                "timing": "host wall clock (the call synchronises)"}
        p2.device_status()
    # FBP comparator on 2 of the slices (n^2 x angles work per slice)
    fb = G.FBP(n, a, th, max_slices=2, device=dev.index or 0)
    t = timed(lambda: fb.reconstruct(src[:2], stream=stream), 2)
    out["fbp_comparator"] = {"slices_per_s": 2 / t, "ms_per_slice": 1000.0 * t / 2}
    fb.close()
    # cross-correlation axis search: two n x 512 projections, 41 x 5 translations
    tpl = src[0, :512].contiguous()
    roi = (n // 8, n - n // 8 - 1, 64, 447)
    troi = tpl[roi[2]:roi[3] + 1, roi[0]:roi[1] + 1].contiguous()
    t0 = time.perf_counter()
    G.xcorr_scores(troi, src[1, :512].contiguous(), roi, -20.0, -2.0, 1.0, 1.0, 41, 5,
                   stream=stream)
    out["xcorr_search"] = {"ms": 1000.0 * (time.perf_counter() - t0), "translations": 205,
                           "image": f"{n}x512", "roi": list(roi),
                           "timing": "host wall clock (the call synchronises)"}
    del x, src
    return out


def measure_single_pair(G, sinos, th, n, a, dev, stream):
    """The reference's own call pattern: one slice pair per call.  Device time of
    gr_reconstruct_pair on resident buffers (a one-pair plan, CUDA events over 20
    calls, with its stage split), and host-to-host time of GridRec.reconstruct()
    -- the GridRec call surface over gr_reconstruct_pair_host -- on the caller's
    pageable float32 arrays (wall clock over 10 calls; each call synchronises)."""
    import torch
    if sinos.dtype != torch.float32:
        return None
    s1, s2 = sinos[0].contiguous(), sinos[1].contiguous()
    with G.Plan(n, a, th, filter=G.FILTER_HANN, max_pairs=1, device=dev.index or 0) as plan:
        o = torch.empty((2, plan.M0, plan.M0), device=dev)
        for _ in range(3):
            plan.reconstruct_pair(s1, s2, o[0], o[1], stream=stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(20):
            plan.reconstruct_pair(s1, s2, o[0], o[1], stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        dev_us = e0.elapsed_time(e1) / 20 * 1000.0
        plan.set_timing(True)
        for _ in range(10):
            plan.reconstruct_pair(s1, s2, o[0], o[1], stream=stream)
        st, nch = plan.stage_times()
        plan.set_timing(False)
        kernel = plan.grid_kernel(1)
    gr = G.GridRec()
    gr.setSinogramDimensions(n, a)
    gr.setThetaList(np.asarray(th, np.float32), a)
    gr.setFilter(G.FILTER_HANN)
    gr.setGPUDeviceID(dev.index or 0)
    gr.init()
    h1, h2 = s1.cpu().numpy(), s2.cpu().numpy()
    r1 = np.zeros((n, n), np.float32)
    r2 = np.zeros((n, n), np.float32)
    gr.setSinoAndReconBuffers(1, h1, r1)
    gr.setSinoAndReconBuffers(2, h2, r2)
    for _ in range(2):
        gr.reconstruct()
    t0 = time.perf_counter()
    for _ in range(10):
        gr.reconstruct()
    h2h_ms = (time.perf_counter() - t0) / 10 * 1000.0
    gr.destroy()
    return {"device_us_per_pair": dev_us,
            "stages_us": {k: 1000.0 * v / max(nch, 1) for k, v in st.items()},
            "grid_kernel": kernel,
            "host_to_host_ms_per_call": h2h_ms,
            "host_bytes_per_call": {"in": 2 * a * n * 4, "out": 2 * n * n * 4},
            "call": "GridRec.setSinoAndReconBuffers(1|2, sinogram, reconstruction); reconstruct() "
                    "on pageable float32 arrays (gr_reconstruct_pair_host)",
            "note": "stage times are taken with events between the stages (eager); the phase "
                    "stage is host time when its ramps are cached"}


def measure_learned(sinos, th, n, a, dev, stream, args, centers_d):
    """The learned narrow-kernel path on the same resident slices, one row per narrow
    width (PSWF C = 4 and 5, networks projects_b200/correction_c4.npy and _c5.npy):
    narrow gridrec alone and narrow + the fused correction network, timed with CUDA
    events; their relative L2 against full-width gridrec on two held-out slices decides
    the fallback (tolerance 1e-3), as LearnedGridrec does.  The network's own cost is
    the fused inference kernel (gr_cnn_infer) on S resident normalised images, with its
    fractions of the HBM roof (x read, y written: 8 bytes per pixel) and of the
    sustained BF16 tensor roof (5184 useful FLOP per pixel: 2 (9 x 16 + 9 x 16 x 16 +
    16 x 9))."""
    import torch

    from projects_b200 import learned as Lrn
    if sinos.dtype != torch.float32:
        return None
    S = min(64, sinos.shape[0])
    x = sinos[:S]
    c = centers_d[:S]

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1000.0 / reps

    rows, cnn = [], None
    for C in (4.0, 5.0):
        lg = Lrn.LearnedGridrec(n, a, th, max_pairs=args.max_pairs, device=dev.index or 0,
                                pswf_c=C)
        raw = torch.empty((S, lg.M0, lg.M0), device=dev)
        t_narrow = timed(lambda: lg.narrow.reconstruct_batch(x, raw, centers=c, stream=stream))
        t_learned = timed(lambda: lg.corrected(x, centers=c, stream=stream))
        if cnn is None:
            xn = (raw / Lrn.LearnedGridrec.scales(raw)).contiguous()
            t_cnn = timed(lambda: lg.net.infer(xn, stream=stream), reps=5) / S
            lg.net.infer_status(stream)
            px = lg.M0 * lg.M0
            hbm, _ = peaks()
            tf = bf16_sustained_tflops()
            cnn = {"kernel": "cnn_fused_kernel (conv1, conv2, conv3's partials as tcgen05 MMAs)",
                   "us_per_slice": t_cnn * 1e6,
                   "hbm_frac": 8.0 * px / t_cnn / (hbm * 1e9),
                   "bf16_sustained_frac": 5184.0 * px / t_cnn / (tf * 1e12),
                   "bound": "shared-memory bandwidth: every N = 16 MMA reads a 4 KB A tile "
                            "(54 conv2 MMAs per 8 x 64 tile)"}
            del xn
        _, info = lg.reconstruct_batch(x[:4], centers=c[:4], stream=stream)
        ref = torch.empty((2, lg.M0, lg.M0), device=dev)
        lg.full.reconstruct_batch(x[:2], ref, centers=c[:2], stream=stream)
        e_narrow = float(torch.linalg.vector_norm(raw[:2] - ref) / torch.linalg.vector_norm(ref))
        rows.append({"pswf_c": C, "narrow_slices_per_s": S / t_narrow,
                     "narrow_plus_cnn_slices_per_s": S / t_learned,
                     "held_out_rel_l2_vs_full_width": {"narrow": e_narrow,
                                                       "narrow_plus_cnn": info["held_out_rel_l2"]},
                     "fallback_to_full_width": info["fallback"]})
        del raw, ref
        lg.close()
    return {"widths": rows, "cnn": cnn, "tolerance": 1e-3,
            "network": "3-layer 16-channel 3x3 residual CNN, BF16 tensor-core layers with FP32 "
                       "accumulators, trained on 4096 slices of 1024 x 900 per narrow width "
                       "(projects_b200/train_correction.py)"}


# ------------------------------------------------------------------ arms

def run_reference(args, rank):
    if rank != 0:
        return
    per_step = []
    for i in range(args.warmup + args.steps):
        v, info = cpu_reference(args.n_det, args.n_ang, 0, steps=1)
        if i >= args.warmup:
            per_step.append((v, info))
    pairs = sum(i["pairs"] for _, i in per_step)
    wall = sum(i["wall_s"] for _, i in per_step)
    value = 2.0 * pairs / wall
    info = per_step[0][1]
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * wall / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"reference CPU GridRec (FP32, NR FFT), {args.n_det} det x "
                   f"{args.n_ang} angles, Hann; each step = one slice pair per host thread",
                   "n_det": args.n_det, "n_ang": args.n_ang},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": info["cores"],
                         "kind": info["kind"],
                         "sample": f"{args.steps} steps x {info['cores']} threads x 1 pair"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def run_b200(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from projects_b200 import gridrec as G
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    S, n, a = args.slices, args.n_det, args.n_ang
    th, sinos, centers = make_sinograms(S, n, a, rank_first_seed(rank, S), dev)
    tdt = {"f32": torch.float32, "f16": torch.float16, "bf16": torch.bfloat16}[args.dtype]
    if tdt != torch.float32:
        sinos = sinos.to(tdt)
    in_bytes = sinos.element_size()
    plan = G.Plan(n, a, th, filter=G.FILTER_HANN, max_pairs=args.max_pairs, device=local_rank)
    tuning = plan.autotune() if not args.no_autotune else plan.tuning()
    outs = torch.empty((S, plan.M0, n), dtype=torch.float32, device=dev)
    centers_d = torch.from_numpy(centers).to(dev)
    stream = torch.cuda.current_stream()

    def step():
        plan.reconstruct_batch(sinos, outs, centers=centers_d, stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # the whole step (all chunks of the batch) as one CUDA graph, replayed per step
    graph = plan.capture_batch(sinos, outs, centers=centers_d)
    graph.launch(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    with ClockSampler(local_rank) as clk:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            graph.launch(stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        elapsed = ev0.elapsed_time(ev1) / 1000.0
        # per-stage CUDA events (eager launches of the same step) for the roofline
        stage_steps = min(args.steps, 8)
        plan.set_timing(True)
        t0 = time.perf_counter()
        for _ in range(stage_steps):
            step()
        stage_ms, chunks = plan.stage_times()
        stage_wall = time.perf_counter() - t0
        plan.set_timing(False)
    launches = graph.launches() * args.steps
    graph.close()
    if world > 1:
        dist.barrier()
    elapsed = max_over_ranks(elapsed, dev, world)
    value = S * args.steps * world / elapsed

    # roofline of the dominant kernel
    bpp = algorithmic_bytes_per_pair(n, a, plan.pdim, plan.M, plan.M0, in_bytes)
    pairs_timed = stage_steps * ((S + 1) // 2)
    dominant = max(stage_ms, key=stage_ms.get)
    n_launch = chunks
    bytes_total = bpp[dominant] * pairs_timed
    achieved = bytes_total / (stage_ms[dominant] / 1000.0) / 1e9
    peak, peak_src = peaks()
    traffic = traffic_from_profile(dominant, min(args.max_pairs, (S + 1) // 2), n, a)
    traffic_note = ("ncu DRAM read + write of one launch (profiles/traffic_%dx%d.txt)" % (n, a))
    gk = plan.grid_kernel(args.max_pairs)
    if dominant == "grid" and gk == "wide32":
        traffic_note += ("; includes the 32-pair kernel's table indices (24 bytes per sample "
                         "and 4x8 sub-tile, read once per launch for its 32 pairs)")
    elif dominant == "grid" and gk == "wide":
        traffic_note += ("; includes the 16-pair kernel's precomputed weights (48 bytes per "
                         "sample and 4x8 sub-tile, read once per launch for its 16 pairs)")
    per_launch_bytes = bytes_total / max(n_launch, 1)
    stages = {k: {"ms_per_pair": v / pairs_timed,
                  "gbs": bpp[k] * pairs_timed / max(v / 1000.0, 1e-12) / 1e9}
              for k, v in stage_ms.items()}
    model_bytes_slice = (bpp["spectra"] + bpp["grid"] + bpp["cols"] + bpp["rows_deapod"]) / 2
    # the staged byte model of the task description: sinogram in, spectrum out/in,
    # H out, 2-D IFFT as 4 passes over H, H in, images out (per slice)
    survey_model = (2 * a * n * in_bytes + 2 * a * (plan.pdim // 2) * 8 * 2 + plan.M ** 2 * 8
                    + 4 * plan.M ** 2 * 8 + plan.M ** 2 * 8 + 2 * plan.M0 ** 2 * 4) / 2

    # end to end through the host-buffer entry point
    e2e = None
    if not args.no_e2e:
        with gpu_local_cpus(local_rank) as host_node:
            h_in = torch.empty(sinos.shape, dtype=sinos.dtype).pin_memory()
            h_out = torch.empty(outs.shape, dtype=torch.float32).pin_memory()
        h_in.copy_(sinos.cpu())
        # the host path is bound by the PCIe links: its own plan streams smaller chunks,
        # so that less of the first copy-in and the last copy-out is left without overlap
        plan_h = G.Plan(n, a, th, filter=G.FILTER_HANN, max_pairs=args.e2e_max_pairs,
                        device=local_rank)
        if not args.no_autotune:
            plan_h.autotune()
        plan_h.reconstruct_host(h_in, h_out, centers=centers, stream=int(stream.cuda_stream))
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            plan_h.reconstruct_host(h_in, h_out, centers=centers, stream=int(stream.cuda_stream))
            float(h_out[0, plan_h.M0 // 2, plan_h.M0 // 2])   # read the result on the host
        te = max_over_ranks(time.perf_counter() - t0, dev, world)
        e2e = {"value": S * args.e2e_steps * world / te, "unit": UNIT,
               "h2d_bytes_per_step": int(h_in.numel() * h_in.element_size()),
               "d2h_bytes_per_step": int(h_out.numel() * h_out.element_size()),
               "steps": args.e2e_steps, "path": "gr_reconstruct_host, pinned host buffers",
               "pairs_per_chunk": args.e2e_max_pairs,
               "grid_kernel": plan_h.grid_kernel(args.e2e_max_pairs),
               "host_buffers_on_cpus": host_node.cpus}
        plan_h.close()
        del h_in, h_out

    learned = None
    if rank == 0 and not args.no_pipeline:
        learned = measure_learned(sinos, th, n, a, dev, stream, args, centers_d)

    pipe = single = None
    if rank == 0 and not args.no_pipeline:
        pipe = measure_slice_pipeline(G, sinos, th, n, a, dev, stream, peaks()[0])
        single = measure_single_pair(G, sinos, th, n, a, dev, stream)

    # BASELINE configs 3 and 5 on the same box (one GPU): the uneven batch (one graph
    # launch per step, raw u16 / f32 / f16 storage) and 128 slices of the streaming volume
    uneven = stream_cfg = uneven_checks = None
    if world == 1 and not args.no_configs:
        uneven, _, _, uneven_checks = measure_uneven(args, rank, world, local_rank, steps=2)
        stream_cfg, _ = measure_stream(args, rank, world, local_rank, total=128)

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the CPU leg: the oracle checks two of the timed images, then the reference's
        # own CPU GridRec is timed on the host cores
        parity = parity_check(sinos, outs, centers, th, plan.M0)
        if uneven_checks is not None:
            uneven["float64_check"] = uneven_float64_check(uneven_checks)
        v, info = cpu_reference(n, a, args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": info["cores"], "kind": info["kind"],
               "sample": f"{info['pairs']} slice pairs of {n}x{a} (Hann) over "
                         f"{info['wall_s']:.1f} s on {info['cores']} host threads"}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"f32": "f32", "f16": "f16 storage, f32 compute",
                      "bf16": "bf16 storage, f32 compute"}[args.dtype],
            "data": "synthetic (seeded random-ellipse phantoms, Poisson 1e4 photons)",
            "config": {"workload": f"plain full-width gridrec (C=6, L={plan.L:.3f}), {S} slices "
                                   f"of {n} det x {a} angles per step, Hann, per-slice centres "
                                   f"{n // 2}+U[-2,2], output {plan.M0}^2 in {n}-stride f32",
                       "n_det": n, "n_ang": a, "slices_per_step": S,
                       "pairs_per_launch": args.max_pairs, "grid_kernel": gk,
                       "parallelism": f"slices x{world}",
                       "launch": f"one CUDA graph per step ({launches // args.steps} kernels); "
                                 f"stage times from {stage_steps} eager steps with events",
                       "tuning": tuning,
                       "l2": f"inputs larger than L2 ({S * a * n * in_bytes / 1e9:.1f} GB/step)"},
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_src,
                         "traffic": traffic, "traffic_note": traffic_note,
                         "algorithmic_bytes_per_launch": per_launch_bytes},
            "stages": stages,
            "pipeline": {"algorithmic_bytes_per_slice": model_bytes_slice,
                         "frac_of_hbm": model_bytes_slice * value / world / 1e9 / peak,
                         "survey_staged_model_bytes_per_slice": survey_model,
                         "survey_model_frac_of_hbm": survey_model * value / world / 1e9 / peak},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "e2e": e2e,
            "cpu_baseline": cpu,
            "parity": parity,
            "slice_pipeline": pipe,
            "single_pair": single,
            "learned": learned,
            "uneven": uneven,
            "stream": stream_cfg,
        }
        print(json.dumps(out), flush=True)
    plan.close()


UNEVEN_SHAPES = ((1024, 720, 256), (2048, 1500, 171), (4096, 3000, 85))


def measure_uneven(args, rank, world, local_rank, steps):
    """512 slices of three shapes (3:2:1), raw uint16 counts with per-slice flat/dark
    rows fused on load, reconstructed by one CUDA-graph launch per step; plus the
    same slices pre-normalised and stored as f32 and as f16.  Returns (result,
    clocks, launches, checks); checks holds the first 1024 x 720 pair's f32
    sinograms and its images from the three paths, for the float64 check."""
    import torch
    import torch.distributed as dist

    from projects_b200 import gridrec as G
    from projects_b200 import phantom as ph
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream()
    groups = []
    seed0 = rank * 100000
    for n, a, S in UNEVEN_SHAPES:
        th = ph.angles_deg(a)
        raw = torch.empty((S, a, n), dtype=torch.int16, device=dev)
        flat = torch.empty((S, n), dtype=torch.float32, device=dev)
        dark = torch.empty((S, n), dtype=torch.float32, device=dev)
        centers = np.zeros(S, np.float32)
        for i in range(S):
            r, f, d, c = ph.random_ellipse_raw(seed0 + n + i, n, a, dev)
            raw[i].copy_(r)
            flat[i].copy_(f)
            dark[i].copy_(d)
            centers[i] = c
        plan = G.Plan(n, a, th, filter=G.FILTER_HANN, max_pairs=32, device=local_rank)
        tuning = plan.autotune() if not args.no_autotune else plan.tuning()
        outs = torch.empty((S, plan.M0, plan.M0), dtype=torch.float32, device=dev)
        # the same slices normalised once (log, as the fused load) for the f32/f16 variants
        v = raw.to(torch.int32).remainder(65536).to(torch.float32) - dark[:, None, :]
        rr = (flat - dark)[:, None, :] / v
        norm = torch.where((v > 0) & (rr > 0), torch.log(rr), torch.zeros_like(v))
        groups.append({"n": n, "a": a, "S": S, "th": th, "plan": plan, "tuning": tuning,
                       "raw": raw, "flat": flat, "dark": dark, "centers": centers,
                       "centers_d": torch.from_numpy(centers).to(dev), "outs": outs,
                       "f32": norm.contiguous(), "f16": norm.half().contiguous()})
        del v, rr, norm

    def graph_for(kind):
        items = []
        for g in groups:
            p = g["plan"]
            if kind == "raw":
                b = p.batch_desc(g["raw"], g["outs"], centers=g["centers_d"], flat=g["flat"],
                                 dark=g["dark"], dtype=G.DTYPE_U16_RAW)
            else:
                b = p.batch_desc(g[kind], g["outs"], centers=g["centers_d"])
            items.append((p, b))
        return G.Graph(items)

    def timed(graph):
        for _ in range(max(args.warmup, 1)):
            graph.launch(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            graph.launch(stream)
        e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1) / 1000.0, dev, world)

    total = sum(g["S"] for g in groups)
    g_raw = graph_for("raw")
    with ClockSampler(local_rank) as clk:
        t_raw = timed(g_raw)
    launches = g_raw.launches() * steps
    g_raw.close()
    ref = [g["outs"][:4].clone() for g in groups]  # raw-path images of 4 slices per shape
    g0 = groups[0]
    checks = {"n": g0["n"], "a": g0["a"], "th": g0["th"], "centers": g0["centers"][:2].copy(),
              "sinos": g0["f32"][:2].cpu().numpy(), "raw": ref[0][:2].cpu().numpy()}
    res = {"raw_u16": {"slices_per_s": total * steps * world / t_raw}}
    for kind in ("f32", "f16"):
        gk = graph_for(kind)
        t = timed(gk)
        gk.close()
        errs = {}
        for g, r in zip(groups, ref):
            o = g["outs"][:4]
            errs[f"{g['n']}x{g['a']}"] = float(torch.linalg.vector_norm(o - r)
                                             / torch.linalg.vector_norm(r))
        res[kind] = {"slices_per_s": total * steps * world / t,
                     "rel_l2_vs_raw_path_images": errs}
        checks[kind] = groups[0]["outs"][:2].cpu().numpy()
    result = {
        "value": total * steps * world / t_raw, "unit": UNIT, "steps": steps,
        "ms_per_step": 1000.0 * t_raw / steps,
        "workload": "uneven batch: " + ", ".join(
            f"{g['S']} x {g['n']} det x {g['a']} angles" for g in groups) +
            "; raw uint16 with per-slice flat/dark fused on load (log); Hann; per-slice "
            "centres; one CUDA-graph launch of all three shapes per step",
        "slices_per_step": total,
        "grid_kernels": {f"{g['n']}x{g['a']}": g["plan"].grid_kernel() for g in groups},
        "tuning": {f"{g['n']}x{g['a']}": g["tuning"] for g in groups},
        "storage_variants": res,
        "l2": f"inputs larger than L2 ({sum(g['raw'].numel() * 2 for g in groups) / 1e9:.1f} "
              "GB/step)"}
    for g in groups:
        g["plan"].close()
    del groups
    torch.cuda.empty_cache()
    return result, clk.summary(), launches, checks


def uneven_float64_check(checks):
    """relL2 of the first 1024 x 720 pair's images from the raw-u16, f32 and f16 paths
    against float64 gridrec of the f32-normalised sinograms (the oracle as the checker)."""
    from oracle import oracle as O
    from projects_b200 import phantom as ph
    s, c = checks["sinos"], checks["centers"]
    r1, r2 = O.port_gridrec_pair(s[0], s[1], checks["th"], center1=float(c[0]),
                                 center2=float(c[1]), filter=2)
    M0 = checks["raw"].shape[1]
    out = {}
    for kind in ("raw", "f32", "f16"):
        g = checks[kind]
        out[kind] = max(ph.rel_l2(g[0], r1[:, :M0]), ph.rel_l2(g[1], r2[:, :M0]))
    return {"pair": f"first {checks['n']}x{checks['a']} pair", "worst_rel_l2": out,
            "reference": "float64 gridrec of the f32-normalised sinograms"}


def run_uneven(args, rank, world, local_rank):
    """--config uneven: the uneven batch as its own JSON line."""
    import torch
    torch.cuda.set_device(local_rank)
    steps = max(1, min(args.steps, 10))
    result, clocks, launches, checks = measure_uneven(args, rank, world, local_rank, steps)
    if rank == 0:
        out = {
            "metric": METRIC, "value": result["value"], "unit": UNIT,
            "n_gpus": world, "steps": steps, "warmup": args.warmup,
            "ms_per_step": result["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u16 raw in, f32 compute",
            "data": "synthetic (seeded random-ellipse phantoms, Poisson counts, per-slice "
                    "flat/dark rows)",
            "config": {"workload": result["workload"], "slices_per_step": result["slices_per_step"],
                       "parallelism": f"slices x{world}", "tuning": result["tuning"],
                       "grid_kernels": result["grid_kernels"], "l2": result["l2"]},
            "gpu_launches": launches,
            "storage_variants": result["storage_variants"],
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            out["float64_check"] = uneven_float64_check(checks)
        print(json.dumps(out), flush=True)


def measure_stream(args, rank, world, local_rank, total, ring=64):
    """Streaming volume: 4096 x 3000 raw uint16 slices with per-slice flat/dark rows,
    streamed from pinned host memory through gr_reconstruct_host (double-buffered
    chunks of 8 pairs, H2D and D2H on their own streams beside the kernels), the
    4095^2 float32 images streamed back into pinned host memory.  A host ring of
    `ring` slices is cycled to move `total` slices; kernel-only slices/s is measured
    on the same slices resident in HBM."""
    import torch
    import torch.distributed as dist

    from projects_b200 import gridrec as G
    from projects_b200 import phantom as ph
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream()
    n, a, K = 4096, 3000, ring
    total = max(K, (total // K) * K)
    th = ph.angles_deg(a)
    raw = torch.empty((K, a, n), dtype=torch.int16, device=dev)
    flat = torch.empty((K, n), dtype=torch.float32, device=dev)
    dark = torch.empty((K, n), dtype=torch.float32, device=dev)
    for i in range(K):
        r, f, d, _ = ph.random_ellipse_raw(rank * 100000 + i, n, a, dev)
        raw[i].copy_(r)
        flat[i].copy_(f)
        dark[i].copy_(d)
    plan = G.Plan(n, a, th, filter=G.FILTER_HANN, max_pairs=8, device=local_rank)
    tuning = plan.autotune() if not args.no_autotune else plan.tuning()
    outs = torch.empty((K, plan.M0, plan.M0), dtype=torch.float32, device=dev)
    # kernel-only: resident in HBM
    for _ in range(2):
        plan.reconstruct_batch(raw, outs, flat=flat, dark=dark, dtype=G.DTYPE_U16_RAW,
                               stream=stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(3):
        plan.reconstruct_batch(raw, outs, flat=flat, dark=dark, dtype=G.DTYPE_U16_RAW,
                               stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    kernel_only = 3 * K / (e0.elapsed_time(e1) / 1000.0)
    with gpu_local_cpus(local_rank) as host_node:
        h_in = torch.empty(raw.shape, dtype=torch.int16).pin_memory()
        h_out = torch.empty(outs.shape, dtype=torch.float32).pin_memory()
    h_in.copy_(raw.cpu())
    h_flat, h_dark = flat.cpu().numpy(), dark.cpu().numpy()
    del raw, outs
    torch.cuda.empty_cache()
    plan.reconstruct_host(h_in, h_out, flat=h_flat, dark=h_dark, dtype=G.DTYPE_U16_RAW,
                          stream=int(stream.cuda_stream))
    if world > 1:
        dist.barrier()
    with ClockSampler(local_rank) as clk:
        t0 = time.perf_counter()
        for _ in range(total // K):
            plan.reconstruct_host(h_in, h_out, flat=h_flat, dark=h_dark, dtype=G.DTYPE_U16_RAW,
                                  stream=int(stream.cuda_stream))
            float(h_out[K - 1, plan.M0 // 2, plan.M0 // 2])
        te = time.perf_counter() - t0
    te = max_over_ranks(te, dev, world)
    in_b = int(h_in.numel() * 2) * (total // K)
    out_b = int(h_out.numel() * 4) * (total // K)
    result = {
        "value": total * world / te, "unit": UNIT, "slices": total, "ring_slices": K,
        "ms_per_ring": 1000.0 * te / (total // K),
        "workload": f"streaming volume: {total} slices of {n} det x {a} angles raw uint16 from "
                    f"pinned host memory, images {plan.M0}^2 f32 streamed back (host ring of {K} "
                    f"slices cycled)",
        "e2e": {"value": total * world / te, "unit": UNIT,
                "h2d_bytes_per_step": in_b // (total // K),
                "d2h_bytes_per_step": out_b // (total // K),
                "path": "gr_reconstruct_host, double-buffered, separate H2D/D2H streams",
                "host_buffers_on_cpus": host_node.cpus},
        "kernel_only_slices_per_s": kernel_only,
        "pcie_gbs": {"h2d": in_b / te / 1e9, "d2h": out_b / te / 1e9},
        "tuning": tuning,
        "path": "plain gridrec (the learned path falls back to it)"}
    plan.close()
    del h_in, h_out
    return result, clk.summary()


def run_stream(args, rank, world, local_rank):
    """--config stream: the streaming volume as its own JSON line."""
    import torch
    torch.cuda.set_device(local_rank)
    result, clocks = measure_stream(args, rank, world, local_rank, args.stream_slices)
    if rank == 0:
        K = result["ring_slices"]
        steps = result["slices"] // K
        out = {
            "metric": METRIC, "value": result["value"], "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": 1, "ms_per_step": result["ms_per_ring"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u16 raw in, f32 compute, f32 out",
            "data": "synthetic (seeded random-ellipse phantoms, Poisson counts, per-slice "
                    "flat/dark rows)",
            "config": {"workload": result["workload"], "slices": result["slices"],
                       "parallelism": f"slices x{world}", "tuning": result["tuning"],
                       "path": result["path"]},
            "e2e": result["e2e"],
            "kernel_only_slices_per_s": result["kernel_only_slices_per_s"],
            "pcie_gbs": result["pcie_gbs"],
            "clocks": clocks,
        }
        print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import datetime

    import torch.distributed as dist
    if world > 1:
        import torch
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.config == "uneven":
            run_uneven(args, rank, world, local_rank)
        elif args.config == "stream":
            run_stream(args, rank, world, local_rank)
        else:
            run_b200(args, rank, world, local_rank)
    finally:
        if world > 1:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
