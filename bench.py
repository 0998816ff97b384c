#!/usr/bin/env python3
"""Benchmark: two-stage V-BM3D on 1920x1080 x 30 frames (GRAYS float32).

Workload (the reference's V-BM3D recipe, README.md:44-53): vbasic =
BM3Dv2(src, radius=2) then vfinal = BM3Dv2(src, ref=vbasic, radius=2), sigma 5,
block_step 8, bm_range 9, ps_num 2, ps_range 4, extractor_exp 6, on a seeded
synthetic clip (band-limited texture moving by integer steps in [-3, 3] px,
AWGN 5/255). One step = the whole two-stage pass over the 30 frames.

  value  Mpix/s with the clip resident in HBM (device buffers in, out), all
         frames of each stage batched into one launch per kernel, block
         matching by learned proposals (--mode learned, the default; the
         proposer is first trained on the GPU from the exhaustive search)
  e2e    the same through bm3d_b200_clip_twostage_host from pinned host
         buffers: the host->device copy of the 30 frames and the
         device->host copy of the result are inside the timed region
  plain_gpu  the same clip with the exhaustive (reference) search, for the
         metric's learned-vs-plain ratio and PSNR delta

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU (torchrun): every rank denoises its own 30-frame clip (weak
scaling, no data-path collective); time = max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "vapoursynth-bm3dcuda_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "V-BM3D 1080p Mpix/s, learned+batched vs plain GPU at ≤0.05 dB PSNR loss"
UNIT = "Mpix/s"
W, H, FRAMES = 1920, 1080, 30
SETTINGS = dict(sigma=5.0, block_step=8, bm_range=9, radius=2, ps_num=2, ps_range=4,
                extractor_exp=6)
SSD_FLOP = 192  # 64 subtractions + 64 fused multiply-adds (2 FLOP) per candidate


def workload_config(frames: int) -> dict:
    return {
        "workload": f"V-BM3D two-stage (BM3Dv2 basic -> BM3Dv2 final), GRAYS float32 "
                    f"{W}x{H} x {frames} frames",
        "width": W, "height": H, "frames": frames, **SETTINGS,
        "l2": "inputs larger than L2 (249 MB clip per step)",
    }


def candidates_per_window(width: int, height: int, bs: int, bm_range: int, radius: int,
                          ps_num: int, ps_range: int) -> int:
    """Distance evaluations of the exhaustive reference algorithm for one
    window: exact clamped spatial counts, temporal windows at their nominal
    size ps_num * (2 ps_range + 1)^2 per neighbour frame."""
    xs = [min(x, width - 8) for x in range(0, width - 8 + bs, bs)]
    ys = [min(y, height - 8) for y in range(0, height - 8 + bs, bs)]
    cx = sum(min(x + bm_range, width - 8) - max(x - bm_range, 0) + 1 for x in xs)
    cy = sum(min(y + bm_range, height - 8) - max(y - bm_range, 0) + 1 for y in ys)
    spatial = cx * cy
    temporal = len(xs) * len(ys) * 2 * radius * ps_num * (2 * ps_range + 1) ** 2
    return spatial + temporal


# --------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples every 200 ms, each stamped with its arrival time so
    that only the samples taken inside the timed region count."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.rows = []
        self.thread = None

    def start(self):
        import threading
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-i", str(self.dev), "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return

        def reader():
            for line in self.proc.stdout:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    self.rows.append((time.perf_counter(), parts))

        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()

    def stop(self, t0: float | None = None, t1: float | None = None) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)
        rows = [r for t, r in self.rows
                if (t0 is None or t >= t0) and (t1 is None or t <= t1 + 0.25)]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------------------
# CPU baseline: the reference's own CPU implementation on the host cores
# --------------------------------------------------------------------------
def cpu_reference_sample(noisy: np.ndarray, seconds: float = 12.0, threads: int | None = None,
                         nframes: int | None = None):
    """Time the reference bm3dcpu (oracle/_ref, stock build) on a bounded
    sample of the two-stage workload: every thread denoises whole output
    frames (basic window + final window, radius 2) of the same clip.
    Falls back to the project's C restatement when the reference build is
    absent. nframes: sample size; if None, sized from a one-frame calibration
    to about `seconds`. Returns (Mpix/s, info dict)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle as O
    kind = "reference" if O.ref_available("stock") else "port"
    threads = threads or os.cpu_count() or 1
    r = SETTINGS["radius"]
    kw = {k: SETTINGS[k] for k in ("sigma", "block_step", "bm_range", "radius", "ps_num", "ps_range")}

    def one_frame(n: int):
        win = O.clip_window(noisy[:, None], n % noisy.shape[0], r)
        if kind == "reference":
            raw = O.ref_bm3d(win, kind="stock", **kw)
            # final stage with the basic estimate of the centre slot as ref
            est = raw[:, :, 0] / np.maximum(raw[:, :, 1], 1e-12)
            O.ref_bm3d(win, est.astype(np.float32), kind="stock", **kw)
        else:
            raw = O.port_bm3d(win, **kw)
            est = raw[:, :, 0] / np.maximum(raw[:, :, 1], 1e-12)
            O.port_bm3d(win, est.astype(np.float32), **kw)

    if nframes is None:
        t0 = time.perf_counter()
        one_frame(0)
        per_frame = time.perf_counter() - t0
        nframes = max(threads, int(seconds / per_frame) * threads)
        nframes = min(nframes, threads * 64)
    with ThreadPoolExecutor(max_workers=threads) as ex:
        t0 = time.perf_counter()
        list(ex.map(one_frame, range(nframes)))
        dt = time.perf_counter() - t0
    mpix = nframes * W * H / 1e6 / dt
    return mpix, {"cores": threads, "kind": kind,
                  "sample": f"{nframes} output frames of the {W}x{H} radius-2 two-stage workload "
                            f"(basic + final window each), {threads} threads, {dt:.1f} s"}


def reference_gpu_sample(frames: int = FRAMES, reps: int = 5) -> dict | None:
    """The reference's own CUDA kernel (source/kernel.cu, release flags
    --use_fast_math, built unchanged into oracle/_ref/) on this GPU:

      kernel  the bm3d kernel alone on device-resident 1080p radius-2 windows
              (basic, then final), CUDA events; Mpix/s = one output frame per
              basic + final window pair (the host VAggregate not counted)
      e2e     the plugin's own pipeline for the whole two-stage clip: worker
              threads, 4 GPU resources (fast=True), pinned staging, graph per
              frame (HtoD, memset, kernel, DtoH) and the host VAggregate

    None when the build or a CUDA device is missing."""
    from oracle import oracle as O
    if not O.refgpu_available("fast"):
        return None
    import torch
    if not torch.cuda.is_available():
        return None
    from bm3dcuda import synthetic as S
    lib = O.refgpu_lib("fast")
    r = SETTINGS["radius"]
    tw = 2 * r + 1
    stride = (W + 31) // 32 * 32
    noisy, _ = S.texture_clip(frames, H, W, seed=0)
    d_src = torch.zeros((2, tw, H, stride), dtype=torch.float32, device="cuda")
    d_src[0, :, :, :W] = torch.from_numpy(noisy[:tw]).cuda()
    d_src[1] = d_src[0]
    d_res = torch.zeros((tw, 2, H, stride), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    ext = float(2.0 ** SETTINGS["extractor_exp"])
    ms = {}
    for final in (0, 1):
        sig = O.scale_sigma(SETTINGS["sigma"], bool(final))

        def launch():
            d_res.zero_()
            O._refgpu_check(lib, lib.refgpu_kernel(
                d_res.data_ptr(), d_src.data_ptr(), W, H, stride, sig, SETTINGS["block_step"],
                SETTINGS["bm_range"], r, SETTINGS["ps_num"], SETTINGS["ps_range"], 0, 0.0, 0.0,
                final, ext, ctypes.c_void_p(stream.cuda_stream)), "refgpu_kernel")
        for _ in range(2):
            launch()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            launch()
        e1.record(stream)
        e1.synchronize()
        ms["final" if final else "basic"] = e0.elapsed_time(e1) / reps
    del d_src, d_res
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    _, secs = O.refgpu_twostage(noisy, sigma=SETTINGS["sigma"], block_step=SETTINGS["block_step"],
                                bm_range=SETTINGS["bm_range"], radius=r,
                                ps_num=SETTINGS["ps_num"], ps_range=SETTINGS["ps_range"],
                                extractor_exp=SETTINGS["extractor_exp"], resources=4,
                                kind="fast")
    wall = time.perf_counter() - t0
    return {
        "what": "the reference's source/kernel.cu compiled unchanged for sm_100a with its "
                "release flags (--use_fast_math), on this GPU",
        "kernel": {"value": W * H / 1e6 / ((ms["basic"] + ms["final"]) * 1e-3), "unit": UNIT,
                   "basic_window_ms": ms["basic"], "final_window_ms": ms["final"],
                   "note": "device-resident windows; zeroing of the accumulators included"},
        "e2e": {"value": frames * W * H / 1e6 / sum(secs), "unit": UNIT, "frames": frames,
                "stage_seconds": {"basic": secs[0], "vaggregate_basic": secs[1],
                                  "final": secs[2], "vaggregate_final": secs[3]},
                "wall_seconds": wall, "resources": 4, "threads": os.cpu_count(),
                "note": "plugin pipeline: graph per output frame (HtoD, memset, kernel, DtoH) "
                        "from pinned staging, host VAggregate, 4 resources (fast=True)"},
    }


def cpu_parity_sample(noisy: np.ndarray, basic: np.ndarray, out: np.ndarray, n: int) -> dict:
    """The checker beside the CPU baseline: output frame n of the GPU's plain
    (exhaustive) arm against the reference's bm3dcpu (exact-reciprocal build)
    on the same frames - the basic stage, and the final stage fed the GPU's
    basic estimate (the final stage matches on it, so both sides get the
    same one). Windows run on the host threads; VAggregate as the plugin."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle as O
    if not O.ref_available("exact"):
        return {"unavailable": "reference bm3dcpu build (oracle/_ref) missing"}
    r = SETTINGS["radius"]
    N = noisy.shape[0]
    kw = {k: SETTINGS[k] for k in ("sigma", "block_step", "bm_range", "ps_num", "ps_range")}
    wins = sorted({min(max(n + i, 0), N - 1) for i in range(-r, r + 1)})
    clip = noisy[:, None]

    def one(args_):
        w, final = args_
        return O.ref_bm3d(O.clip_window(clip, w, r),
                          O.clip_window(basic[:, None], w, r) if final else None,
                          radius=r, **kw)

    jobs = [(w, f) for f in (False, True) for w in wins]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as ex:
        raws = dict(zip(jobs, ex.map(one, jobs)))
    res = {"frame": n, "windows": wins, "seconds": time.perf_counter() - t0,
           "reference": "bm3dcpu (cpu_source/source.cpp), exact-reciprocal build",
           "note": "GPU arm pre-rounds its sums (extractor_exp 6), bm3dcpu does not"}
    for name, got, final in (("basic", basic, False), ("final", out, True)):
        idx = [min(max(n + i, 0), N - 1) for i in range(-r, r + 1)]
        want = O.port_vaggregate(np.stack([raws[(w, final)][0] for w in idx]), n, N)
        res[f"max_abs_{name}"] = float(np.abs(got[n] - want).max())
    return res


def run_reference_arm(args, rank: int, world: int):
    if rank != 0:
        return None
    from bm3dcuda import synthetic as S
    noisy, _ = S.texture_clip(8, H, W, seed=0)
    threads = os.cpu_count() or 1
    # one sample of `threads` frames (one per thread) per warm-up step; timed
    # steps sized so the whole run stays near 150 s of CPU time
    t0 = time.perf_counter()
    cpu_reference_sample(noisy, threads=threads, nframes=threads)
    per_round = time.perf_counter() - t0
    rounds = max(1, int(150.0 / max(per_round, 1e-3) / max(1, args.steps + args.warmup)))
    for _ in range(max(0, args.warmup - 1)):
        cpu_reference_sample(noisy, threads=threads, nframes=threads)
    vals, infos = [], []
    for _ in range(args.steps):
        v, info = cpu_reference_sample(noisy, threads=threads, nframes=threads * rounds)
        vals.append(v)
        infos.append(info)
    value = float(np.median(vals))
    ms_per_step = FRAMES * W * H / 1e6 / value * 1e3
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(FRAMES), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": infos[-1]["cores"],
                         "kind": infos[-1]["kind"], "sample": infos[-1]["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    try:
        line["reference_gpu"] = reference_gpu_sample()
    except Exception as exc:  # the CPU line stands on its own
        line["reference_gpu"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
    return line


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
def fp32_peak_tflops(torch) -> float:
    """Measured FP32 (SIMT) throughput: cuBLAS SGEMM 8192^3 with TF32 off."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, device="cuda")
    b = torch.randn(n, n, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    return 2 * n ** 3 / (best * 1e-3) / 1e12


def load_traffic() -> dict:
    """DRAM bytes per 30-window launch of each kernel, from the committed
    summary of one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum
    on the 16-window case, scaled by windows; the capture command is in the
    file)."""
    p = os.path.join(ROOT, "profiles", "dram_traffic_vbm3d_1080p.json")
    try:
        with open(p) as f:
            return json.load(f).get("kernels", {})
    except (OSError, ValueError):
        return {}


def load_peaks() -> dict:
    """HBM and dense BF16 peaks measured on this pool (MEASURED_PEAKS.json),
    else the pool's earlier fallback figures."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]),
                "source": "MEASURED_PEAKS.json (measured on this pool)"}
    except (OSError, ValueError, KeyError, TypeError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0,
                "source": "fallback: 6.65 TB/s, 1.59 PFLOP/s (earlier measurement on this pool; "
                          "MEASURED_PEAKS.json absent)"}


def train_proposer(prop, seed: int = 100):
    """The proposer used by the learned runs: trained on the GPU (the engine's
    own FP32 forward/backward kernels) by distillation from the exhaustive
    search on six config-1-style clips (moving piecewise scenes, 320x240 x 5
    frames, noise 10/255: 7200 reference blocks x 5 frames)."""
    from bm3dcuda import synthetic as S
    train = [S.moving_piecewise_clip(5, 240, 320, seed=seed + i)[0] for i in range(6)]
    t0 = time.perf_counter()
    losses = prop.fit(train, radius=SETTINGS["radius"], sigma=10.0, steps=300, lr=2e-3)
    return {"clips": "6 x moving piecewise 320x240x5, noise 10/255", "steps": 300,
            "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
            "seconds": time.perf_counter() - t0}


# filter transform arithmetic (bm3d_b200_clip_set_precision)
PRECISIONS = {"fp32": 0, "split-bf16": 1, "tc-f16": 2}


def run_our_arm(args, rank: int, world: int, dist):
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    from bm3dcuda.learned import Proposer
    L = _lib.lib()
    dev = torch.cuda.current_device()
    frames = args.frames

    noisy, clean = S.texture_clip(frames, H, W, seed=rank)
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    for i in range(3):
        p.sigma[i] = SETTINGS["sigma"]
        p.block_step[i] = SETTINGS["block_step"]
        p.bm_range[i] = SETTINGS["bm_range"]
        p.ps_num[i] = SETTINGS["ps_num"]
        p.ps_range[i] = SETTINGS["ps_range"]
    p.radius = SETTINGS["radius"]
    p.extractor_exp = SETTINGS["extractor_exp"]
    # h: the timed clip; h2: a second clip of the same configuration, so that
    # the end-to-end figure can keep two clips in flight (one computing while
    # the other's frames cross PCIe)
    h, h2 = ctypes.c_void_p(), ctypes.c_void_p()
    clips = [h] if args.profile else [h, h2]
    for c in clips:
        _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), W, H, 1, 0, 0, frames,
                                           ctypes.byref(p), dev))
        _lib.check(L.bm3d_b200_clip_set_precision(c, PRECISIONS[args.precision]))
    stride = L.bm3d_b200_clip_stride(h)
    ff = L.bm3d_b200_clip_frame_floats(h)
    host = np.zeros((frames, ff), np.float32)
    host.reshape(frames, H, stride)[:, :, :W] = noisy
    h_src = torch.from_numpy(host).pin_memory()
    h_dst = torch.empty_like(h_src).pin_memory()
    h_dst2 = torch.empty_like(h_src).pin_memory()
    d_src = h_src.cuda()
    d_basic = torch.empty_like(d_src)
    d_dst = torch.empty_like(d_src)
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    stream2 = torch.cuda.Stream()
    sp2 = ctypes.c_void_p(stream2.cuda_stream)

    prop = None
    training = None
    if args.mode == "learned":
        prop = Proposer(device=dev)
        training = train_proposer(prop)

    final_mode = {"search": 0, "basic-lists": 1, "basic-order": 2}[args.final_matching]

    def set_learned(on: bool):
        for c in clips:
            if on:
                _lib.check(L.bm3d_b200_clip_set_proposer(c, prop.handle, args.cells_spatial,
                                                         args.cells_temporal, args.fallback_tau))
                _lib.check(L.bm3d_b200_clip_set_final_matching(c, final_mode))
            else:
                _lib.check(L.bm3d_b200_clip_set_proposer(c, None, 1, 1, 0.0))

    def step_device():
        _lib.check(L.bm3d_b200_clip_twostage(h, d_src.data_ptr(), d_basic.data_ptr(),
                                             d_dst.data_ptr(), sp))

    def step_e2e():
        _lib.check(L.bm3d_b200_clip_twostage_host(h, h_src.data_ptr(), h_dst.data_ptr(), sp))

    # two clips in turn, each on its own stream, through the asynchronous
    # host-buffer entry point: step k copies its frames in, filters them and
    # copies the result out, while step k + 1's copies already run
    inflight = [(h, h_dst, sp), (h2, h_dst2, sp2)]
    turn = [0]

    def step_e2e_async():
        c, dst, s_ = inflight[turn[0] % 2]
        turn[0] += 1
        _lib.check(L.bm3d_b200_clip_twostage_host_async(c, h_src.data_ptr(), dst.data_ptr(), s_))

    def join_e2e():
        stream.wait_stream(stream2)

    if args.profile:
        set_learned(prop is not None)
        for _ in range(args.warmup + args.steps):
            step_device()
        torch.cuda.synchronize()
        L.bm3d_b200_clip_destroy(h)
        return None

    peak = fp32_peak_tflops(torch) if rank == 0 else 0.0

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps, finish=None):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        if finish is not None:
            finish()  # the timing stream waits for every stream the steps used
        e1.record(stream)
        barrier()
        ms = e0.elapsed_time(e1)
        if dist is not None:
            from bm3dcuda.distributed import max_over_ranks
            ms = max_over_ranks(ms, dist)
        return ms

    def repeated(fn, finish=None):
        """The timed region: exactly args.steps steps between barriers and
        device synchronisations, repeated back to back until the repeats
        cover at least args.min_timed_s seconds (so that the clock sampler
        sees the GPU under load); returns the median region time (ms) and the
        number of repeats."""
        regions = [timed(fn, args.steps, finish)]
        reps = min(64, max(1, int(np.ceil(args.min_timed_s * 1e3 / max(regions[0], 1e-3)))))
        if dist is not None:  # every rank runs the same number of collectives
            from bm3dcuda.distributed import max_over_ranks
            reps = int(max_over_ranks(float(reps), dist))
        for _ in range(reps - 1):
            regions.append(timed(fn, args.steps, finish))
        return float(np.median(regions)), len(regions)

    def measure_device(sampler=None):
        """Warm-up, then the device-resident timed regions with per-stage events."""
        for _ in range(args.warmup):
            step_device()
        torch.cuda.synchronize()
        if sampler is not None:
            sampler.start()
            time.sleep(0.5)  # nvidia-smi's first sample lands inside the timed region
        L.bm3d_b200_clip_stage_times(h, None, None, 1)
        L.bm3d_b200_clip_learned_stats(h, None, None, 1)
        L.bm3d_b200_clip_set_profiling(h, 1)
        t0 = time.perf_counter()
        ms, reps = repeated(step_device)
        t1 = time.perf_counter()
        L.bm3d_b200_clip_set_profiling(h, 0)
        stage_ms = (ctypes.c_double * _lib.NUM_STAGES)()
        stage_n = (ctypes.c_longlong * _lib.NUM_STAGES)()
        _lib.check(L.bm3d_b200_clip_stage_times(h, stage_ms, stage_n, 1))
        blocks, fell = ctypes.c_longlong(), ctypes.c_longlong()
        _lib.check(L.bm3d_b200_clip_learned_stats(h, ctypes.byref(blocks), ctypes.byref(fell), 1))
        clk = sampler.stop(t0, t1) if sampler is not None else None
        basic = d_basic.cpu().numpy().reshape(frames, H, stride)[:, :, :W]
        out = d_dst.cpu().numpy().reshape(frames, H, stride)[:, :, :W]
        # stage times and launches per repeat of the timed region
        return {"ms": ms, "reps": reps, "wall_s": t1 - t0,
                "stage_ms": [v / reps for v in stage_ms],
                "stage_n": [v // reps for v in stage_n], "clocks": clk,
                "psnr": S.psnr(out, clean), "blocks": blocks.value // reps,
                "fallbacks": fell.value // reps, "basic": basic, "out": out}

    clock_dev = (int(os.environ.get("CUDA_VISIBLE_DEVICES", str(dev)).split(",")[0])
                 if os.environ.get("CUDA_VISIBLE_DEVICES", "").isdigit() else dev)

    # plain GPU drop-in: the exhaustive search (reference algorithm), batched
    set_learned(False)
    plain = measure_device(None if prop is not None else ClockSampler(clock_dev))
    # learned + batched (headline when --mode learned)
    head = plain
    if prop is not None:
        set_learned(True)
        head = measure_device(ClockSampler(clock_dev))

    # end-to-end through the host-buffer entry points, headline configuration:
    # one call at a time (synchronous), then two clips in flight (asynchronous)
    for _ in range(max(1, args.warmup // 2)):
        step_e2e()
    ms_e2e_sync, _ = repeated(step_e2e)
    for _ in range(max(2, args.warmup)):
        step_e2e_async()
    join_e2e()
    torch.cuda.synchronize()
    ms_e2e, reps_e2e = repeated(step_e2e_async, join_e2e)
    torch.cuda.synchronize()
    for c in (h, h2):
        _lib.check(L.bm3d_b200_clip_status(c))
    out = h_dst.numpy().reshape(frames, H, stride)[:, :, :W]
    out2 = h_dst2.numpy().reshape(frames, H, stride)[:, :, :W]
    e2e_psnr = S.psnr(out, clean)
    e2e_same = bool(np.array_equal(out, out2))
    in_psnr = S.psnr(noisy, clean)
    L.bm3d_b200_clip_destroy(h)
    L.bm3d_b200_clip_destroy(h2)
    if prop is not None:
        prop.close()

    mpix_step = frames * W * H / 1e6
    value = world * mpix_step * args.steps / (head["ms"] * 1e-3)
    plain_value = world * mpix_step * args.steps / (plain["ms"] * 1e-3)
    e2e = world * mpix_step * args.steps / (ms_e2e * 1e-3)
    e2e_sync = world * mpix_step * args.steps / (ms_e2e_sync * 1e-3)
    if rank != 0:
        return None

    names = ["match", "filter", "aggregate", "propose", "match_final", "filter_final",
             "fallback"]

    def per_step(m):
        return {names[i]: float(m["stage_ms"][i]) / args.steps for i in range(_lib.NUM_STAGES)}

    def per_launch(m, i):
        n = m["stage_n"][i]
        return float(m["stage_ms"][i]) / n if n else None

    cand = candidates_per_window(W, H, SETTINGS["block_step"], SETTINGS["bm_range"],
                                 SETTINGS["radius"], SETTINGS["ps_num"], SETTINGS["ps_range"])
    nbx = len(range(0, W - 8 + SETTINGS["block_step"], SETTINGS["block_step"]))
    nby = len(range(0, H - 8 + SETTINGS["block_step"], SETTINGS["block_step"]))
    groups = nbx * nby * frames  # reference blocks (groups) of one launch over the clip
    r_ = SETTINGS["radius"]
    traffic = load_traffic()
    peaks = load_peaks()

    def entry(kernel, work, unit, ms, peak_, peak_src, basis, bound="fp32"):
        if ms is None:
            return None
        achieved = work / (ms * 1e-3) / 1e12 if unit != "GB/s" else work / (ms * 1e-3) / 1e9
        t = traffic.get(kernel)
        return {"kernel": kernel, "bound": bound, "achieved": achieved, "peak": peak_,
                "unit": unit, "frac": achieved / peak_ if peak_ else None,
                "traffic": t["bytes_per_launch"] if t else None,
                "algorithmic_work_per_launch": work, "avg_launch_ms": ms, "basis": basis,
                "peak_source": peak_src}

    fp32_src = ("measured live in this run: cuBLAS SGEMM 8192^3, TF32 off (MEASURED_PEAKS.json "
                "holds no FP32 figure)")
    kernels = {}
    if prop is not None:
        cells_nominal = ((SETTINGS["bm_range"] + 1) ** 2
                         + 2 * r_ * SETTINGS["ps_num"] * (SETTINGS["ps_range"] + 1) ** 2)
        scored = 4 * (args.cells_spatial + 2 * r_ * args.cells_temporal)
        ops = groups * (SSD_FLOP * scored + 48 * cells_nominal)
        kernels["learned_match_kernel"] = entry(
            "learned_match_kernel", ops, "TFLOP/s", per_launch(head, 0), peak, fp32_src,
            "executed work per launch: %d exact block distances per block (4 origins of %d "
            "spatial + %d x %d temporal kept cells) x 192 FLOP, plus %d ranked cells per block "
            "(nominal window sizes) x 48 integer operations (16 byte differences, 16 "
            "multiply-adds of 4-way dot products), over %d blocks; FP32 peak as the SIMT "
            "issue-rate bound" % (scored, args.cells_spatial, 2 * r_, args.cells_temporal,
                                  cells_nominal, groups))
        kernels["learned_match_kernel"]["exhaustive_equivalent"] = {
            "flop_per_launch": SSD_FLOP * cand * frames,
            "tflops": SSD_FLOP * cand * frames / (per_launch(head, 0) * 1e-3) / 1e12,
            "note": "the exhaustive search's distance FLOP for the same windows: pruning "
                    "counted as speed at equal work, not a roofline"}
        if args.final_matching == "basic-lists":
            kernels["rescore_kernel"] = entry(
                "rescore_kernel", groups * 8 * SSD_FLOP, "TFLOP/s", per_launch(head, 4), peak,
                fp32_src, "8 block distances x 192 FLOP per block")
        kernels["embed_umma_kernel"] = entry(
            "embed_umma_kernel", 2 * 4752 * (W // 2) * (H // 2) * frames, "TFLOP/s",
            per_launch(head, 3), peaks["bf16_tflops"], peaks["source"],
            "4752 MAC per half-resolution pixel, three 3x3 16-channel layers", bound="tensor")
    if args.precision == "tc-f16":
        fb, ff_ = "filter_tc_kernel<0>", "filter_tc_kernel<1>"
        kernels[fb] = entry(
            fb, groups * 131072, "TFLOP/s", per_launch(head, 1), peaks["bf16_tflops"],
            peaks["source"], "131,072 tensor FLOP per group (forward and inverse 2-D transforms "
            "of 8 patches as 64 x 64 FP16 MMAs); the group transforms and the scatter are SIMT",
            bound="tensor")
        kernels[ff_] = entry(
            ff_, groups * 196608, "TFLOP/s", per_launch(head, 5), peaks["bf16_tflops"],
            peaks["source"], "196,608 tensor FLOP per group (two forward 2-D transforms and "
            "the inverse)", bound="tensor")
    else:
        fb, ff_ = "filter_kernel<0,0,0>", "filter_kernel<1,0,0>"
        kernels[fb] = entry(
            fb, groups * 18240, "TFLOP/s", per_launch(head, 1), peak, fp32_src,
            "18,240 FLOP per group (3-D DCT forward + inverse, FFTW operation counts x 192 "
            "one-dimensional transforms)")
        kernels[ff_] = entry(
            ff_, groups * 26688, "TFLOP/s", per_launch(head, 5), peak, fp32_src,
            "26,688 FLOP per group (two forward 3-D DCTs + inverse)")
    kernels["aggregate_kernel"] = entry(
        "aggregate_kernel", 12 * W * H * frames, "GB/s", per_launch(head, 2),
        peaks["hbm_gbs"], peaks["source"],
        "12 B per pixel (weighted sum and corner weights read, output written)", bound="hbm")
    kernels["match_kernel<10,0>"] = entry(
        "match_kernel<10,0>", SSD_FLOP * cand * frames, "TFLOP/s", per_launch(plain, 0), peak,
        fp32_src, "exhaustive search (plain arm): 192 FLOP per candidate")
    kernels = {k: v for k, v in kernels.items() if v is not None}
    # the headline roofline: the kernel with the largest share of the headline step
    share = {}
    for k, i in (("learned_match_kernel", 0), ("rescore_kernel", 4), ("embed_umma_kernel", 3),
                 (fb, 1), (ff_, 5),
                 ("aggregate_kernel", 2)):
        if k in kernels:
            share[k] = float(head["stage_ms"][i])
    if prop is None:
        share["match_kernel<10,0>"] = float(head["stage_ms"][0])
    top = max(share, key=share.get)
    roofline = dict(kernels[top])
    roofline["share_of_step"] = share[top] / sum(head["stage_ms"])
    roofline["kernels"] = {k: v for k, v in kernels.items() if k != top}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {**workload_config(frames), "parallelism": f"replicas x{world}",
                   "filter_precision": args.precision,
                   "matching": ("learned proposals (cells %d spatial, %d temporal), fallback "
                                "tau %g, final stage: %s" % (
                                    args.cells_spatial, args.cells_temporal, args.fallback_tau,
                                    args.final_matching)) if prop is not None
                   else "exhaustive"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(frames * ff * 4),
                "d2h_bytes_per_step": int(frames * ff * 4),
                "ms_per_step": ms_e2e / args.steps,
                "api": "bm3d_b200_clip_twostage_host_async, two clips in turn on two streams "
                       "(pinned host buffers; every step copies its 30 frames in and its 30 "
                       "results out inside the timed region)",
                "outputs_of_both_clips_identical": e2e_same,
                "one_call_at_a_time": {"value": e2e_sync, "ms_per_step": ms_e2e_sync / args.steps,
                                       "api": "bm3d_b200_clip_twostage_host (synchronous)"}},
        "roofline": roofline,
        "gpu_launches": int(sum(head["stage_n"])),
        "stage_ms_per_step": per_step(head),
        "stage_launches": {names[i]: int(head["stage_n"][i]) for i in range(_lib.NUM_STAGES)},
        "quality": {"psnr_in_db": in_psnr, "psnr_out_db": head["psnr"],
                    "psnr_e2e_out_db": e2e_psnr},
        "clocks": head["clocks"],
        "timing": {"steps_per_region": args.steps, "regions": head["reps"],
                   "statistic": "median region", "timed_wall_s": head["wall_s"],
                   "e2e_regions": reps_e2e},
        "_plain_frames": (noisy, plain["basic"], plain["out"]),
    }
    if prop is not None:
        line["plain_gpu"] = {
            "value": plain_value, "unit": UNIT, "ms_per_step": plain["ms"] / args.steps,
            "psnr_out_db": plain["psnr"], "stage_ms_per_step": per_step(plain),
            "matching": "exhaustive (the reference algorithm, bit-exact lists)"}
        line["learned"] = {
            "speedup_vs_plain_gpu": value / plain_value,
            "psnr_delta_db": head["psnr"] - plain["psnr"],
            "fallback_fraction": head["fallbacks"] / max(1, head["blocks"]),
            "training": training}
    return line


# --------------------------------------------------------------------------
# further workloads (one JSON line each; --workload)
# --------------------------------------------------------------------------
def _device_timer(torch, fn, warmup: int, steps: int) -> float:
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def run_cbm3d(args) -> dict:
    """CBM3D (chroma=True) YUV444PS 1920x1080 x 16, radius 1, sigma [10, 7, 7],
    two-stage: FP32 transforms (the reference's factorisation) against the
    split-BF16 tensor-core transforms. Accuracy against the FP64 oracle on a
    256x192 x 4 crop of the same scene (basic and final stage accumulators,
    the GPU's match lists injected into the oracle)."""
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    from oracle import oracle as O
    L = _lib.lib()
    N, Hc, Wc, r = 16, 1080, 1920, 1
    sig = [10.0, 7.0, 7.0]

    def make(w, h, n, prec):
        p = _lib.Params()
        L.bm3d_b200_params_default(ctypes.byref(p))
        for i in range(3):
            p.sigma[i] = sig[i]
        p.radius = r
        p.chroma = 1
        c = ctypes.c_void_p()
        _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), w, h, 3, 0, 0, n, ctypes.byref(p), 0))
        _lib.check(L.bm3d_b200_clip_set_precision(c, prec))
        return c

    noisy, clean = S.chroma_clip(N, Hc, Wc, seed=3)
    res = {}
    for prec, name in ((0, "fp32"), (1, "split_bf16")):
        c = make(Wc, Hc, N, prec)
        stride = L.bm3d_b200_clip_stride(c)
        hbuf = np.zeros((N, 3, Hc, stride), np.float32)
        hbuf[..., :Wc] = noisy
        d_src = torch.from_numpy(hbuf).cuda()
        d_b, d_d = torch.zeros_like(d_src), torch.zeros_like(d_src)
        step = lambda: _lib.check(L.bm3d_b200_clip_twostage(c, d_src.data_ptr(), d_b.data_ptr(),
                                                          d_d.data_ptr(), None))
        ms = _device_timer(torch, step, args.warmup, max(3, args.steps // 6))
        L.bm3d_b200_clip_stage_times(c, None, None, 1)
        L.bm3d_b200_clip_set_profiling(c, 1)
        step()
        L.bm3d_b200_clip_set_profiling(c, 0)
        sm = (ctypes.c_double * _lib.NUM_STAGES)()
        L.bm3d_b200_clip_stage_times(c, sm, None, 1)
        out = d_d.cpu().numpy()[..., :Wc]
        L.bm3d_b200_clip_destroy(c)
        res[name] = {"mpix_s": N * Wc * Hc / 1e6 / (ms * 1e-3), "ms_per_step": ms,
                     "filter_ms": sm[1] + sm[5], "psnr_db": [S.psnr(out[:, q], clean[:, q]) for q in range(3)]}
    # accuracy against the FP64 oracle on a crop
    n, h, w = 4, 192, 256
    crop = np.ascontiguousarray(noisy[:n, :, :h, :w])
    for prec, name in ((0, "fp32"), (1, "split_bf16")):
        c = make(w, h, n, prec)
        stride = L.bm3d_b200_clip_stride(c)
        rf = L.bm3d_b200_clip_raw_frame_floats(c)
        hb = np.zeros((n, 3, h, stride), np.float32)
        hb[..., :w] = crop
        d_src = torch.from_numpy(hb).cuda()
        d_raw = torch.zeros((n, rf), dtype=torch.float32, device="cuda")
        _lib.check(L.bm3d_b200_clip_run(c, d_src.data_ptr(), None, d_raw.data_ptr(),
                                        _lib.DST_RAW, None))
        torch.cuda.synchronize()
        raw = d_raw.cpu().numpy().reshape(n, 3, 2 * r + 1, 2, h, stride)[..., :w]
        nb = ctypes.c_int()
        L.bm3d_b200_clip_matches(c, 0, None, 0, ctypes.byref(nb))
        err = np.zeros(3)
        scale = np.zeros(3)
        for f in range(n):
            lists = np.zeros((nb.value, 8, 3), np.int32)
            _lib.check(L.bm3d_b200_clip_matches(c, f, lists.ctypes.data, nb.value,
                                                ctypes.byref(nb)))
            want = O.port_bm3d(O.clip_window(crop, f, r), sigma=sig, radius=r, chroma=True,
                               fp64=True, match_in=lists)
            err = np.maximum(err, np.abs(raw[f] - want).max(axis=(1, 2, 3, 4)))
            scale = np.maximum(scale, np.abs(want).max(axis=(1, 2, 3, 4)))
        L.bm3d_b200_clip_destroy(c)
        res[name]["vs_fp64_max_abs_per_plane"] = err.tolist()
        res[name]["vs_fp64_rel_per_plane"] = (err / scale).tolist()
    return {"metric": "CBM3D 1080p Mpix/s, split-BF16 tensor-core transforms vs FP32",
            "value": res["split_bf16"]["mpix_s"], "unit": UNIT, "n_gpus": 1,
            "higher_is_better": True, "dtype": "bf16x3 split (FP32 accumulation)",
            "data": "synthetic", "workload": "cbm3d-1080p",
            "config": {"workload": "CBM3D two-stage, YUV444PS 1920x1080 x 16, chroma=True, "
                                   "radius 1, sigma [10, 7, 7]",
                       "accuracy_crop": "256x192 x 4 frames, basic-stage accumulators vs the "
                                        "FP64 oracle with the GPU's match lists"},
            "fp32": res["fp32"], "split_bf16": res["split_bf16"]}


def run_batched(args) -> dict:
    """64 GRAYS clips of seeded sizes from {320x240, 640x480, 1280x720,
    1920x1080, 3840x2160}, 8 frames each, radius in {0..3}, block_step in
    {4, 6, 8}, noise in U[3, 15]/255: the whole two-stage batch in one CUDA
    graph of persistent launches, match tiles chosen by the autotuner."""
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    L = _lib.lib()
    rng = np.random.default_rng(4)
    sizes = [(320, 240), (640, 480), (1280, 720), (1920, 1080), (3840, 2160)]
    b = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_batch_create(ctypes.byref(b), 0))
    bufs, pix = [], 0
    for i in range(64):
        w, h = sizes[int(rng.integers(0, len(sizes)))]
        r = int(rng.integers(0, 4))
        bs = int(rng.choice([4, 6, 8]))
        sigma = float(rng.uniform(3, 15))
        stride = (w + 31) // 32 * 32
        tex = S.texture_clip(8, h, w, noise=sigma / 255, seed=1000 + i)[0]
        host = np.zeros((8, h, stride), np.float32)
        host[..., :w] = tex
        d_src = torch.from_numpy(host).cuda()
        d_dst = torch.zeros_like(d_src)
        p = _lib.Params()
        L.bm3d_b200_params_default(ctypes.byref(p))
        p.sigma[0] = sigma
        p.block_step[0] = bs
        p.radius = r
        p.extractor_exp = 6
        idx = ctypes.c_int()
        _lib.check(L.bm3d_b200_batch_add(b, w, h, 8, ctypes.byref(p), d_src.data_ptr(),
                                         d_dst.data_ptr(), ctypes.byref(idx)))
        bufs.append((d_src, d_dst))
        pix += 8 * w * h
    t0 = time.perf_counter()
    _lib.check(L.bm3d_b200_batch_autotune(b, None))
    tune_s = time.perf_counter() - t0
    wx, k = ctypes.c_int(), ctypes.c_int()
    L.bm3d_b200_batch_config(b, ctypes.byref(wx), ctypes.byref(k))
    gb, gf, ga = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    L.bm3d_b200_batch_grids(b, ctypes.byref(gb), ctypes.byref(gf), ctypes.byref(ga))
    ms = _device_timer(torch, lambda: _lib.check(L.bm3d_b200_batch_run(b, None)),
                       max(1, args.warmup // 2), max(2, args.steps // 15))
    lat = (ctypes.c_double * 64)()
    _lib.check(L.bm3d_b200_batch_latencies(b, lat, 64))
    L.bm3d_b200_batch_destroy(b)
    lat = np.array(lat[:])
    return {"metric": "Batched uneven V-BM3D two-stage Mpix/s (one graph, persistent launches)",
            "value": pix / 1e6 / (ms * 1e-3), "unit": UNIT, "n_gpus": 1,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "workload": "batched-uneven", "ms_per_run": ms,
            "config": {"clips": 64, "frames_per_clip": 8, "megapixels_per_run": pix / 1e6,
                       "autotuned": {"cta_warps": wx.value, "strip": k.value,
                                     "filter_ctas_per_sm": [gb.value, gf.value],
                                     "aggregate_ctas_per_sm": ga.value,
                                     "seconds": tune_s}},
            "latency_ms": {"p50": float(np.percentile(lat, 50)),
                           "p99": float(np.percentile(lat, 99)), "max": float(lat.max())}}


def stream_measure(args, threads: int | None = None, reps: int = 3) -> dict:
    """Frame-by-frame V-BM3D through bm3d_b200_stream, the engine behind the
    VapourSynth plugin's BM3Dv2 with radius > 0: GRAYS 1920x1080 x 30, radius
    2, sigma 5, extractor_exp 6, a basic pass over the clip, then a final pass
    with the basic frames as its reference. Each output frame is one call that
    receives the 4r + 1 pageable host frames around it (as the plugin's
    getFrame does) and writes one host frame; `threads` host threads take the
    requests in order at once (VapourSynth's fmParallel), as many as the
    stream runs concurrently by default. Throughput = output pixels of the
    final pass / wall time of both passes; stream creation and destruction
    (device allocations) are timed apart. Beside it the whole-clip host path
    (bm3d_b200_clip_twostage_host) on the same frames, pinned buffers."""
    import threading

    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    L = _lib.lib()
    N, H, W, r = 30, 1080, 1920, 2
    noisy, _ = S.texture_clip(N, H, W, seed=7)
    noisy = np.ascontiguousarray(noisy, np.float32)

    def params():
        p = _lib.Params()
        L.bm3d_b200_params_default(ctypes.byref(p))
        for i in range(3):
            p.sigma[i] = 5.0
        p.radius = r
        p.extractor_exp = 6
        return p

    def create(final: bool):
        p = params()
        s = ctypes.c_void_p()
        _lib.check(L.bm3d_b200_stream_create(ctypes.byref(s), W, H, 1, 0, 0, N, ctypes.byref(p),
                                             int(final), 0))
        return s

    def stream_pass(s, src, ref, out, nthreads):
        nw = 4 * r + 1
        nxt = iter(range(N))
        lock = threading.Lock()
        errors = []

        def worker():
            while True:
                with lock:
                    n = next(nxt, None)
                if n is None:
                    return
                hs = (ctypes.c_void_p * (nw * 3))()
                hr = (ctypes.c_void_p * (nw * 3))()
                st = (ctypes.c_int * (nw * 3))()
                for i in range(nw):
                    f = min(max(n - 2 * r + i, 0), N - 1)
                    hs[i * 3] = src[f].ctypes.data
                    st[i * 3] = W * 4
                    if ref is not None:
                        hr[i * 3] = ref[f].ctypes.data
                hd = (ctypes.c_void_p * 3)()
                ds = (ctypes.c_int * 3)()
                hd[0] = out[n].ctypes.data
                ds[0] = W * 4
                rc = L.bm3d_b200_stream_frame(s, n, hs, hr if ref is not None else None, st, hd,
                                              ds)
                if rc:
                    errors.append(_lib.last_error())
        ts = [threading.Thread(target=worker) for _ in range(nthreads)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        if errors:
            raise RuntimeError(errors[0])

    t0 = time.perf_counter()
    sb, sf = create(False), create(True)
    setup_s = time.perf_counter() - t0
    nthreads = threads or L.bm3d_b200_stream_concurrency(sb)
    basic = np.empty_like(noisy)
    out = np.empty_like(noisy)
    try:
        for _ in range(max(1, args.warmup // 2)):
            stream_pass(sb, noisy, None, basic, nthreads)
            stream_pass(sf, noisy, basic, out, nthreads)
        # the rings now hold the clip's frames and windows: start every timed
        # repetition from empty rings, as a new clip would
        times, breakdown = [], []
        for _ in range(reps):
            for s in (sb, sf):
                L.bm3d_b200_stream_destroy(s)
            sb, sf = None, None
            sb, sf = create(False), create(True)
            t0 = time.perf_counter()
            stream_pass(sb, noisy, None, basic, nthreads)
            stream_pass(sf, noisy, basic, out, nthreads)
            times.append(time.perf_counter() - t0)
            per = {}
            for name, s in (("basic", sb), ("final", sf)):
                ms = (ctypes.c_double * 3)()
                calls = ctypes.c_longlong()
                _lib.check(L.bm3d_b200_stream_timings(s, ms, ctypes.byref(calls), 1))
                per[name] = {"calls": calls.value,
                             "upload_ms_per_call": ms[0] / max(1, calls.value),
                             "filter_ms_per_call": ms[1] / max(1, calls.value),
                             "output_ms_per_call": ms[2] / max(1, calls.value)}
            breakdown.append(per)
        up, win = ctypes.c_longlong(), ctypes.c_longlong()
        _lib.check(L.bm3d_b200_stream_stats(sb, ctypes.byref(up), ctypes.byref(win)))
    finally:
        for s in (sb, sf):
            if s is not None:
                L.bm3d_b200_stream_destroy(s)
    dt = float(np.median(times))
    mpix = N * W * H / 1e6

    # the whole-clip host path on the same frames (pinned buffers)
    p = params()
    c = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), W, H, 1, 0, 0, N, ctypes.byref(p), 0))
    try:
        stride = L.bm3d_b200_clip_stride(c)
        ff = L.bm3d_b200_clip_frame_floats(c)
        host = np.zeros((N, ff), np.float32)
        host.reshape(N, H, stride)[:, :, :W] = noisy
        h_src = torch.from_numpy(host).pin_memory()
        h_dst = torch.empty_like(h_src).pin_memory()

        def clip():
            _lib.check(L.bm3d_b200_clip_twostage_host(c, h_src.data_ptr(), h_dst.data_ptr(),
                                                      None))
        ms_clip = _device_timer(torch, clip, max(1, args.warmup), reps)
        same = bool(np.array_equal(h_dst.numpy().reshape(N, H, stride)[:, :, :W], out))
    finally:
        L.bm3d_b200_clip_destroy(c)
    return {"value": mpix / dt, "unit": "Mpix/s", "ms_per_clip": dt * 1e3,
            "host_threads": nthreads, "repetitions": reps,
            "setup_ms": setup_s * 1e3,
            "per_call_device_ms": breakdown[len(breakdown) // 2],
            "frames_uploaded_per_pass": up.value, "windows_per_pass": win.value,
            "identical_to_whole_clip": same,
            "whole_clip_host_path": {"mpix_s": mpix / (ms_clip / 1e3), "ms_per_clip": ms_clip},
            "matching": "exhaustive (the reference algorithm)"}


def run_stream(args) -> dict:
    res = stream_measure(args, reps=max(1, min(args.steps, 5)))
    single = stream_measure(args, threads=1, reps=2)
    return {"metric": "Frame-by-frame V-BM3D (the VapourSynth plugin's BM3Dv2 engine) Mpix/s",
            "value": res["value"], "unit": "Mpix/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic", "workload": "stream-1080p",
            "config": {"workload": "BM3Dv2 basic then final, GRAYS 1920x1080 x 30, radius 2, "
                                   "sigma 5, one call per output frame from pageable host "
                                   "frames, requests from %d host threads" % res["host_threads"],
                       "matching": "exhaustive (the reference algorithm)"},
            **{k: v for k, v in res.items() if k not in ("value", "unit")},
            "single_host_thread": {"mpix_s": single["value"], "ms_per_clip": single["ms_per_clip"],
                                   "per_call_device_ms": single["per_call_device_ms"]}}


def run_learned_4k(args) -> dict:
    """3840x2160 x 16 GRAYS, V-BM3D radius 2, bm_range 16, sigma 10: learned
    proposals (proposer trained on config-1-style clips) against the
    exhaustive search - two-stage Mpix/s, PSNR, and match recall of four
    basic-stage windows."""
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    from bm3dcuda.learned import Proposer, exhaustive_matches, learned_match, recall
    L = _lib.lib()
    N, Hc, Wc, r, R = 16, 2160, 3840, 2, 16
    noisy, clean = S.texture_clip(N, Hc, Wc, noise=10 / 255, seed=5)
    prop = Proposer()
    training = train_proposer(prop)
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    p.sigma[0] = 10.0
    p.bm_range[0] = R
    p.radius = r
    p.extractor_exp = 6
    c = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), Wc, Hc, 1, 0, 0, N, ctypes.byref(p), 0))
    stride = L.bm3d_b200_clip_stride(c)
    hb = np.zeros((N, Hc, stride), np.float32)
    hb[..., :Wc] = noisy
    d_src = torch.from_numpy(hb).cuda()
    d_b, d_d = torch.zeros_like(d_src), torch.zeros_like(d_src)
    step = lambda: _lib.check(L.bm3d_b200_clip_twostage(c, d_src.data_ptr(), d_b.data_ptr(),
                                                      d_d.data_ptr(), None))
    res = {}
    for name, on in (("exhaustive", False), ("learned", True)):
        if on:
            _lib.check(L.bm3d_b200_clip_set_proposer(c, prop.handle, args.cells_spatial,
                                                     args.cells_temporal, args.fallback_tau))
        ms = _device_timer(torch, step, 2, max(2, args.steps // 20))
        out = d_d.cpu().numpy()[..., :Wc]
        res[name] = {"mpix_s": N * Wc * Hc / 1e6 / (ms * 1e-3), "ms_per_step": ms,
                     "psnr_db": S.psnr(out, clean)}
    L.bm3d_b200_clip_destroy(c)
    recs = []
    for n in (2, 5, 9, 13):
        win = np.ascontiguousarray(noisy[n - r:n + r + 1])
        ex = exhaustive_matches(win, bm_range=R, radius=r)
        lm, _ = learned_match(prop, win, bm_range=R, radius=r, cells_spatial=args.cells_spatial,
                              cells_temporal=args.cells_temporal)
        recs.append(recall(lm, ex))
    prop.close()
    return {"metric": "Learned proposals vs exhaustive, V-BM3D 4K Mpix/s",
            "value": res["learned"]["mpix_s"], "unit": UNIT, "n_gpus": 1,
            "higher_is_better": True, "dtype": "f32 (int8 embeddings)", "data": "synthetic",
            "workload": "learned-4k",
            "config": {"workload": "V-BM3D two-stage GRAYS 3840x2160 x 16, radius 2, "
                                   "bm_range 16, sigma 10",
                       "cells": [args.cells_spatial, args.cells_temporal],
                       "fallback_tau": args.fallback_tau},
            "exhaustive": res["exhaustive"], "learned": res["learned"],
            "speedup": res["learned"]["mpix_s"] / res["exhaustive"]["mpix_s"],
            "psnr_delta_db": res["learned"]["psnr_db"] - res["exhaustive"]["psnr_db"],
            "match_recall": float(np.mean(recs)), "training": training}


def run_shard_frames(args, rank: int, world: int, dist) -> dict | None:
    """Frame shards of ONE clip of 30 x N frames (weak scaling: 30 output
    frames per rank): rank k denoises output frames [a_k, b_k) of the clip
    from source frames [a_k - 4r, b_k + 4r) clamped to the clip (the halo is
    recomputed, there is no data-path collective), through the host entry
    point bm3d_b200_clip_twostage_host from pinned buffers; the matching is
    the headline's. value = the clip's output pixels / the slowest rank's
    time; the only collectives are barriers and the max of the timings."""
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    from bm3dcuda.distributed import halo_range, max_over_ranks, shard_range
    from bm3dcuda.learned import Proposer
    L = _lib.lib()
    dev = torch.cuda.current_device()
    N = FRAMES * world
    r = SETTINGS["radius"]
    noisy, clean = S.texture_clip(N, H, W, seed=11)
    a, b = shard_range(N, world, rank)
    lo, hi = halo_range(a, b, N, r)
    n = hi - lo
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    p.sigma[0] = SETTINGS["sigma"]
    p.radius = r
    p.extractor_exp = SETTINGS["extractor_exp"]
    h = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(h), W, H, 1, 0, 0, n, ctypes.byref(p), dev))
    prop = None
    try:
        if args.mode == "learned":
            prop = Proposer(device=dev)
            train_proposer(prop)
            _lib.check(L.bm3d_b200_clip_set_proposer(h, prop.handle, args.cells_spatial,
                                                     args.cells_temporal, args.fallback_tau))
            _lib.check(L.bm3d_b200_clip_set_final_matching(
                h, {"search": 0, "basic-lists": 1, "basic-order": 2}[args.final_matching]))
        stride = L.bm3d_b200_clip_stride(h)
        ff = L.bm3d_b200_clip_frame_floats(h)
        host = np.zeros((n, ff), np.float32)
        host.reshape(n, H, stride)[:, :, :W] = noisy[lo:hi]
        h_src = torch.from_numpy(host).pin_memory()
        h_dst = torch.empty_like(h_src).pin_memory()
        stream = torch.cuda.current_stream()
        sp = ctypes.c_void_p(stream.cuda_stream)

        def step():
            _lib.check(L.bm3d_b200_clip_twostage_host(h, h_src.data_ptr(), h_dst.data_ptr(), sp))

        for _ in range(args.warmup):
            step()

        def barrier():
            if dist is not None:
                dist.barrier()
            torch.cuda.synchronize()

        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        barrier()
        ms = e0.elapsed_time(e1)
        if dist is not None:
            ms = max_over_ranks(ms, dist)
        out = h_dst.numpy().reshape(n, H, stride)[a - lo:b - lo, :, :W]
        psnr = S.psnr(out, clean[a:b])
    finally:
        L.bm3d_b200_clip_destroy(h)
        if prop is not None:
            prop.close()
    if rank != 0:
        return None
    mpix = N * W * H / 1e6
    return {"metric": METRIC, "value": mpix * args.steps / (ms * 1e-3), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "workload": "vbm3d-1080p-frame-shards",
            "config": {**workload_config(N), "parallelism": f"frame shards x{world}",
                       "halo_frames": 4 * r, "shard_of_rank0": [a, b],
                       "matching": args.mode},
            "e2e": {"value": mpix * args.steps / (ms * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": int(n * ff * 4), "d2h_bytes_per_step": int(n * ff * 4),
                    "note": "rank 0's copies; the timed region is the host entry point"},
            "quality": {"psnr_out_db_rank0": psnr}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--profile", action="store_true",
                    help="device two-stage only (for ncu): no CPU baseline, no peak GEMM, "
                         "no e2e pass, no JSON line")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--shard", choices=["replicas", "frames"], default="replicas",
                    help="multi-GPU layout: every rank its own clip (default), or frame shards "
                         "of one clip with a recomputed halo")
    ap.add_argument("--frames", type=int, default=FRAMES)
    ap.add_argument("--min-timed-s", type=float, default=2.0,
                    help="repeat the timed region of --steps steps until the repeats cover "
                         "this many seconds; the reported time is the median repeat")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-uneven figure of the headline line")
    ap.add_argument("--no-stream", action="store_true",
                    help="skip the frame-by-frame (plugin path) figure of the headline line")
    ap.add_argument("--mode", choices=["learned", "plain"], default="learned",
                    help="headline matching: learned proposals (default) or exhaustive")
    ap.add_argument("--cells-spatial", type=int, default=None,
                    help="learned matching: cells scored per centre-frame search "
                         "(default 1 for vbm3d-1080p, 4 for learned-4k)")
    ap.add_argument("--cells-temporal", type=int, default=None,
                    help="cells scored per neighbour frame (default 2 / 4)")
    ap.add_argument("--fallback-tau", type=float, default=None,
                    help="exhaustive re-search threshold (default 4 / 2)")
    ap.add_argument("--precision", choices=list(PRECISIONS), default="fp32",
                    help="headline filter transforms: FP32 (the reference's factorisation), "
                         "split-BF16 tensor cores, or FP16 Kronecker-form tcgen05 MMAs")
    ap.add_argument("--final-matching", choices=["search", "basic-lists", "basic-order"],
                    default="basic-lists",
                    help="learned runs: final-stage matching by the learned search on the basic "
                         "estimate, the basic stage's lists re-scored on it, or the basic "
                         "stage's lists in their basic order")
    ap.add_argument("--workload", default="vbm3d-1080p",
                    choices=["vbm3d-1080p", "cbm3d-1080p", "batched-uneven", "learned-4k",
                             "stream-1080p"],
                    help="vbm3d-1080p: the headline line; the others print their own line")
    args = ap.parse_args()
    # learned operating points: 1080p r 2 (bm_range 9) keeps the fallback
    # active on ~0.2% of blocks; the 4K bm_range-16 windows rank 4x the cells
    learned_defaults = {"learned-4k": (4, 4, 2.0)}.get(args.workload, (1, 2, 4.0))
    if args.cells_spatial is None:
        args.cells_spatial = learned_defaults[0]
    if args.cells_temporal is None:
        args.cells_temporal = learned_defaults[1]
    if args.fallback_tau is None:
        args.fallback_tau = learned_defaults[2]

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        line = run_reference_arm(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return

    import torch
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    if args.shard == "frames":
        dist = None
        if world > 1:
            import datetime
            import torch.distributed as td
            td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
            dist = td
        line = run_shard_frames(args, rank, world, dist)
        if line is not None:
            print(json.dumps(line), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.workload != "vbm3d-1080p":
        fn = {"cbm3d-1080p": run_cbm3d, "batched-uneven": run_batched,
              "learned-4k": run_learned_4k, "stream-1080p": run_stream}[args.workload]
        if rank == 0:
            print(json.dumps(fn(args)), flush=True)
        return
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as td
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = td

    # CPU baseline first (host threads only, before heavy GPU work), rank 0 at N=1
    cpu_base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.profile:
        from bm3dcuda import synthetic as S
        noisy, _ = S.texture_clip(5, H, W, seed=100)
        v, info = cpu_reference_sample(noisy, seconds=12.0)
        cpu_base = {"value": v, "unit": UNIT, **info}

    line = run_our_arm(args, rank, world, dist)
    if line is not None:
        noisy, basic, out = line.pop("_plain_frames")
        if cpu_base is not None:
            try:
                cpu_base["parity"] = cpu_parity_sample(noisy, basic, out, noisy.shape[0] // 2)
            except Exception as exc:  # the baseline figure stands on its own
                cpu_base["parity"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
        line["cpu_baseline"] = cpu_base
        if world == 1 and not args.no_batched:
            # the batched uneven workload (64 clips, one graph of persistent launches)
            try:
                bl = run_batched(args)
                line["batched_uneven"] = {k: bl[k] for k in ("value", "unit", "ms_per_run",
                                                             "config", "latency_ms")}
            except Exception as exc:
                line["batched_uneven"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
        if world == 1 and not args.no_stream:
            # the VapourSynth plugin's own path (frame-by-frame BM3Dv2), same clip size
            try:
                line["stream_1080p"] = stream_measure(args)
            except Exception as exc:
                line["stream_1080p"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
