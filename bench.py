#!/usr/bin/env python3
"""Benchmark: two-stage V-BM3D on 1920x1080 x 30 frames (GRAYS float32).

Workload (the reference's V-BM3D recipe, README.md:44-53): vbasic =
BM3Dv2(src, radius=2) then vfinal = BM3Dv2(src, ref=vbasic, radius=2), sigma 5,
block_step 8, bm_range 9, ps_num 2, ps_range 4, extractor_exp 6, on a seeded
synthetic clip (band-limited texture moving by integer steps in [-3, 3] px,
AWGN 5/255). One step = the whole two-stage pass over the 30 frames.

  value  Mpix/s with the clip resident in HBM (device buffers in, out)
  e2e    Mpix/s through bm3d_b200_clip_twostage_host from pinned host
         buffers: the host->device copy of the 30 frames and the
         device->host copy of the result are inside the timed region

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
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            self.fh = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-i", str(self.dev), "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
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


def load_traffic():
    p = os.path.join(ROOT, "profiles", "match_kernel_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def run_our_arm(args, rank: int, world: int, dist):
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
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
    h = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(h), W, H, 1, 0, 0, frames, ctypes.byref(p), dev))
    stride = L.bm3d_b200_clip_stride(h)
    ff = L.bm3d_b200_clip_frame_floats(h)
    host = np.zeros((frames, ff), np.float32)
    host.reshape(frames, H, stride)[:, :, :W] = noisy
    h_src = torch.from_numpy(host).pin_memory()
    h_dst = torch.empty_like(h_src).pin_memory()
    d_src = h_src.cuda()
    d_basic = torch.empty_like(d_src)
    d_dst = torch.empty_like(d_src)
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)

    if args.profile:
        for _ in range(args.warmup + args.steps):
            _lib.check(L.bm3d_b200_clip_twostage(h, d_src.data_ptr(), d_basic.data_ptr(),
                                                 d_dst.data_ptr(), sp))
        torch.cuda.synchronize()
        L.bm3d_b200_clip_destroy(h)
        return None

    peak = fp32_peak_tflops(torch) if rank == 0 else 0.0

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def step_device():
        _lib.check(L.bm3d_b200_clip_twostage(h, d_src.data_ptr(), d_basic.data_ptr(),
                                             d_dst.data_ptr(), sp))

    def step_e2e():
        _lib.check(L.bm3d_b200_clip_twostage_host(h, h_src.data_ptr(), h_dst.data_ptr(), sp))

    def timed(fn, steps):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        barrier()
        ms = e0.elapsed_time(e1)
        if dist is not None:
            from bm3dcuda.distributed import max_over_ranks
            ms = max_over_ranks(ms, dist)
        return ms

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()

    # device-resident timed region, with per-stage events and clock samples
    clocks = ClockSampler(int(os.environ.get("CUDA_VISIBLE_DEVICES", str(dev)).split(",")[0])
                          if os.environ.get("CUDA_VISIBLE_DEVICES", "").isdigit() else dev)
    clocks.start()
    L.bm3d_b200_clip_stage_times(h, None, None, 1)
    L.bm3d_b200_clip_set_profiling(h, 1)
    ms_dev = timed(step_device, args.steps)
    L.bm3d_b200_clip_set_profiling(h, 0)
    stage_ms = (ctypes.c_double * _lib.NUM_STAGES)()
    stage_n = (ctypes.c_longlong * _lib.NUM_STAGES)()
    _lib.check(L.bm3d_b200_clip_stage_times(h, stage_ms, stage_n, 1))
    clock_info = clocks.stop()

    # end-to-end through the host-buffer entry point
    for _ in range(max(1, args.warmup // 2)):
        step_e2e()
    ms_e2e = timed(step_e2e, args.steps)

    # quality check of the last result (PSNR against the clean clip)
    out = h_dst.numpy().reshape(frames, H, stride)[:, :, :W]
    q_psnr = S.psnr(out, clean)
    in_psnr = S.psnr(noisy, clean)
    _lib.lib().bm3d_b200_clip_destroy(h)

    mpix_step = frames * W * H / 1e6
    value = world * mpix_step * args.steps / (ms_dev * 1e-3)
    e2e = world * mpix_step * args.steps / (ms_e2e * 1e-3)
    if rank != 0:
        return None

    names = ["match", "filter", "aggregate", "propose"]
    launches = {names[i]: int(stage_n[i]) for i in range(_lib.NUM_STAGES)}
    per_stage = {names[i]: float(stage_ms[i]) / args.steps for i in range(_lib.NUM_STAGES)}
    cand = candidates_per_window(W, H, SETTINGS["block_step"], SETTINGS["bm_range"],
                                 SETTINGS["radius"], SETTINGS["ps_num"], SETTINGS["ps_range"])
    flop_launch = SSD_FLOP * cand * frames  # one match launch covers every window of the clip
    match_ms = float(stage_ms[0]) / max(1, int(stage_n[0]))
    achieved = flop_launch / (match_ms * 1e-3) / 1e12
    traffic = load_traffic()
    roofline = {
        "kernel": "match_kernel (block matching, FP32 SIMT)",
        "bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
        "frac": achieved / peak if peak else None,
        "peak_source": "measured live in this run: cuBLAS SGEMM 8192^3, TF32 off (no FP32 "
                       "entry in MEASURED_PEAKS.json)",
        "traffic": traffic.get("bytes_per_launch") if traffic else None,
        "algorithmic_flop_per_launch": flop_launch,
        "avg_launch_ms": match_ms,
    }
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_dev / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {**workload_config(frames), "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(frames * ff * 4),
                "d2h_bytes_per_step": int(frames * ff * 4)},
        "roofline": roofline,
        "gpu_launches": int(sum(stage_n)),
        "stage_ms_per_step": per_stage,
        "stage_launches": launches,
        "quality": {"psnr_in_db": in_psnr, "psnr_out_db": q_psnr},
        "clocks": clock_info,
    }
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--profile", action="store_true",
                    help="device two-stage only (for ncu): no CPU baseline, no peak GEMM, "
                         "no e2e pass, no JSON line")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--frames", type=int, default=FRAMES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()

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
        line["cpu_baseline"] = cpu_base
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
