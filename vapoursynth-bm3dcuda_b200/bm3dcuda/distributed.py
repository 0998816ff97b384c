"""Multi-GPU use of the engine: one process per GPU, no data-path collective.

Two ways to spread work:

* replicas - every rank denoises its own clips (what ``bench.py --gpus N``
  measures, weak scaling);
* frame shards of one long clip - rank k owns output frames [a_k, b_k) and
  runs the pipeline on source frames [a_k - h, b_k + h) clamped to the clip,
  with h = 2r per BM3Dv2 stage (4r for the two-stage V-BM3D). Output frame m
  of a BM3Dv2 stage depends only on input frames m-2r .. m+2r (its VAggregate
  reads windows m-r .. m+r, each window frames +-r), so the owned frames come
  out identical to an unsharded run; the halo is recomputed, not exchanged.

The only cross-rank operations are the final gather of owned frames (by the
caller) and the max-over-ranks of timings.
"""
from __future__ import annotations

from typing import Callable

import numpy as np


def shard_range(num_frames: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced output-frame range [a, b) of `rank`."""
    base, extra = divmod(num_frames, world)
    a = rank * base + min(rank, extra)
    return a, a + base + (1 if rank < extra else 0)


def halo_range(a: int, b: int, num_frames: int, radius: int, stages: int = 2) -> tuple[int, int]:
    """Source frames [lo, hi) needed to produce output frames [a, b)."""
    h = stages * 2 * radius
    return max(0, a - h), min(num_frames, b + h)


def run_sharded(frames: np.ndarray, radius: int, world: int, rank: int,
                run: Callable[[np.ndarray], np.ndarray], stages: int = 2) -> tuple[int, np.ndarray]:
    """Runs `run` (a whole-clip pipeline over [N, ...] frames) on this rank's
    shard plus halo and returns (a, owned output frames [a, b))."""
    n = frames.shape[0]
    a, b = shard_range(n, world, rank)
    if b <= a:
        return a, frames[a:a]
    lo, hi = halo_range(a, b, n, radius, stages)
    out = run(np.ascontiguousarray(frames[lo:hi]))
    return a, out[a - lo:b - lo]


def engine_twostage(frames: np.ndarray, *, sigma: float = 5.0, radius: int = 2,
                    block_step: int = 8, bm_range: int = 9, ps_num: int = 2, ps_range: int = 4,
                    extractor_exp: int = 6) -> np.ndarray:
    """Two-stage V-BM3D of a GRAYS clip [N, H, W] on this rank's current CUDA
    device through the engine's host entry point (bm3d_b200_clip_twostage_host):
    the per-rank work of a frame-sharded run."""
    from . import Clip, twostage
    return twostage(Clip.from_array(frames), sigma=sigma, radius=radius, block_step=block_step,
                    bm_range=bm_range, ps_num=ps_num, ps_range=ps_range,
                    extractor_exp=extractor_exp).to_array()


def max_over_ranks(value: float, dist) -> float:
    """Maximum of a per-rank timing over all ranks (CPU tensor for gloo,
    CUDA tensor for nccl)."""
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
