"""Multi-process paths (gloo, world size 2).

What is under test is the sharding logic the multi-GPU runs use: frame
shards with a recomputed 4r halo must reproduce the unsharded two-stage
V-BM3D bit for bit, and timings reduce to the max. On CPU the compute inside
each rank is the CPU oracle (the restatement of bm3dcpu); the GPU test runs
the engine's own host entry point in each rank (both ranks on one device:
their kernels never wait on each other, only the gloo collectives join them).
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "vapoursynth-bm3dcuda_b200")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _twostage_oracle(frames: np.ndarray, radius: int) -> np.ndarray:
    from oracle import oracle as O
    kw = dict(sigma=5.0, radius=radius, extractor_exp=6)
    basic = O.clip_bm3d_v2(O.port_bm3d, frames[:, None], None, chroma=False, **kw)
    return O.clip_bm3d_v2(O.port_bm3d, frames[:, None], basic, chroma=False, **kw)[:, 0]


def _engine_twostage(frames: np.ndarray, radius: int) -> np.ndarray:
    from bm3dcuda.distributed import engine_twostage
    return engine_twostage(frames, sigma=5.0, radius=radius, extractor_exp=6)


def _worker(rank, world, port, radius, frames, q, engine=False):
    for p in (ROOT, PKG):
        sys.path.insert(0, p)
    import torch.distributed as dist
    from bm3dcuda import distributed as D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        fn = _engine_twostage if engine else _twostage_oracle
        a, owned = D.run_sharded(frames, radius, world, rank, lambda f: fn(f, radius))
        gathered = [None] * world
        dist.all_gather_object(gathered, (a, owned))
        slowest = D.max_over_ranks(1.0 + rank, dist)
        if rank == 0:
            q.put((gathered, slowest))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("radius", [1, 2])
def test_sharded_twostage_equals_unsharded(radius, oracle):
    from bm3dcuda import synthetic as S
    frames, _ = S.texture_clip(11, 24, 32, seed=60 + radius)
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, radius, frames, q))
             for r in range(world)]
    for p in procs:
        p.start()
    gathered, slowest = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert slowest == float(world)
    out = np.zeros_like(frames)
    covered = np.zeros(frames.shape[0], bool)
    for a, owned in gathered:
        out[a:a + owned.shape[0]] = owned
        covered[a:a + owned.shape[0]] = True
    assert covered.all()
    np.testing.assert_array_equal(out, _twostage_oracle(frames, radius))


def test_shard_and_halo_ranges():
    from bm3dcuda.distributed import halo_range, shard_range
    ranges = [shard_range(30, 4, r) for r in range(4)]
    assert ranges == [(0, 8), (8, 16), (16, 23), (23, 30)]
    assert halo_range(8, 16, 30, 2) == (0, 24)
    assert halo_range(23, 30, 30, 2, stages=1) == (19, 30)


@pytest.mark.gpu
def test_sharded_engine_twostage_equals_unsharded(cuda, engine_lib):
    """Two gloo ranks each run the engine's host two-stage entry point on
    their frame shard plus halo; the gathered frames equal the unsharded
    engine run bit for bit (pre-rounded sums)."""
    from bm3dcuda import synthetic as S
    radius = 2
    frames, _ = S.texture_clip(14, 48, 64, seed=63)
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, radius, frames, q, True))
             for r in range(world)]
    for p in procs:
        p.start()
    gathered, _ = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out = np.zeros_like(frames)
    for a, owned in gathered:
        out[a:a + owned.shape[0]] = owned
    np.testing.assert_array_equal(out, _engine_twostage(frames, radius))
