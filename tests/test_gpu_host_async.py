"""Asynchronous host-buffer two-stage entry point (bm3d_b200_clip_twostage_host_async).

Two clips used in turn on two streams, several calls queued before any wait:
every output equals the synchronous call's bit for bit (pre-rounded sums), for
the single-plane chunked pipeline and for the multi-plane path.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _clip(L, N, H, W, planes, r):
    from bm3dcuda import _lib
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    for i in range(3):
        p.sigma[i] = 8.0
    p.radius = r
    p.extractor_exp = 6
    p.chroma = 1 if planes == 3 else 0
    c = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), W, H, planes, 0, 0, N, ctypes.byref(p), 0))
    return c


@pytest.mark.parametrize("planes", [1, 3])
def test_async_two_clips_in_flight_equal_sync(cuda, engine_lib, planes):
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    L = engine_lib
    N, H, W, r = 9, 72, 104, 2
    if planes == 3:
        noisy, _ = S.chroma_clip(N, H, W, seed=81)
    else:
        noisy, _ = S.moving_piecewise_clip(N, H, W, seed=82)
        noisy = noisy[:, None]
    a, b = _clip(L, N, H, W, planes, r), _clip(L, N, H, W, planes, r)
    try:
        stride = L.bm3d_b200_clip_stride(a)
        host = np.zeros((N, planes, H, stride), np.float32)
        host[..., :W] = noisy
        h_src = torch.from_numpy(host).pin_memory()
        want = torch.empty_like(h_src).pin_memory()
        _lib.check(L.bm3d_b200_clip_twostage_host(a, h_src.data_ptr(), want.data_ptr(), None))
        s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
        outs = [torch.zeros_like(h_src).pin_memory() for _ in range(4)]
        for k, dst in enumerate(outs):
            c, s = (a, s1) if k % 2 == 0 else (b, s2)
            _lib.check(L.bm3d_b200_clip_twostage_host_async(c, h_src.data_ptr(), dst.data_ptr(),
                                                            ctypes.c_void_p(s.cuda_stream)))
        torch.cuda.synchronize()
        for c in (a, b):
            _lib.check(L.bm3d_b200_clip_status(c))
        for k, dst in enumerate(outs):
            assert torch.equal(dst[..., :W], want[..., :W]), k
    finally:
        L.bm3d_b200_clip_destroy(a)
        L.bm3d_b200_clip_destroy(b)


def test_async_calls_on_one_clip_from_different_streams_run_in_order(cuda, engine_lib):
    """One clip, calls queued on alternating streams without waiting: each
    waits for the clip's previous call, so every output is the synchronous one."""
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    L = engine_lib
    N, H, W, r = 9, 72, 104, 2
    noisy, _ = S.moving_piecewise_clip(N, H, W, seed=83)
    a = _clip(L, N, H, W, 1, r)
    try:
        stride = L.bm3d_b200_clip_stride(a)
        host = np.zeros((N, 1, H, stride), np.float32)
        host[..., :W] = noisy[:, None]
        h_src = torch.from_numpy(host).pin_memory()
        want = torch.empty_like(h_src).pin_memory()
        _lib.check(L.bm3d_b200_clip_twostage_host(a, h_src.data_ptr(), want.data_ptr(), None))
        streams = [torch.cuda.Stream() for _ in range(3)]
        outs = [torch.zeros_like(h_src).pin_memory() for _ in range(6)]
        for k, dst in enumerate(outs):
            s = streams[k % 3]
            _lib.check(L.bm3d_b200_clip_twostage_host_async(a, h_src.data_ptr(), dst.data_ptr(),
                                                            ctypes.c_void_p(s.cuda_stream)))
        torch.cuda.synchronize()
        _lib.check(L.bm3d_b200_clip_status(a))
        for k, dst in enumerate(outs):
            assert torch.equal(dst[..., :W], want[..., :W]), k
    finally:
        L.bm3d_b200_clip_destroy(a)
