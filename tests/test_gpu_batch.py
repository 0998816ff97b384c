"""Batches of uneven clips (persistent launches, one CUDA graph per run).

Every clip of a batch must come out exactly as when it runs alone through the
clip pipeline (pre-rounded sums make both bit-identical), across repeated
graph launches and after the autotuner changes the match tile shape.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CLIPS = [  # width, height, frames, radius, block_step, sigma
    (64, 48, 4, 0, 8, 6.0),
    (96, 72, 5, 1, 4, 9.0),
    (80, 40, 6, 2, 6, 5.0),
    (120, 88, 3, 3, 8, 12.0),
    (40, 40, 7, 1, 8, 3.0),
]


def params(L, radius, bs, sigma):
    from bm3dcuda import _lib
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    p.sigma[0] = sigma
    p.block_step[0] = bs
    p.radius = radius
    p.extractor_exp = 6
    return p


def clip_alone(L, torch, d_src, w, h, n, p):
    from bm3dcuda import _lib
    c = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), w, h, 1, 0, 0, n, ctypes.byref(p), 0))
    try:
        d_basic = torch.zeros_like(d_src)
        d_dst = torch.zeros_like(d_src)
        _lib.check(L.bm3d_b200_clip_twostage(c, d_src.data_ptr(), d_basic.data_ptr(),
                                             d_dst.data_ptr(), None))
        torch.cuda.synchronize()
        return d_dst.cpu().numpy()
    finally:
        L.bm3d_b200_clip_destroy(c)


def test_batch_equals_clips_run_alone(cuda, engine_lib):
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    L = engine_lib
    b = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_batch_create(ctypes.byref(b), 0))
    try:
        srcs, dsts, want = [], [], []
        for i, (w, h, n, r, bs, sg) in enumerate(CLIPS):
            stride = (w + 31) // 32 * 32
            noisy, _ = S.texture_clip(n, h, w, seed=70 + i)
            host = np.zeros((n, h, stride), np.float32)
            host[:, :, :w] = noisy
            d_src = torch.from_numpy(host).cuda()
            d_dst = torch.zeros_like(d_src)
            p = params(L, r, bs, sg)
            idx = ctypes.c_int()
            _lib.check(L.bm3d_b200_batch_add(b, w, h, n, ctypes.byref(p), d_src.data_ptr(),
                                             d_dst.data_ptr(), ctypes.byref(idx)))
            assert idx.value == i
            srcs.append(d_src)
            dsts.append(d_dst)
            want.append(clip_alone(L, torch, d_src, w, h, n, p))
        for run in range(2):
            for d in dsts:
                d.zero_()
            torch.cuda.synchronize()
            _lib.check(L.bm3d_b200_batch_run(b, None))
            torch.cuda.synchronize()
            for i, (d, w_) in enumerate(zip(dsts, want)):
                np.testing.assert_array_equal(d.cpu().numpy()[..., :CLIPS[i][0]],
                                              w_[..., :CLIPS[i][0]], err_msg=f"clip {i} run {run}")
        lat = (ctypes.c_double * len(CLIPS))()
        _lib.check(L.bm3d_b200_batch_latencies(b, lat, len(CLIPS)))
        assert all(v > 0 for v in lat)
        _lib.check(L.bm3d_b200_batch_autotune(b, None))
        wx, k = ctypes.c_int(), ctypes.c_int()
        _lib.check(L.bm3d_b200_batch_config(b, ctypes.byref(wx), ctypes.byref(k)))
        assert wx.value in (1, 2, 4) and 8 <= k.value <= 12
        fb, ff, ag = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(L.bm3d_b200_batch_grids(b, ctypes.byref(fb), ctypes.byref(ff),
                                           ctypes.byref(ag)))
        assert 1 <= fb.value <= 4 and 1 <= ff.value <= 4 and ag.value in (1, 2, 4, 8)
        for d in dsts:
            d.zero_()
        _lib.check(L.bm3d_b200_batch_run(b, None))
        torch.cuda.synchronize()
        for i, (d, w_) in enumerate(zip(dsts, want)):
            np.testing.assert_array_equal(d.cpu().numpy()[..., :CLIPS[i][0]],
                                          w_[..., :CLIPS[i][0]], err_msg=f"clip {i} tuned")
    finally:
        L.bm3d_b200_batch_destroy(b)
