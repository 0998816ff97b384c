"""Helpers that drive the engine through its C ABI with device buffers."""
from __future__ import annotations

import ctypes

import numpy as np


def sigma3(sigma):
    s = [float(v) for v in np.atleast_1d(sigma)]
    while len(s) < 3:
        s.append(s[-1])
    return s[:3]


def graph_run(window, ref_window=None, *, sigma=3.0, block_step=8, bm_range=9, radius=0,
              ps_num=2, ps_range=4, chroma=False, extractor_exp=0, host=False,
              return_matches=False, bm_error=0, transform_2d=0, transform_1d=0):
    """One window through bm3d_b200_graph_* (the reference graph replacement;
    bm3d_b200_graph_create_rtc when a run-time-compiled plugin variant is set).

    window/ref_window: [planes][2r+1][H][W]. Returns the accumulators
    [planes][2r+1][2][H][W] (and the match lists [nb][8][3])."""
    import torch
    from bm3dcuda import _lib
    L = _lib.lib()
    np_, tw, H, W = window.shape
    stride = (W + 31) // 32 * 32
    final = ref_window is not None
    src = np.zeros((2 if final else 1, np_, tw, H, stride), np.float32)
    if final:
        src[0, ..., :W] = ref_window
        src[1, ..., :W] = window
    else:
        src[0, ..., :W] = window
    d_res = torch.zeros((np_, tw, 2, H, stride), dtype=torch.float32, device="cuda")
    s = [L.bm3d_b200_scale_sigma(v, int(final)) for v in sigma3(sigma)]
    ext = float(np.ldexp(np.float32(1.0), extractor_exp)) if extractor_exp else 0.0
    h = ctypes.c_void_p()
    if host:
        size = max(src.size, d_res.numel())
        h_res = torch.zeros(size, dtype=torch.float32).pin_memory()
        h_res[: src.size] = torch.from_numpy(src.reshape(-1))
        d_src = torch.zeros(src.shape, dtype=torch.float32, device="cuda")
        hp = h_res.data_ptr()
    else:
        d_src = torch.from_numpy(src).cuda()
        hp = None
    torch.cuda.synchronize()
    if bm_error or transform_2d or transform_1d:
        _lib.check(L.bm3d_b200_graph_create_rtc(
            ctypes.byref(h), d_res.data_ptr(), d_src.data_ptr(), hp, W, H, stride, s[0], block_step,
            bm_range, radius, ps_num, ps_range, int(chroma), s[1], s[2], int(final), ext,
            bm_error, transform_2d, transform_1d))
    else:
        _lib.check(L.bm3d_b200_graph_create(ctypes.byref(h), d_res.data_ptr(), d_src.data_ptr(),
                                            hp, W, H, stride, s[0], block_step, bm_range, radius,
                                            ps_num, ps_range, int(chroma), s[1], s[2], int(final),
                                            ext))
    try:
        if host:
            # the create-time warm-up already ran the device part; run the full graph
            d_res.zero_()
            torch.cuda.synchronize()
            _lib.check(L.bm3d_b200_graph_launch(h, None))
            torch.cuda.synchronize()
            res = h_res[: d_res.numel()].numpy().reshape(d_res.shape)[..., :W].copy()
        else:
            _lib.check(L.bm3d_b200_graph_launch_device(h, None))
            torch.cuda.synchronize()
            res = d_res.cpu().numpy()[..., :W].copy()
        matches = None
        if return_matches:
            nb = ctypes.c_int()
            dummy = np.zeros(3, np.int32)
            L.bm3d_b200_graph_matches(h, dummy.ctypes.data, 0, ctypes.byref(nb))  # reports the count
            buf = np.zeros((nb.value, 8, 3), np.int32)
            _lib.check(L.bm3d_b200_graph_matches(h, buf.ctypes.data, nb.value, ctypes.byref(nb)))
            matches = buf
    finally:
        L.bm3d_b200_graph_destroy(h)
    return (res, matches) if return_matches else res


def aggregate(acc):
    """Host Aggregation of a radius-0 accumulator [planes][1][2][H][W]."""
    return (acc[:, 0, 0] / acc[:, 0, 1]).astype(np.float32)


def psnr(a, b):
    from bm3dcuda.synthetic import psnr as p
    return p(a, b)
