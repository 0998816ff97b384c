"""The allocation-free entry point, bm3d_b200_window_noalloc.

It serves callers that cannot let the library allocate device memory while
processing (a host that owns the device-memory budget, or a pipeline that
cannot absorb cudaMalloc's synchronisation). Its scratch lives in a fixed
array inside the library that every call reuses, so each case runs it twice
in a row and compares both results with the existing entry point
(bm3d_b200_graph_launch_device) on the same inputs: accumulators within the
rtol 1e-5 used for accumulators elsewhere, and bit-identical when the sums are
pre-rounded (extractor_exp 6), where the summation order cannot matter.
"""
import ctypes

import numpy as np
import pytest

from gpu_util import graph_run, sigma3

pytestmark = pytest.mark.gpu


def noalloc_run(window, ref_window=None, *, sigma=3.0, block_step=8, bm_range=9, radius=0,
                ps_num=2, ps_range=4, chroma=False, extractor_exp=0):
    """Calls bm3d_b200_window_noalloc; the test (not the library) owns the buffers."""
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
    d_src = torch.from_numpy(src).cuda()
    d_res = torch.full((np_, tw, 2, H, stride), 7.0, dtype=torch.float32, device="cuda")
    s = [L.bm3d_b200_scale_sigma(v, int(final)) for v in sigma3(sigma)]
    ext = float(np.ldexp(np.float32(1.0), extractor_exp)) if extractor_exp else 0.0
    torch.cuda.synchronize()
    _lib.check(L.bm3d_b200_window_noalloc(d_res.data_ptr(), d_src.data_ptr(), W, H, stride, s[0],
                                          block_step, bm_range, radius, ps_num, ps_range,
                                          int(chroma), s[1], s[2], int(final), ext, None))
    torch.cuda.synchronize()
    return d_res.cpu().numpy()[..., :W].copy()


def cases():
    from bm3dcuda import synthetic as S
    noisy, _ = S.texture_clip(5, 56, 72, seed=31)
    basic = noisy * 0.5 + 0.25
    ch, _ = S.chroma_clip(3, 40, 48, seed=32)
    cw = np.ascontiguousarray(ch.transpose(1, 0, 2, 3))
    return [
        ("spatial_basic", noisy[None, 2:3], None, dict(sigma=5.0)),
        ("temporal_basic", noisy[None], None, dict(sigma=5.0, radius=2)),
        ("temporal_final", noisy[None, 1:4], basic[None, 1:4], dict(sigma=5.0, radius=1)),
        ("chroma_temporal", cw, None, dict(sigma=[10.0, 7.0, 0.0], radius=1, chroma=True)),
    ]


@pytest.mark.parametrize("idx", range(4))
def test_noalloc_equals_graph_entry_point_twice(cuda, engine_lib, idx):
    name, w, r, kw = cases()[idx]
    want = graph_run(w, r, **kw)
    first = noalloc_run(w, r, **kw)
    second = noalloc_run(w, r, **kw)
    np.testing.assert_allclose(first, want, rtol=1e-5, atol=1e-5, err_msg=name)
    np.testing.assert_allclose(second, want, rtol=1e-5, atol=1e-5, err_msg=name)
    want_x = graph_run(w, r, extractor_exp=6, **kw)
    for _ in range(2):
        np.testing.assert_array_equal(noalloc_run(w, r, extractor_exp=6, **kw), want_x)


def test_noalloc_rejects_frames_beyond_its_scratch(cuda, engine_lib):
    import torch
    from bm3dcuda import _lib
    L = _lib.lib()
    # 4096 x 4096 at block_step 4 is 1 046 529 reference blocks: over the limit.
    d = torch.zeros(16, dtype=torch.float32, device="cuda")
    rc = L.bm3d_b200_window_noalloc(d.data_ptr(), d.data_ptr(), 4096, 4096, 4096, 1.0, 4, 9, 0,
                                    2, 4, 0, 0.0, 0.0, 0, 0.0, None)
    assert rc == _lib.ERR_UNSUPPORTED
    assert "allocation-free" in _lib.last_error()


def test_noalloc_captured_into_a_cuda_graph(cuda, engine_lib):
    """After one eager call on the device, a call captured into a CUDA graph on
    a side stream replays to the graph entry point's result, twice."""
    import torch
    from bm3dcuda import _lib
    L = _lib.lib()
    name, w, r, kw = cases()[1]  # temporal_basic
    want = graph_run(w, r, extractor_exp=6, **kw)
    noalloc_run(w, r, extractor_exp=6, **kw)  # first call outside any capture
    np_, tw, H, W = w.shape
    stride = (W + 31) // 32 * 32
    src = np.zeros((1, np_, tw, H, stride), np.float32)
    src[0, ..., :W] = w
    d_src = torch.from_numpy(src).cuda()
    d_res = torch.full((np_, tw, 2, H, stride), 7.0, dtype=torch.float32, device="cuda")
    s = [L.bm3d_b200_scale_sigma(v, 0) for v in sigma3(kw["sigma"])]
    ext = float(np.ldexp(np.float32(1.0), 6))
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    rc = []
    with torch.cuda.graph(g, stream=side):
        cs = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc.append(L.bm3d_b200_window_noalloc(d_res.data_ptr(), d_src.data_ptr(), W, H, stride,
                                             s[0], 8, 9, kw["radius"], 2, 4, 0, s[1], s[2], 0,
                                             ext, cs))
    assert rc == [_lib.OK], _lib.last_error()
    for _ in range(2):
        d_res.fill_(7.0)
        g.replay()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(d_res.cpu().numpy()[..., :W], want, err_msg=name)
