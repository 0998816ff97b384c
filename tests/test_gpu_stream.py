"""Frame-by-frame V-BM3D through bm3d_b200_stream (the streamed BM3Dv2 of
the VapourSynth plugin): same output as the whole-clip pipeline, each source
frame uploaded once and each window filtered once when requests move through
the clip in order, and the same frames whatever the request order (pre-rounded
sums make recomputed windows bit-identical)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(L, _lib, radius, sigma, extractor_exp=6, chroma=False):
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    s = list(np.atleast_1d(sigma).astype(float)) + [None] * 3
    for i in range(3):
        p.sigma[i] = s[i] if s[i] is not None else p.sigma[i - 1]
    p.radius = radius
    p.chroma = int(chroma)
    p.extractor_exp = extractor_exp
    return p


def stream_frames(planes, radius, sigma, order, ref=None, chroma=False):
    """planes: list of [N][H_p][W_p] float32 arrays; returns frames in `order`."""
    from bm3dcuda import _lib
    L = _lib.lib()
    n_frames, h, w = planes[0].shape
    np_ = len(planes)
    ssw = 1 if np_ == 3 and planes[1].shape[2] * 2 == w else 0
    ssh = 1 if np_ == 3 and planes[1].shape[1] * 2 == h else 0
    p = _params(L, _lib, radius, sigma, chroma=chroma)
    s = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_stream_create(ctypes.byref(s), w, h, np_, ssw, ssh, n_frames,
                                         ctypes.byref(p), int(ref is not None), 0))
    out = [np.zeros_like(pl) for pl in planes]
    try:
        nw = 4 * radius + 1
        for n in order:
            hs = (ctypes.c_void_p * (nw * 3))()
            hr = (ctypes.c_void_p * (nw * 3))()
            st = (ctypes.c_int * (nw * 3))()
            for i in range(nw):
                f = min(max(n - 2 * radius + i, 0), n_frames - 1)
                for q in range(np_):
                    hs[i * 3 + q] = planes[q][f].ctypes.data
                    st[i * 3 + q] = planes[q].shape[2] * 4
                    if ref is not None:
                        hr[i * 3 + q] = ref[q][f].ctypes.data
            hd = (ctypes.c_void_p * 3)()
            ds = (ctypes.c_int * 3)()
            for q in range(np_):
                hd[q] = out[q][n].ctypes.data
                ds[q] = planes[q].shape[2] * 4
            _lib.check(L.bm3d_b200_stream_frame(s, n, hs, hr if ref is not None else None, st,
                                                hd, ds))
        up, win = ctypes.c_longlong(), ctypes.c_longlong()
        _lib.check(L.bm3d_b200_stream_stats(s, ctypes.byref(up), ctypes.byref(win)))
    finally:
        L.bm3d_b200_stream_destroy(s)
    return out, up.value, win.value


@pytest.mark.parametrize("radius,frames", [(1, 6), (2, 9)])
def test_stream_equals_clip_pipeline_and_uploads_once(cuda, engine_lib, radius, frames):
    from bm3dcuda import BM3Dv2, Clip
    from bm3dcuda import synthetic as S
    noisy, _ = S.texture_clip(frames, 40, 56, seed=60 + radius)
    got, uploads, windows = stream_frames([noisy], radius, 5.0, range(frames))
    want = BM3Dv2(Clip.from_array(noisy), sigma=5.0, radius=radius, extractor_exp=6).to_array()
    np.testing.assert_array_equal(got[0], want)
    assert uploads == frames and windows == frames


def test_stream_final_stage_equals_clip_pipeline(cuda, engine_lib):
    from bm3dcuda import BM3Dv2, Clip
    from bm3dcuda import synthetic as S
    noisy, _ = S.texture_clip(7, 40, 56, seed=64)
    src = Clip.from_array(noisy)
    basic = BM3Dv2(src, sigma=5.0, radius=2, extractor_exp=6)
    want = BM3Dv2(src, ref=basic, sigma=5.0, radius=2, extractor_exp=6).to_array()
    got, _, _ = stream_frames([noisy], 2, 5.0, range(7), ref=[basic.to_array()])
    np.testing.assert_array_equal(got[0], want)


def test_stream_any_request_order(cuda, engine_lib):
    from bm3dcuda import synthetic as S
    noisy, _ = S.texture_clip(10, 40, 56, seed=65)
    a, _, _ = stream_frames([noisy], 2, 5.0, range(10))
    order = list(np.random.default_rng(0).permutation(10)) + [3, 3, 9, 0]
    b, _, windows = stream_frames([noisy], 2, 5.0, order)
    np.testing.assert_array_equal(a[0], b[0])
    assert windows >= 10


def test_stream_chroma_and_subsampled_planes(cuda, engine_lib):
    from bm3dcuda import BM3Dv2, Clip
    from bm3dcuda import synthetic as S
    noisy, _ = S.chroma_clip(5, 40, 48, seed=66)
    planes = [np.ascontiguousarray(noisy[:, i]) for i in range(3)]
    got, _, _ = stream_frames(planes, 1, [10.0, 7.0], range(5), chroma=True)
    want = BM3Dv2(Clip(planes, "YUV444PS"), sigma=[10.0, 7.0], radius=1, chroma=True,
                  extractor_exp=6)
    for q in range(3):
        np.testing.assert_array_equal(got[q], want.planes[q])
    y, _ = S.piecewise_clip(4, 48, 64, seed=67)
    u, _ = S.piecewise_clip(4, 24, 32, seed=68)
    v, _ = S.piecewise_clip(4, 24, 32, seed=69)
    got420, _, _ = stream_frames([y, u, v], 1, [8.0, 0.0, 4.0], range(4))
    want420 = BM3Dv2(Clip([y, u, v], "YUV420PS"), sigma=[8.0, 0.0, 4.0], radius=1,
                     extractor_exp=6)
    np.testing.assert_array_equal(got420[0], want420.planes[0])
    np.testing.assert_array_equal(got420[2], want420.planes[2])
    assert not got420[1].any()  # unprocessed plane left to the caller


def stream_frames_threaded(planes, radius, sigma, threads, ref=None):
    """As stream_frames, the requests 0 .. N-1 taken in order by `threads`
    host threads at once (VapourSynth's fmParallel getFrame)."""
    import threading

    from bm3dcuda import _lib
    L = _lib.lib()
    n_frames, h, w = planes[0].shape
    p = _params(L, _lib, radius, sigma)
    s = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_stream_create(ctypes.byref(s), w, h, 1, 0, 0, n_frames,
                                         ctypes.byref(p), int(ref is not None), 0))
    out = np.zeros_like(planes[0])
    nxt = iter(range(n_frames))
    lock = threading.Lock()
    errors = []

    def worker():
        nw = 4 * radius + 1
        while True:
            with lock:
                n = next(nxt, None)
            if n is None:
                return
            hs = (ctypes.c_void_p * (nw * 3))()
            hr = (ctypes.c_void_p * (nw * 3))()
            st = (ctypes.c_int * (nw * 3))()
            for i in range(nw):
                f = min(max(n - 2 * radius + i, 0), n_frames - 1)
                hs[i * 3] = planes[0][f].ctypes.data
                st[i * 3] = w * 4
                if ref is not None:
                    hr[i * 3] = ref[0][f].ctypes.data
            hd = (ctypes.c_void_p * 3)()
            ds = (ctypes.c_int * 3)()
            hd[0] = out[n].ctypes.data
            ds[0] = w * 4
            rc = L.bm3d_b200_stream_frame(s, n, hs, hr if ref is not None else None, st, hd, ds)
            if rc != 0:
                errors.append((n, rc, _lib.last_error()))
    try:
        ts = [threading.Thread(target=worker) for _ in range(threads)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        up, win = ctypes.c_longlong(), ctypes.c_longlong()
        _lib.check(L.bm3d_b200_stream_stats(s, ctypes.byref(up), ctypes.byref(win)))
        ms = (ctypes.c_double * 3)()
        calls = ctypes.c_longlong()
        _lib.check(L.bm3d_b200_stream_timings(s, ms, ctypes.byref(calls), 1))
        conc = L.bm3d_b200_stream_concurrency(s)
    finally:
        L.bm3d_b200_stream_destroy(s)
    assert not errors, errors
    return out, up.value, win.value, calls.value, conc


@pytest.mark.parametrize("threads", [2, 4, 8])
def test_stream_concurrent_requests_equal_sequential(cuda, engine_lib, threads):
    """Requests from several host threads at once: the same frames as one
    caller in order, every frame uploaded and every window filtered once."""
    from bm3dcuda import synthetic as S
    N, r = 12, 2
    noisy, _ = S.texture_clip(N, 40, 56, seed=70 + threads)
    want, _, _ = stream_frames([noisy], r, 5.0, range(N))
    got, uploads, windows, calls, conc = stream_frames_threaded([noisy], r, 5.0, threads)
    np.testing.assert_array_equal(got, want[0])
    assert uploads == N and windows == N and calls == N and conc == 4
    # final stage, concurrent
    basic = want[0]
    fin_want, _, _ = stream_frames([noisy], r, 5.0, range(N), ref=[basic])
    fin, _, _, _, _ = stream_frames_threaded([noisy], r, 5.0, threads, ref=[basic])
    np.testing.assert_array_equal(fin, fin_want[0])
