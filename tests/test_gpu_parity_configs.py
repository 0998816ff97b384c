"""GPU parity at the sizes of the benchmark configurations, against the
reference's own bm3dcpu (cpu_source/source.cpp:769-911, exact-reciprocal
build in oracle/_ref) on the GPU box's host cores.

  C1  BM3D basic, 640x360 x 8, radius 0, sigma 10, piecewise scene
  C2  V-BM3D two-stage 1920x1080 x 30, radius 2, sigma 5: the basic stage and
      the final stage fed the ENGINE's basic estimate on both sides (the final
      stage matches on its reference, so both sides must see the same one), on
      the first, five middle and the last windows of the clip
  C3  CBM3D YUV444 1920x1080, radius 1, sigma [10, 7, 7], against bm3dcpu and
      against the FP64 oracle per plane, with FP32 and split-BF16 transforms
      (against FP64 the bar is the reference's own FP32 distance to FP64:
      hard-threshold decisions of near-threshold coefficients flip between
      FP32 and FP64 arithmetic)
  C4  a batch of uneven clips (3840x2160, block_step 4 and 6, radius up to 3)
      in one persistent launch, against bm3dcpu, basic and final stage

Bars (the parity target of this path): match lists identical, denoised
output max-abs <= 1e-4 and PSNR within 0.01 dB of bm3dcpu, raw accumulators
rtol 1e-5. The oracle windows run in a thread pool (bm3dcpu is
single-threaded per call, as under VapourSynth's fmParallel).
"""
import ctypes
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from gpu_util import aggregate, graph_run, psnr

pytestmark = pytest.mark.gpu

MAX_ABS = 1e-4
PSNR_DB = 0.01


@pytest.fixture(scope="module")
def ref(oracle):
    if not oracle.ref_available("exact"):
        pytest.fail("the reference bm3dcpu build (oracle/_ref) is missing: make -C oracle ref")
    return oracle


def pool_map(fn, items):
    with ThreadPoolExecutor(max_workers=max(1, min(len(items), os.cpu_count() or 1))) as ex:
        return list(ex.map(fn, items))


def clampi(v, n):
    return min(max(v, 0), n - 1)


def ref_raw_windows(O, noisy, ref_clip, ns, radius, **kw):
    """bm3dcpu raw outputs {n: [planes][2r+1][2][H][W]} of windows ns.
    noisy / ref_clip: [N][planes][H][W]."""
    def one(n):
        w = O.clip_window(noisy, n, radius)
        r = None if ref_clip is None else O.clip_window(ref_clip, n, radius)
        return O.ref_bm3d(w, r, radius=radius, **kw)
    return dict(zip(ns, pool_map(one, list(ns))))


def vaggregate_frame(O, raws, n, N, radius, plane=0):
    """VAggregate of output frame n from raw window outputs (replication
    padding at the clip ends, source/source.cpp:814-850)."""
    idx = [clampi(n + i, N) for i in range(-radius, radius + 1)]
    return O.port_vaggregate(np.stack([raws[i][plane] for i in idx]), n, N)


def windows_for(frames, N, radius):
    return sorted({clampi(n + i, N) for n in frames for i in range(-radius, radius + 1)})


# --------------------------------------------------------------------------
# C1: BM3D basic 640x360 x 8
# --------------------------------------------------------------------------
def test_c1_bm3d_640x360x8_vs_bm3dcpu(cuda, engine_lib, ref):
    from bm3dcuda import BM3D, Clip
    from bm3dcuda import synthetic as S
    O = ref
    noisy, clean = S.piecewise_clip(8, 360, 640, noise=10 / 255, seed=101)
    kw = dict(sigma=10.0, block_step=8, bm_range=9, radius=0, ps_num=2, ps_range=4)
    want = np.stack(pool_map(lambda n: O.ref_bm3d(noisy[n][None, None], **kw)[0], range(8)))
    lists = pool_map(lambda n: O.ref_match_lists(noisy[n][None], block_step=8, bm_range=9)[2],
                     range(8))
    for n in range(8):
        acc, m = graph_run(noisy[n][None, None], return_matches=True, **kw)
        np.testing.assert_array_equal(m, lists[n], err_msg=f"frame {n} match lists")
        assert np.abs(aggregate(acc)[0] - want[n]).max() <= MAX_ABS, f"frame {n}"
    out = BM3D(Clip.from_array(noisy), sigma=10.0).to_array()
    assert np.abs(out - want).max() <= MAX_ABS
    assert abs(psnr(out, clean) - psnr(want, clean)) <= PSNR_DB
    # final stage (BM3D with ref) fed the engine's basic estimate on both sides
    fin = BM3D(Clip.from_array(noisy), ref=Clip.from_array(out), sigma=10.0).to_array()
    want_f = np.stack(pool_map(
        lambda n: O.ref_bm3d(noisy[n][None, None], out[n][None, None], **kw)[0], range(8)))
    assert np.abs(fin - want_f).max() <= MAX_ABS
    assert abs(psnr(fin, clean) - psnr(want_f, clean)) <= PSNR_DB


# --------------------------------------------------------------------------
# C2: V-BM3D two-stage 1080p x 30, radius 2
# --------------------------------------------------------------------------
C2_FRAMES = (0, 12, 29)  # output frames checked: first, middle, last


@pytest.fixture(scope="module")
def c2(cuda, engine_lib):
    from bm3dcuda import BM3Dv2, Clip
    from bm3dcuda import synthetic as S
    noisy, clean = S.texture_clip(30, 1080, 1920, noise=5 / 255, seed=102)
    basic = BM3Dv2(Clip.from_array(noisy), sigma=5.0, radius=2).to_array()
    final = BM3Dv2(Clip.from_array(noisy), ref=Clip.from_array(basic), sigma=5.0,
                   radius=2).to_array()
    return noisy, clean, basic, final


C2_KW = dict(sigma=5.0, block_step=8, bm_range=9, ps_num=2, ps_range=4)


def test_c2_basic_stage_1080p_vs_bm3dcpu(c2, ref):
    O = ref
    noisy, clean, basic, _ = c2
    r, N = 2, 30
    ws = windows_for(C2_FRAMES, N, r)
    raws = ref_raw_windows(O, noisy[:, None], None, ws, r, **C2_KW)
    for n in C2_FRAMES:
        want = vaggregate_frame(O, raws, n, N, r)
        err = np.abs(basic[n] - want).max()
        assert err <= MAX_ABS, f"basic frame {n}: max-abs {err}"
        assert abs(psnr(basic[n], clean[n]) - psnr(want, clean[n])) <= PSNR_DB


def test_c2_final_stage_1080p_same_basic_vs_bm3dcpu(c2, ref):
    """Final (Wiener) stage fed the engine's basic estimate on both sides: the
    raw window outputs, every block's match list (on 5 consecutive windows and
    the clip's first and last) and the aggregated output frames."""
    O = ref
    noisy, clean, basic, final = c2
    r, N = 2, 30
    ws = windows_for(C2_FRAMES, N, r)
    raws = ref_raw_windows(O, noisy[:, None], basic[:, None], ws, r, **C2_KW)
    for n in C2_FRAMES:
        want = vaggregate_frame(O, raws, n, N, r)
        err = np.abs(final[n] - want).max()
        assert err <= MAX_ABS, f"final frame {n}: max-abs {err}"
        assert abs(psnr(final[n], clean[n]) - psnr(want, clean[n])) <= PSNR_DB
    check = [0, 10, 11, 12, 13, 14, 29]
    lists = dict(zip(check, pool_map(
        lambda n: O.ref_match_lists(O.clip_window(basic[:, None], n, r)[0], block_step=8,
                                    bm_range=9, radius=r, ps_num=2, ps_range=4)[2], check)))
    for n in check:
        acc, m = graph_run(O.clip_window(noisy[:, None], n, r),
                           O.clip_window(basic[:, None], n, r), radius=r, return_matches=True,
                           **C2_KW)
        np.testing.assert_array_equal(m, lists[n], err_msg=f"window {n} match lists")
        np.testing.assert_allclose(acc, raws[n], rtol=1e-5, atol=1e-5,
                                   err_msg=f"window {n} accumulators")


# --------------------------------------------------------------------------
# C3: CBM3D 1080p, radius 1, sigma [10, 7, 7]
# --------------------------------------------------------------------------
def _clip_chroma_run(L, noisy, sig, r, precision):
    """Raw V-BM3D stacks of a chroma clip through the clip pipeline and the
    match lists of every window."""
    import torch
    from bm3dcuda import _lib
    n, _, h, w = noisy.shape
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    for i in range(3):
        p.sigma[i] = sig[i]
    p.radius = r
    p.chroma = 1
    c = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), w, h, 3, 0, 0, n, ctypes.byref(p), 0))
    try:
        _lib.check(L.bm3d_b200_clip_set_precision(c, precision))
        stride = L.bm3d_b200_clip_stride(c)
        rf = L.bm3d_b200_clip_raw_frame_floats(c)
        hb = np.zeros((n, 3, h, stride), np.float32)
        hb[..., :w] = noisy
        d_src = torch.from_numpy(hb).cuda()
        d_raw = torch.zeros((n, rf), dtype=torch.float32, device="cuda")
        _lib.check(L.bm3d_b200_clip_run(c, d_src.data_ptr(), None, d_raw.data_ptr(),
                                        _lib.DST_RAW, None))
        torch.cuda.synchronize()
        raw = d_raw.cpu().numpy().reshape(n, 3, 2 * r + 1, 2, h, stride)[..., :w]
        nb = ctypes.c_int()
        L.bm3d_b200_clip_matches(c, 0, None, 0, ctypes.byref(nb))
        lists = []
        for f in range(n):
            buf = np.zeros((nb.value, 8, 3), np.int32)
            _lib.check(L.bm3d_b200_clip_matches(c, f, buf.ctypes.data, nb.value,
                                                ctypes.byref(nb)))
            lists.append(buf)
        return raw, lists
    finally:
        L.bm3d_b200_clip_destroy(c)


def test_c3_cbm3d_1080p_vs_bm3dcpu_and_fp64(cuda, engine_lib, ref):
    from bm3dcuda import synthetic as S
    O = ref
    L = engine_lib
    N, r = 3, 1
    sig = [10.0, 7.0, 7.0]
    noisy, clean = S.chroma_clip(N, 1080, 1920, seed=103)
    kw = dict(sigma=sig, block_step=8, bm_range=9, ps_num=2, ps_range=4, chroma=True)
    raws_ref = ref_raw_windows(O, noisy, None, list(range(N)), r, **kw)
    ymatch = O.ref_match_lists(O.clip_window(noisy, 1, r)[0], radius=r)[2]
    res = {}
    for prec, name in ((0, "fp32"), (1, "split_bf16")):
        raw, lists = _clip_chroma_run(L, noisy, sig, r, prec)
        np.testing.assert_array_equal(lists[1], ymatch, err_msg=f"{name} match lists")
        raw_d = {f: raw[f] for f in range(N)}
        fp64 = dict(zip(range(N), pool_map(
            lambda f: O.port_bm3d(O.clip_window(noisy, f, r), sigma=sig, radius=r, chroma=True,
                                  fp64=True, match_in=lists[f]), list(range(N)))))
        for pl in range(3):
            got = vaggregate_frame(O, raw_d, 1, N, r, pl)
            want = vaggregate_frame(O, raws_ref, 1, N, r, pl)
            want64 = O.port_vaggregate(np.stack([fp64[clampi(1 + i, N)][pl]
                                                 for i in range(-r, r + 1)]), 1, N, fp64=True)
            e_ref = float(np.abs(got - want).max())
            d64 = np.abs(got.astype(np.float64) - want64)
            # the reference's own FP32 arithmetic against FP64 on the same
            # lists: hard-threshold decisions of coefficients within rounding
            # of the threshold flip between FP32 and FP64, so neither FP32
            # path is within 1e-4 of FP64 everywhere
            r64 = np.abs(want.astype(np.float64) - want64)
            res[(name, pl)] = {"vs_bm3dcpu": e_ref, "vs_fp64": float(d64.max()),
                               "bm3dcpu_vs_fp64": float(r64.max()),
                               "mean_vs_fp64": float(d64.mean()),
                               "bm3dcpu_mean_vs_fp64": float(r64.mean())}
            if prec == 0:
                assert e_ref <= MAX_ABS, f"{name} plane {pl}: {e_ref} vs bm3dcpu"
                assert d64.max() <= r64.max() + MAX_ABS, (name, pl, res[(name, pl)])
            else:
                # split-BF16 transforms: as close to FP64 as FP32 is
                assert d64.max() <= 2 * r64.max() + MAX_ABS, (name, pl, res[(name, pl)])
                assert d64.mean() <= 2 * r64.mean() + 1e-6, (name, pl, res[(name, pl)])
            assert abs(psnr(got, clean[1, pl]) - psnr(want, clean[1, pl])) <= PSNR_DB
    print("C3 per plane:", res)


# --------------------------------------------------------------------------
# C4: batched uneven clips, one persistent launch per stage
# --------------------------------------------------------------------------
C4_CLIPS = [  # width, height, frames, radius, block_step, sigma
    (3840, 2160, 3, 1, 8, 10.0),
    (640, 480, 4, 3, 4, 7.0),
    (1280, 720, 3, 2, 6, 12.0),
    (320, 240, 4, 0, 6, 5.0),
]


def test_c4_batched_uneven_vs_bm3dcpu(cuda, engine_lib, ref):
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    O = ref
    L = engine_lib
    b = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_batch_create(ctypes.byref(b), 0))
    try:
        clips = []
        for i, (w, h, n, r, bs, sg) in enumerate(C4_CLIPS):
            stride = (w + 31) // 32 * 32
            noisy, clean = S.texture_clip(n, h, w, noise=sg / 255, seed=110 + i)
            host = np.zeros((n, h, stride), np.float32)
            host[..., :w] = noisy
            d_src = torch.from_numpy(host).cuda()
            d_dst = torch.zeros_like(d_src)
            p = _lib.Params()
            L.bm3d_b200_params_default(ctypes.byref(p))
            p.sigma[0] = sg
            p.block_step[0] = bs
            p.radius = r
            idx = ctypes.c_int()
            _lib.check(L.bm3d_b200_batch_add(b, w, h, n, ctypes.byref(p), d_src.data_ptr(),
                                             d_dst.data_ptr(), ctypes.byref(idx)))
            clips.append((noisy, clean, d_src, d_dst))
        _lib.check(L.bm3d_b200_batch_run(b, None))
        torch.cuda.synchronize()
        for i, ((w, h, n, r, bs, sg), (noisy, clean, d_src, d_dst)) in enumerate(
                zip(C4_CLIPS, clips)):
            d_basic = torch.zeros_like(d_src)
            _lib.check(L.bm3d_b200_batch_basic(b, i, d_basic.data_ptr(), None))
            torch.cuda.synchronize()
            basic = d_basic.cpu().numpy()[..., :w]
            final = d_dst.cpu().numpy()[..., :w]
            kw = dict(sigma=sg, block_step=bs, bm_range=9, ps_num=2, ps_range=4)
            ws = list(range(n))
            for stage, got, refc in (("basic", basic, None), ("final", final, basic)):
                raws = ref_raw_windows(O, noisy[:, None], None if refc is None else refc[:, None],
                                       ws, r, **kw)
                for f in range(n):
                    want = raws[f][0] if r == 0 else vaggregate_frame(O, raws, f, n, r)
                    err = np.abs(got[f] - want).max()
                    assert err <= MAX_ABS, f"clip {i} ({w}x{h}) {stage} frame {f}: {err}"
                    assert abs(psnr(got[f], clean[f]) - psnr(want, clean[f])) <= PSNR_DB
    finally:
        L.bm3d_b200_batch_destroy(b)
