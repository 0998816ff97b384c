"""Learned match proposal on the GPU.

* inference: the fused tensor-core network (tcgen05, BF16 operands, FP32 sums, 8-bit
  out) against the oracle's BF16 restatement, and the FP32 training network
  against the FP64 numpy network;
* training: teacher distances, loss and gradient of the FP32 forward/backward
  kernels against the FP64 oracle (itself pinned by finite differences);
* learned matching: lists and fallback flags identical to the C oracle for
  the same 8-bit embeddings; all-fallback lists identical to the exhaustive
  matcher's;
* what training gains: PSNR of the trained network above the coarse
  (downsampled-SSD) network on held-out clips at the same proposal counts;
* the clip pipeline with a proposer attached: PSNR at most 0.05 dB below
  the exhaustive search, host pipelined path identical to the device path.
"""
import ctypes

import numpy as np
import pytest

from oracle import proposer_ref as P

pytestmark = pytest.mark.gpu


def _frames(torch, arr):
    from bm3dcuda.learned import _device_frames
    return _device_frames(np.asarray(arr, np.float32))


@pytest.fixture(scope="module")
def prop(cuda, engine_lib):
    from bm3dcuda.learned import Proposer
    p = Proposer()
    yield p
    p.close()


def test_tensor_core_embeddings_vs_oracle(cuda, oracle, prop):
    from bm3dcuda import synthetic as S
    rng = np.random.default_rng(3)
    theta = (P.init_params(4.0) + rng.normal(0, 0.03, P.NPARAMS)).astype(np.float32)
    prop.set_params(theta)
    # sizes that cut the 122 x 12 output tiles unevenly, odd plane sides, a
    # width two columns past two whole tiles
    for (h, w) in [(70, 130), (45, 37), (200, 260), (96, 492)]:
        noisy, _ = S.texture_clip(2, h, w, seed=h + w)
        d_f = _frames(cuda, noisy)
        quant = prop.calibrate(d_f, w, h)
        got = prop.embed(d_f, w, h).cpu().numpy().astype(np.int32)
        assert got.min() >= 0 and got.max() <= 255 and got.std() > 4
        for f in range(2):
            want = oracle.quantize_embedding(oracle.port_proposer_embed_bf16(noisy[f], theta),
                                             quant).astype(np.int32)
            err = np.abs(got[f] - want)
            assert err.max() <= 2, (h, w, err.max())
            assert err.mean() <= 0.05
    prop.set_params(None)
    prop.set_quant(None)


def test_tensor_core_embeddings_full_size_vs_oracle(cuda, oracle, prop):
    """Two 1080p frames: 480 CTAs per frame, three per SM sharing the tensor
    memory, every accumulator slot of the ring reused many times. The oracle
    sums exactly and the tensor cores in FP32, so a last-place difference can
    flip the BF16 rounding of an intermediate activation; over 8.3 M outputs a
    frame then has a few tens of values off by 2 or 3 levels (measured: mean
    9e-5 levels, 65 values above 1, 13 at 3), spread over every tile position
    and repeatable run to run, which a race or an indexing error would not
    be. Hence a bound on the tail rather than on the single worst value."""
    from bm3dcuda import synthetic as S
    rng = np.random.default_rng(5)
    theta = (P.init_params(4.0) + rng.normal(0, 0.03, P.NPARAMS)).astype(np.float32)
    prop.set_params(theta)
    noisy, _ = S.texture_clip(2, 1080, 1920, seed=77)
    d_f = _frames(cuda, noisy)
    quant = prop.calibrate(d_f, 1920, 1080)
    got = prop.embed(d_f, 1920, 1080).cpu().numpy().astype(np.int32)
    try:
        for f in range(2):
            want = oracle.quantize_embedding(oracle.port_proposer_embed_bf16(noisy[f], theta),
                                             quant).astype(np.int32)
            err = np.abs(got[f] - want)
            assert err.max() <= 4, (f, err.max())
            assert (err > 1).sum() <= 2e-5 * err.size, (f, int((err > 1).sum()))
            assert err.mean() <= 1e-3, (f, err.mean())
        again = prop.embed(d_f, 1920, 1080).cpu().numpy().astype(np.int32)
        np.testing.assert_array_equal(again, got)  # deterministic
    finally:
        prop.set_params(None)
        prop.set_quant(None)


def test_fp32_training_network_vs_fp64(cuda, prop):
    rng = np.random.default_rng(4)
    theta = (P.init_params(2.0) + rng.normal(0, 0.05, P.NPARAMS)).astype(np.float32)
    prop.set_params(theta)
    frames = rng.random((2, 34, 50)).astype(np.float32)
    got = prop.embed_f32(_frames(cuda, frames), 50, 34).cpu().numpy()
    for f in range(2):
        want = P.forward(theta.astype(np.float64), P.down2(frames[f]))
        np.testing.assert_allclose(got[f], want, rtol=1e-4, atol=1e-4 * np.abs(want).max())
    prop.set_params(None)


def test_teacher_loss_and_gradient_vs_oracle(cuda, prop):
    from bm3dcuda.learned import teacher_distances
    rng = np.random.default_rng(5)
    H, W, U, T = 40, 56, 4, 0.5
    theta = (P.init_params(2.0) + rng.normal(0, 0.05, P.NPARAMS)).astype(np.float32)
    prop.set_params(theta)
    frames = rng.random((3, H, W)).astype(np.float32)
    n = 40
    samples = np.array([(int(rng.integers(0, 3)), int(rng.integers(0, 3)),
                         int(rng.integers(0, W - 7)), int(rng.integers(0, H - 7)))
                        for _ in range(n - 2)] + [(0, 1, 0, 0), (2, 2, W - 8, H - 8)], np.int32)
    d_f = _frames(cuda, frames)
    d_s = cuda.from_numpy(samples).cuda()
    tch = teacher_distances(d_f, W, H, d_s, U)
    want_t = P.teacher(list(frames), samples, U, W, H)
    got_t = tch.cpu().numpy()
    assert (np.isinf(got_t) == np.isinf(want_t)).all()
    fin = np.isfinite(want_t)
    np.testing.assert_allclose(got_t[fin], want_t[fin], rtol=1e-5, atol=1e-5)
    loss, grad = prop.loss_grad(d_f, W, H, d_s, tch, U, T)
    halves = [P.down2(f) for f in frames]
    want_loss, want_grad = P.loss_and_grad(theta.astype(np.float64), halves, samples, want_t, U, T)
    assert abs(loss - want_loss) <= 1e-3 * abs(want_loss) + 1e-6
    gs = np.abs(want_grad).max()
    assert np.abs(grad - want_grad).max() <= 2e-3 * gs
    # the parameter blocks all receive gradient
    assert np.abs(grad[:144]).max() > 0 and np.abs(grad[2480:4784]).max() > 0
    prop.set_params(None)


def _window(kind, r, h, w, seed):
    from bm3dcuda import synthetic as S
    fn = S.texture_clip if kind == "texture" else S.moving_piecewise_clip
    noisy, _ = fn(2 * r + 1, h, w, seed=seed)
    return noisy


@pytest.mark.parametrize("r,bs,cells", [(0, 8, (4, 4)), (2, 8, (4, 4)), (2, 8, (2, 2)), (1, 4, (2, 3)),
                                        (2, 6, (8, 1))])
def test_learned_lists_identical_to_oracle(cuda, oracle, prop, r, bs, cells):
    from bm3dcuda.learned import learned_match
    rng = np.random.default_rng(6 + r)
    prop.set_params((P.init_params(8.0) + rng.normal(0, 0.02, P.NPARAMS)).astype(np.float32))
    win = _window("texture", r, 52, 76, seed=20 + r)
    d_f = _frames(cuda, win)
    prop.calibrate(d_f, 76, 52)
    emb = prop.embed(d_f, 76, 52)
    e8 = emb.cpu().numpy()
    mixed = False
    for fb in (0.0, 0.04, 0.08):
        kw = dict(block_step=bs, radius=r, cells_spatial=cells[0], cells_temporal=cells[1],
                  fallback_ssd=fb)
        got, gfell = learned_match(prop, win, embeddings=emb, **kw)
        want, wfell = oracle.port_learned_match(win, e8, **kw)
        np.testing.assert_array_equal(got, want, err_msg=f"fallback_ssd {fb}")
        np.testing.assert_array_equal(gfell, wfell)
        mixed |= 0 < wfell.sum() < len(wfell)
    assert mixed  # both the learned and the fallback path were exercised
    prop.set_params(None)
    prop.set_quant(None)


@pytest.mark.parametrize("r", [0, 2])
def test_all_fallback_is_the_exhaustive_matcher(cuda, prop, r):
    from bm3dcuda.learned import exhaustive_matches, learned_match
    win = _window("texture", r, 48, 64, seed=30 + r)
    got, fell = learned_match(prop, win, radius=r, fallback_ssd=1e-30)
    assert fell.all()
    np.testing.assert_array_equal(got, exhaustive_matches(win, radius=r))


def _twostage_psnr(L, torch, prop, noisy, clean, sigma, cells):
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    N, H, W = noisy.shape
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    p.sigma[0] = sigma
    p.radius = 2
    p.extractor_exp = 6
    c = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), W, H, 1, 0, 0, N, ctypes.byref(p), 0))
    try:
        host = np.zeros((N, H, L.bm3d_b200_clip_stride(c)), np.float32)
        host[..., :W] = noisy
        d_src = torch.from_numpy(host).cuda()
        d_b, d_d = torch.zeros_like(d_src), torch.zeros_like(d_src)
        if prop is not None:
            _lib.check(L.bm3d_b200_clip_set_proposer(c, prop.handle, cells[0], cells[1], 0.0))
        _lib.check(L.bm3d_b200_clip_twostage(c, d_src.data_ptr(), d_b.data_ptr(),
                                             d_d.data_ptr(), None))
        torch.cuda.synchronize()
        return S.psnr(d_d.cpu().numpy()[..., :W], clean)
    finally:
        L.bm3d_b200_clip_destroy(c)


def test_training_gains_over_coarse_network(cuda, engine_lib, prop):
    """Trained on config-1-style clips (moving piecewise scenes, noise 10/255),
    the network must denoise held-out clips of that kind better than the
    coarse network (downsampled SSD) at the same proposal counts; training
    from the exhaustive search's distances must also lower the loss."""
    from bm3dcuda import synthetic as S
    r = 2
    train = [S.moving_piecewise_clip(5, 240, 320, seed=100 + i)[0] for i in range(6)]
    noisy, clean = S.moving_piecewise_clip(8, 240, 320, seed=901)
    prop.set_params(None)
    prop.set_quant(None)
    coarse = [_twostage_psnr(engine_lib, cuda, prop, noisy, clean, 10.0, c)
              for c in [(2, 2), (4, 4)]]
    losses = prop.fit(train, radius=r, sigma=10.0, steps=300, lr=2e-3)
    trained = [_twostage_psnr(engine_lib, cuda, prop, noisy, clean, 10.0, c)
               for c in [(2, 2), (4, 4)]]
    assert losses[-1] < 0.5 * losses[0]
    for a, b in zip(coarse, trained):
        assert b >= a + 0.03, (coarse, trained)
    prop.set_params(None)
    prop.set_quant(None)


def test_clip_pipeline_with_proposer(cuda, engine_lib, prop):
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    L = engine_lib
    N, H, W, r = 7, 72, 96, 2
    noisy, clean = S.texture_clip(N, H, W, seed=40)
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    p.sigma[0] = 5.0
    p.radius = r
    p.extractor_exp = 6
    c = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), W, H, 1, 0, 0, N, ctypes.byref(p), 0))
    try:
        stride = L.bm3d_b200_clip_stride(c)
        host = np.zeros((N, H, stride), np.float32)
        host[..., :W] = noisy
        d_src = torch.from_numpy(host).cuda()
        d_basic, d_dst = torch.zeros_like(d_src), torch.zeros_like(d_src)

        def run():
            _lib.check(L.bm3d_b200_clip_twostage(c, d_src.data_ptr(), d_basic.data_ptr(),
                                                 d_dst.data_ptr(), None))
            torch.cuda.synchronize()
            return d_dst.cpu().numpy()[..., :W].copy()

        exh = run()
        _lib.check(L.bm3d_b200_clip_set_proposer(c, prop.handle, 4, 4, 0.0))
        lrn = run()
        blocks, fb = ctypes.c_longlong(), ctypes.c_longlong()
        _lib.check(L.bm3d_b200_clip_learned_stats(c, ctypes.byref(blocks), ctypes.byref(fb), 1))
        assert blocks.value == 2 * N * 12 * 9 and fb.value == 0
        assert S.psnr(lrn, clean) >= S.psnr(exh, clean) - 0.05
        # with the fallback on, some blocks take the exhaustive search
        _lib.check(L.bm3d_b200_clip_set_proposer(c, prop.handle, 4, 4, 1.0))
        lrn_fb = run()
        _lib.check(L.bm3d_b200_clip_learned_stats(c, ctypes.byref(blocks), ctypes.byref(fb), 1))
        assert 0 < fb.value < blocks.value
        assert S.psnr(lrn_fb, clean) >= S.psnr(exh, clean) - 0.05
        # the pipelined host path computes the same frames
        h_src = torch.from_numpy(host.copy()).pin_memory()
        h_dst = torch.zeros_like(h_src).pin_memory()
        _lib.check(L.bm3d_b200_clip_twostage_host(c, h_src.data_ptr(), h_dst.data_ptr(), None))
        np.testing.assert_array_equal(h_dst.numpy()[..., :W], lrn_fb)
        _lib.check(L.bm3d_b200_clip_set_proposer(c, None, 4, 4, 0.0))
        np.testing.assert_array_equal(run(), exh)
    finally:
        L.bm3d_b200_clip_destroy(c)


@pytest.mark.parametrize("precision", [0, 1])
def test_final_stage_reuses_basic_lists(cuda, engine_lib, prop, precision):
    """BASIC_LISTS: every final-stage list is the block's basic-stage list
    ordered by the reference's block distance on the basic estimate, ties
    keeping the basic order - equal to the oracle's re-scoring of the same
    lists on the same basic estimate (whatever the filter precision that made
    that estimate); the pipelined host path computes the same frames as the
    device path."""
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    from oracle import oracle as O
    L = engine_lib
    N, H, W, r = 6, 64, 88, 2
    noisy, clean = S.texture_clip(N, H, W, seed=41)
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    p.sigma[0] = 5.0
    p.radius = r
    p.extractor_exp = 6
    c = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), W, H, 1, 0, 0, N, ctypes.byref(p), 0))
    try:
        _lib.check(L.bm3d_b200_clip_set_precision(c, precision))
        stride = L.bm3d_b200_clip_stride(c)
        host = np.zeros((N, H, stride), np.float32)
        host[..., :W] = noisy
        d_src = torch.from_numpy(host).cuda()
        d_basic, d_dst = torch.zeros_like(d_src), torch.zeros_like(d_src)
        _lib.check(L.bm3d_b200_clip_set_proposer(c, prop.handle, 2, 2, 4.0))
        _lib.check(L.bm3d_b200_clip_set_final_matching(c, 1))
        nb = ctypes.c_int()

        def lists():
            L.bm3d_b200_clip_matches(c, 0, None, 0, ctypes.byref(nb))
            out = []
            for n in range(N):
                buf = np.zeros((nb.value, 8, 3), np.int32)
                _lib.check(L.bm3d_b200_clip_matches(c, n, buf.ctypes.data, nb.value,
                                                    ctypes.byref(nb)))
                out.append(buf)
            return out

        _lib.check(L.bm3d_b200_clip_run(c, d_src.data_ptr(), None, d_basic.data_ptr(),
                                        _lib.DST_AGGREGATED, None))
        torch.cuda.synchronize()
        basic_lists = lists()
        _lib.check(L.bm3d_b200_clip_twostage(c, d_src.data_ptr(), d_basic.data_ptr(),
                                             d_dst.data_ptr(), None))
        torch.cuda.synchronize()
        _lib.check(L.bm3d_b200_clip_status(c))
        final_lists = lists()
        basic = d_basic.cpu().numpy()[..., :W].copy()
        out = d_dst.cpu().numpy()[..., :W].copy()
        moved = 0
        for n in range(N):
            win = O.clip_window(basic[:, None], n, r)[0]  # [2r+1][H][W]
            want = O.port_rescore(win, basic_lists[n])
            np.testing.assert_array_equal(final_lists[n], want, err_msg=f"window {n}")
            moved += int((want != basic_lists[n]).any(axis=(1, 2)).sum())
        assert moved > 0  # the basic estimate re-orders some lists
        # the pipelined host path re-scores the same lists
        h_src = torch.from_numpy(host.copy()).pin_memory()
        h_dst = torch.zeros_like(h_src).pin_memory()
        _lib.check(L.bm3d_b200_clip_twostage_host(c, h_src.data_ptr(), h_dst.data_ptr(), None))
        np.testing.assert_array_equal(h_dst.numpy()[..., :W], out)
        assert S.psnr(out, clean) > S.psnr(noisy, clean) + 2.0
    finally:
        L.bm3d_b200_clip_destroy(c)


def test_final_stage_basic_order_keeps_the_basic_lists(cuda, engine_lib, prop):
    """BASIC_ORDER: the final stage filters with the basic stage's lists as
    they are (same positions, same order); the pipelined host path computes
    the same frames as the device path."""
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    L = engine_lib
    N, H, W, r = 6, 64, 88, 2
    noisy, clean = S.texture_clip(N, H, W, seed=43)
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    p.sigma[0] = 5.0
    p.radius = r
    p.extractor_exp = 6
    c = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), W, H, 1, 0, 0, N, ctypes.byref(p), 0))
    try:
        assert L.bm3d_b200_clip_set_final_matching(c, 3) == _lib.ERR_INVALID
        stride = L.bm3d_b200_clip_stride(c)
        host = np.zeros((N, H, stride), np.float32)
        host[..., :W] = noisy
        d_src = torch.from_numpy(host).cuda()
        d_basic, d_dst = torch.zeros_like(d_src), torch.zeros_like(d_src)
        _lib.check(L.bm3d_b200_clip_set_proposer(c, prop.handle, 2, 2, 4.0))
        _lib.check(L.bm3d_b200_clip_set_final_matching(c, 2))
        nb = ctypes.c_int()

        def lists():
            L.bm3d_b200_clip_matches(c, 0, None, 0, ctypes.byref(nb))
            out = np.zeros((N, nb.value, 8, 3), np.int32)
            for n in range(N):
                _lib.check(L.bm3d_b200_clip_matches(c, n, out[n].ctypes.data, nb.value,
                                                    ctypes.byref(nb)))
            return out

        _lib.check(L.bm3d_b200_clip_run(c, d_src.data_ptr(), None, d_basic.data_ptr(),
                                        _lib.DST_AGGREGATED, None))
        torch.cuda.synchronize()
        basic_lists = lists()
        _lib.check(L.bm3d_b200_clip_twostage(c, d_src.data_ptr(), d_basic.data_ptr(),
                                             d_dst.data_ptr(), None))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(lists(), basic_lists)
        out = d_dst.cpu().numpy()[..., :W].copy()
        h_src = torch.from_numpy(host.copy()).pin_memory()
        h_dst = torch.zeros_like(h_src).pin_memory()
        _lib.check(L.bm3d_b200_clip_twostage_host(c, h_src.data_ptr(), h_dst.data_ptr(), None))
        np.testing.assert_array_equal(h_dst.numpy()[..., :W], out)
        assert S.psnr(out, clean) > S.psnr(noisy, clean) + 2.0
    finally:
        L.bm3d_b200_clip_destroy(c)


def test_c5_learned_4k_bm_range16_recall_and_psnr(cuda, engine_lib):
    """C5: 3840x2160, V-BM3D radius 2, bm_range 16, sigma 10 (5 frames of the
    seeded texture scene). A proposer trained on the GPU (config-1-style
    clips) scores 4 cells per search: match recall of the basic stage's
    centre window against the exhaustive lists, and the two-stage PSNR
    against the exhaustive search (the metric allows a loss of 0.05 dB), with
    the final stage searching again and re-scoring the basic lists."""
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    from bm3dcuda.learned import Proposer, exhaustive_matches, learned_match, recall
    L = engine_lib
    N, H, W, r, R = 5, 2160, 3840, 2, 16
    noisy, clean = S.texture_clip(N, H, W, noise=10 / 255, seed=5)
    prop = Proposer()
    try:
        train = [S.moving_piecewise_clip(5, 240, 320, seed=100 + i)[0] for i in range(6)]
        prop.fit(train, radius=r, sigma=10.0, steps=300, lr=2e-3)
        win = np.ascontiguousarray(noisy[N // 2 - r:N // 2 + r + 1])
        ex = exhaustive_matches(win, bm_range=R, radius=r)
        lm, _ = learned_match(prop, win, bm_range=R, radius=r, cells_spatial=4, cells_temporal=4)
        rec = recall(lm, ex)
        assert rec >= 0.9, rec
        p = _lib.Params()
        L.bm3d_b200_params_default(ctypes.byref(p))
        p.sigma[0] = 10.0
        p.bm_range[0] = R
        p.radius = r
        p.extractor_exp = 6
        c = ctypes.c_void_p()
        _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), W, H, 1, 0, 0, N, ctypes.byref(p), 0))
        try:
            stride = L.bm3d_b200_clip_stride(c)
            host = np.zeros((N, H, stride), np.float32)
            host[..., :W] = noisy
            d_src = torch.from_numpy(host).cuda()
            d_b, d_d = torch.zeros_like(d_src), torch.zeros_like(d_src)

            def run():
                _lib.check(L.bm3d_b200_clip_twostage(c, d_src.data_ptr(), d_b.data_ptr(),
                                                     d_d.data_ptr(), None))
                torch.cuda.synchronize()
                return S.psnr(d_d.cpu().numpy()[..., :W], clean)

            exhaustive = run()
            _lib.check(L.bm3d_b200_clip_set_proposer(c, prop.handle, 4, 4, 2.0))
            for mode in (0, 1):
                _lib.check(L.bm3d_b200_clip_set_final_matching(c, mode))
                delta = run() - exhaustive
                assert delta >= -0.05, (mode, delta)
        finally:
            L.bm3d_b200_clip_destroy(c)
        print(f"C5: recall {rec:.4f}")
    finally:
        prop.close()


@pytest.mark.parametrize("tau", [0.0, 2.0])
def test_clip_learned_lists_equal_the_standalone_matcher(cuda, engine_lib, prop, tau):
    """The clip's learned lists (its own embeddings of the whole clip, windows
    batched in one launch, fallback threshold from fallback_tau) equal those of
    bm3d_b200_learned_match on each window's frames alone (first, middle and
    last windows: replicated borders included)."""
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    from bm3dcuda.learned import learned_match
    L = engine_lib
    N, H, W, r, sigma = 7, 72, 104, 2, 5.0
    noisy, _ = S.moving_piecewise_clip(N, H, W, seed=45)
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    p.sigma[0] = sigma
    p.radius = r
    c = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), W, H, 1, 0, 0, N, ctypes.byref(p), 0))
    try:
        _lib.check(L.bm3d_b200_clip_set_proposer(c, prop.handle, 2, 2, tau))
        stride = L.bm3d_b200_clip_stride(c)
        host = np.zeros((N, H, stride), np.float32)
        host[..., :W] = noisy
        d_src = torch.from_numpy(host).cuda()
        d_dst = torch.zeros_like(d_src)
        _lib.check(L.bm3d_b200_clip_run(c, d_src.data_ptr(), None, d_dst.data_ptr(),
                                        _lib.DST_AGGREGATED, None))
        torch.cuda.synchronize()
        _lib.check(L.bm3d_b200_clip_status(c))
        nb = ctypes.c_int()
        L.bm3d_b200_clip_matches(c, 0, None, 0, ctypes.byref(nb))
        sg = np.float32(sigma) / np.float32(255.0)  # the clip's FP32 threshold
        fb = float(np.float32(tau) * np.float32(128.0) * sg * sg)
        for n in (0, 3, N - 1):
            got = np.zeros((nb.value, 8, 3), np.int32)
            _lib.check(L.bm3d_b200_clip_matches(c, n, got.ctypes.data, nb.value,
                                                ctypes.byref(nb)))
            win = np.stack([noisy[min(max(n - r + z, 0), N - 1)] for z in range(2 * r + 1)])
            want, _ = learned_match(prop, win, radius=r, cells_spatial=2, cells_temporal=2,
                                    fallback_ssd=fb)
            np.testing.assert_array_equal(got, want, err_msg=f"window {n}")
    finally:
        L.bm3d_b200_clip_destroy(c)
