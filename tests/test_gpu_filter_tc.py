"""FP16 Kronecker-form filter on tcgen05 (precision TC_F16) against the FP32 path.

The 2-D transforms run as 128-patch x 64 x 64 MMAs with FP16 operands, so
the result is not the reference's arithmetic; these tests bound its distance:
the same match lists go into the FP64 oracle (per-slot estimates within
55 dB basic, 70 dB final, on [0, 1] data), and the filtered clips stay within 0.05 dB PSNR of the FP32
path's against the clean clip, at sizes whose group count is no multiple of
the 16 groups of a CTA.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIGMA = [10.0, 7.0, 7.0]


def _clip(L, N, H, W, r, precision, planes=3, chroma=1, sigma=SIGMA):
    from bm3dcuda import _lib
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    for i in range(3):
        p.sigma[i] = sigma[i]
    p.radius = r
    p.chroma = chroma
    c = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), W, H, planes, 0, 0, N, ctypes.byref(p), 0))
    _lib.check(L.bm3d_b200_clip_set_precision(c, precision))
    return c


def _twostage(L, torch, c, noisy, N, P, H, W):
    from bm3dcuda import _lib
    stride = L.bm3d_b200_clip_stride(c)
    h = np.zeros((N, P, H, stride), np.float32)
    h[..., :W] = noisy.reshape(N, P, H, W)
    d_src = torch.from_numpy(h).cuda()
    d_b, d_d = torch.zeros_like(d_src), torch.zeros_like(d_src)
    _lib.check(L.bm3d_b200_clip_twostage(c, d_src.data_ptr(), d_b.data_ptr(), d_d.data_ptr(),
                                         None))
    torch.cuda.synchronize()
    _lib.check(L.bm3d_b200_clip_status(c))
    return d_b.cpu().numpy()[..., :W], d_d.cpu().numpy()[..., :W]


def test_precision_tc_f16_is_accepted_and_reported(cuda, engine_lib):
    from bm3dcuda import _lib
    L = engine_lib
    c = _clip(L, 2, 32, 32, 0, _lib.PRECISION_TC_F16, planes=1, chroma=0)
    try:
        assert L.bm3d_b200_clip_set_precision(c, 3) == _lib.ERR_INVALID
        assert L.bm3d_b200_clip_status(c) == _lib.OK
    finally:
        L.bm3d_b200_clip_destroy(c)


@pytest.mark.parametrize("radius", [0, 1])
def test_tc_f16_raw_accumulators_close_to_fp64(cuda, engine_lib, oracle, radius):
    """Basic and final stage accumulators (numerator and weight planes) of
    the tensor-core filter against the FP64 oracle given the GPU's lists."""
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    L = engine_lib
    N, H, W, r = 3, 40, 56, radius
    noisy, _ = S.chroma_clip(N, H, W, seed=71)

    def raw_stage(c, src, ref):
        stride = L.bm3d_b200_clip_stride(c)
        rf = L.bm3d_b200_clip_raw_frame_floats(c)

        def dev(a):
            h = np.zeros((N, 3, H, stride), np.float32)
            h[..., :W] = a
            return cuda.from_numpy(h).cuda()

        d_src = dev(src)
        d_ref = dev(ref) if ref is not None else None
        d_dst = cuda.zeros((N, rf), dtype=cuda.float32, device="cuda")
        _lib.check(L.bm3d_b200_clip_run(c, d_src.data_ptr(),
                                        d_ref.data_ptr() if ref is not None else None,
                                        d_dst.data_ptr(), _lib.DST_RAW, None))
        cuda.cuda.synchronize()
        _lib.check(L.bm3d_b200_clip_status(c))
        if r == 0:  # radius 0: the aggregated frames (no per-slot accumulators)
            ff = L.bm3d_b200_clip_frame_floats(c)
            raw = d_dst.cpu().numpy().reshape(-1)[:N * ff].reshape(N, 3, H, stride)[..., :W]
        else:
            raw = d_dst.cpu().numpy().reshape(N, 3, 2 * r + 1, 2, H, stride)[..., :W]
        nb = ctypes.c_int()
        L.bm3d_b200_clip_matches(c, 0, None, 0, ctypes.byref(nb))
        lists = []
        for n in range(N):
            buf = np.zeros((nb.value, 8, 3), np.int32)
            _lib.check(L.bm3d_b200_clip_matches(c, n, buf.ctypes.data, nb.value,
                                                ctypes.byref(nb)))
            lists.append(buf)
        return raw, lists

    c = _clip(L, N, H, W, r, _lib.PRECISION_TC_F16)
    try:
        raw, lists = raw_stage(c, noisy, None)
        basic = raw.copy() if r == 0 else np.stack(
            [raw[n, :, r, 0] / np.maximum(raw[n, :, r, 1], 1e-12)
             for n in range(N)]).astype(np.float32)
        raw_f, lists_f = raw_stage(c, noisy, basic)
    finally:
        L.bm3d_b200_clip_destroy(c)
    # per-slot estimates numerator / weight where the oracle's weight is
    # positive: hard thresholds flip coefficients that sit within the FP16
    # error of the threshold, which moves a group's weight by a whole
    # 1/nnz step, so the estimates (not the raw planes) carry the bound
    worst = {}
    for n in range(N):
        win = oracle.clip_window(noisy, n, r)
        want = oracle.port_bm3d(win, sigma=SIGMA, radius=r, chroma=True, fp64=True,
                                match_in=lists[n])
        rwin = oracle.clip_window(basic, n, r)
        want_f = oracle.port_bm3d(win, rwin, sigma=SIGMA, radius=r, chroma=True, fp64=True,
                                  match_in=lists_f[n])
        for stage, got, ref in (("basic", raw[n], want), ("final", raw_f[n], want_f)):
            for p in range(3):
                if r == 0:
                    e_got, e_ref = got[p], ref[p]
                else:
                    m = ref[p, :, 1] > 0
                    assert (got[p, :, 1][m] > 0).all()
                    e_got = got[p, :, 0][m] / got[p, :, 1][m]
                    e_ref = ref[p, :, 0][m] / ref[p, :, 1][m]
                mse = float(np.mean((e_got - e_ref) ** 2))
                db = 10 * np.log10(1.0 / max(mse, 1e-30))
                worst[(stage, p)] = min(worst.get((stage, p), 1e9), db)
    print("tc_f16 vs fp64 estimates, dB:", {k: round(v, 1) for k, v in worst.items()})
    for (stage, p), db in worst.items():
        assert db >= (70.0 if stage == "final" else 55.0), (stage, p, db)


@pytest.mark.parametrize("shape", [(4, 64, 96, 1, 3), (5, 72, 88, 2, 1), (3, 56, 120, 0, 1)])
def test_tc_f16_two_stage_psnr_matches_fp32(cuda, engine_lib, shape):
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    L = engine_lib
    N, H, W, r, P = shape
    if P == 3:
        noisy, clean = S.chroma_clip(N, H, W, seed=72)
    else:
        noisy, clean = S.piecewise_clip(N, H, W, seed=73)
        noisy, clean = noisy[:, None], clean[:, None]
    outs = {}
    for prec in (_lib.PRECISION_FP32, _lib.PRECISION_TC_F16):
        c = _clip(L, N, H, W, r, prec, planes=P, chroma=1 if P == 3 else 0)
        try:
            outs[prec] = _twostage(L, cuda, c, noisy, N, P, H, W)
        finally:
            L.bm3d_b200_clip_destroy(c)
    for stage in (0, 1):
        a, b = outs[_lib.PRECISION_FP32][stage], outs[_lib.PRECISION_TC_F16][stage]
        assert np.isfinite(b).all()
        for p in range(P):
            pa, pb = S.psnr(a[:, p], clean[:, p]), S.psnr(b[:, p], clean[:, p])
            assert pb >= pa - 0.05, (stage, p, pa, pb)
            # distance between the two paths far below the denoising error
            assert S.psnr(b[:, p], a[:, p]) >= pa + 15.0, (stage, p, S.psnr(b[:, p], a[:, p]), pa)


def test_tc_f16_host_pipeline_equals_device_path(cuda, engine_lib):
    """The chunked host-buffer pipeline runs the same tensor-core filter
    launches over its chunks: its frames equal the device path's."""
    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    L = engine_lib
    N, H, W, r = 9, 64, 96, 2
    noisy, _ = S.moving_piecewise_clip(N, H, W, seed=74)
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    p.sigma[0] = 8.0
    p.radius = r
    p.extractor_exp = 6
    c = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(c), W, H, 1, 0, 0, N, ctypes.byref(p), 0))
    try:
        _lib.check(L.bm3d_b200_clip_set_precision(c, _lib.PRECISION_TC_F16))
        stride = L.bm3d_b200_clip_stride(c)
        host = np.zeros((N, H, stride), np.float32)
        host[..., :W] = noisy
        d_src = torch.from_numpy(host).cuda()
        d_b, d_d = torch.zeros_like(d_src), torch.zeros_like(d_src)
        _lib.check(L.bm3d_b200_clip_twostage(c, d_src.data_ptr(), d_b.data_ptr(), d_d.data_ptr(),
                                             None))
        torch.cuda.synchronize()
        h_src = torch.from_numpy(host.copy()).pin_memory()
        h_dst = torch.zeros_like(h_src).pin_memory()
        _lib.check(L.bm3d_b200_clip_twostage_host(c, h_src.data_ptr(), h_dst.data_ptr(), None))
        np.testing.assert_array_equal(h_dst.numpy()[..., :W], d_d.cpu().numpy()[..., :W])
    finally:
        L.bm3d_b200_clip_destroy(c)
