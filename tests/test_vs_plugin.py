"""The native VapourSynth filter layer (libbm3dcuda_vs.so), driven through an
in-process fake VapourSynth core (tests/vs_fakecore).

CPU tests: plugin identity, registered argument strings and the create-time
argument errors (all raised before any device call, source/source.cpp:476-595).
GPU tests: frames produced through the plugin against the oracle and against
the Python mirror of the same functions.
"""
import numpy as np
import pytest

import vs_fakecore as vsf

# the reference's argument string (source/source.cpp:1001-1017), then the
# optional learned-proposal arguments this engine adds
BM3D_ARGS = ("clip:clip;ref:clip:opt;sigma:float[]:opt;block_step:int[]:opt;bm_range:int[]:opt;"
             "radius:int:opt;ps_num:int[]:opt;ps_range:int[]:opt;chroma:int:opt;device_id:int:opt;"
             "fast:int:opt;extractor_exp:int:opt;zero_init:int:opt;"
             "proposer:data:opt;proposer_cells:int[]:opt;proposer_tau:float:opt;")


@pytest.fixture(scope="module")
def core(engine_lib):
    vsf.build()
    return vsf.Core()


def test_plugin_identity_and_signatures(core):
    assert core.plugin_id == "com.wolframrhodium.bm3dcuda"
    assert core.namespace == "bm3dcuda"
    assert core.function_args("BM3D") == BM3D_ARGS
    assert core.function_args("BM3Dv2") == BM3D_ARGS
    assert core.function_args("VAggregate") == "clip:clip;src:clip;planes:int[];"


@pytest.mark.parametrize("kw,msg", [
    (dict(sigma=-1.0), '"sigma" must be non-negative'),
    (dict(block_step=9), '"block_step" must be in range [1, 8]'),
    (dict(bm_range=0), '"bm_range" must be positive'),
    (dict(radius=-1), '"radius" must be non-negative'),
    (dict(ps_num=0), '"ps_num" must be in range [1, 8]'),
    (dict(ps_range=0), '"ps_range" must be positive'),
    (dict(chroma=1), 'clip format must be YUV444 when "chroma" is true'),
])
def test_plugin_argument_errors(core, kw, msg):
    c = core.clip(np.zeros((2, 24, 32), np.float32))
    with pytest.raises(vsf.VSError) as e:
        core.invoke("BM3D", clip=c, **kw)
    assert str(e.value) == "BM3D: " + msg
    core.free(c)


def test_plugin_format_and_ref_errors(core):
    c8 = core.clip(np.zeros((2, 16, 16), np.uint8), "GRAY8")
    with pytest.raises(vsf.VSError, match="only constant format 32bit float input supported"):
        core.invoke("BM3D", clip=c8)
    c = core.clip(np.zeros((2, 16, 16), np.float32))
    r_fmt = core.clip([np.zeros((2, 16, 16), np.float32)] * 3, "YUV444PS")
    with pytest.raises(vsf.VSError, match='"ref" must be of the same format as "clip"'):
        core.invoke("BM3D", clip=c, ref=r_fmt)
    r_dim = core.clip(np.zeros((2, 16, 24), np.float32))
    with pytest.raises(vsf.VSError, match='"ref" must be of the same dimensions as "clip"'):
        core.invoke("BM3D", clip=c, ref=r_dim)
    r_len = core.clip(np.zeros((3, 16, 16), np.float32))
    with pytest.raises(vsf.VSError, match='"ref" must be of the same number of frames as "clip"'):
        core.invoke("BM3Dv2", clip=c, ref=r_len)
    for n in (c8, c, r_fmt, r_dim, r_len):
        core.free(n)


def test_bm3dv2_passthrough_without_device(core):
    data = np.random.default_rng(0).random((2, 16, 16)).astype(np.float32)
    c = core.clip(data)
    out = core.invoke("BM3Dv2", clip=c, sigma=0.0)
    planes, _ = core.frames(out)
    np.testing.assert_array_equal(planes[0], data)
    core.free(out)
    core.free(c)


# ---------------------------------------------------------------------------
# GPU: frames through the plugin
# ---------------------------------------------------------------------------
gpu = pytest.mark.gpu


@gpu
def test_plugin_bm3d_spatial_vs_oracle(core, cuda, oracle):
    from bm3dcuda import synthetic as S
    noisy, _ = S.piecewise_clip(3, 48, 64, seed=51)
    c = core.clip(noisy)
    basic = core.invoke("BM3D", clip=c, sigma=10.0)
    got, props = core.frames(basic)
    assert props == {}
    for n in range(3):
        want = oracle.port_bm3d(noisy[n][None, None], sigma=10.0)[0]
        assert np.abs(got[0][n] - want).max() <= 1e-4
    final = core.invoke("BM3D", clip=c, ref=basic, sigma=10.0, fast=0)
    got_f, _ = core.frames(final)
    for n in range(3):
        want = oracle.port_bm3d(noisy[n][None, None], got[0][n][None, None], sigma=10.0)[0]
        assert np.abs(got_f[0][n] - want).max() <= 1e-4
    for nd in (final, basic, c):
        core.free(nd)


@gpu
def test_plugin_raw_vbm3d_and_vaggregate_vs_oracle(core, cuda, oracle):
    from bm3dcuda import synthetic as S
    noisy, _ = S.texture_clip(5, 40, 48, seed=52)
    r = 2
    c = core.clip(noisy)
    raw = core.invoke("BM3D", clip=c, sigma=5.0, radius=r)
    w, h, n, _ = core.info(raw)
    assert (w, h, n) == (48, 40 * 2 * (2 * r + 1), 5)
    raw_planes, props = core.frames(raw)
    assert props == {"BM3D_V_radius": r, "BM3D_V_process": [1, 1, 1]}
    raws = raw_planes[0].reshape(5, 2 * r + 1, 2, 40, 48)
    for k in range(5):
        want = oracle.port_bm3d(oracle.clip_window(noisy[:, None], k, r), sigma=5.0, radius=r)[0]
        np.testing.assert_allclose(raws[k], want, rtol=1e-5, atol=1e-5)
    # The fake core caches no frames: VAggregate re-requests (recomputes) the
    # raw frames, so use pre-rounded, order-independent sums to compare exactly.
    raw = core.invoke("BM3D", clip=c, sigma=5.0, radius=r, extractor_exp=6)
    raws = core.frames(raw)[0][0].reshape(5, 2 * r + 1, 2, 40, 48)
    agg = core.invoke("VAggregate", clip=raw, src=c, planes=[0])
    got, _ = core.frames(agg)
    for k in range(5):
        idx = [min(max(k - r + i, 0), 4) for i in range(2 * r + 1)]
        want = oracle.port_vaggregate(np.stack([raws[i] for i in idx]), k, 5)
        np.testing.assert_array_equal(got[0][k], want)  # same slabs in, same sums out
    v2 = core.invoke("BM3Dv2", clip=c, sigma=5.0, radius=r)
    got2, _ = core.frames(v2)
    want2 = oracle.clip_bm3d_v2(oracle.port_bm3d, noisy[:, None], None, radius=r, chroma=False,
                                sigma=5.0)[:, 0]
    assert np.abs(got2[0] - want2).max() <= 1e-4
    for nd in (v2, agg, raw, c):
        core.free(nd)


@gpu
def test_plugin_chroma_and_subsampled(core, cuda):
    from bm3dcuda import BM3D, BM3Dv2, Clip
    from bm3dcuda import synthetic as S
    noisy, _ = S.chroma_clip(3, 40, 48, seed=53)
    planes = [noisy[:, i] for i in range(3)]
    c = core.clip(planes, "YUV444PS")
    out = core.invoke("BM3Dv2", clip=c, sigma=[10.0, 7.0], radius=1, chroma=1, extractor_exp=6)
    got, _ = core.frames(out, 3)
    want = BM3Dv2(Clip(planes, "YUV444PS"), sigma=[10.0, 7.0], radius=1, chroma=True,
                  extractor_exp=6)
    for p in range(3):
        np.testing.assert_array_equal(got[p], want.planes[p])
    y, _ = S.piecewise_clip(2, 48, 64, seed=54)
    u, _ = S.piecewise_clip(2, 24, 32, seed=55)
    v, _ = S.piecewise_clip(2, 24, 32, seed=56)
    c420 = core.clip([y, u, v], "YUV420PS")
    o420 = core.invoke("BM3D", clip=c420, sigma=[8.0, 0.0, 4.0], extractor_exp=6)
    got420, _ = core.frames(o420, 3)
    want420 = BM3D(Clip([y, u, v], "YUV420PS"), sigma=[8.0, 0.0, 4.0], extractor_exp=6)
    for p in range(3):
        np.testing.assert_array_equal(got420[p], want420.planes[p])
    np.testing.assert_array_equal(got420[1], u)  # unprocessed plane copied
    for nd in (o420, c420, out, c):
        core.free(nd)


@gpu
def test_plugin_learned_proposer_argument(core, cuda, tmp_path):
    """BM3Dv2 with the optional proposer argument (a saved trained proposer):
    the streamed plugin path matches blocks with it exactly as the clip
    pipeline with the same proposer attached; the argument is rejected where
    it does not apply and for unreadable files."""
    import ctypes

    import torch
    from bm3dcuda import _lib
    from bm3dcuda import synthetic as S
    from bm3dcuda.learned import Proposer
    L = _lib.lib()
    prop = Proposer()
    train = [S.moving_piecewise_clip(5, 64, 96, seed=90 + i)[0] for i in range(2)]
    prop.fit(train, radius=2, sigma=10.0, steps=20, lr=2e-3)
    path = str(tmp_path / "proposer.bin")
    prop.save(path)
    again = Proposer.load(path)
    np.testing.assert_array_equal(again.params(), prop.params())
    np.testing.assert_array_equal(again.quant(), prop.quant())
    again.close()
    N, H, W, r = 6, 48, 72, 2
    noisy, _ = S.texture_clip(N, H, W, seed=58)
    c = core.clip(noisy)
    out = core.invoke("BM3Dv2", clip=c, sigma=5.0, radius=r, extractor_exp=6, proposer=path,
                      proposer_cells=[2, 1], proposer_tau=4.0)
    got, _ = core.frames(out)
    p = _lib.Params()
    L.bm3d_b200_params_default(ctypes.byref(p))
    p.sigma[0] = 5.0
    p.radius = r
    p.extractor_exp = 6
    h = ctypes.c_void_p()
    _lib.check(L.bm3d_b200_clip_create(ctypes.byref(h), W, H, 1, 0, 0, N, ctypes.byref(p), 0))
    try:
        _lib.check(L.bm3d_b200_clip_set_proposer(h, prop.handle, 2, 1, 4.0))
        stride = L.bm3d_b200_clip_stride(h)
        host = np.zeros((N, H, stride), np.float32)
        host[..., :W] = noisy
        d_src = torch.from_numpy(host).cuda()
        d_dst = torch.zeros_like(d_src)
        _lib.check(L.bm3d_b200_clip_run(h, d_src.data_ptr(), None, d_dst.data_ptr(),
                                        _lib.DST_AGGREGATED, None))
        torch.cuda.synchronize()
        want = d_dst.cpu().numpy()[..., :W]
    finally:
        L.bm3d_b200_clip_destroy(h)
    np.testing.assert_array_equal(got[0], want)
    # the Python mirror with the same optional arguments (file or object)
    from bm3dcuda import BM3Dv2, Clip
    for src in (path, prop):
        mirror = BM3Dv2(Clip.from_array(noisy), sigma=5.0, radius=r, extractor_exp=6,
                        proposer=src, proposer_cells=[2, 1], proposer_tau=4.0)
        np.testing.assert_array_equal(mirror.planes[0], want)
    plain = core.frames(core.invoke("BM3Dv2", clip=c, sigma=5.0, radius=r, extractor_exp=6))[0]
    assert not np.array_equal(plain[0], got[0])  # the proposer changed the matching
    with pytest.raises(vsf.VSError, match='"proposer" applies to BM3Dv2 with radius > 0'):
        core.invoke("BM3D", clip=c, sigma=5.0, proposer=path)
    with pytest.raises(vsf.VSError, match='cannot open "proposer" file'):
        core.invoke("BM3Dv2", clip=c, sigma=5.0, radius=1, proposer=path + ".missing")
    with pytest.raises(vsf.VSError, match='"proposer_cells" must be in range'):
        core.invoke("BM3Dv2", clip=c, sigma=5.0, radius=1, proposer=path, proposer_cells=9)
    core.free(out)
    core.free(c)
    prop.close()


# ---------------------------------------------------------------------------
# the run-time-compiled plugin's surface (libbm3dcuda_rtc_vs.so)
# ---------------------------------------------------------------------------
RTC_ARGS = BM3D_ARGS.replace(
    "extractor_exp:int:opt;",
    "extractor_exp:int:opt;bm_error_s:data[]:opt;transform_2d_s:data[]:opt;"
    "transform_1d_s:data[]:opt;")


@pytest.fixture(scope="module")
def rtc_core(engine_lib):
    vsf.build()
    return vsf.Core(vsf.RTC_PLUGIN_SO)


def test_rtc_plugin_identity_and_signatures(rtc_core):
    assert rtc_core.plugin_id == "com.wolframrhodium.bm3dcuda_rtc"
    assert rtc_core.namespace == "bm3dcuda_rtc"
    assert rtc_core.function_args("BM3D") == RTC_ARGS
    assert rtc_core.function_args("BM3Dv2") == RTC_ARGS
    assert rtc_core.function_args("VAggregate") == "clip:clip;src:clip;planes:int[];"


def test_rtc_plugin_argument_errors(rtc_core):
    c = rtc_core.clip(np.zeros((2, 24, 32), np.float32))
    with pytest.raises(vsf.VSError) as e:
        rtc_core.invoke("BM3D", clip=c, sigma=-1.0)
    assert str(e.value) == 'BM3D_RTC: "sigma" must be non-negative'
    rtc_core.free(c)


@gpu
def test_rtc_plugin_variants_vs_python_mirror(rtc_core, cuda):
    from bm3dcuda import Clip
    from bm3dcuda import rtc as R
    from bm3dcuda import synthetic as S
    noisy, _ = S.texture_clip(4, 40, 48, seed=57)
    c = rtc_core.clip(noisy)
    with pytest.raises(vsf.VSError, match="BM3D_RTC: invalid 'transform_2d_s': dft"):
        rtc_core.invoke("BM3D", clip=c, transform_2d_s="DFT")
    kw = dict(sigma=6.0, radius=1, extractor_exp=6)
    out = rtc_core.invoke("BM3Dv2", clip=c, bm_error_s=["ZSAD"], transform_2d_s=["bior1.5"],
                          transform_1d_s=["Haar"], **kw)
    got, _ = rtc_core.frames(out)
    want = R.BM3Dv2(Clip.from_array(noisy), bm_error_s=["zsad"], transform_2d_s=["bior1.5"],
                    transform_1d_s=["haar"], **kw)
    np.testing.assert_array_equal(got[0], want.planes[0])
    for nd in (out, c):
        rtc_core.free(nd)
