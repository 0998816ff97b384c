"""Argument handling of the Python mirror of BM3D / BM3Dv2 / VAggregate.

Messages and checks follow BM3DCreate (source/source.cpp:457-634); these
errors are raised before any device work, so they run without a GPU.
"""
import numpy as np
import pytest

from bm3dcuda import BM3D, BM3Dv2, BM3DError, Clip


def gray(n=3, h=24, w=32):
    return Clip.from_array(np.zeros((n, h, w), np.float32))


@pytest.mark.parametrize("kw,msg", [
    (dict(sigma=-1.0), '"sigma" must be non-negative'),
    (dict(sigma=[3.0, -2.0]), '"sigma" must be non-negative'),
    (dict(block_step=0), '"block_step" must be in range [1, 8]'),
    (dict(block_step=[8, 9]), '"block_step" must be in range [1, 8]'),
    (dict(bm_range=0), '"bm_range" must be positive'),
    (dict(radius=-1), '"radius" must be non-negative'),
    (dict(ps_num=0), '"ps_num" must be in range [1, 8]'),
    (dict(ps_num=9), '"ps_num" must be in range [1, 8]'),
    (dict(ps_range=0), '"ps_range" must be positive'),
    (dict(chroma=True), 'clip format must be YUV444 when "chroma" is true'),
])
def test_bm3d_argument_errors(kw, msg):
    with pytest.raises(BM3DError) as e:
        BM3D(gray(), **kw)
    assert str(e.value) == "BM3D: " + msg


def test_format_errors():
    integer = Clip([np.zeros((2, 16, 16), np.uint8)], "GRAY8")
    with pytest.raises(BM3DError, match="only constant format 32bit float input supported"):
        BM3D(integer)
    half = Clip([np.zeros((2, 16, 16), np.float16)], "GRAYH")
    with pytest.raises(BM3DError, match="only constant format 32bit float input supported"):
        BM3D(half)


def test_ref_mismatch_errors():
    c = gray()
    with pytest.raises(BM3DError, match='"ref" must be of the same format as "clip"'):
        BM3D(c, ref=Clip.from_array(np.zeros((3, 3, 24, 32), np.float32)))
    with pytest.raises(BM3DError, match='"ref" must be of the same dimensions as "clip"'):
        BM3D(c, ref=gray(3, 24, 40))
    with pytest.raises(BM3DError, match='"ref" must be of the same number of frames as "clip"'):
        BM3D(c, ref=gray(4))


def test_bm3dv2_passes_through_when_nothing_is_processed():
    c = gray()
    assert BM3Dv2(c, sigma=0.0) is c
    yuv = Clip.from_array(np.zeros((2, 3, 16, 16), np.float32))
    assert BM3Dv2(yuv, sigma=[0.0]) is yuv  # carry-forward of the last sigma


def test_sigma_carry_forward_and_process_flags():
    from bm3dcuda import _parse
    yuv = Clip.from_array(np.zeros((2, 3, 16, 16), np.float32))
    try:
        a = _parse(yuv, None, [5.0, 0.0], None, None, None, None, None, None, None, None, None, None)
    except BM3DError as e:  # no device here: everything before the device check passed
        assert "invalid device ID" in str(e)
        return
    assert a.sigma == [5.0, 0.0, 0.0]
    assert a.process == [True, False, False]
