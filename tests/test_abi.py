"""The C ABI library: loads, exports every declared symbol, validates on the host.

No compute calls here (no GPU needed): only functions that touch no device.
"""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bm3d_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"BM3D_B200_API[^;(]*?\b(bm3d_b200_\w+)\s*\(", text)))


def test_header_declares_the_surface():
    names = declared_functions()
    assert "bm3d_b200_graph_create" in names
    assert "bm3d_b200_clip_twostage_host" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(engine_lib):
    for name in declared_functions():
        assert hasattr(engine_lib, name), f"{name} not exported"


def test_python_binding_covers_header(engine_lib):
    from bm3dcuda import _lib
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_scale_sigma_matches_reference_expression(engine_lib, oracle):
    L = oracle.port_lib()
    L.port_scale_sigma.restype = ctypes.c_float
    L.port_scale_sigma.argtypes = [ctypes.c_float, ctypes.c_int]
    for s in (0.0, 1.0, 3.0, 5.0, 10.0, 33.3):
        for final in (0, 1):
            assert engine_lib.bm3d_b200_scale_sigma(s, final) == L.port_scale_sigma(s, final)


def test_params_default_are_the_reference_defaults(engine_lib):
    from bm3dcuda import _lib
    p = _lib.Params()
    engine_lib.bm3d_b200_params_default(ctypes.byref(p))
    assert list(p.sigma) == [3.0, 3.0, 3.0]
    assert list(p.block_step) == [8, 8, 8]
    assert list(p.bm_range) == [9, 9, 9]
    assert list(p.ps_num) == [2, 2, 2]
    assert list(p.ps_range) == [4, 4, 4]
    assert (p.radius, p.chroma, p.extractor_exp, p.zero_init) == (0, 0, 0, 1)


@pytest.mark.parametrize("field,value,msg", [
    ("block_step", 0, '"block_step" must be in range [1, 8]'),
    ("block_step", 9, '"block_step" must be in range [1, 8]'),
    ("bm_range", 0, '"bm_range" must be positive'),
    ("ps_num", 9, '"ps_num" must be in range [1, 8]'),
    ("ps_range", 0, '"ps_range" must be positive'),
])
def test_clip_create_rejects_bad_search_args_without_a_device(engine_lib, field, value, msg):
    from bm3dcuda import _lib
    p = _lib.Params()
    engine_lib.bm3d_b200_params_default(ctypes.byref(p))
    getattr(p, field)[0] = value
    h = ctypes.c_void_p()
    rc = engine_lib.bm3d_b200_clip_create(ctypes.byref(h), 64, 48, 1, 0, 0, 4, ctypes.byref(p), 0)
    assert rc == _lib.ERR_INVALID
    assert msg in _lib.last_error()


def test_clip_create_rejects_radius_and_format(engine_lib):
    from bm3dcuda import _lib
    p = _lib.Params()
    engine_lib.bm3d_b200_params_default(ctypes.byref(p))
    h = ctypes.c_void_p()
    p.radius = -1
    assert engine_lib.bm3d_b200_clip_create(ctypes.byref(h), 64, 48, 1, 0, 0, 4, ctypes.byref(p), 0) == _lib.ERR_INVALID
    assert '"radius" must be non-negative' in _lib.last_error()
    p.radius = 8
    assert engine_lib.bm3d_b200_clip_create(ctypes.byref(h), 64, 48, 1, 0, 0, 4, ctypes.byref(p), 0) == _lib.ERR_UNSUPPORTED
    p.radius = 1
    p.chroma = 1
    assert engine_lib.bm3d_b200_clip_create(ctypes.byref(h), 64, 48, 1, 0, 0, 4, ctypes.byref(p), 0) == _lib.ERR_INVALID
    assert 'YUV444' in _lib.last_error()
    p.chroma = 0
    p.sigma[1] = -1.0
    assert engine_lib.bm3d_b200_clip_create(ctypes.byref(h), 64, 48, 3, 0, 0, 4, ctypes.byref(p), 0) == _lib.ERR_INVALID
    assert '"sigma" must be non-negative' in _lib.last_error()


def test_graph_create_rejects_null_buffers(engine_lib):
    from bm3dcuda import _lib
    h = ctypes.c_void_p()
    rc = engine_lib.bm3d_b200_graph_create(ctypes.byref(h), None, None, None, 64, 48, 64, 1.0, 8,
                                           9, 0, 2, 4, 0, 0.0, 0.0, 0, 0.0)
    assert rc == _lib.ERR_INVALID
    assert not h


def test_tiny_planes_rejected(engine_lib):
    from bm3dcuda import _lib
    p = _lib.Params()
    engine_lib.bm3d_b200_params_default(ctypes.byref(p))
    h = ctypes.c_void_p()
    assert engine_lib.bm3d_b200_clip_create(ctypes.byref(h), 7, 48, 1, 0, 0, 4, ctypes.byref(p), 0) == _lib.ERR_INVALID
    assert "at least 8x8" in _lib.last_error()


@pytest.mark.parametrize("args,code,words", [
    (dict(frames=0), "ERR_INVALID", "no frames"),
    (dict(planes=2), "ERR_INVALID", "1 or 3 planes"),
    (dict(width=7), "ERR_INVALID", "8x8"),
    (dict(height=7), "ERR_INVALID", "8x8"),
    (dict(width=16384), "ERR_UNSUPPORTED", "16383"),
    (dict(height=16384), "ERR_UNSUPPORTED", "16383"),
    (dict(sigma=-1.0), "ERR_INVALID", "non-negative"),
    (dict(chroma=1), "ERR_INVALID", "YUV444"),
    (dict(block_step=9), "ERR_INVALID", "[1, 8]"),
    (dict(subsampling=3), "ERR_INVALID", "subsampling"),
])
def test_clip_create_rejects_before_touching_the_device(engine_lib, args, code, words):
    """Empty clips, wrong plane counts and sizes outside [8, 16383] fail with
    the reference's wording, on the host (no device needed)."""
    from bm3dcuda import _lib
    p = _lib.Params()
    engine_lib.bm3d_b200_params_default(ctypes.byref(p))
    p.sigma[0] = args.get("sigma", 5.0)
    p.chroma = args.get("chroma", 0)
    p.block_step[0] = args.get("block_step", 8)
    c = ctypes.c_void_p()
    ss = args.get("subsampling", 0)
    rc = engine_lib.bm3d_b200_clip_create(ctypes.byref(c), args.get("width", 64),
                                          args.get("height", 48), args.get("planes", 1), ss, ss,
                                          args.get("frames", 4), ctypes.byref(p), 0)
    assert rc == getattr(_lib, code), (rc, _lib.last_error())
    assert words in _lib.last_error()
    assert not c.value
