"""The run-time-compiled plugin's variants (bm3dcuda_rtc) in the oracle, on CPU:
the transforms' round trips, the block distances' invariances, and the
plugin's string arguments (rtc_source/source.cpp:854-911)."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O


def tx(v, kind, forward, fp64=False):
    lib = O.port_lib()
    a = np.array(v, np.float64 if fp64 else np.float32)
    fn = lib.port_tx8_f64 if fp64 else lib.port_tx8_f32
    fn(a.ctypes.data, ctypes.c_int(kind), ctypes.c_int(int(forward)))
    return a


@pytest.mark.parametrize("kind", [0, 2, 3])
def test_dct_wht_bior_round_trip_is_16x(kind):
    rng = np.random.default_rng(kind)
    for _ in range(20):
        x = rng.standard_normal(8)
        y = tx(tx(x, kind, True, True), kind, False, True)
        np.testing.assert_allclose(y, 16.0 * x, rtol=1e-12, atol=1e-12)


def test_haar_inverse_is_the_references():
    """The reference's inverse Haar (rtc_source/kernel.hpp:226-252) reads
    coefficients 0, 1, 2 and 4 only; a drop-in keeps that."""
    for k in (3, 5, 6, 7):
        e = np.zeros(8)
        e[k] = 1.0
        np.testing.assert_array_equal(tx(e, 1, False, True), np.zeros(8))
    # so forward then inverse is not 16x the identity in general
    x = np.random.default_rng(1).standard_normal(8)
    y = tx(tx(x, 1, True, True), 1, False, True)
    assert not np.allclose(y, 16.0 * x)


def test_haar_forward_is_orthogonal_up_to_scale():
    m = np.stack([tx(e, 1, True, True) for e in np.eye(8)], 1)
    g = m @ m.T
    np.testing.assert_allclose(g, np.diag(np.diag(g)), atol=1e-9)


def _block_window(seed=0):
    rng = np.random.default_rng(seed)
    return rng.random((1, 1, 24, 24)).astype(np.float32)


@pytest.mark.parametrize("metric", [2, 3])
def test_zero_mean_distances_ignore_a_constant_offset(metric):
    """ZSSD/ZSAD of a candidate that is the reference plus a constant is ~0:
    the block matches an offset copy of itself before anything else."""
    rng = np.random.default_rng(3)
    base = rng.random((16, 16)).astype(np.float32)
    img = np.zeros((24, 40), np.float32)
    img[4:20, 0:16] = base
    img[4:20, 20:36] = base + 0.25
    w = img[None, None]
    _, m = O.port_bm3d(w, sigma=10, block_step=8, bm_range=20, bm_error=metric,
                       return_matches=True)
    nb = O.num_blocks(40, 24, 8)
    assert m.shape == (nb, 8, 3)
    # block at (0, 8) has its offset copy at (20, 8) among its matches
    xs = O.num_blocks(40, 8, 8)  # blocks per row
    b = 1 * xs + 0
    pos = {(int(x), int(y)) for x, y, _ in m[b]}
    assert (20, 8) in pos


def test_ssd_norm_matches_a_scaled_copy():
    rng = np.random.default_rng(4)
    base = rng.random((16, 16)).astype(np.float32) + 0.1
    img = np.zeros((24, 40), np.float32)
    img[4:20, 0:16] = base
    img[4:20, 20:36] = 0.5 * base
    _, m = O.port_bm3d(img[None, None], sigma=10, block_step=8, bm_range=20, bm_error=4,
                       return_matches=True)
    xs = O.num_blocks(40, 8, 8)
    pos = {(int(x), int(y)) for x, y, _ in m[1 * xs + 0]}
    assert (20, 8) in pos


def test_default_variant_is_the_plain_port():
    w = _block_window(5)
    a = O.port_bm3d(w, sigma=10)
    b = O.port_bm3d(w, sigma=10, bm_error=0, transform_2d=0, transform_1d=0)
    np.testing.assert_array_equal(a, b)


def test_rtc_string_arguments():
    from bm3dcuda import BM3DError
    from bm3dcuda.rtc import BM_ERRORS, TRANSFORMS, _variant_strings
    assert _variant_strings(None, BM_ERRORS, "bm_error_s") == [0, 0, 0]
    assert _variant_strings(["SAD"], BM_ERRORS, "bm_error_s") == [1, 1, 1]
    assert _variant_strings(["ssd", "SSD/NORM"], BM_ERRORS, "bm_error_s") == [0, 4, 4]
    assert _variant_strings(["Bior1.5", "haar", "wht"], TRANSFORMS, "transform_2d_s") == [3, 1, 2]
    with pytest.raises(BM3DError, match="BM3D_RTC: invalid 'bm_error_s': l1"):
        _variant_strings(["l1"], BM_ERRORS, "bm_error_s")
    with pytest.raises(BM3DError, match="BM3D_RTC: invalid 'transform_1d_s': dft"):
        _variant_strings(["dct", "DFT"], TRANSFORMS, "transform_1d_s")
