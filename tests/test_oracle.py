"""The CPU oracle, pinned against the reference's own outputs.

golden.npz holds outputs of the reference bm3dcpu code (cpu_source/source.cpp,
exact-reciprocal build) on seeded inputs; tests/golden/make_golden.py made it.
The project's C restatement must reproduce every one of them bit for bit.
"""
import ast
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")


def golden_cases():
    g = np.load(GOLDEN)
    names = sorted({k.split("/")[0] for k in g.files})
    return g, names


G, NAMES = golden_cases()


def case(name):
    kw = ast.literal_eval(str(G[f"{name}/kwargs"]))
    ref = G[f"{name}/ref"] if f"{name}/ref" in G.files else None
    return G[f"{name}/window"], ref, kw


@pytest.mark.parametrize("name", NAMES)
def test_port_matches_reference_bitwise(oracle, name):
    w, r, kw = case(name)
    got = oracle.port_bm3d(w, r, **kw)
    np.testing.assert_array_equal(got, G[f"{name}/exact"])


@pytest.mark.parametrize("name", NAMES)
def test_port_match_lists_equal_reference(oracle, name):
    w, r, kw = case(name)
    _, m = oracle.port_bm3d(w, r, return_matches=True, **kw)
    np.testing.assert_array_equal(m, G[f"{name}/post"])


@pytest.mark.parametrize("name", NAMES)
def test_stock_build_distance_is_small(name):
    # the shipped ~12-bit reciprocal only perturbs the output slightly
    exact, stock = G[f"{name}/exact"], G[f"{name}/stock"]
    assert np.abs(exact - stock).max() < 2e-3


def test_live_reference_when_available(oracle):
    """Against the compiled reference directly on a fresh seeded input."""
    if not oracle.ref_available("exact"):
        pytest.skip("reference bm3dcpu not built here")
    from bm3dcuda import synthetic as S
    noisy, _ = S.texture_clip(3, 56, 72, seed=99)
    w = noisy[None]
    kw = dict(sigma=7.0, radius=1, ps_num=2, ps_range=3, block_step=6, bm_range=7)
    np.testing.assert_array_equal(oracle.port_bm3d(w, **kw), oracle.ref_bm3d(w, **kw))
    basic = oracle.port_bm3d(w[:, 1:2], sigma=7.0)
    np.testing.assert_array_equal(oracle.port_bm3d(w[:, 1:2], basic[:, None], sigma=7.0),
                                  oracle.ref_bm3d(w[:, 1:2], basic[:, None], sigma=7.0))


def test_dct_round_trip_is_16x(oracle):
    # fwd(inv(x)) = 16 x per dimension; 4096 x for the 3-D transform
    rng = np.random.default_rng(0)
    x = rng.normal(size=8)
    y = oracle.port_dct8(oracle.port_dct8(x, True, fp64=True), False, fp64=True)
    np.testing.assert_allclose(y, 16 * x, rtol=1e-12, atol=1e-12)
    xf = x.astype(np.float32)
    yf = oracle.port_dct8(oracle.port_dct8(xf, True), False)
    np.testing.assert_allclose(yf, 16 * xf, rtol=1e-5, atol=1e-5)


def test_dct_matches_orthonormal_dct_ii(oracle):
    # the scaled DCT-II: X_k = 2 sum x_n cos(pi (2n+1) k / 16), X_0 divided by sqrt(2)
    rng = np.random.default_rng(1)
    x = rng.normal(size=8)
    n = np.arange(8)
    ref = np.array([2 * np.sum(x * np.cos(np.pi * (2 * n + 1) * k / 16)) for k in range(8)])
    ref[0] /= np.sqrt(2)
    got = oracle.port_dct8(x, True, fp64=True)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_constant_image_is_a_fixed_point(oracle):
    w = np.full((1, 1, 32, 40), 0.37, np.float32)
    out = oracle.port_bm3d(w, sigma=10.0)
    np.testing.assert_allclose(out, 0.37, atol=1e-6)


def test_fp64_oracle_tracks_fp32(oracle):
    w, r, kw = case("spatial_basic")
    f32, m = oracle.port_bm3d(w, r, return_matches=True, **kw)
    f64 = oracle.port_bm3d(w, r, fp64=True, match_in=m, **kw)
    assert np.abs(f32 - f64).max() < 1e-5


def test_vaggregate_replication_padding(oracle):
    """Slab (f, s) of frame f holds the value 100*f + s: VAggregate of frame n
    then reads exactly the slabs of source/source.cpp:834-836."""
    N, r, H, W = 4, 2, 2, 3
    tw = 2 * r + 1
    raw = np.zeros((N, tw, 2, H, W), np.float64)
    for f in range(N):
        for s in range(tw):
            raw[f, s, 0] = 100 * f + s
            raw[f, s, 1] = 1.0
    for n in range(N):
        idx = [min(max(n - r + i, 0), N - 1) for i in range(tw)]
        got = oracle.port_vaggregate(np.stack([raw[i] for i in idx]), n, N, fp64=True)
        want = 0.0
        for i in range(tw):
            s = min(max(2 * r - i, n - N + 1 + r), n + r)
            want += 100 * idx[i] + s
        np.testing.assert_allclose(got, want / tw)


def test_rescore_orders_by_distance_and_keeps_ties(oracle):
    """port_rescore (the checker of the engine's BASIC_LISTS final matching):
    the same entries, ascending by the block distance to the block's own
    origin in the centre plane, equal distances in their given order."""
    rng = np.random.default_rng(12)
    h, w, r = 24, 32, 1
    win = rng.random((2 * r + 1, h, w)).astype(np.float32)
    xs = [min(x, w - 8) for x in range(0, w - 8 + 8, 8)]
    ys = [min(y, h - 8) for y in range(0, h - 8 + 8, 8)]
    nb = len(xs) * len(ys)
    lists = np.zeros((nb, 8, 3), np.int32)
    for b in range(nb):
        for i in range(8):
            lists[b, i] = (rng.integers(0, w - 7), rng.integers(0, h - 7), rng.integers(0, 2 * r + 1))
        lists[b, 5] = lists[b, 2]  # an exact tie: entry 2 must stay before entry 5
    out = oracle.port_rescore(win, lists)
    for b in range(nb):
        x, y = xs[b % len(xs)], ys[b // len(xs)]
        ref = win[r, y:y + 8, x:x + 8].astype(np.float64)
        d = [((ref - win[z, v:v + 8, u:u + 8].astype(np.float64)) ** 2).sum() for u, v, z in out[b]]
        assert sorted(map(tuple, out[b])) == sorted(map(tuple, lists[b]))
        assert all(d[i] <= d[i + 1] * (1 + 1e-5) for i in range(7)), b
        # the two tied entries are identical rows: both present, adjacent
        k = [i for i in range(8) if tuple(out[b, i]) == tuple(lists[b, 2])]
        assert len(k) == 2 and k[1] == k[0] + 1
