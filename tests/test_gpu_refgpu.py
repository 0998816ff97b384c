"""GPU parity against the reference's own CUDA kernel.

The reference's source/kernel.cu is compiled unchanged into oracle/_ref/
(``make -C oracle refgpu``) and run through its own get_graphexec graph, the
way the plugin runs it. Two builds: ``exact`` (IEEE division) and ``fast``
(--use_fast_math, the flags of the reference's release build).

Tolerances: the same bars as against bm3dcpu —
  * raw accumulators rtol 1e-5 / atol 1e-5 (only the order of the atomic
    sums differs); radius-0 outputs max-abs <= 1e-4;
  * with extractor_exp > 0 (pre-rounded, order-independent sums) the exact
    build and this engine agree to the same bars on every case; on a larger
    textured clip this engine equals bm3dcpu exactly while the reference's
    CUDA kernel is within one pre-rounding quantum of both;
  * the fast build differs from both by its approximate division only
    (max-abs <= 1e-4 on radius-0 outputs, PSNR within 0.01 dB).
"""
import ast
import os

import numpy as np
import pytest

from gpu_util import aggregate, graph_run, psnr

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")
G = np.load(GOLDEN)
NAMES = sorted({k.split("/")[0] for k in G.files})


def case(name):
    kw = ast.literal_eval(str(G[f"{name}/kwargs"]))
    ref = G[f"{name}/ref"] if f"{name}/ref" in G.files else None
    return G[f"{name}/window"], ref, kw


@pytest.fixture(scope="module")
def refgpu(cuda, engine_lib, oracle):
    if not (oracle.refgpu_available("exact") and oracle.refgpu_available("fast")):
        pytest.fail("reference CUDA build missing: run make -C oracle refgpu where the "
                    "reference tree is present")
    return oracle


def compare(a, b, radius):
    if radius == 0:
        assert np.abs(aggregate(a) - aggregate(b)).max() <= 1e-4
    else:
        np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("name", NAMES)
def test_reference_kernel_agrees_with_bm3dcpu(refgpu, name):
    """The reference's two implementations agree on the golden cases: its
    CUDA kernel (exact build) against the bm3dcpu results in the fixture
    (radius 0: the denoised planes; radius > 0: the raw accumulators)."""
    w, r, kw = case(name)
    got = refgpu.refgpu_window(w, r, kind="exact", **kw)
    golden = G[f"{name}/exact"]
    if kw.get("radius", 0) == 0:
        assert np.abs(aggregate(got) - golden).max() <= 1e-4
    else:
        np.testing.assert_allclose(got, golden, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("name", NAMES)
def test_engine_equals_reference_kernel(refgpu, name):
    w, r, kw = case(name)
    ours = graph_run(w, r, **kw)
    ref = refgpu.refgpu_window(w, r, kind="exact", **kw)
    compare(ours, ref, kw.get("radius", 0))


@pytest.mark.parametrize("name", NAMES)
def test_engine_equals_reference_kernel_pre_rounded(refgpu, name):
    w, r, kw = case(name)
    ours = graph_run(w, r, extractor_exp=6, **kw)
    ref = refgpu.refgpu_window(w, r, kind="exact", extractor_exp=6, **kw)
    compare(ours, ref, kw.get("radius", 0))


@pytest.mark.parametrize("name", ["spatial_basic", "spatial_final", "odd_bs5_r4"])
def test_engine_vs_shipped_reference_build(refgpu, name):
    w, r, kw = case(name)
    ours = aggregate(graph_run(w, r, **kw))
    ref = aggregate(refgpu.refgpu_window(w, r, kind="fast", **kw))
    assert np.abs(ours - ref).max() <= 1e-4


def test_reference_kernel_is_within_one_quantum_of_bm3dcpu(refgpu, oracle):
    """With pre-rounded sums (extractor_exp 6: multiples of 2^-17), this
    engine equals the bm3dcpu restatement exactly on every window of a
    textured clip, while the reference's own CUDA kernel differs from both in
    a handful of pixels by one quantum (its transform arithmetic rounds a
    last bit differently)."""
    from bm3dcuda import synthetic as S
    noisy, _ = S.texture_clip(7, 64, 96, seed=21)
    kw = dict(sigma=5.0, block_step=8, bm_range=9, radius=2, ps_num=2, ps_range=4)
    quantum = 2.0 ** -17
    for n in range(7):
        win = oracle.clip_window(noisy[:, None], n, 2)
        ours = graph_run(win, extractor_exp=6, **kw)
        port = oracle.port_bm3d(win, extractor_exp=6, return_acc=True, **kw)
        ref = refgpu.refgpu_window(win, kind="exact", extractor_exp=6, **kw)
        np.testing.assert_array_equal(ours, port)
        d = np.abs(ours - ref)
        assert d.max() <= quantum
        assert np.count_nonzero(d) <= 1e-3 * d.size


def test_twostage_equals_reference_plugin_pipeline(refgpu):
    """BM3Dv2 basic then final over a clip: this engine's device-resident
    pipeline against the reference plugin's host pipeline (graph per frame,
    host VAggregate) around the reference's own kernel. The one-quantum
    differences of the basic estimate may move a rare near-tie match of the
    final stage, hence mean and PSNR bars rather than equality."""
    from bm3dcuda import Clip, twostage
    from bm3dcuda import synthetic as S
    noisy, clean = S.texture_clip(7, 64, 96, seed=21)
    ours = twostage(Clip.from_array(noisy), sigma=5.0, radius=2, extractor_exp=6).to_array()
    for kind in ("exact", "fast"):
        ref, _ = refgpu.refgpu_twostage(noisy, sigma=5.0, radius=2, extractor_exp=6,
                                        threads=4, resources=4, kind=kind)
        d = np.abs(ours - ref)
        assert np.mean(d) <= 1e-5, kind
        assert np.count_nonzero(d > 1e-4) <= 1e-2 * d.size, kind
        assert abs(psnr(ours, clean) - psnr(ref, clean)) <= 0.01, kind
