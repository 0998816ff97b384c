"""CPU checks of the learned-proposal oracles (no GPU).

* oracle/proposer_ref.py: its analytic gradient against central finite
  differences (this pins the gradient oracle the GPU kernels are held to).
* oracle/learned_port.c: with every block forced to fall back, the learned
  matcher must return the reference bm3dcpu's exhaustive lists exactly; with
  the coarse network, proposals must recover most exhaustive matches.
* The BF16 inference restatement stays within BF16 rounding of the FP64
  network.
"""
import numpy as np
import pytest

from oracle import proposer_ref as P


def test_gradient_oracle_matches_finite_differences():
    rng = np.random.default_rng(0)
    H, W = 36, 44
    frames = [rng.random((H, W)) for _ in range(2)]
    halves = [P.down2(f) for f in frames]
    theta = P.init_params(2.0).astype(np.float64) + rng.normal(0, 0.05, P.NPARAMS)
    U = 3
    samples = np.array([(i % 2, (i // 2) % 2, int(rng.integers(0, W - 7)),
                         int(rng.integers(0, H - 7))) for i in range(10)])
    tch = P.teacher(frames, samples, U, W, H)
    T = 0.5

    def loss(t):
        return P.loss_and_grad(t, halves, samples, tch, U, T)[0]

    _, g = P.loss_and_grad(theta, halves, samples, tch, U, T)
    eps = 1e-6
    for k in rng.choice(P.NPARAMS, 30, replace=False):
        t1, t2 = theta.copy(), theta.copy()
        t1[k] += eps
        t2[k] -= eps
        fd = (loss(t1) - loss(t2)) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * (abs(fd) + abs(g[k])), (k, fd, g[k])


def test_teacher_is_the_cellwise_minimum_distance():
    rng = np.random.default_rng(7)
    H, W, U = 30, 38, 2
    frames = [rng.random((H, W)) for _ in range(2)]
    samples = np.array([(0, 1, 5, 7), (1, 0, 0, 0), (0, 0, W - 8, H - 8)])
    tch = P.teacher(frames, samples, U, W, H)
    side = 2 * U + 1
    for i, (fc, fz, x, y) in enumerate(samples):
        ref = frames[fc][y:y + 8, x:x + 8]
        for v in range(H - 7):
            for u in range(W - 7):
                du, dv = (u >> 1) - (x >> 1), (v >> 1) - (y >> 1)
                if abs(du) > U or abs(dv) > U:
                    continue
                d = float(((ref - frames[fz][v:v + 8, u:u + 8]) ** 2).sum())
                assert tch[i, (dv + U) * side + du + U] <= d + 1e-12
        # the sample's own block in its own frame is at distance 0
        if fc == fz:
            assert tch[i, U * side + U] == 0.0
    # cells with no block origin in the plane are excluded
    assert np.isinf(tch[1, 0]) and np.isinf(tch[2, -1])


def test_coarse_network_copies_the_block_footprint():
    rng = np.random.default_rng(1)
    plane = rng.random((24, 32))
    half = P.down2(plane)
    e = P.forward(P.init_params(8.0).astype(np.float64), half)
    # channel k at pixel (cy+2, cx+2) = 8 * (half[cy + k//4, cx + k%4] + 1): the +1
    # (first-layer bias, keeps the copies positive) cancels in every distance
    for cy, cx in [(3, 4), (5, 7), (8, 10)]:
        want = 8.0 * (half[cy:cy + 4, cx:cx + 4].ravel() + 1.0)
        np.testing.assert_allclose(e[cy + 2, cx + 2], want, rtol=1e-12, atol=1e-12)


def test_bf16_inference_restatement_close_to_fp64(oracle):
    rng = np.random.default_rng(2)
    plane = rng.random((30, 46)).astype(np.float32)
    theta = (P.init_params(4.0) + rng.normal(0, 0.02, P.NPARAMS)).astype(np.float32)
    ref = P.forward(theta.astype(np.float64), P.down2(plane))
    got = oracle.port_proposer_embed_bf16(plane, theta)
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 0.03 * scale


@pytest.mark.parametrize("radius", [0, 1])
def test_oracle_fallback_is_the_reference_exhaustive_search(oracle, radius):
    from bm3dcuda import synthetic as S
    noisy, _ = S.texture_clip(2 * radius + 1, 40, 56, seed=11)
    embs = np.zeros((2 * radius + 1, 20, 28, 16), np.uint8)
    lists, fell = oracle.port_learned_match(noisy, embs, radius=radius, fallback_ssd=1e-30)
    assert fell.all()
    if oracle.ref_available():
        _, _, want = oracle.ref_match_lists(noisy, radius=radius)
    else:
        _, want = oracle.port_bm3d(noisy[None], radius=radius, return_matches=True)
    np.testing.assert_array_equal(lists, want)


def test_oracle_coarse_proposals_recover_exhaustive_matches(oracle):
    from bm3dcuda import synthetic as S
    from bm3dcuda.learned import recall
    # texture: distinct best matches (flat regions have many equivalent ones)
    noisy, _ = S.texture_clip(3, 48, 64, seed=12)
    theta = P.init_params(8.0)
    quant = np.array([20.0] + [-100.0] * 16, np.float32)  # the coarse network's
    embs = np.stack([oracle.quantize_embedding(oracle.port_proposer_embed_bf16(f, theta), quant)
                     for f in noisy])
    lists, fell = oracle.port_learned_match(noisy, embs, radius=1)
    assert not fell.any()
    _, want = oracle.port_bm3d(noisy[None], radius=1, return_matches=True)
    assert recall(lists, want) > 0.8
    # every list starts from the block itself (centre insertion)
    from bm3dcuda.learned import block_origins
    org = block_origins(64, 48, 8)
    assert all((l[:, :2] == o).all(axis=1).any() for l, o in zip(lists, org))


def test_training_set_pairs_every_block_with_every_window_frame():
    from bm3dcuda.learned import training_set, block_origins
    windows = [np.zeros((3, 24, 32), np.float32), np.ones((3, 24, 32), np.float32)]
    frames, samples = training_set(windows, radius=1)
    org = block_origins(32, 24, 8)
    assert frames.shape == (6, 24, 32)
    assert samples.shape == (2 * len(org) * 3, 4)
    assert set(samples[:, 0]) == {1, 4}  # centre frames of the two windows
    for w in range(2):
        part = samples[samples[:, 0] == 3 * w + 1]
        assert set(part[:, 1]) == {3 * w, 3 * w + 1, 3 * w + 2}
        assert {tuple(v) for v in part[:, 2:]} == {tuple(v) for v in org}
