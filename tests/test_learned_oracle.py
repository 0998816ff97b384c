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


def _pos_masks(rng, n, U, k=4):
    side = 2 * U + 1
    words = (side * side + 63) // 64
    out = np.zeros((n, words), np.uint64)
    for i in range(n):
        for c in rng.choice(side * side, k, replace=False):
            out[i, c >> 6] |= np.uint64(1 << (int(c) & 63))
    return out


def test_gradient_oracle_matches_finite_differences():
    rng = np.random.default_rng(0)
    H, W = 36, 44
    halves = [P.down2(rng.random((H, W))) for _ in range(2)]
    theta = P.init_params(2.0).astype(np.float64) + rng.normal(0, 0.05, P.NPARAMS)
    U = 3
    samples = np.array([(i % 2, (i // 2) % 2, int(rng.integers(0, W - 7)),
                         int(rng.integers(0, H - 7))) for i in range(10)])
    pos = _pos_masks(rng, len(samples), U)
    _, g = P.loss_and_grad(theta, halves, samples, pos, U, W, H)
    eps = 1e-6
    for k in rng.choice(P.NPARAMS, 30, replace=False):
        t1, t2 = theta.copy(), theta.copy()
        t1[k] += eps
        t2[k] -= eps
        fd = (P.loss_and_grad(t1, halves, samples, pos, U, W, H)[0] -
              P.loss_and_grad(t2, halves, samples, pos, U, W, H)[0]) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * (abs(fd) + abs(g[k])), (k, fd, g[k])


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


def test_training_set_marks_the_cells_of_exhaustive_matches():
    from bm3dcuda.learned import training_set, block_origins
    window = np.zeros((3, 24, 32), np.float32)
    org = block_origins(32, 24, 8)
    lists = np.zeros((len(org), 8, 3), np.int32)
    for b, (x, y) in enumerate(org):
        lists[b, :, 0], lists[b, :, 1], lists[b, :, 2] = x, y, 1  # the block itself
        lists[b, 1] = (min(x + 3, 24), y, 0)   # a match in frame 0
        lists[b, 2] = (x, min(y + 2, 16), 2)   # a match in frame 2
    frames, samples, pos = training_set([window], [lists], radius=1, U=6)
    assert frames.shape == (3, 24, 32)
    assert len(samples) == 2 * len(org)
    side = 13
    for (fc, fz, x, y), m in zip(samples, pos):
        assert fc == 1 and fz in (0, 2)
        u, v, _ = lists[list(map(tuple, org)).index((x, y)), 1 if fz == 0 else 2]
        bit = int(((v >> 1) - (y >> 1) + 6) * side + ((u >> 1) - (x >> 1) + 6))
        assert int(m[bit >> 6]) >> (bit & 63) & 1
        assert sum(bin(int(w)).count("1") for w in m) == 1
