"""Generates tests/golden/golden.npz from the reference's own CPU implementation.

The reference repository ships no tests and no golden vectors, so the pins
come from running the reference's bm3dcpu code itself (cpu_source/source.cpp,
compiled unchanged by oracle/Makefile into oracle/_ref/) on small seeded
inputs. The exact-reciprocal build is the parity target; the stock build's
output is stored too, to record its distance.

Run in a container that has the reference tree:
    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "vapoursynth-bm3dcuda_b200"))

from oracle import oracle as O  # noqa: E402
from bm3dcuda import synthetic as S  # noqa: E402


def cases():
    """(name, window [planes][2r+1][H][W], ref window or None, kwargs)."""
    out = []
    noisy, _ = S.piecewise_clip(1, 48, 64, seed=11)
    w = noisy[None, :1]
    out.append(("spatial_basic", w, None, dict(sigma=10.0, block_step=8, bm_range=9)))
    basic = O.ref_bm3d(w, sigma=10.0, block_step=8, bm_range=9)
    out.append(("spatial_final", w, basic[:, None], dict(sigma=10.0, block_step=8, bm_range=9)))
    noisy, _ = S.piecewise_clip(1, 29, 37, seed=12)
    out.append(("odd_bs5_r4", noisy[None, :1], None, dict(sigma=12.0, block_step=5, bm_range=4)))
    tex, _ = S.texture_clip(5, 40, 56, seed=13)
    tw = tex[None]
    kw = dict(sigma=5.0, block_step=8, bm_range=9, radius=2, ps_num=2, ps_range=4)
    out.append(("temporal_basic", tw, None, kw))
    raw = O.ref_bm3d(tw, **kw)
    # a plausible basic estimate for the final stage: the centre-slot estimate
    est = (raw[0, :, 0] / np.maximum(raw[0, :, 1], 1e-6)).astype(np.float32)
    out.append(("temporal_final", tw, est[None], kw))
    kw3 = dict(sigma=6.0, block_step=4, bm_range=5, radius=1, ps_num=3, ps_range=2)
    out.append(("temporal_bs4_ps3", tw[:, 1:4], None, kw3))
    ch, _ = S.chroma_clip(3, 40, 48, seed=14)
    cw = np.ascontiguousarray(ch.transpose(1, 0, 2, 3))  # [3][3][H][W]
    out.append(("chroma_spatial", cw[:, 1:2], None, dict(sigma=[10.0, 7.0, 7.0], chroma=True)))
    out.append(("chroma_temporal_skip", cw, None,
                dict(sigma=[10.0, 0.0, 7.0], chroma=True, radius=1)))
    return out


def main():
    if not O.ref_available("exact"):
        raise SystemExit("build the reference first: make -C oracle ref")
    data = {}
    for name, w, r, kw in cases():
        data[f"{name}/window"] = w
        if r is not None:
            data[f"{name}/ref"] = r
        data[f"{name}/exact"] = O.ref_bm3d(w, r, kind="exact", **kw)
        data[f"{name}/stock"] = O.ref_bm3d(w, r, kind="stock", **kw)
        data[f"{name}/kwargs"] = np.array(repr(kw))
        mkw = {k: kw[k] for k in ("block_step", "bm_range", "radius", "ps_num", "ps_range") if k in kw}
        mwin = (r if r is not None else w)[0]
        pre, err, post = O.ref_match_lists(mwin, **mkw)
        data[f"{name}/pre"] = pre
        data[f"{name}/pre_err"] = err
        data[f"{name}/post"] = post
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")
    np.savez_compressed(path, **data)
    print(f"wrote {path}: {len(data)} arrays, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
