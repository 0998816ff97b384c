"""Test infrastructure only: CPU oracle of the learned match proposer.

The proposer has no counterpart in the reference; this module restates the
project's own definition of it in float64 numpy, as the checker of the CUDA
kernels (forward, backward, loss):

* ``down2``: 2x2 mean of a plane (half-resolution input).
* ``forward``: three 3x3 convolutions (1 -> 16 -> 16 -> 16 channels, zero
  padding, ReLU after the first two). Parameters are one flat float32 vector
  of 4800 values: w1 [3][3][1][16], b1 [16], w2 [3][3][16][16], b2 [16],
  w3 [3][3][16][16], b3 [16]; w[dy][dx][ci][co] multiplies input pixel
  (y + dy - 1, x + dx - 1).
* ``teacher`` / ``loss_and_grad``: the distillation loss of the training
  samples. A sample (fc, fz, x, y) is a reference block at full-resolution
  origin (x, y) of frame fc, with candidate cells (x/2 + u, y/2 + v),
  |u|, |v| <= U, of frame fz; a cell's embedding is the network output at
  half-resolution pixel (cell + 2), its teacher distance the smallest exact
  block distance to its block origins. loss = mean over samples of
  KL(softmax(-(s - min s) / T) || softmax(-d)), d the squared embedding
  distances.
* ``init_params``: the "coarse" initialisation, whose 16 output channels are
  the 4x4 half-resolution pixels of the block scaled by ``scale``.
"""
from __future__ import annotations

import numpy as np

C = 16
SIZES = [("w1", (3, 3, 1, C)), ("b1", (C,)), ("w2", (3, 3, C, C)), ("b2", (C,)),
         ("w3", (3, 3, C, C)), ("b3", (C,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(theta: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(theta[o:o + n], np.float64).reshape(shape)
        o += n
    return out


def pack(p: dict) -> np.ndarray:
    return np.concatenate([np.asarray(p[name], np.float64).ravel() for name, _ in SIZES])


def init_params(scale: float = 8.0) -> np.ndarray:
    """Channel k = scale * half-resolution pixel at offset (dy, dx) = (k/4 - 2, k%4 - 2)
    from the cell + 2, routed through the three layers in steps of at most 1."""
    p = {name: np.zeros(shape) for name, shape in SIZES}
    p["b1"][:] = 1.0  # keeps the pixel copies positive through the ReLUs
    for k in range(C):
        dy, dx = k // 4 - 2, k % 4 - 2
        s1 = (max(-1, min(1, dy)), max(-1, min(1, dx)))
        r1 = (dy - s1[0], dx - s1[1])
        s2 = (max(-1, min(1, r1[0])), max(-1, min(1, r1[1])))
        s3 = (r1[0] - s2[0], r1[1] - s2[1])
        p["w1"][1 + s1[0], 1 + s1[1], 0, k] = 1.0
        p["w2"][1 + s2[0], 1 + s2[1], k, k] = 1.0
        p["w3"][1 + s3[0], 1 + s3[1], k, k] = scale
    return pack(p).astype(np.float32)


def down2(plane: np.ndarray) -> np.ndarray:
    h2, w2 = plane.shape[0] // 2, plane.shape[1] // 2
    f = np.asarray(plane, np.float64)[:2 * h2, :2 * w2]
    return 0.25 * ((f[0::2, 0::2] + f[0::2, 1::2]) + (f[1::2, 0::2] + f[1::2, 1::2]))


def _conv(x: np.ndarray, w: np.ndarray, b: np.ndarray) -> np.ndarray:
    """x [H][W][Cin], w [3][3][Cin][Cout] -> [H][W][Cout], zero padding."""
    h, wd, _ = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (0, 0)))
    out = np.broadcast_to(b, (h, wd, w.shape[3])).copy()
    for dy in range(3):
        for dx in range(3):
            out += xp[dy:dy + h, dx:dx + wd] @ w[dy, dx]
    return out


def _conv_back(x: np.ndarray, w: np.ndarray, g: np.ndarray):
    """Gradients of _conv: (dx, dw, db) for output gradient g."""
    h, wd, _ = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (0, 0)))
    gp = np.pad(g, ((1, 1), (1, 1), (0, 0)))
    dw = np.zeros_like(w)
    dxv = np.zeros_like(x)
    for dy in range(3):
        for dx in range(3):
            dw[dy, dx] = xp[dy:dy + h, dx:dx + wd].reshape(-1, x.shape[2]).T @ g.reshape(-1, g.shape[2])
            # out[y][x] uses in[y+dy-1][x+dx-1]  =>  din[y][x] gets g[y-dy+1][x-dx+1]
            dxv += gp[2 - dy:2 - dy + h, 2 - dx:2 - dx + wd] @ w[dy, dx].T
    return dxv, dw, g.sum(axis=(0, 1))


def forward(theta: np.ndarray, half: np.ndarray, keep: bool = False):
    """half [H2][W2] -> embedding [H2][W2][16] (and the activations if keep)."""
    p = unpack(theta)
    x0 = np.asarray(half, np.float64)[..., None]
    a1 = _conv(x0, p["w1"], p["b1"])
    r1 = np.maximum(a1, 0.0)
    a2 = _conv(r1, p["w2"], p["b2"])
    r2 = np.maximum(a2, 0.0)
    e = _conv(r2, p["w3"], p["b3"])
    if keep:
        return e, (x0, a1, r1, a2, r2)
    return e


def teacher(frames: list, samples: np.ndarray, U: int, width: int, height: int) -> np.ndarray:
    """Teacher distances [n][(2U+1)^2]: per sample (fc, fz, x, y) and cell
    (x/2 + u, y/2 + v) of frame fz, the smallest exact block distance to the
    cell's block origins in the plane (+inf when it has none)."""
    side = 2 * U + 1
    out = np.full((len(samples), side * side), np.inf)
    for i, (fc, fz, x, y) in enumerate(samples):
        ref = np.asarray(frames[fc], np.float64)[y:y + 8, x:x + 8]
        for c in range(side * side):
            gx, gy = (x >> 1) + c % side - U, (y >> 1) + c // side - U
            best = np.inf
            for dv in range(2):
                for du in range(2):
                    u, v = 2 * gx + du, 2 * gy + dv
                    if u < 0 or v < 0 or u > width - 8 or v > height - 8:
                        continue
                    d = ref - np.asarray(frames[fz], np.float64)[v:v + 8, u:u + 8]
                    best = min(best, float((d * d).sum()))
            out[i, c] = best
    return out


def sample_loss(embs: list, samples: np.ndarray, tch: np.ndarray, U: int, temperature: float):
    """Distillation loss and d(loss)/d(emb) per frame: mean over samples of
    KL(q || p), p = softmax(-d) over the sample's cells (d: squared embedding
    distance), q = softmax(-(s - min s) / temperature) over the teacher
    distances s (cells with s = inf excluded)."""
    side = 2 * U + 1
    grads = [np.zeros_like(e) for e in embs]
    terms, keep = [], []
    for i, (fc, fz, x, y) in enumerate(samples):
        cx, cy = x >> 1, y >> 1
        er = embs[fc][cy + 2, cx + 2]
        cells, dists, ts = [], [], []
        for c in range(side * side):
            if not np.isfinite(tch[i, c]):
                continue
            yy, xx = cy + c // side - U + 2, cx + c % side - U + 2
            diff = er - embs[fz][yy, xx]
            cells.append((yy, xx, diff))
            dists.append(float(diff @ diff))
            ts.append(float(tch[i, c]))
        if not cells:
            continue
        d, t = np.array(dists), np.array(ts)
        lp = -d - np.log(np.exp(-d - (-d).max()).sum()) - (-d).max()
        z = (t - t.min()) / temperature
        q = np.exp(-z) / np.exp(-z).sum()
        terms.append(float(np.where(q > 0, q * (np.log(np.maximum(q, 1e-300)) - lp), 0.0).sum()))
        keep.append((fc, cy + 2, cx + 2, cells, q - np.exp(lp), fz))
    n = len(terms)
    if n == 0:
        return 0.0, grads
    for fc, ry, rx, cells, g, fz in keep:
        for (yy, xx, diff), gd in zip(cells, g):
            grads[fc][ry, rx] += 2.0 * gd / n * diff
            grads[fz][yy, xx] -= 2.0 * gd / n * diff
    return float(np.sum(terms) / n), grads


def loss_and_grad(theta: np.ndarray, halves: list, samples: np.ndarray, tch: np.ndarray, U: int,
                  temperature: float):
    """Full loss and parameter gradient (float64) over frames `halves`."""
    p = unpack(theta)
    embs, acts = [], []
    for h in halves:
        e, a = forward(theta, h, keep=True)
        embs.append(e)
        acts.append(a)
    loss, gembs = sample_loss(embs, samples, tch, U, temperature)
    g = {name: np.zeros(shape) for name, shape in SIZES}
    for ge, (x0, a1, r1, a2, r2) in zip(gembs, acts):
        d2, dw3, db3 = _conv_back(r2, p["w3"], ge)
        d2 = d2 * (a2 > 0)
        d1, dw2, db2 = _conv_back(r1, p["w2"], d2)
        d1 = d1 * (a1 > 0)
        _, dw1, db1 = _conv_back(x0, p["w1"], d1)
        for k, v in (("w3", dw3), ("b3", db3), ("w2", dw2), ("b2", db2), ("w1", dw1), ("b1", db1)):
            g[k] += v
    return loss, pack(g)
