"""Learned match proposal (no counterpart in the reference).

A :class:`Proposer` owns the engine's proposal network (include/bm3d_b200.h,
section 5) on one device. It is trained by distillation from the exhaustive
search: for every reference block of a temporal window and every frame of
the window, the exact block distances of the candidate cells around the
block (what the exhaustive search ranks) define the target distribution
over those cells. Training, inference and learned matching all run on the
GPU through the C ABI; nothing here computes on the CPU beyond bookkeeping.

    prop = Proposer()
    windows = [clip_window(...), ...]             # [2r+1][H][W] numpy
    prop.fit(windows, radius=2)                    # exhaustive lists -> training
    lists, fell = learned_match(prop, window, radius=2)
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

__all__ = ["Proposer", "exhaustive_matches", "training_set", "teacher_distances",
           "learned_match", "recall",
           "DEFAULT_CELLS_SPATIAL", "DEFAULT_CELLS_TEMPORAL", "DEFAULT_U"]

DEFAULT_CELLS_SPATIAL = 4   # 16 candidate offsets in the centre frame
DEFAULT_CELLS_TEMPORAL = 4  # 16 candidate offsets per neighbour frame
DEFAULT_U = 6               # training candidates: cells within +-6 of the block's cell


def _stride(width: int) -> int:
    return (width + 31) // 32 * 32


def _device_frames(frames: np.ndarray):
    """[F][H][W] numpy -> contiguous [F][H][stride] float32 CUDA tensor."""
    import torch
    f, h, w = frames.shape
    host = np.zeros((f, h, _stride(w)), np.float32)
    host[..., :w] = frames
    return torch.from_numpy(host).cuda()


class Proposer:
    """The proposal network on a device (FP32 master parameters)."""

    def __init__(self, params: np.ndarray | None = None, device: int = 0):
        self._L = _lib.lib()
        self._h = ctypes.c_void_p()
        ptr = None
        if params is not None:
            params = np.ascontiguousarray(params, np.float32)
            assert params.size == _lib.PROPOSER_PARAMS
            ptr = params.ctypes.data
        _lib.check(self._L.bm3d_b200_proposer_create(ctypes.byref(self._h), ptr, device))
        self.device = device

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def close(self) -> None:
        if self._h:
            self._L.bm3d_b200_proposer_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.zeros(_lib.PROPOSER_PARAMS, np.float32)
        _lib.check(self._L.bm3d_b200_proposer_get_params(self._h, out.ctypes.data))
        return out

    def set_params(self, params: np.ndarray | None) -> None:
        """New parameters (None: the coarse network); resets Adam."""
        ptr = None
        if params is not None:
            params = np.ascontiguousarray(params, np.float32)
            ptr = params.ctypes.data
        _lib.check(self._L.bm3d_b200_proposer_set_params(self._h, ptr))

    def quant(self) -> np.ndarray:
        """Embedding quantisation: qscale, qoff[16]."""
        out = np.zeros(17, np.float32)
        _lib.check(self._L.bm3d_b200_proposer_get_quant(self._h, out.ctypes.data))
        return out

    def set_quant(self, quant: np.ndarray | None) -> None:
        ptr = None
        if quant is not None:
            quant = np.ascontiguousarray(quant, np.float32)
            assert quant.size == 17
            ptr = quant.ctypes.data
        _lib.check(self._L.bm3d_b200_proposer_set_quant(self._h, ptr))

    def save(self, path: str) -> None:
        """Writes the parameters and the embedding quantisation (float32,
        little-endian) to `path`: the file the VapourSynth plugin's optional
        ``proposer`` argument reads."""
        np.concatenate([self.params(), self.quant()]).astype("<f4").tofile(path)

    @classmethod
    def load(cls, path: str, device: int = 0) -> "Proposer":
        """A proposer from a file written by :meth:`save`."""
        data = np.fromfile(path, dtype="<f4")
        if data.size != _lib.PROPOSER_PARAMS + 17:
            raise ValueError(f"{path} is not a saved proposer")
        p = cls(data[:_lib.PROPOSER_PARAMS], device=device)
        p.set_quant(data[_lib.PROPOSER_PARAMS:])
        return p

    def calibrate(self, frames, width: int, height: int) -> np.ndarray:
        """Quantisation from the embeddings of device frames [F][H][stride]."""
        _lib.check(self._L.bm3d_b200_proposer_calibrate(self._h, frames.data_ptr(),
                                                        frames.shape[0], width, height,
                                                        frames.shape[-1], None))
        return self.quant()

    def embed(self, frames, width: int, height: int):
        """8-bit embeddings [F][H/2][W/2][16] of device frames [F][H][stride] (torch)."""
        import torch
        n = frames.shape[0]
        out = torch.empty((n, height // 2, width // 2, 16), dtype=torch.uint8,
                          device=frames.device)
        _lib.check(self._L.bm3d_b200_proposer_embed(self._h, frames.data_ptr(), n, width, height,
                                                    frames.shape[-1], out.data_ptr(), None))
        torch.cuda.synchronize()
        _lib.check(self._L.bm3d_b200_proposer_status(self._h))
        return out

    def embed_f32(self, frames, width: int, height: int):
        """The FP32 training network's embeddings, same layout."""
        import torch
        n = frames.shape[0]
        out = torch.empty((n, height // 2, width // 2, 16), dtype=torch.float32,
                          device=frames.device)
        _lib.check(self._L.bm3d_b200_proposer_embed_f32(self._h, frames.data_ptr(), n, width,
                                                        height, frames.shape[-1], out.data_ptr(),
                                                        None))
        return out

    def loss_grad(self, frames, width: int, height: int, samples, teacher, U: int,
                  temperature: float):
        """Loss and FP32 gradient at the current parameters (device tensors in)."""
        loss = ctypes.c_float()
        grad = np.zeros(_lib.PROPOSER_PARAMS, np.float32)
        _lib.check(self._L.bm3d_b200_proposer_loss_grad(
            self._h, frames.data_ptr(), frames.shape[0], width, height, frames.shape[-1],
            samples.data_ptr(), teacher.data_ptr(), samples.shape[0], U,
            ctypes.c_float(temperature), ctypes.byref(loss), grad.ctypes.data, None))
        return float(loss.value), grad

    def train(self, frames, width: int, height: int, samples, teacher, U: int,
              temperature: float, steps: int, lr: float = 2e-3) -> np.ndarray:
        losses = np.zeros(max(1, steps), np.float32)
        _lib.check(self._L.bm3d_b200_proposer_train(
            self._h, frames.data_ptr(), frames.shape[0], width, height, frames.shape[-1],
            samples.data_ptr(), teacher.data_ptr(), samples.shape[0], U,
            ctypes.c_float(temperature), steps, ctypes.c_float(lr), losses.ctypes.data, None))
        return losses[:steps]

    def fit(self, windows: list, *, radius: int, block_step: int = 8, sigma: float = 10.0,
            U: int = DEFAULT_U, steps: int = 200, lr: float = 2e-3) -> np.ndarray:
        """Trains on `windows` ([2r+1][H][W] each): every reference block of a
        window's centre frame against every frame of the window, distilled
        from the exhaustive distances at the noise level of `sigma` (the
        temperature is the expected distance of two noisy copies of one
        block, 2 * 64 * (sigma / 255)^2)."""
        import torch
        frames, samples = training_set(windows, radius=radius, block_step=block_step)
        h, w = frames.shape[1:]
        d_frames = _device_frames(frames)
        d_samples = torch.from_numpy(samples).cuda()
        d_teacher = teacher_distances(d_frames, w, h, d_samples, U)
        return self.train(d_frames, w, h, d_samples, d_teacher, U,
                          2.0 * 64.0 * (sigma / 255.0) ** 2, steps, lr)


def teacher_distances(frames, width: int, height: int, samples, U: int):
    """Teacher distances [n][(2U+1)^2] of device samples (GPU)."""
    import torch
    n = samples.shape[0]
    out = torch.empty((n, (2 * U + 1) ** 2), dtype=torch.float32, device=frames.device)
    _lib.check(_lib.lib().bm3d_b200_proposer_teacher(frames.data_ptr(), frames.shape[0], width,
                                                     height, frames.shape[-1], samples.data_ptr(),
                                                     n, U, out.data_ptr(), None))
    return out


def exhaustive_matches(window: np.ndarray, *, block_step: int = 8, bm_range: int = 9,
                       radius: int = 0, ps_num: int = 2, ps_range: int = 4) -> np.ndarray:
    """Exhaustive match lists [nb][8][3] of one window [2r+1][H][W] (GPU)."""
    import torch
    L = _lib.lib()
    tw, h, w = window.shape
    stride = _stride(w)
    src = np.zeros((1, tw, h, stride), np.float32)
    src[0, :, :, :w] = window
    d_src = torch.from_numpy(src).cuda()
    d_res = torch.zeros((1, tw, 2, h, stride), dtype=torch.float32, device="cuda")
    g = ctypes.c_void_p()
    s = L.bm3d_b200_scale_sigma(10.0, 0)
    _lib.check(L.bm3d_b200_graph_create(ctypes.byref(g), d_res.data_ptr(), d_src.data_ptr(), None,
                                        w, h, stride, s, block_step, bm_range, radius, ps_num,
                                        ps_range, 0, s, s, 0, 0.0))
    try:
        nb = ctypes.c_int()
        _lib.check(L.bm3d_b200_graph_launch_device(g, None))
        dummy = np.zeros(3, np.int32)
        L.bm3d_b200_graph_matches(g, dummy.ctypes.data, 0, ctypes.byref(nb))
        out = np.zeros((nb.value, 8, 3), np.int32)
        _lib.check(L.bm3d_b200_graph_matches(g, out.ctypes.data, nb.value, ctypes.byref(nb)))
    finally:
        L.bm3d_b200_graph_destroy(g)
    return out


def block_origins(width: int, height: int, block_step: int) -> np.ndarray:
    """[nb][2] (x, y) reference-block origins in scan order (source/kernel.cu:389-400)."""
    xs = [min(x, width - 8) for x in range(0, width - 8 + block_step, block_step)]
    ys = [min(y, height - 8) for y in range(0, height - 8 + block_step, block_step)]
    return np.array([(x, y) for y in ys for x in xs], np.int32)


def training_set(windows: list, *, radius: int, block_step: int = 8):
    """Training frames and samples: frames [F][H][W] (all windows' frames) and
    samples int32 [n][4] = (fc, fz, x, y), every reference block (x, y) of each
    window's centre frame fc paired with every frame fz of its window."""
    frames, samples = [], []
    for window in windows:
        tw, h, w = window.shape
        assert tw == 2 * radius + 1
        base = len(frames)
        frames.extend(list(window))
        for x, y in block_origins(w, h, block_step).tolist():
            for z in range(tw):
                samples.append((base + radius, base + z, x, y))
    return (np.ascontiguousarray(np.stack(frames), np.float32),
            np.asarray(samples, np.int32).reshape(-1, 4))


def learned_match(proposer: Proposer, window: np.ndarray, *, block_step: int = 8,
                  bm_range: int = 9, radius: int = 0, ps_num: int = 2, ps_range: int = 4,
                  cells_spatial: int = DEFAULT_CELLS_SPATIAL,
                  cells_temporal: int = DEFAULT_CELLS_TEMPORAL, fallback_ssd: float = 0.0,
                  embeddings=None):
    """Learned match lists [nb][8][3] and fallback flags [nb] of one window
    (GPU). embeddings: optional uint8 device tensor [2r+1][H/2][W/2][16]."""
    tw, h, w = window.shape
    d_frames = _device_frames(window)
    emb = embeddings if embeddings is not None else proposer.embed(d_frames, w, h)
    fptr = (ctypes.c_void_p * tw)(*[d_frames[z].data_ptr() for z in range(tw)])
    eptr = (ctypes.c_void_p * tw)(*[emb[z].data_ptr() for z in range(tw)])
    nb = len(block_origins(w, h, block_step))
    out = np.zeros((nb, 8, 3), np.int32)
    fell = np.zeros(nb, np.int32)
    n = ctypes.c_int()
    _lib.check(_lib.lib().bm3d_b200_learned_match(
        fptr, eptr, w, h, d_frames.shape[-1], block_step, bm_range, radius, ps_num, ps_range,
        cells_spatial, cells_temporal, ctypes.c_float(fallback_ssd), out.ctypes.data,
        fell.ctypes.data, nb, ctypes.byref(n)))
    return out, fell


def recall(learned: np.ndarray, exhaustive: np.ndarray) -> float:
    """Fraction of the exhaustive lists' distinct entries found in the learned lists."""
    hit = tot = 0
    for a, b in zip(learned, exhaustive):
        sa = {tuple(e) for e in a}
        sb = {tuple(e) for e in b}
        hit += len(sa & sb)
        tot += len(sb)
    return hit / max(1, tot)
