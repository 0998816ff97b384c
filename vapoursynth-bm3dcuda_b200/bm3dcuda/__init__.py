"""bm3dcuda — host-side mirror of the reference plugin's interface on numpy clips.

The reference is a VapourSynth plugin (namespace ``bm3dcuda``) registering
``BM3D``, ``VAggregate`` and ``BM3Dv2`` (source/source.cpp:991-1027). This
module exposes the same three functions, the same argument names, defaults,
carry-forward rules and error messages (source/source.cpp:457-634, 880-989),
over :class:`Clip` objects holding float32 numpy planes, and runs them on the
B200 engine through its C ABI (include/bm3d_b200.h). There is no CPU path.

    basic = BM3D(src, radius=0)
    final = BM3D(src, ref=basic, radius=0)
    vbasic = BM3Dv2(src, radius=r)
    vfinal = BM3Dv2(src, ref=vbasic, radius=r)
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import BM3DError, Params

__all__ = ["Clip", "BM3D", "BM3Dv2", "VAggregate", "BM3DError", "FORMATS", "twostage"]

FLT_EPSILON = float(np.finfo(np.float32).eps)

# name -> (sample type, bits, planes, subsampling_w, subsampling_h)
FORMATS = {
    "GRAYS": ("float", 32, 1, 0, 0),
    "YUV444PS": ("float", 32, 3, 0, 0),
    "RGBS": ("float", 32, 3, 0, 0),
    "YUV420PS": ("float", 32, 3, 1, 1),
    "YUV422PS": ("float", 32, 3, 1, 0),
    "GRAYH": ("float", 16, 1, 0, 0),
    "GRAY8": ("integer", 8, 1, 0, 0),
    "YUV420P8": ("integer", 8, 3, 1, 1),
}


@dataclass
class Clip:
    """A clip: one array per plane, each [num_frames, height_p, width_p]."""
    planes: list
    format: str = "GRAYS"
    props: list = field(default_factory=list)  # one dict of frame properties per frame

    def __post_init__(self):
        if self.format not in FORMATS:
            raise ValueError(f"unknown format {self.format}")
        self.planes = [np.asarray(p) for p in self.planes]
        if len(self.planes) != FORMATS[self.format][2]:
            raise ValueError("plane count does not match the format")
        if not self.props:
            self.props = [dict() for _ in range(self.num_frames)]

    @classmethod
    def from_array(cls, frames: np.ndarray, format: str | None = None) -> "Clip":
        """frames: [N, H, W] (gray) or [N, planes, H, W]."""
        frames = np.asarray(frames, np.float32)
        if frames.ndim == 3:
            return cls([frames], format or "GRAYS")
        return cls([frames[:, i] for i in range(frames.shape[1])], format or "YUV444PS")

    @property
    def num_frames(self) -> int:
        return self.planes[0].shape[0]

    @property
    def width(self) -> int:
        return self.planes[0].shape[2]

    @property
    def height(self) -> int:
        return self.planes[0].shape[1]

    @property
    def num_planes(self) -> int:
        return len(self.planes)

    @property
    def subsampling(self) -> tuple[int, int]:
        f = FORMATS[self.format]
        return f[3], f[4]

    def to_array(self) -> np.ndarray:
        if self.num_planes == 1:
            return self.planes[0]
        return np.stack(self.planes, axis=1)


# --------------------------------------------------------------------------
# argument parsing with the reference's rules
# --------------------------------------------------------------------------
def _arr(v):
    if v is None:
        return []
    if isinstance(v, (list, tuple, np.ndarray)):
        return list(v)
    return [v]


def _per_plane(values, default, check, message):
    vals = _arr(values)
    out = []
    for i in range(3):
        if i < len(vals):
            v = vals[i]
            if not check(v):
                raise BM3DError("BM3D: " + message)
        else:
            v = default if i == 0 else out[i - 1]
        out.append(v)
    return out


@dataclass
class _Args:
    sigma: list
    block_step: list
    bm_range: list
    radius: int
    ps_num: list
    ps_range: list
    chroma: bool
    device_id: int
    fast: bool
    extractor_exp: int
    zero_init: bool
    final: bool
    process: list


def _parse(clip: Clip, ref: Clip | None, sigma, block_step, bm_range, radius, ps_num, ps_range,
           chroma, device_id, fast, extractor_exp, zero_init) -> _Args:
    kind, bits = FORMATS[clip.format][:2]
    if kind != "float" or bits != 32:
        raise BM3DError("BM3D: only constant format 32bit float input supported")
    final = ref is not None
    if final:
        if ref.format != clip.format:
            raise BM3DError('BM3D: "ref" must be of the same format as "clip"')
        if ref.width != clip.width or ref.height != clip.height:
            raise BM3DError('BM3D: "ref" must be of the same dimensions as "clip"')
        if ref.num_frames != clip.num_frames:
            raise BM3DError('BM3D: "ref" must be of the same number of frames as "clip"')
    sig = _per_plane(sigma, 3.0, lambda v: float(v) >= 0.0, '"sigma" must be non-negative')
    sig = [float(np.float32(s)) for s in sig]
    process = [not (s < FLT_EPSILON) for s in sig]
    bs = _per_plane(block_step, 8, lambda v: 0 < int(v) <= 8, '"block_step" must be in range [1, 8]')
    bmr = _per_plane(bm_range, 9, lambda v: int(v) > 0, '"bm_range" must be positive')
    r = 0 if radius is None else int(radius)
    if r < 0:
        raise BM3DError('BM3D: "radius" must be non-negative')
    psn = _per_plane(ps_num, 2, lambda v: 0 < int(v) <= 8, '"ps_num" must be in range [1, 8]')
    psr = _per_plane(ps_range, 4, lambda v: int(v) > 0, '"ps_range" must be positive')
    ch = bool(chroma) if chroma is not None else False
    if ch and clip.format != "YUV444PS":
        raise BM3DError('BM3D: clip format must be YUV444 when "chroma" is true')
    dev = 0 if device_id is None else int(device_id)
    import torch  # device count only
    if not (0 <= dev < torch.cuda.device_count()):
        raise BM3DError(f"BM3D: invalid device ID ({dev})")
    return _Args(sig, [int(v) for v in bs], [int(v) for v in bmr], r, [int(v) for v in psn],
                 [int(v) for v in psr], ch, dev, True if fast is None else bool(fast),
                 0 if extractor_exp is None else int(extractor_exp),
                 True if zero_init is None else bool(zero_init), final, process)


def _params(a: _Args) -> Params:
    p = Params()
    _lib.lib().bm3d_b200_params_default(ctypes.byref(p))
    for i in range(3):
        p.sigma[i] = a.sigma[i]
        p.block_step[i] = a.block_step[i]
        p.bm_range[i] = a.bm_range[i]
        p.ps_num[i] = a.ps_num[i]
        p.ps_range[i] = a.ps_range[i]
    p.radius = a.radius
    p.chroma = int(a.chroma)
    p.extractor_exp = a.extractor_exp
    p.zero_init = int(a.zero_init)
    return p


class _Engine:
    """One bm3d_b200_clip handle (device-resident clip pipeline). variant:
    optional (bm_error, transform_2d, transform_1d) per-plane int lists of the
    run-time-compiled plugin (bm3dcuda.rtc)."""

    def __init__(self, clip: Clip, a: _Args, variant=None):
        L = _lib.lib()
        self.h = ctypes.c_void_p()
        ssw, ssh = clip.subsampling
        p = _params(a)
        _lib.check(L.bm3d_b200_clip_create(ctypes.byref(self.h), clip.width, clip.height,
                                           clip.num_planes, ssw, ssh, clip.num_frames,
                                           ctypes.byref(p), a.device_id))
        if variant is not None:
            arrs = [(ctypes.c_int * 3)(*v) for v in variant]
            try:
                _lib.check(L.bm3d_b200_clip_set_variant(self.h, *arrs))
            except Exception:
                L.bm3d_b200_clip_destroy(self.h)
                self.h = ctypes.c_void_p()
                raise
        self.stride = L.bm3d_b200_clip_stride(self.h)
        self.frame_floats = L.bm3d_b200_clip_frame_floats(self.h)
        self.raw_frame_floats = L.bm3d_b200_clip_raw_frame_floats(self.h)
        self.clip = clip
        self.radius = a.radius

    def close(self):
        if self.h:
            _lib.lib().bm3d_b200_clip_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pack(self, clip: Clip) -> np.ndarray:
        buf = np.zeros((clip.num_frames, self.frame_floats), np.float32)
        off = 0
        for pl in clip.planes:
            n, h, w = pl.shape
            view = buf[:, off:off + h * self.stride].reshape(n, h, self.stride)
            view[:, :, :w] = pl
            off += h * self.stride
        return buf

    def unpack(self, buf: np.ndarray, raw: bool) -> list:
        planes = []
        off = 0
        tw = 2 * self.radius + 1
        for pl in self.clip.planes:
            n, h, w = pl.shape
            rows = h * 2 * tw if raw else h
            view = buf[:, off:off + rows * self.stride].reshape(n, rows, self.stride)
            planes.append(np.ascontiguousarray(view[:, :, :w]))
            off += rows * self.stride
        return planes

    def run(self, src: Clip, ref: Clip | None, raw: bool) -> list:
        L = _lib.lib()
        hs = self.pack(src)
        hr = self.pack(ref) if ref is not None else None
        n = src.num_frames
        dst = np.zeros((n, self.raw_frame_floats if raw else self.frame_floats), np.float32)
        _lib.check(L.bm3d_b200_clip_run_host(
            self.h, hs.ctypes.data, hr.ctypes.data if hr is not None else None, dst.ctypes.data,
            _lib.DST_RAW if raw else _lib.DST_AGGREGATED, None))
        return self.unpack(dst, raw)


def BM3D(clip: Clip, ref: Clip | None = None, sigma=None, block_step=None, bm_range=None,
         radius=None, ps_num=None, ps_range=None, chroma=None, device_id=None, fast=None,
         extractor_exp=None, zero_init=None) -> Clip:
    """bm3dcuda.BM3D (source/source.cpp:457-720, 206-441).

    radius == 0: the denoised clip (unprocessed planes copied from ``clip``).
    radius  > 0: the raw V-BM3D clip of height H * 2 * (2r+1) per plane, with
    frame properties BM3D_V_radius / BM3D_V_process, to be fed to VAggregate.
    """
    a = _parse(clip, ref, sigma, block_step, bm_range, radius, ps_num, ps_range, chroma,
               device_id, fast, extractor_exp, zero_init)
    eng = _Engine(clip, a)
    try:
        raw = a.radius > 0
        planes = eng.run(clip, ref, raw)
    finally:
        eng.close()
    props = [dict(p) for p in clip.props]
    if a.radius > 0:
        for p in props:
            p["BM3D_V_radius"] = a.radius
            p["BM3D_V_process"] = [int(v) for v in a.process]
    return Clip(planes, clip.format, props)


def VAggregate(clip: Clip, src: Clip, planes) -> Clip:
    """bm3dcuda.VAggregate (source/source.cpp:722-909): temporal aggregation of
    a raw V-BM3D clip. The radius is inferred from the heights
    (source/source.cpp:892)."""
    import torch

    radius = (clip.height // src.height - 2) // 4
    process = [False, False, False]
    for p in _arr(planes):
        process[int(p)] = True
    L = _lib.lib()
    tw = 2 * radius + 1
    n_frames = src.num_frames
    out = []
    for pi, sp in enumerate(src.planes):
        if pi >= len(process) or not process[pi]:
            out.append(np.array(sp, np.float32, copy=True))
            continue
        n, h, w = sp.shape
        raw = np.ascontiguousarray(clip.planes[pi], np.float32)  # [N][2*tw*h][w]
        d_raw = torch.from_numpy(raw).cuda()
        d_dst = torch.empty((n, h, w), dtype=torch.float32, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        for k in range(n):
            ptrs = (ctypes.c_void_p * tw)()
            for i in range(tw):
                f = min(max(k - radius + i, 0), n_frames - 1)
                ptrs[i] = d_raw[f].data_ptr()
            _lib.check(L.bm3d_b200_vaggregate(d_dst[k].data_ptr(), w, ptrs, w, w, h, radius, k,
                                              n_frames, ctypes.c_void_p(stream)))
        torch.cuda.synchronize()
        out.append(d_dst.cpu().numpy())
    return Clip(out, src.format, [dict(p) for p in src.props])


def BM3Dv2(clip: Clip, ref: Clip | None = None, sigma=None, block_step=None, bm_range=None,
           radius=None, ps_num=None, ps_range=None, chroma=None, device_id=None, fast=None,
           extractor_exp=None, zero_init=None, proposer=None, proposer_cells=None,
           proposer_tau=None) -> Clip:
    """bm3dcuda.BM3Dv2 (source/source.cpp:911-989): BM3D followed by VAggregate
    when radius > 0. Here the VAggregate sum is fused into the device scatter,
    so the raw stack never leaves the GPU.

    proposer, proposer_cells, proposer_tau: the plugin's optional learned
    match proposal (no counterpart in the reference): a trained
    :class:`bm3dcuda.learned.Proposer` (or the path of a file it saved), the
    cells scored per spatial / temporal search (default 2, 2) and the
    exhaustive re-search threshold (default 4). Radius > 0 only."""
    process = [True, True, True]
    sig = _arr(sigma)
    for i in range(min(3, len(sig))):
        if float(sig[i]) < FLT_EPSILON:
            process[i] = False
    if len(sig) > 0:
        for i in range(len(sig), 3):
            process[i] = process[i - 1]
    if all(not process[i] for i in range(clip.num_planes)):
        return clip
    a = _parse(clip, ref, sigma, block_step, bm_range, radius, ps_num, ps_range, chroma,
               device_id, fast, extractor_exp, zero_init)
    owned = None
    if proposer is not None:
        if a.radius == 0:
            raise BM3DError('BM3D: "proposer" applies to BM3Dv2 with radius > 0')
        from .learned import Proposer
        cells = [2, 2] if proposer_cells is None else [int(v) for v in _arr(proposer_cells)]
        if len(cells) == 1:
            cells.append(cells[0])
        if not all(1 <= v <= 8 for v in cells[:2]):
            raise BM3DError('BM3D: "proposer_cells" must be in range [1, 8]')
        tau = 4.0 if proposer_tau is None else float(proposer_tau)
        if not tau >= 0.0:
            raise BM3DError('BM3D: "proposer_tau" must be non-negative')
        if not isinstance(proposer, Proposer):
            owned = proposer = Proposer.load(str(proposer), device=a.device_id)
    eng = _Engine(clip, a)
    try:
        if proposer is not None:
            _lib.check(_lib.lib().bm3d_b200_clip_set_proposer(eng.h, proposer.handle, cells[0],
                                                              cells[1], tau))
        planes = eng.run(clip, ref, raw=False)
    finally:
        eng.close()
        if owned is not None:
            owned.close()
    return Clip(planes, clip.format, [dict(p) for p in clip.props])


def twostage(clip: Clip, **kw) -> Clip:
    """V-BM3D basic + final (README.md:44-53) with the intermediate kept on the
    device: BM3Dv2(src, ref=BM3Dv2(src))."""
    a = _parse(clip, None, kw.get("sigma"), kw.get("block_step"), kw.get("bm_range"),
               kw.get("radius"), kw.get("ps_num"), kw.get("ps_range"), kw.get("chroma"),
               kw.get("device_id"), kw.get("fast"), kw.get("extractor_exp"), kw.get("zero_init"))
    eng = _Engine(clip, a)
    try:
        hs = eng.pack(clip)
        dst = np.zeros_like(hs)
        _lib.check(_lib.lib().bm3d_b200_clip_twostage_host(eng.h, hs.ctypes.data, dst.ctypes.data,
                                                           None))
        planes = eng.unpack(dst, raw=False)
    finally:
        eng.close()
    return Clip(planes, clip.format, [dict(p) for p in clip.props])
