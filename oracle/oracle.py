"""Test infrastructure only: ctypes front-end of the CPU oracle.

Two oracles live here, both driven with numpy arrays:

* ``ref_*`` run the reference's own bm3dcpu code (cpu_source/source.cpp),
  compiled unchanged by ``oracle/Makefile`` into ``oracle/_ref/``. The
  ``exact`` build replaces the ~12-bit ``_mm256_rcp_ps`` with an IEEE division
  and is the parity target; the ``stock`` build is the shipped arithmetic.
* ``refgpu_*`` run the reference's own CUDA kernel (source/kernel.cu),
  compiled unchanged with nvcc into ``oracle/_ref/libbm3dcuda_ref_{fast,exact}.so``
  (``fast``: --use_fast_math as the reference ships; ``exact``: IEEE division),
  through its own ``get_graphexec`` graph and the plugin's host pipeline.
  These need a GPU; they are a checker and the GPU reference timing.
* ``port_*`` run this project's C restatement (``oracle/bm3d_port*.{c,h}``):
  FP32 (bit-identical to the exact bm3dcpu build, optionally with the CUDA
  kernel's pre-rounded accumulation) and FP64.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline
use this module, always as the checker.

Array conventions (numpy, C-contiguous float32):
  window: [planes][2r+1][H][W]   -- planes is 3 with chroma, else 1
  radius == 0 result: [planes][H][W]
  radius  > 0 result: [planes][2r+1][2][H][W]  (wdst slab, weight slab)
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "libbm3d_port.so")
REF_SO = {
    "exact": os.path.join(HERE, "_ref", "libbm3dcpu_ref_exact.so"),
    "stock": os.path.join(HERE, "_ref", "libbm3dcpu_ref_stock.so"),
}

REFRTC_SO = os.path.join(HERE, "_ref", "libbm3dcuda_rtc_ref.so")
REFGPU_SO = {
    "fast": os.path.join(HERE, "_ref", "libbm3dcuda_ref_fast.so"),
    "exact": os.path.join(HERE, "_ref", "libbm3dcuda_ref_exact.so"),
}

_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_pp = ctypes.POINTER(ctypes.c_void_p)


def build_port() -> str:
    """Compile the C restatement (needs only gcc)."""
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    return PORT_SO


def build_ref() -> bool:
    """Compile the reference checkers when the reference tree is present (the
    recipe in oracle/Makefile knows its location; BM3D_REF_DIR overrides);
    True when the bm3dcpu build exists afterwards."""
    subprocess.run(["make", "-s", "-C", HERE, "refs"], check=True)
    return os.path.exists(REF_SO["exact"])


_libs: dict[str, ctypes.CDLL] = {}


def _load(path: str) -> ctypes.CDLL:
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library missing: {path} (run make -C oracle)")
        _libs[path] = ctypes.CDLL(path)
    return _libs[path]


def port_lib() -> ctypes.CDLL:
    if not os.path.exists(PORT_SO):
        build_port()
    return _load(PORT_SO)


def ref_available(kind: str = "exact") -> bool:
    return os.path.exists(REF_SO[kind])


def ref_lib(kind: str = "exact") -> ctypes.CDLL:
    return _load(REF_SO[kind])


def refgpu_available(kind: str = "fast") -> bool:
    return os.path.exists(REFGPU_SO[kind])


def refgpu_lib(kind: str = "fast") -> ctypes.CDLL:
    lib = _load(REFGPU_SO[kind])
    if not getattr(lib, "_typed", False):
        c_int, c_float, c_vp = ctypes.c_int, ctypes.c_float, ctypes.c_void_p
        lib.refgpu_last_error.restype = ctypes.c_char_p
        lib.refgpu_graph_create.restype = c_vp
        lib.refgpu_graph_create.argtypes = [c_vp, c_vp, c_vp] + [c_int] * 3 + [c_float] + \
            [c_int] * 6 + [c_float, c_float, c_int, c_float]
        lib.refgpu_graph_launch.argtypes = [c_vp, c_vp]
        lib.refgpu_graph_destroy.argtypes = [c_vp]
        lib.refgpu_kernel.argtypes = [c_vp, c_vp] + [c_int] * 3 + [c_float] + [c_int] * 6 + \
            [c_float, c_float, c_int, c_float, c_vp]
        lib.refgpu_vbm3d_twostage.argtypes = [c_vp, c_vp] + [c_int] * 4 + [c_float] + \
            [c_int] * 9 + [c_vp]
        lib._typed = True
    return lib


def _refgpu_check(lib, rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what}: {lib.refgpu_last_error().decode()}")


def scale_sigma(sigma: float, final_: bool) -> float:
    """The plugin's sigma scaling (source/source.cpp:520-523), in float32."""
    s = np.float32(sigma) * np.float32(3.0 / 4.0) / np.float32(255.0) * np.float32(64.0)
    return float(np.float32(s * np.float32(1.0 if final_ else 2.7)))


def refgpu_window(window: np.ndarray, ref_window: np.ndarray | None = None, *, sigma=3.0,
                  block_step=8, bm_range=9, radius=0, ps_num=2, ps_range=4, chroma=False,
                  extractor_exp=0, kind: str = "fast") -> np.ndarray:
    """One frame window through the reference's own graph (get_graphexec:
    HtoD, memset, bm3d kernel, DtoH) on the current CUDA device, exactly as
    the plugin launches it. window/ref_window: [planes][2r+1][H][W].
    Returns the raw accumulators [planes][2r+1][2][H][W] (host copy)."""
    import torch
    lib = refgpu_lib(kind)
    np_, h, w = _check_window(window, radius, chroma)
    stride = (w + 31) // 32 * 32  # a 128-byte pitch, as cudaMallocPitch gives
    final = ref_window is not None
    tw = 2 * radius + 1
    src = np.zeros((2 if final else 1, np_, tw, h, stride), np.float32)
    if final:
        src[0, ..., :w] = ref_window
        src[1, ..., :w] = window
    else:
        src[0, ..., :w] = window
    res_floats = np_ * tw * 2 * h * stride
    h_res = torch.zeros(max(src.size, res_floats), dtype=torch.float32).pin_memory()
    h_res[: src.size] = torch.from_numpy(src.reshape(-1))
    d_src = torch.zeros(src.size, dtype=torch.float32, device="cuda")
    d_res = torch.zeros(res_floats, dtype=torch.float32, device="cuda")
    s = [float(v) for v in np.atleast_1d(sigma)]
    while len(s) < 3:
        s.append(s[-1])
    sig = [scale_sigma(v, final) for v in s[:3]]
    ext = float(np.ldexp(np.float32(1.0), extractor_exp)) if extractor_exp else 0.0
    torch.cuda.synchronize()
    g = lib.refgpu_graph_create(d_res.data_ptr(), d_src.data_ptr(), h_res.data_ptr(), w, h,
                                stride, sig[0], block_step, bm_range, radius, ps_num, ps_range,
                                int(chroma), sig[1], sig[2], int(final), ext)
    if not g:
        raise RuntimeError("get_graphexec returned no graph")
    try:
        _refgpu_check(lib, lib.refgpu_graph_launch(g, None), "cudaGraphLaunch")
        torch.cuda.synchronize()
    finally:
        lib.refgpu_graph_destroy(g)
    out = h_res[:res_floats].numpy().reshape(np_, tw, 2, h, stride)[..., :w].copy()
    return out


def refrtc_available() -> bool:
    return os.path.exists(REFRTC_SO)


def refrtc_window(window: np.ndarray, ref_window: np.ndarray | None = None, *, sigma=3.0,
                  block_step=8, bm_range=9, radius=0, ps_num=2, ps_range=4, chroma=False,
                  extractor_exp=0, bm_error=0, transform_2d=0, transform_1d=0) -> np.ndarray:
    """One frame window through the reference's run-time-compiled kernel
    (rtc_source/kernel.hpp, compiled with NVRTC as the rtc plugin does) on the
    current CUDA device. Returns the raw accumulators [planes][2r+1][2][H][W]."""
    import torch
    lib = _load(REFRTC_SO)
    if not getattr(lib, "_typed", False):
        c_int, c_float, c_vp = ctypes.c_int, ctypes.c_float, ctypes.c_void_p
        lib.refrtc_last_error.restype = ctypes.c_char_p
        lib.refrtc_window.argtypes = [c_vp, c_vp] + [c_int] * 3 + [c_float] + [c_int] * 6 + \
            [c_float, c_float, c_int, c_float, c_int, c_int, c_int, c_vp]
        lib._typed = True
    np_, h, w = _check_window(window, radius, chroma)
    stride = (w + 31) // 32 * 32
    final = ref_window is not None
    tw = 2 * radius + 1
    src = np.zeros((2 if final else 1, np_, tw, h, stride), np.float32)
    if final:
        src[0, ..., :w] = ref_window
        src[1, ..., :w] = window
    else:
        src[0, ..., :w] = window
    d_src = torch.from_numpy(src).cuda()
    d_res = torch.zeros((np_, tw, 2, h, stride), dtype=torch.float32, device="cuda")
    s = [float(v) for v in np.atleast_1d(sigma)]
    while len(s) < 3:
        s.append(s[-1])
    sig = [scale_sigma(v, final) for v in s[:3]]
    ext = float(np.ldexp(np.float32(1.0), extractor_exp)) if extractor_exp else 0.0
    stream = torch.cuda.current_stream()
    rc = lib.refrtc_window(d_res.data_ptr(), d_src.data_ptr(), w, h, stride, sig[0], block_step,
                           bm_range, radius, ps_num, ps_range, int(chroma), sig[1], sig[2],
                           int(final), ext, bm_error, transform_2d, transform_1d,
                           ctypes.c_void_p(stream.cuda_stream))
    if rc != 0:
        raise RuntimeError(f"refrtc_window: {lib.refrtc_last_error().decode()}")
    torch.cuda.synchronize()
    return d_res.cpu().numpy()[..., :w].copy()


def refgpu_twostage(noisy: np.ndarray, *, sigma=5.0, block_step=8, bm_range=9, radius=2,
                    ps_num=2, ps_range=4, extractor_exp=0, threads: int | None = None,
                    resources: int = 4, kind: str = "fast", device: int = 0):
    """BM3Dv2(src) then BM3Dv2(src, ref=vbasic) on a GRAYS clip [N][H][W]
    with the reference plugin's host pipeline around its own kernel
    (resources=4 is fast=True). Returns (vfinal [N][H][W], stage seconds
    [basic, its VAggregate, final, its VAggregate])."""
    lib = refgpu_lib(kind)
    n, h, w = noisy.shape
    stride = w
    src = np.ascontiguousarray(noisy, np.float32)
    dst = np.zeros_like(src)
    secs = (ctypes.c_double * 4)()
    threads = threads or os.cpu_count() or 1
    _refgpu_check(lib, lib.refgpu_vbm3d_twostage(
        src.ctypes.data, dst.ctypes.data, n, w, h, stride, float(sigma), block_step, bm_range,
        radius, ps_num, ps_range, extractor_exp, threads, resources, device, secs),
        "refgpu_vbm3d_twostage")
    return dst, list(secs)


# --------------------------------------------------------------------------
# padded, aligned plane buffers
# --------------------------------------------------------------------------
def padded_stride(width: int) -> int:
    return (width + 7) // 8 * 8


def aligned_empty(shape, dtype=np.float32, align: int = 64) -> np.ndarray:
    dtype = np.dtype(dtype)
    n = int(np.prod(shape))
    raw = np.zeros(n * dtype.itemsize + align, dtype=np.uint8)
    off = (-raw.ctypes.data) % align
    return raw[off:off + n * dtype.itemsize].view(dtype).reshape(shape)


def _to_planes(arr: np.ndarray, stride: int) -> np.ndarray:
    """[..., H, W] float32 -> aligned [..., H, stride] copy (zero padded)."""
    shape = arr.shape[:-1] + (stride,)
    out = aligned_empty(shape)
    out[..., : arr.shape[-1]] = arr
    return out


def _ptr_array(planes: np.ndarray):
    """[n, H, stride] -> (c_void_p * n) of plane pointers."""
    n = planes.shape[0]
    arr = (ctypes.c_void_p * n)()
    step = planes.strides[0]
    base = planes.ctypes.data
    for i in range(n):
        arr[i] = base + i * step
    return arr


def _check_window(window: np.ndarray, radius: int, chroma: bool) -> tuple[int, int, int]:
    if window.ndim != 4:
        raise ValueError("window must be [planes][2r+1][H][W]")
    np_, tw, h, w = window.shape
    if np_ != (3 if chroma else 1) or tw != 2 * radius + 1:
        raise ValueError("window shape does not match radius/chroma")
    return np_, h, w


def _sigma3(sigma, np_: int) -> "ctypes.Array":
    s = list(np.atleast_1d(np.asarray(sigma, dtype=np.float64)))
    while len(s) < 3:
        s.append(s[-1])
    return (ctypes.c_float * 3)(*[float(v) for v in s[:3]]) if np_ == 3 else (ctypes.c_float * 3)(float(s[0]), 0.0, 0.0)


# --------------------------------------------------------------------------
# reference bm3dcpu
# --------------------------------------------------------------------------
def ref_bm3d(window: np.ndarray, ref_window: np.ndarray | None = None, *, sigma=3.0,
             block_step=8, bm_range=9, radius=0, ps_num=2, ps_range=4, chroma=False,
             kind: str = "exact") -> np.ndarray:
    """One bm3dcpu call over a temporal window (cpu_source/source.cpp:769-911)."""
    lib = ref_lib(kind)
    np_, h, w = _check_window(window, radius, chroma)
    stride = padded_stride(w)
    tw = 2 * radius + 1
    src = _to_planes(np.ascontiguousarray(window, np.float32).reshape(np_ * tw, h, w), stride)
    refp = None
    if ref_window is not None:
        refp = _to_planes(np.ascontiguousarray(ref_window, np.float32).reshape(np_ * tw, h, w), stride)
    if radius == 0:
        dst = aligned_empty((np_, h, stride))
    else:
        dst = aligned_empty((np_, tw, 2, h, stride))
    dptrs = (ctypes.c_void_p * np_)(*[dst.ctypes.data + i * dst.strides[0] for i in range(np_)])
    rc = lib.ref_bm3d(dptrs, _ptr_array(src), _ptr_array(refp) if refp is not None else None,
                      ctypes.c_int(w), ctypes.c_int(h), ctypes.c_int(stride), _sigma3(sigma, np_),
                      ctypes.c_int(block_step), ctypes.c_int(bm_range), ctypes.c_int(radius),
                      ctypes.c_int(ps_num), ctypes.c_int(ps_range), ctypes.c_int(int(chroma)))
    if rc != 0:
        raise ValueError("ref_bm3d rejected its arguments")
    return np.ascontiguousarray(dst[..., :w])


def num_blocks(width: int, height: int, block_step: int) -> int:
    nx = len(range(0, width - 8 + block_step, block_step))
    ny = len(range(0, height - 8 + block_step, block_step))
    return nx * ny


def ref_match_lists(mwindow: np.ndarray, *, block_step=8, bm_range=9, radius=0, ps_num=2,
                    ps_range=4, kind: str = "exact"):
    """Block-matching lists of bm3dcpu for every reference block.

    mwindow: [2r+1][H][W] matching planes (src for basic, ref for final).
    Returns (pre [nb,8,3], pre_err [nb,8], post [nb,8,3]) with columns (x, y, z).
    """
    lib = ref_lib(kind)
    tw, h, w = mwindow.shape
    stride = padded_stride(w)
    planes = _to_planes(np.ascontiguousarray(mwindow, np.float32), stride)
    nb = num_blocks(w, h, block_step)
    pre = np.zeros((nb, 8, 3), np.int32)
    post = np.zeros((nb, 8, 3), np.int32)
    err = np.zeros((nb, 8), np.float32)
    got = lib.ref_match_lists(pre.ctypes.data_as(_ip), err.ctypes.data_as(_fp),
                              post.ctypes.data_as(_ip), _ptr_array(planes), ctypes.c_int(w),
                              ctypes.c_int(h), ctypes.c_int(stride), ctypes.c_int(block_step),
                              ctypes.c_int(bm_range), ctypes.c_int(radius), ctypes.c_int(ps_num),
                              ctypes.c_int(ps_range))
    assert got == nb
    return pre, err, post


# --------------------------------------------------------------------------
# project C restatement
# --------------------------------------------------------------------------
def port_bm3d(window: np.ndarray, ref_window: np.ndarray | None = None, *, sigma=3.0,
              block_step=8, bm_range=9, radius=0, ps_num=2, ps_range=4, chroma=False,
              extractor_exp: int = 0, fp64: bool = False, match_in: np.ndarray | None = None,
              return_matches: bool = False, return_acc: bool = False, bm_error: int = 0,
              transform_2d: int = 0, transform_1d: int = 0):
    """One BM3D call of the C restatement. Same shapes as :func:`ref_bm3d`.

    extractor_exp > 0 switches the FP32 accumulation to the CUDA kernel's
    pre-rounded terms (value + 2^e) - 2^e. fp64 runs the FP64 oracle.
    return_acc: return the [planes][2r+1][2][H][W] accumulators even for radius 0.
    match_in: optional [nb,8,3] match lists to use instead of searching.
    bm_error / transform_2d / transform_1d: the run-time-compiled plugin's
    variants (0-4: ssd, sad, zssd, zsad, ssd/norm; 0-3: dct, haar, wht,
    bior1.5), FP32 only.
    """
    lib = port_lib()
    np_, h, w = _check_window(window, radius, chroma)
    stride = padded_stride(w)
    tw = 2 * radius + 1
    src = _to_planes(np.ascontiguousarray(window, np.float32).reshape(np_ * tw, h, w), stride)
    refp = None
    if ref_window is not None:
        refp = _to_planes(np.ascontiguousarray(ref_window, np.float32).reshape(np_ * tw, h, w), stride)
    dt = np.float64 if fp64 else np.float32
    acc = aligned_empty((np_, tw, 2, h, stride), dt)
    out = aligned_empty((np_, h, stride), dt)
    aptrs = (ctypes.c_void_p * np_)(*[acc.ctypes.data + i * acc.strides[0] for i in range(np_)])
    optrs = (ctypes.c_void_p * np_)(*[out.ctypes.data + i * out.strides[0] for i in range(np_)])
    nb = num_blocks(w, h, block_step)
    mout = np.zeros((nb, 8, 3), np.int32)
    min_ptr = None
    if match_in is not None:
        match_in = np.ascontiguousarray(match_in, np.int32)
        assert match_in.shape == (nb, 8, 3)
        min_ptr = match_in.ctypes.data_as(_ip)
    common = (ctypes.c_int(w), ctypes.c_int(h), ctypes.c_int(stride), _sigma3(sigma, np_),
              ctypes.c_int(block_step), ctypes.c_int(bm_range), ctypes.c_int(radius),
              ctypes.c_int(ps_num), ctypes.c_int(ps_range), ctypes.c_int(int(chroma)))
    sp = _ptr_array(src)
    rp = _ptr_array(refp) if refp is not None else None
    if bm_error or transform_2d or transform_1d:
        if fp64:
            raise ValueError("the variants have an FP32 restatement only")
        ext = float(np.ldexp(1.0, extractor_exp)) if extractor_exp else 0.0
        rc = lib.port_bm3d_rtc_f32(aptrs, optrs, sp, rp, *common, ctypes.c_float(ext),
                                   ctypes.c_int(bm_error), ctypes.c_int(transform_2d),
                                   ctypes.c_int(transform_1d), min_ptr, mout.ctypes.data_as(_ip))
    elif fp64:
        rc = lib.port_bm3d_f64(aptrs, optrs, sp, rp, *common, min_ptr, mout.ctypes.data_as(_ip))
    else:
        ext = float(np.ldexp(1.0, extractor_exp)) if extractor_exp else 0.0
        rc = lib.port_bm3d_f32(aptrs, optrs, sp, rp, *common, ctypes.c_float(ext), min_ptr,
                               mout.ctypes.data_as(_ip))
    if rc < 0:
        raise ValueError("port_bm3d rejected its arguments")
    if radius == 0 and not return_acc:
        res = np.ascontiguousarray(out[..., :w])
    else:
        res = np.ascontiguousarray(acc[..., :w])
    if return_matches:
        return res, mout
    return res


def port_rescore(window: np.ndarray, lists: np.ndarray, *, block_step: int = 8) -> np.ndarray:
    """Final-stage lists from basic lists (FP32, the reference's block distance,
    stable ascending order). window: [2r+1][H][W] matching planes (the basic
    estimate); lists: [nb][8][3] (x, y, slot). Returns the re-ordered lists."""
    lib = port_lib()
    tw, h, w = window.shape
    radius = (tw - 1) // 2
    stride = padded_stride(w)
    planes = _to_planes(np.asarray(window, np.float32)[None], stride)[0]
    out = np.ascontiguousarray(lists, np.int32).copy()
    ptrs = (ctypes.c_void_p * tw)(*[planes.ctypes.data + z * planes.strides[0] for z in range(tw)])
    lib.port_rescore_f32(out.ctypes.data_as(_ip), ptrs, ctypes.c_int(w), ctypes.c_int(h),
                         ctypes.c_int(stride), ctypes.c_int(block_step), ctypes.c_int(radius))
    return out


def port_vaggregate(vframes: np.ndarray, n: int, num_frames: int, fp64: bool = False) -> np.ndarray:
    """VAggregate of output frame n. vframes: [2r+1][2r+1][2][H][W] raw outputs of
    frames clamp(n-r..n+r) (cpu_source/source.cpp:1507-1544)."""
    lib = port_lib()
    tw, tw2, two, h, w = vframes.shape
    assert tw == tw2 and two == 2
    radius = (tw - 1) // 2
    stride = padded_stride(w)
    dt = np.float64 if fp64 else np.float32
    v = aligned_empty((tw, tw, 2, h, stride), dt)
    v[..., :w] = vframes
    dst = aligned_empty((h, stride), dt)
    ptrs = (ctypes.c_void_p * tw)(*[v.ctypes.data + i * v.strides[0] for i in range(tw)])
    fn = lib.port_vaggregate_f64 if fp64 else lib.port_vaggregate_f32
    fn(dst.ctypes.data_as(_dp if fp64 else _fp), ptrs, ctypes.c_int(w), ctypes.c_int(h),
       ctypes.c_int(stride), ctypes.c_int(radius), ctypes.c_int(n), ctypes.c_int(num_frames))
    return np.ascontiguousarray(dst[:, :w])


def port_dct8(v: np.ndarray, forward: bool = True, fp64: bool = False) -> np.ndarray:
    lib = port_lib()
    a = np.ascontiguousarray(v, np.float64 if fp64 else np.float32).copy()
    if fp64:
        lib.port_dct8_f64(a.ctypes.data_as(_dp), ctypes.c_int(int(forward)))
    else:
        lib.port_dct8_f32(a.ctypes.data_as(_fp), ctypes.c_int(int(forward)))
    return a


# --------------------------------------------------------------------------
# whole-clip drivers (the filter graph of BM3D / VAggregate / BM3Dv2)
# --------------------------------------------------------------------------
def clip_window(clip: np.ndarray, n: int, radius: int) -> np.ndarray:
    """clip [N][planes][H][W] -> window [planes][2r+1][H][W] with clamped indices
    (source/source.cpp:240-264)."""
    N = clip.shape[0]
    idx = [min(max(n + i, 0), N - 1) for i in range(-radius, radius + 1)]
    return np.ascontiguousarray(np.stack([clip[i] for i in idx], axis=1))


def clip_bm3d_v2(bm3d_fn, clip: np.ndarray, ref: np.ndarray | None, *, radius: int, chroma: bool,
                 vagg_fn=None, **kw) -> np.ndarray:
    """BM3Dv2 over a whole clip: BM3D per frame, then VAggregate when radius > 0
    (source/source.cpp:911-989). clip: [N][planes][H][W]."""
    N = clip.shape[0]
    if radius == 0:
        return np.stack([bm3d_fn(clip_window(clip, n, 0), None if ref is None else clip_window(ref, n, 0),
                                 radius=0, chroma=chroma, **kw) for n in range(N)])
    raw = [bm3d_fn(clip_window(clip, n, radius), None if ref is None else clip_window(ref, n, radius),
                   radius=radius, chroma=chroma, **kw) for n in range(N)]
    vagg_fn = vagg_fn or port_vaggregate
    planes = clip.shape[1]
    out = np.empty_like(clip)
    for n in range(N):
        for p in range(planes):
            idx = [min(max(n + i, 0), N - 1) for i in range(-radius, radius + 1)]
            out[n, p] = vagg_fn(np.stack([raw[i][p] for i in idx]), n, N)
    return out


# --------------------------------------------------------------------------
# learned match proposal (the project's own definition; no reference code)
# --------------------------------------------------------------------------
def port_learned_match(mwindow: np.ndarray, embs: np.ndarray, *, block_step=8, bm_range=9,
                       radius=0, ps_num=2, ps_range=4, cells_spatial=4, cells_temporal=4,
                       fallback_ssd: float = 0.0):
    """Learned match lists of one window (oracle/learned_port.c).

    mwindow: [2r+1][H][W] matching planes; embs: [2r+1][H/2][W/2][16] uint8
    embeddings. Returns (lists [nb][8][3], fallback flags [nb])."""
    lib = port_lib()
    tw, h, w = mwindow.shape
    stride = padded_stride(w)
    planes = _to_planes(np.ascontiguousarray(mwindow, np.float32), stride)
    e8 = np.ascontiguousarray(embs, np.uint8)
    eptrs = (ctypes.c_void_p * tw)(*[e8[z].ctypes.data for z in range(tw)])
    nb = num_blocks(w, h, block_step)
    out = np.zeros((nb, 8, 3), np.int32)
    fell = np.zeros(nb, np.int32)
    got = lib.port_learned_match(_ptr_array(planes), eptrs, ctypes.c_int(w), ctypes.c_int(h),
                                 ctypes.c_int(stride), ctypes.c_int(block_step),
                                 ctypes.c_int(bm_range), ctypes.c_int(radius),
                                 ctypes.c_int(ps_num), ctypes.c_int(ps_range),
                                 ctypes.c_int(cells_spatial), ctypes.c_int(cells_temporal),
                                 ctypes.c_float(fallback_ssd), out.ctypes.data_as(_ip),
                                 fell.ctypes.data_as(_ip))
    if got != nb:
        raise ValueError("port_learned_match rejected its arguments")
    return out, fell


def port_proposer_embed_bf16(plane: np.ndarray, params: np.ndarray) -> np.ndarray:
    """The proposer's inference arithmetic on one plane [H][W] with BF16
    operands and exact sums: [H/2][W/2][16] float32 before quantisation."""
    lib = port_lib()
    h, w = plane.shape
    stride = padded_stride(w)
    p = aligned_empty((h, stride))
    p[:, :w] = plane
    prm = np.ascontiguousarray(params, np.float32)
    out = np.zeros((h // 2, w // 2, 16), np.float32)
    lib.port_proposer_embed_bf16(p.ctypes.data_as(_fp), ctypes.c_int(w), ctypes.c_int(h),
                                 ctypes.c_int(stride), prm.ctypes.data_as(_fp),
                                 out.ctypes.data_as(_fp))
    return out


def quantize_embedding(v: np.ndarray, quant: np.ndarray) -> np.ndarray:
    """q = clamp(rint(v * qscale + qoff[c]), 0, 255) with one FP32 rounding of
    the product-sum (the inference kernel's fused multiply-add)."""
    v64 = np.asarray(v, np.float64) * np.float64(np.float32(quant[0])) + \
        np.asarray(quant[1:], np.float32).astype(np.float64)
    return np.clip(np.rint(v64.astype(np.float32)), 0, 255).astype(np.uint8)
