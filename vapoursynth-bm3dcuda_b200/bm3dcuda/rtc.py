"""The run-time-compiled plugin's interface (namespace ``bm3dcuda_rtc``).

bm3dcuda_rtc.BM3D / BM3Dv2 take the arguments of bm3dcuda plus three
experimental per-plane strings (README.md:118-135; parsed at
rtc_source/source.cpp:854-911, registered at 1370-1387):

  bm_error_s      "ssd" (default), "sad", "zssd", "zsad", "ssd/norm"
  transform_2d_s  "dct" (default), "haar", "wht", "bior1.5"  (rows, columns)
  transform_1d_s  "dct" (default), "haar", "wht", "bior1.5"  (across the group)

Values are case-insensitive, missing planes repeat the previous plane's value,
and errors carry the plugin's "BM3D_RTC: " prefix. The reference compiles one
kernel per plane with NVRTC; here the same variants are template and
run-time choices of the engine's sm_100a kernels (no run-time compilation).
VAggregate is the bm3dcuda one.
"""
from __future__ import annotations

from . import BM3DError, Clip, FLT_EPSILON, VAggregate, _arr, _Engine, _parse

__all__ = ["BM3D", "BM3Dv2", "VAggregate", "BM_ERRORS", "TRANSFORMS"]

BM_ERRORS = {"ssd": 0, "sad": 1, "zssd": 2, "zsad": 3, "ssd/norm": 4}
TRANSFORMS = {"dct": 0, "haar": 1, "wht": 2, "bior1.5": 3}


def _variant_strings(values, table, name):
    out = []
    vals = _arr(values)
    for i in range(3):
        if i < len(vals):
            v = vals[i]
            v = v.decode() if isinstance(v, bytes) else str(v)
            v = v.lower()
            if v not in table:
                raise BM3DError(f"BM3D_RTC: invalid '{name}': {v}")
            out.append(table[v])
        else:
            out.append(0 if i == 0 else out[i - 1])
    return out


def _rtc_call(fn):
    try:
        return fn()
    except BM3DError as e:
        msg = str(e)
        if msg.startswith("BM3D: "):
            msg = "BM3D_RTC: " + msg[len("BM3D: "):]
        raise BM3DError(msg) from None


def BM3D(clip: Clip, ref: Clip | None = None, sigma=None, block_step=None, bm_range=None,
         radius=None, ps_num=None, ps_range=None, chroma=None, device_id=None, fast=None,
         extractor_exp=None, bm_error_s=None, transform_2d_s=None, transform_1d_s=None,
         zero_init=None) -> Clip:
    """bm3dcuda_rtc.BM3D (rtc_source/source.cpp:700-1100): as bm3dcuda.BM3D
    with the block distance and transforms chosen per plane."""
    def run():
        a = _parse(clip, ref, sigma, block_step, bm_range, radius, ps_num, ps_range, chroma,
                   device_id, fast, extractor_exp, zero_init)
        variant = (_variant_strings(bm_error_s, BM_ERRORS, "bm_error_s"),
                   _variant_strings(transform_2d_s, TRANSFORMS, "transform_2d_s"),
                   _variant_strings(transform_1d_s, TRANSFORMS, "transform_1d_s"))
        eng = _Engine(clip, a, variant)
        try:
            planes = eng.run(clip, ref, a.radius > 0)
        finally:
            eng.close()
        props = [dict(p) for p in clip.props]
        if a.radius > 0:
            for p in props:
                p["BM3D_V_radius"] = a.radius
                p["BM3D_V_process"] = [int(v) for v in a.process]
        return Clip(planes, clip.format, props)
    return _rtc_call(run)


def BM3Dv2(clip: Clip, ref: Clip | None = None, sigma=None, block_step=None, bm_range=None,
           radius=None, ps_num=None, ps_range=None, chroma=None, device_id=None, fast=None,
           extractor_exp=None, bm_error_s=None, transform_2d_s=None, transform_1d_s=None,
           zero_init=None) -> Clip:
    """bm3dcuda_rtc.BM3Dv2 (rtc_source/source.cpp:1290-1357): BM3D then
    VAggregate for radius > 0, the aggregation fused on the device."""
    sig = _arr(sigma)
    process = [True, True, True]
    for i in range(min(3, len(sig))):
        if float(sig[i]) < FLT_EPSILON:
            process[i] = False
    if len(sig) > 0:
        for i in range(len(sig), 3):
            process[i] = process[i - 1]
    if all(not process[i] for i in range(clip.num_planes)):
        return clip

    def run():
        a = _parse(clip, ref, sigma, block_step, bm_range, radius, ps_num, ps_range, chroma,
                   device_id, fast, extractor_exp, zero_init)
        variant = (_variant_strings(bm_error_s, BM_ERRORS, "bm_error_s"),
                   _variant_strings(transform_2d_s, TRANSFORMS, "transform_2d_s"),
                   _variant_strings(transform_1d_s, TRANSFORMS, "transform_1d_s"))
        eng = _Engine(clip, a, variant)
        try:
            planes = eng.run(clip, ref, raw=False)
        finally:
            eng.close()
        return Clip(planes, clip.format, [dict(p) for p in clip.props])
    return _rtc_call(run)
