"""ctypes binding of libbm3d_b200.so (the C ABI declared in include/bm3d_b200.h).

The library is built in-tree (``make -C vapoursynth-bm3dcuda_b200``). There is
no CPU fallback: if the library or a CUDA device is missing, calls raise.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "libbm3d_b200.so")

OK = 0
ERR_INVALID = 1
ERR_CUDA = 2
ERR_UNSUPPORTED = 3
ERR_NOMEM = 4
DST_AGGREGATED = 0
DST_RAW = 1
MAX_DIM = 16383
MAX_RADIUS = 7

c_int = ctypes.c_int
c_float = ctypes.c_float
c_void_p = ctypes.c_void_p
c_ll = ctypes.c_longlong


class Params(ctypes.Structure):
    """struct bm3d_b200_params."""
    _fields_ = [
        ("sigma", c_float * 3),
        ("block_step", c_int * 3),
        ("bm_range", c_int * 3),
        ("ps_num", c_int * 3),
        ("ps_range", c_int * 3),
        ("radius", c_int),
        ("chroma", c_int),
        ("extractor_exp", c_int),
        ("zero_init", c_int),
    ]


# name -> (restype, argtypes); the exported surface of include/bm3d_b200.h
SIGNATURES = {
    "bm3d_b200_last_error": (ctypes.c_char_p, []),
    "bm3d_b200_abi_version": (c_int, []),
    "bm3d_b200_scale_sigma": (c_float, [c_float, c_int]),
    "bm3d_b200_graph_create": (c_int, [ctypes.POINTER(c_void_p), c_void_p, c_void_p, c_void_p,
                                       c_int, c_int, c_int, c_float, c_int, c_int, c_int, c_int,
                                       c_int, c_int, c_float, c_float, c_int, c_float]),
    "bm3d_b200_graph_create_rtc": (c_int, [ctypes.POINTER(c_void_p), c_void_p, c_void_p, c_void_p,
                                       c_int, c_int, c_int, c_float, c_int, c_int, c_int, c_int,
                                       c_int, c_int, c_float, c_float, c_int, c_float, c_int, c_int, c_int]),
    "bm3d_b200_graph_launch": (c_int, [c_void_p, c_void_p]),
    "bm3d_b200_graph_launch_device": (c_int, [c_void_p, c_void_p]),
    "bm3d_b200_graph_matches": (c_int, [c_void_p, c_void_p, c_int, ctypes.POINTER(c_int)]),
    "bm3d_b200_graph_destroy": (None, [c_void_p]),
    "bm3d_b200_window_noalloc": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_float, c_int,
                                         c_int, c_int, c_int, c_int, c_int, c_float, c_float,
                                         c_int, c_float, c_void_p]),
    "bm3d_b200_aggregate": (c_int, [c_void_p, c_int, c_void_p, c_int, c_int, c_int, c_void_p]),
    "bm3d_b200_vaggregate": (c_int, [c_void_p, c_int, ctypes.POINTER(c_void_p), c_int, c_int,
                                     c_int, c_int, c_int, c_int, c_void_p]),
    "bm3d_b200_params_default": (None, [ctypes.POINTER(Params)]),
    "bm3d_b200_clip_create": (c_int, [ctypes.POINTER(c_void_p), c_int, c_int, c_int, c_int, c_int,
                                      c_int, ctypes.POINTER(Params), c_int]),
    "bm3d_b200_clip_frame_floats": (c_ll, [c_void_p]),
    "bm3d_b200_clip_raw_frame_floats": (c_ll, [c_void_p]),
    "bm3d_b200_clip_stride": (c_int, [c_void_p]),
    "bm3d_b200_clip_run": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "bm3d_b200_clip_run_host": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "bm3d_b200_clip_twostage_host": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "bm3d_b200_clip_twostage_host_async": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "bm3d_b200_clip_twostage": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "bm3d_b200_clip_set_profiling": (c_int, [c_void_p, c_int]),
    "bm3d_b200_clip_stage_times": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "bm3d_b200_clip_destroy": (None, [c_void_p]),
    "bm3d_b200_selftest_reciprocal": (c_int, [ctypes.c_uint, ctypes.c_uint, c_void_p, c_void_p]),
    "bm3d_b200_batch_create": (c_int, [ctypes.POINTER(c_void_p), c_int]),
    "bm3d_b200_batch_add": (c_int, [c_void_p, c_int, c_int, c_int, ctypes.POINTER(Params),
                                    c_void_p, c_void_p, ctypes.POINTER(c_int)]),
    "bm3d_b200_batch_autotune": (c_int, [c_void_p, c_void_p]),
    "bm3d_b200_batch_config": (c_int, [c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int)]),
    "bm3d_b200_batch_grids": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "bm3d_b200_batch_run": (c_int, [c_void_p, c_void_p]),
    "bm3d_b200_batch_basic": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "bm3d_b200_batch_latencies": (c_int, [c_void_p, c_void_p, c_int]),
    "bm3d_b200_batch_destroy": (None, [c_void_p]),
    "bm3d_b200_proposer_num_params": (c_int, []),
    "bm3d_b200_proposer_create": (c_int, [ctypes.POINTER(c_void_p), c_void_p, c_int]),
    "bm3d_b200_proposer_get_params": (c_int, [c_void_p, c_void_p]),
    "bm3d_b200_proposer_set_params": (c_int, [c_void_p, c_void_p]),
    "bm3d_b200_proposer_destroy": (None, [c_void_p]),
    "bm3d_b200_proposer_get_quant": (c_int, [c_void_p, c_void_p]),
    "bm3d_b200_proposer_set_quant": (c_int, [c_void_p, c_void_p]),
    "bm3d_b200_proposer_calibrate": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int,
                                             c_void_p]),
    "bm3d_b200_proposer_teacher": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_int,
                                           c_int, c_void_p, c_void_p]),
    "bm3d_b200_proposer_loss_grad": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int,
                                             c_void_p, c_void_p, c_int, c_int, c_float, c_void_p,
                                             c_void_p, c_void_p]),
    "bm3d_b200_proposer_train": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_void_p,
                                         c_void_p, c_int, c_int, c_float, c_int, c_float,
                                         c_void_p, c_void_p]),
    "bm3d_b200_proposer_embed": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_void_p,
                                         c_void_p]),
    "bm3d_b200_proposer_status": (c_int, [c_void_p]),
    "bm3d_b200_proposer_embed_f32": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int,
                                             c_void_p, c_void_p]),
    "bm3d_b200_learned_match": (c_int, [ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p), c_int,
                                        c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_int,
                                        c_int, c_float, c_void_p, c_void_p, c_int,
                                        ctypes.POINTER(c_int)]),
    "bm3d_b200_clip_set_proposer": (c_int, [c_void_p, c_void_p, c_int, c_int, c_float]),
    "bm3d_b200_clip_set_precision": (c_int, [c_void_p, c_int]),
    "bm3d_b200_clip_status": (c_int, [c_void_p]),
    "bm3d_b200_clip_set_variant": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "bm3d_b200_stream_create": (c_int, [ctypes.POINTER(c_void_p), c_int, c_int, c_int, c_int,
                                        c_int, c_int, c_void_p, c_int, c_int]),
    "bm3d_b200_stream_frame": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_void_p]),
    "bm3d_b200_stream_set_variant": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "bm3d_b200_stream_stats": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_longlong),
                                       ctypes.POINTER(ctypes.c_longlong)]),
    "bm3d_b200_stream_timings": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "bm3d_b200_stream_concurrency": (c_int, [c_void_p]),
    "bm3d_b200_stream_set_concurrency": (c_int, [c_void_p, c_int]),
    "bm3d_b200_stream_set_proposer": (c_int, [c_void_p, c_void_p, c_int, c_int, ctypes.c_float]),
    "bm3d_b200_stream_destroy": (None, [c_void_p]),
    "bm3d_b200_clip_matches": (c_int, [c_void_p, c_int, c_void_p, c_int, ctypes.POINTER(c_int)]),
    "bm3d_b200_clip_set_final_matching": (c_int, [c_void_p, c_int]),
    "bm3d_b200_clip_learned_stats": (c_int, [c_void_p, ctypes.POINTER(c_ll), ctypes.POINTER(c_ll),
                                             c_int]),
}

STAGE_MATCH = 0
STAGE_FILTER = 1
STAGE_AGGREGATE = 2
STAGE_PROPOSE = 3
STAGE_MATCH_FINAL = 4
STAGE_FILTER_FINAL = 5
STAGE_FALLBACK = 6
PRECISION_FP32 = 0
PRECISION_SPLIT_BF16 = 1
PRECISION_TC_F16 = 2
NUM_STAGES = 7
PROPOSER_PARAMS = 4800


class BM3DError(RuntimeError):
    """Raised with the library's error message (the reference's wording)."""


_lib: ctypes.CDLL | None = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", PKG_ROOT], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise BM3DError(f"libbm3d_b200.so not built ({LIB_PATH}); run make -C {PKG_ROOT}")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    msg = lib().bm3d_b200_last_error()
    return msg.decode() if msg else ""


def check(rc: int) -> None:
    if rc != OK:
        raise BM3DError(last_error() or f"bm3d_b200 error {rc}")
