"""ctypes driver of the fake VapourSynth core (fakecore.cpp), test-only."""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PKG = os.path.join(ROOT, "vapoursynth-bm3dcuda_b200")
FAKECORE_SO = os.path.join(HERE, "libfakecore.so")
PLUGIN_SO = os.path.join(PKG, "libbm3dcuda_vs.so")
RTC_PLUGIN_SO = os.path.join(PKG, "libbm3dcuda_rtc_vs.so")

# preset ids of vsapi_min/VapourSynth.h
FORMAT_IDS = {"GRAYS": 1000013, "YUV444PS": 3000021, "RGBS": 2000022, "YUV420PS": 3000020,
              "GRAY8": 1000001, "GRAYH": 1000012}
_vp = ctypes.c_void_p


def build() -> None:
    src = os.path.join(HERE, "fakecore.cpp")
    if not os.path.exists(FAKECORE_SO) or os.path.getmtime(FAKECORE_SO) < os.path.getmtime(src):
        subprocess.run(["g++", "-std=c++17", "-O1", "-fPIC", "-shared",
                        f"-I{os.path.join(PKG, 'csrc', 'vsapi_min')}", src, "-ldl", "-o",
                        FAKECORE_SO], check=True)
    subprocess.run(["make", "-s", "-C", PKG], check=True)


class VSError(RuntimeError):
    pass


class Node:
    """A node reference held by the test (one reference; release with Core.free)."""

    def __init__(self, ptr):
        self.ptr = ptr


class Core:
    """One fake core with the bm3dcuda plugin (or another plugin binary) loaded."""

    def __init__(self, plugin_so: str = PLUGIN_SO):
        L = ctypes.CDLL(FAKECORE_SO)
        sig = {
            "fc_last_error": (ctypes.c_char_p, []),
            "fc_core_new": (_vp, []),
            "fc_load_plugin": (ctypes.c_int, [_vp, ctypes.c_char_p]),
            "fc_plugin_id": (ctypes.c_char_p, [_vp]),
            "fc_plugin_ns": (ctypes.c_char_p, [_vp]),
            "fc_function_args": (ctypes.c_char_p, [_vp, ctypes.c_char_p]),
            "fc_map_new": (_vp, []),
            "fc_map_free": (None, [_vp]),
            "fc_map_set_int": (None, [_vp, ctypes.c_char_p, ctypes.c_longlong, ctypes.c_int]),
            "fc_map_set_float": (None, [_vp, ctypes.c_char_p, ctypes.c_double, ctypes.c_int]),
            "fc_map_set_node": (None, [_vp, ctypes.c_char_p, _vp]),
            "fc_map_set_data": (None, [_vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]),
            "fc_map_error": (ctypes.c_char_p, [_vp]),
            "fc_map_get_node": (_vp, [_vp, ctypes.c_char_p]),
            "fc_invoke": (_vp, [_vp, ctypes.c_char_p, _vp]),
            "fc_clip_new": (_vp, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
            "fc_clip_set_plane": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp]),
            "fc_node_free": (None, [_vp]),
            "fc_video_info": (None, [_vp] + [ctypes.POINTER(ctypes.c_int)] * 4),
            "fc_get_frame": (_vp, [_vp, ctypes.c_int]),
            "fc_frame_dims": (None, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int)]),
            "fc_frame_read": (None, [_vp, ctypes.c_int, _vp]),
            "fc_frame_prop_int": (ctypes.c_longlong, [_vp, ctypes.c_char_p, ctypes.c_int,
                                                      ctypes.POINTER(ctypes.c_int)]),
            "fc_frame_free": (None, [_vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        self.L = L
        self.core = L.fc_core_new()
        if L.fc_load_plugin(self.core, plugin_so.encode()) != 0:
            raise VSError(L.fc_last_error().decode())

    @property
    def plugin_id(self) -> str:
        return self.L.fc_plugin_id(self.core).decode()

    @property
    def namespace(self) -> str:
        return self.L.fc_plugin_ns(self.core).decode()

    def function_args(self, name: str) -> str | None:
        a = self.L.fc_function_args(self.core, name.encode())
        return a.decode() if a else None

    def clip(self, planes, fmt: str = "GRAYS"):
        """planes: list of [N, H_p, W_p] arrays (or a single [N, H, W] array)."""
        if isinstance(planes, np.ndarray):
            planes = [planes]
        n, h, w = planes[0].shape
        dtype = np.uint8 if fmt == "GRAY8" else (np.float16 if fmt == "GRAYH" else np.float32)
        node = self.L.fc_clip_new(FORMAT_IDS[fmt], w, h, n)
        for p, arr in enumerate(planes):
            arr = np.ascontiguousarray(arr, dtype)
            for i in range(n):
                self.L.fc_clip_set_plane(node, i, p, arr[i].ctypes.data)
        return Node(node)

    def invoke(self, name: str, **args):
        m = self.L.fc_map_new()
        for k, v in args.items():
            if v is None:
                continue
            vals = v if isinstance(v, (list, tuple)) else [v]
            for j, x in enumerate(vals):
                if isinstance(x, Node):
                    self.L.fc_map_set_node(m, k.encode(), x.ptr)
                elif isinstance(x, float):
                    self.L.fc_map_set_float(m, k.encode(), x, 1 if j else 0)
                elif isinstance(x, (str, bytes)):
                    self.L.fc_map_set_data(m, k.encode(), x.encode() if isinstance(x, str) else x,
                                           1 if j else 0)
                else:
                    self.L.fc_map_set_int(m, k.encode(), int(x), 1 if j else 0)
        out = self.L.fc_invoke(self.core, name.encode(), m)
        self.L.fc_map_free(m)
        err = self.L.fc_map_error(out)
        if err:
            self.L.fc_map_free(out)
            raise VSError(err.decode())
        node = self.L.fc_map_get_node(out, b"clip")
        self.L.fc_map_free(out)
        return Node(node)

    def info(self, node):
        w, h, n, f = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self.L.fc_video_info(node.ptr, ctypes.byref(w), ctypes.byref(h), ctypes.byref(n), ctypes.byref(f))
        return w.value, h.value, n.value, f.value

    def frames(self, node, num_planes: int = 1):
        """All frames as a list of planes, each [N, H_p, W_p] float32; plus props of frame 0."""
        _, _, n, _ = self.info(node)
        out = [[] for _ in range(num_planes)]
        props = {}
        for i in range(n):
            f = self.L.fc_get_frame(node.ptr, i)
            if not f:
                raise VSError(self.L.fc_last_error().decode())
            for p in range(num_planes):
                w, h = ctypes.c_int(), ctypes.c_int()
                self.L.fc_frame_dims(f, p, ctypes.byref(w), ctypes.byref(h))
                a = np.zeros((h.value, w.value), np.float32)
                self.L.fc_frame_read(f, p, a.ctypes.data)
                out[p].append(a)
            if i == 0:
                for key, cnt in (("BM3D_V_radius", 1), ("BM3D_V_process", 3)):
                    vals = []
                    for k in range(cnt):
                        e = ctypes.c_int()
                        v = self.L.fc_frame_prop_int(f, key.encode(), k, ctypes.byref(e))
                        if not e.value:
                            vals.append(v)
                    if vals:
                        props[key] = vals if cnt > 1 else vals[0]
            self.L.fc_frame_free(f)
        return [np.stack(p) for p in out], props

    def free(self, node):
        self.L.fc_node_free(node.ptr)
