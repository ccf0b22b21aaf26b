"""ctypes binding of liboracle.so (oracle/irt_oracle.cpp).

Test infrastructure: the CPU restatement of lighting.wgsl, sdf.wgsl and
svgf.wgsl used as the parity checker and as the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")

# buffer ids of oracle_buffer()
RES = {("d", 0): 0, ("d", 1): 1, ("d", 2): 2, ("i", 0): 3, ("i", 1): 4, ("i", 2): 5}
ARCHIVE, PREV_DEPTH, PREV_NORMAL, DIRECT, LIGHTING = 6, 7, 8, 9, 10
MOMENTS = (11, 12)
FEEDBACK = (13, 14)
TEMPORAL = 15
SCRATCH = (16, 17)
HISTORIES = (18, 19)


def build_oracle():
    """Compile liboracle.so with its Makefile if it is missing or stale."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


class _Scene(C.Structure):
    _fields_ = [("objects", C.c_void_p), ("meshes", C.c_void_p), ("nodes", C.c_void_p), ("lights", C.c_void_p),
                ("atlas", C.c_void_p), ("atlas_dims", C.c_uint32 * 3)]


class _GBuffer(C.Structure):
    _fields_ = [("depth", C.c_void_p), ("normal", C.c_void_p), ("color", C.c_void_p), ("params", C.c_void_p),
                ("motion", C.c_void_p)]


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build_oracle()
        lib = C.CDLL(LIB_PATH)
        P = C.c_void_p
        lib.oracle_create.restype = P
        lib.oracle_create.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_int, C.c_int]
        lib.oracle_destroy.argtypes = [P]
        lib.oracle_lighting.restype = C.c_int
        lib.oracle_lighting.argtypes = [P, P, C.POINTER(_Scene), C.POINTER(_GBuffer), P, P, C.c_int, C.c_int]
        lib.oracle_svgf.restype = C.c_int
        lib.oracle_svgf.argtypes = [P, P, C.POINTER(_GBuffer), C.c_uint32]
        lib.oracle_end_frame.argtypes = [P, C.POINTER(_GBuffer)]
        lib.oracle_frame.restype = C.c_int
        lib.oracle_frame.argtypes = [P, P, C.POINTER(_Scene), C.POINTER(_GBuffer), P, P, C.c_uint32]
        lib.oracle_buffer.restype = P
        lib.oracle_buffer.argtypes = [P, C.c_int, C.POINTER(C.c_uint64)]
        lib.oracle_counters.argtypes = [P, C.POINTER(C.c_uint64)]
        lib.oracle_threads.restype = C.c_int
        lib.oracle_threads.argtypes = [P]
        lib.oracle_set_rows.argtypes = [P, C.c_uint32, C.c_uint32]
        lib.oracle_f32_to_f16.restype = C.c_uint16
        lib.oracle_f32_to_f16.argtypes = [C.c_float]
        lib.oracle_f16_to_f32.restype = C.c_float
        lib.oracle_f16_to_f32.argtypes = [C.c_uint16]
        lib.oracle_random_stream.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, P, P]
        lib.oracle_signed_box_distance.restype = C.c_float
        lib.oracle_signed_box_distance.argtypes = [C.POINTER(C.c_float)] * 3
        lib.oracle_res_add_u.restype = C.c_int
        lib.oracle_res_add_u.argtypes = [P, C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_uint32,
                                         C.c_uint32, C.c_float]
        lib.oracle_normalization.restype = C.c_float
        lib.oracle_normalization.argtypes = [P]
        lib.oracle_quilez_step.restype = C.c_float
        lib.oracle_quilez_step.argtypes = [C.c_float] * 5
        lib.oracle_set_field_filter.argtypes = [P, C.c_int]
        lib.oracle_sample_field.restype = C.c_float
        lib.oracle_sample_field.argtypes = [P, P, C.POINTER(C.c_uint32), C.POINTER(C.c_float), C.c_int]
        lib.oracle_mesh_distance.restype = C.c_float
        lib.oracle_mesh_distance.argtypes = [P, P, C.POINTER(C.c_uint32), C.POINTER(C.c_float)]
        _lib = lib
    return _lib


def lib():
    return _load()


def sample_field(mesh: np.ndarray, atlas_f32: np.ndarray, q, linear: int) -> float:
    """sample_field of one mesh row (MESH_DTYPE record) at grid-space point q
    over an f32 atlas [z, y, x]."""
    lib = _load()
    a = np.ascontiguousarray(atlas_f32, np.float32)
    m = np.ascontiguousarray(mesh)
    dims = (C.c_uint32 * 3)(a.shape[2], a.shape[1], a.shape[0])
    qq = (C.c_float * 3)(*[float(v) for v in q])
    return float(lib.oracle_sample_field(_p(m), _p(a), dims, qq, int(linear)))


def f16_bits(v: float) -> int:
    return int(_load().oracle_f32_to_f16(float(v)))


def f16_from_bits(h: int) -> float:
    return float(_load().oracle_f16_to_f32(h))


def _p(a):
    assert a.flags["C_CONTIGUOUS"], "oracle inputs must be C-contiguous"
    return C.c_void_p(a.ctypes.data)


class OracleScene:
    """Keeps the numpy arrays of one frame's scene alive for the oracle."""

    def __init__(self, objects, meshes, nodes, lights, atlas_f32):
        self.arrays = [np.ascontiguousarray(a) for a in (objects, meshes, nodes, lights, atlas_f32)]
        o, m, n, li, at = self.arrays
        self.s = _Scene(_p(o).value, _p(m).value, _p(n).value, _p(li).value if len(li) else None, _p(at).value,
                        (C.c_uint32 * 3)(at.shape[2], at.shape[1], at.shape[0]))


def _gb(planes):
    arrs = [np.ascontiguousarray(planes[k], dtype=np.float32) for k in ("depth", "normal", "color", "params", "motion")]
    return _GBuffer(*[_p(a).value for a in arrs]), arrs


class Oracle:
    """One session of the CPU restatement: reservoirs, VPL archive, SVGF
    history, previous depth/normal.  precision: 0 = FP32, 1 = FP64."""

    def __init__(self, width, height, vpl_count, max_history=4, precision=0, radiance_f16=False, threads=0):
        self.lib = _load()
        self.w, self.h = width, height
        self.h_ = self.lib.oracle_create(width, height, vpl_count, max_history, precision, int(radiance_f16), threads)
        self.threads = self.lib.oracle_threads(self.h_)

    def close(self):
        if self.h_:
            self.lib.oracle_destroy(self.h_)
            self.h_ = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_field_filter(self, linear: int):
        """0: point-sampled sample_field (common.wgsl:31-38); 1: the
        reference's hardware-filtered variant (src/renderer.rs:277-286) with
        8-bit weights rounded to nearest; 2: the same with weights
        truncated."""
        self.lib.oracle_set_field_filter(self.h_, int(linear))

    def set_rows(self, row0=0, row1=0xFFFFFFFF):
        """Evaluate only rows [row0, row1) (a timing band of a large frame)."""
        self.lib.oracle_set_rows(self.h_, row0, row1)

    def lighting(self, frame, scene: OracleScene, gbuffer_f32, cur_vpls, prev_vpls, first=0, last=7):
        g, keep = _gb(gbuffer_f32)
        r = self.lib.oracle_lighting(self.h_, C.cast(C.pointer(frame), C.c_void_p), C.byref(scene.s), C.byref(g),
                                     _p(cur_vpls), _p(prev_vpls), first, last)
        if r:
            raise RuntimeError(f"oracle_lighting failed ({r})")
        del keep

    def svgf(self, frame, gbuffer_f32, iterations=4):
        g, keep = _gb(gbuffer_f32)
        self.lib.oracle_svgf(self.h_, C.cast(C.pointer(frame), C.c_void_p), C.byref(g), iterations)
        del keep

    def end_frame(self, gbuffer_f32):
        g, keep = _gb(gbuffer_f32)
        self.lib.oracle_end_frame(self.h_, C.byref(g))
        del keep

    def frame(self, frame, scene, gbuffer_f32, cur_vpls, prev_vpls, iterations=4):
        self.lighting(frame, scene, gbuffer_f32, cur_vpls, prev_vpls)
        self.svgf(frame, gbuffer_f32, iterations)
        self.end_frame(gbuffer_f32)

    def buffer(self, which, dtype=np.float32):
        n = C.c_uint64()
        p = self.lib.oracle_buffer(self.h_, which, C.byref(n))
        raw = (C.c_uint8 * n.value).from_address(p)
        return np.frombuffer(raw, dtype=dtype)

    def reservoirs(self, domain: str, k: int, dtype):
        return self.buffer(RES[(domain, k)], dtype)

    def image(self, which):
        return self.buffer(which, np.float32).reshape(self.h, self.w, 4)

    def counters(self):
        out = (C.c_uint64 * 6)()
        self.lib.oracle_counters(self.h_, out)
        return dict(zip(("march_steps", "nodes", "box_queries", "field_queries", "rays", "evals"), list(out)))
