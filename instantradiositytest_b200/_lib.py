"""ctypes binding of libirt.so (include/irt.h).

The shared library is built in-tree (``make -C instantradiositytest_b200``) and
loaded from this directory.  There is no fallback: importing this module
without the library raises ``ImportError``.  With IRT_LIBRARY=checked in the
environment the checked build (libirt_checked.so, the same C-ABI with every
data-dependent index tested in the kernels) is loaded instead; with
IRT_LIBRARY=host the host-only library (libirt_host.so: workload generator,
CPU producers, scene loader, host logic — no CUDA code), which binds only
the functions it has.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
CHECKED_LIB_PATH = os.path.join(_HERE, "libirt_checked.so")
HOST_LIB_PATH = os.path.join(_HERE, "libirt_host.so")
LIB_PATH = {"checked": CHECKED_LIB_PATH, "host": HOST_LIB_PATH}.get(os.environ.get("IRT_LIBRARY", ""),
                                                                   os.path.join(_HERE, "libirt.so"))
HOST_ONLY = LIB_PATH == HOST_LIB_PATH

IRT_OK = 0
IRT_E_INVALID = -1
IRT_E_CUDA = -2
IRT_E_ADMISSION = -3
IRT_E_NOMEM = -4
IRT_E_STATE = -5
IRT_E_DEVICE = -6
IRT_E_NODEVICE = -7

GBUFFER_F32, GBUFFER_F16, GBUFFER_PACKED = 0, 1, 2
RADIANCE_F32, RADIANCE_F16 = 0, 1
MOMENTS_F32, MOMENTS_F16 = 0, 1
SDF_F32, SDF_F16 = 0, 1
FIELD_POINT, FIELD_LINEAR = 0, 1

BUF_DIRECT, BUF_NOISY, BUF_FILTERED, BUF_MOMENTS = 0, 1, 2, 3
BUF_RES_DIRECT, BUF_RES_INDIRECT, BUF_VPL_ARCHIVE = 4, 5, 6
BUF_PREV_DEPTH, BUF_PREV_NORMAL, BUF_MOMENTS_OLD = 7, 8, 9
BUF_FEEDBACK, BUF_FEEDBACK_OLD, BUF_ERROR = 10, 11, 12
BUF_TEMPORAL, BUF_VARIANCE = 13, 14


class Mat4(C.Structure):
    _fields_ = [("m", C.c_float * 16)]


class Frame(C.Structure):
    _fields_ = [
        ("vp", Mat4), ("inv_vp", Mat4), ("previous_vp", Mat4), ("previous_inv_vp", Mat4),
        ("camera", C.c_float * 4), ("size", C.c_uint32 * 4), ("counts", C.c_uint32 * 4),
        ("restir", C.c_uint32 * 4), ("temporal", C.c_float * 4), ("sdf", C.c_float * 4),
        ("rr", C.c_float * 4), ("flags", C.c_uint32 * 4),
    ]


class Settings(C.Structure):
    _fields_ = [
        ("render_width", C.c_uint32), ("render_height", C.c_uint32),
        ("vpl_count", C.c_uint32), ("vpl_max_bounces", C.c_uint32),
        ("vpl_rr_min_survival", C.c_float), ("vpl_rr_max_survival", C.c_float),
        ("restir_direct_candidates", C.c_uint32), ("restir_vpl_candidates", C.c_uint32),
        ("restir_spatial_neighbors", C.c_uint32), ("restir_spatial_radius", C.c_uint32),
        ("restir_max_history", C.c_uint32), ("svgf_iterations", C.c_uint32),
        ("depth_threshold", C.c_float), ("normal_threshold", C.c_float),
        ("temporal_history_weight", C.c_float), ("temporal_max_history", C.c_uint32),
        ("sdf_max_steps", C.c_uint32), ("sdf_hit_epsilon", C.c_float),
        ("sdf_soft_shadow_k", C.c_float), ("target_frame_ms", C.c_float),
    ]


class Config(C.Structure):
    _fields_ = [("device", C.c_int32), ("hbm_budget_bytes", C.c_uint64)]


class SessionDesc(C.Structure):
    _fields_ = [
        ("settings", Settings), ("gbuffer_format", C.c_int32), ("radiance_format", C.c_int32),
        ("moments_format", C.c_int32), ("fused", C.c_int32), ("keep_candidates", C.c_int32),
        ("exact_march", C.c_int32),
    ]


class GBuffer(C.Structure):
    _fields_ = [
        ("format", C.c_int32), ("depth", C.c_void_p), ("normal", C.c_void_p), ("color", C.c_void_p),
        ("params", C.c_void_p), ("motion", C.c_void_p),
    ]


class WorkloadSpec(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64), ("width", C.c_uint32), ("height", C.c_uint32),
        ("n_boxes", C.c_uint32), ("n_spheres", C.c_uint32), ("room_single_mesh", C.c_int32),
        ("sdf_resolution", C.c_uint32), ("sdf_format", C.c_int32), ("n_lights", C.c_uint32),
        ("radiance_lo", C.c_float), ("radiance_hi", C.c_float),
        ("emitter_size_lo", C.c_float), ("emitter_size_hi", C.c_float),
        ("vpl_count", C.c_uint32), ("vpl_bounces", C.c_uint32),
        ("orbit_deg_per_frame", C.c_float), ("dolly_m_per_frame", C.c_float),
    ]


class BatchDesc(C.Structure):
    _fields_ = [
        ("settings", Settings), ("gbuffer_format", C.c_int32), ("radiance_format", C.c_int32),
        ("moments_format", C.c_int32), ("use_graphs", C.c_int32), ("n_views", C.c_uint32),
        ("widths", C.POINTER(C.c_uint32)), ("heights", C.POINTER(C.c_uint32)),
        ("vpl_counts", C.POINTER(C.c_uint32)),
    ]


class ServerDesc(C.Structure):
    _fields_ = [
        ("hbm_budget_bytes", C.c_uint64), ("max_sessions", C.c_uint32), ("streams", C.c_uint32),
        ("frame_rate", C.c_float), ("gbuffer_format", C.c_int32), ("radiance_format", C.c_int32),
        ("moments_format", C.c_int32), ("fused", C.c_int32),
    ]


class Request(C.Structure):
    _fields_ = [
        ("id", C.c_uint64), ("arrival_s", C.c_double), ("frames", C.c_uint32), ("workload", C.c_void_p),
        ("capture_frame", C.c_uint32), ("capture", C.c_void_p), ("times", C.POINTER(C.c_double)),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("frames", C.c_uint64), ("sessions", C.c_uint64), ("rejected", C.c_uint64),
        ("pixel_frames", C.c_double), ("seconds", C.c_double), ("mpix_frames_per_s", C.c_double),
        ("p50_latency_ms", C.c_float), ("p99_latency_ms", C.c_float),
        ("p50_frame_ms", C.c_float), ("p99_frame_ms", C.c_float),
        ("p50_wait_ms", C.c_float), ("p99_wait_ms", C.c_float),
        ("mean_active", C.c_float), ("peak_active", C.c_float), ("peak_bytes", C.c_uint64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# numpy record layouts of the array-of-struct types (byte-identical to irt.h)
OBJECT_DTYPE = np.dtype([("model", "<f4", 16), ("previous", "<f4", 16), ("inverse", "<f4", 16),
                         ("info", "<u4", 4)])
MESH_DTYPE = np.dtype([("lo", "<f4", 4), ("hi", "<f4", 4), ("geometry", "<u4", 4), ("field", "<u4", 4),
                       ("grid", "<f4", 4), ("geometry_lo", "<f4", 4), ("geometry_hi", "<f4", 4),
                       ("enclosing_sphere", "<f4", 4)])
NODE_DTYPE = np.dtype([("lo", "<f4", 4), ("hi", "<f4", 4), ("info", "<u4", 4)])
LIGHT_DTYPE = np.dtype([("position_strength", "<f4", 4), ("direction_angle", "<f4", 4),
                        ("color_type", "<f4", 4)])
VPL_DTYPE = np.dtype([("position", "<f4", 4), ("normal", "<f4", 4), ("flux", "<f4", 4)])
RESERVOIR_DTYPE = np.dtype([("id", "<u4"), ("source", "<u4"), ("count", "<u4"), ("age", "<u4"),
                            ("sum", "<f4"), ("selected_target", "<f4"), ("pdf", "<f4"),
                            ("generation", "<u4")])
VERTEX_DTYPE = np.dtype([("position", "<f4", 4), ("normal", "<f4", 4), ("tangent", "<f4", 4),
                         ("uv", "<f4", 4)])
MATERIAL_DTYPE = np.dtype([("color", "<f4", 4), ("params", "<f4", 4), ("textures", "<i4", 4),
                           ("channels", "<u4", 4)])

P = C.c_void_p
U32 = C.c_uint32
I32 = C.c_int32
U64 = C.c_uint64

# name: (restype, argtypes)
_PROTOS = {
    "irt_settings_default": (None, [C.POINTER(Settings)]),
    "irt_settings_validate": (I32, [C.POINTER(Settings), C.c_char_p, C.c_size_t]),
    "irt_context_create": (I32, [C.POINTER(Config), C.POINTER(P)]),
    "irt_context_destroy": (None, [P]),
    "irt_last_error": (C.c_char_p, [P]),
    "irt_context_bytes_in_use": (U64, [P]),
    "irt_scene_create": (I32, [P, P, U32, P, C.POINTER(U32), I32, C.POINTER(P)]),
    "irt_scene_update": (I32, [P, P, U32, P, U32, P, U32, P]),
    "irt_scene_destroy": (None, [P]),
    "irt_session_create": (I32, [P, C.POINTER(SessionDesc), C.POINTER(P)]),
    "irt_session_bytes": (U64, [C.POINTER(SessionDesc)]),
    "irt_session_destroy": (None, [P]),
    "irt_frame_lighting": (I32, [P, P, C.POINTER(Frame), C.POINTER(GBuffer), P, P, P]),
    "irt_frame_svgf": (I32, [P, C.POINTER(Frame), C.POINTER(GBuffer), P]),
    "irt_render_frame": (I32, [P, P, C.POINTER(Frame), C.POINTER(GBuffer), P, P, P]),
    "irt_render_frame_host": (I32, [P, P, C.POINTER(Frame), C.POINTER(GBuffer), P, P, P]),
    "irt_session_host_sync": (I32, [P, P]),
    "irt_session_buffer": (I32, [P, I32, C.POINTER(P), C.POINTER(U64)]),
    "irt_session_reservoirs": (I32, [P, I32, I32, C.POINTER(P), C.POINTER(U64)]),
    "irt_session_check": (I32, [P, P]),
    "irt_session_set_profiling": (I32, [P, I32]),
    "irt_session_pass_ms": (I32, [P, C.POINTER(C.c_float)]),
    "irt_session_pass_ms_at": (I32, [P, U32, C.POINTER(C.c_float)]),
    "irt_build_flavour": (C.c_char_p, []),
    "irt_scene_set_field_filter": (I32, [P, I32]),
    "irt_scene_sample_field": (I32, [P, I32, U32, P, U32, P, P]),
    "irt_svgf_spatial_noalloc": (I32, [C.POINTER(Frame), C.POINTER(GBuffer), I32, I32, U32, P, P, P, P, P,
                                       C.c_char_p, C.c_size_t]),
    "irt_is_box_geometry": (I32, [P, U32, P, U32, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "irt_field_lipschitz_bound": (C.c_float, [P, U32, C.POINTER(C.c_float)]),
    "irt_mesh_metadata": (I32, [P, U32, P, U32, P, U32, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                C.POINTER(U32), P]),
    "irt_atlas_layout": (None, [U32, U32, C.POINTER(U32), C.POINTER(U32)]),
    "irt_build_hierarchy": (I32, [P, P, U32, P]),
    "irt_pack_object": (None, [C.POINTER(Mat4), C.POINTER(Mat4), U32, U32, C.POINTER(C.c_float),
                               C.POINTER(C.c_float), U32, P]),
    "irt_workload_preset": (I32, [I32, C.POINTER(WorkloadSpec)]),
    "irt_workload_create": (I32, [C.POINTER(WorkloadSpec), C.POINTER(P)]),
    "irt_workload_load": (I32, [C.c_char_p, C.POINTER(WorkloadSpec), C.POINTER(P), C.c_char_p, U64]),
    "irt_workload_destroy": (None, [P]),
    "irt_workload_mesh_count": (U32, [P]),
    "irt_workload_object_count": (U32, [P]),
    "irt_workload_light_count": (U32, [P]),
    "irt_workload_meshes": (P, [P]),
    "irt_workload_atlas": (P, [P, C.POINTER(U32)]),
    "irt_workload_sdf_format": (I32, [P]),
    "irt_workload_settings": (None, [P, C.POINTER(Settings)]),
    "irt_workload_frame": (I32, [P, U32, U32, C.POINTER(Frame), P, P, P]),
    "irt_workload_gbuffer_cpu": (I32, [P, C.POINTER(Frame), P, I32, P, P, P, P, P]),
    "irt_workload_vpls_cpu": (I32, [P, C.POINTER(Frame), P, P, P]),
    "irt_gbuffer_render": (I32, [P, P, C.POINTER(Frame), P, I32, P, P, P, P, P, P]),
    "irt_vpl_generate": (I32, [P, P, C.POINTER(Frame), P, P]),
    "irt_present": (I32, [P, I32, U32, U32, P, P]),
    "irt_batch_create": (I32, [P, C.POINTER(BatchDesc), C.POINTER(P)]),
    "irt_batch_render": (I32, [P, P, C.POINTER(Frame), C.POINTER(GBuffer), P, P, P]),
    "irt_batch_view": (P, [P, U32]),
    "irt_batch_autotune": (I32, [P, U32]),
    "irt_batch_tuning": (I32, [P, C.c_char_p, C.c_size_t]),
    "irt_batch_set_waves": (I32, [P, U64]),
    "irt_batch_pass_ms": (I32, [P, C.POINTER(C.c_float)]),
    "irt_batch_destroy": (None, [P]),
    "irt_server_create": (I32, [P, C.POINTER(ServerDesc), C.POINTER(P)]),
    "irt_server_submit": (I32, [P, C.POINTER(Request)]),
    "irt_server_run": (I32, [P, C.POINTER(ServerStats)]),
    "irt_server_request_bytes": (U64, [P, C.POINTER(Request)]),
    "irt_server_destroy": (None, [P]),
}


def exported_symbols():
    """Names of every function include/irt.h declares."""
    return sorted(_PROTOS)


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C {_HERE}` (nvcc for sm_100a); "
            "there is no CPU fallback")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _PROTOS.items():
        if HOST_ONLY and not hasattr(lib, name):
            continue  # a device entry point the host-only library does not have
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class IrtError(RuntimeError):
    def __init__(self, status, message=""):
        super().__init__(f"irt status {status}: {message}")
        self.status = status


def check(status, ctx=None, what=""):
    if status != IRT_OK:
        msg = lib.irt_last_error(ctx).decode() if ctx else ""
        raise IrtError(status, f"{what} {msg}".strip())
    return status


def ptr(a):
    """Address of a numpy array's data (C-contiguous) as c_void_p."""
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)
