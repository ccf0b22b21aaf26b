"""Seeded procedural room workloads and their host-side input producers.

A workload is a scene (meshes with SDF grids, objects, materials, lights) plus
a camera path.  Per frame it yields the Frame uniform, objects, BVH nodes and
lights packed as ``Renderer::encode`` packs them (src/renderer.rs:1687-1782),
a G-buffer from analytic primary rays, and VPL pools from a CPU port of
vpl.wgsl with analytic ray casts.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import lib


def preset_spec(which: int, **overrides) -> L.WorkloadSpec:
    spec = L.WorkloadSpec()
    L.check(lib.irt_workload_preset(which, C.byref(spec)), what=f"preset {which}")
    for k, v in overrides.items():
        setattr(spec, k, v)
    return spec


class SceneLoadError(ValueError):
    """A scene file that Scene::load / Scene::validate (src/scene.rs:157-382)
    rejects; the message carries the reference's error context."""


class Workload:
    def __init__(self, spec: L.WorkloadSpec | int = 0, _handle=None, **overrides):
        if isinstance(spec, int):
            spec = preset_spec(spec, **overrides)
        else:
            for k, v in overrides.items():
                setattr(spec, k, v)
        self.spec = spec
        if _handle is None:
            h = C.c_void_p()
            L.check(lib.irt_workload_create(C.byref(spec), C.byref(h)), what="workload create")
        else:
            h = _handle
        self._init_from_handle(h)

    @classmethod
    def load(cls, manifest_path, width: int = 1920, height: int = 1080, vpl_count: int = 1024,
             vpl_bounces: int = 3, sdf_format: int = L.SDF_F32) -> "Workload":
        """Scene::load (src/scene.rs:180-255) of a version-1 scene manifest and
        its binaries: the returned workload renders the file's scene from its
        fixed camera at width x height.  Raises SceneLoadError with the
        reference's error text when the file is rejected."""
        spec = L.WorkloadSpec()
        spec.width, spec.height = width, height
        spec.vpl_count, spec.vpl_bounces = vpl_count, vpl_bounces
        spec.sdf_format = sdf_format
        h = C.c_void_p()
        msg = C.create_string_buffer(1024)
        st = lib.irt_workload_load(str(manifest_path).encode(), C.byref(spec), C.byref(h), msg, len(msg))
        if st != L.IRT_OK:
            if st == L.IRT_E_NOMEM:
                raise MemoryError(msg.value.decode(errors="replace"))
            raise SceneLoadError(msg.value.decode(errors="replace"))
        wl = cls(spec, _handle=h)
        wl.path = str(manifest_path)
        return wl

    def _init_from_handle(self, h):
        spec = self.spec
        self.handle = h
        self.width, self.height = spec.width, spec.height
        self.object_count = lib.irt_workload_object_count(h)
        self.light_count = lib.irt_workload_light_count(h)
        self.mesh_count = lib.irt_workload_mesh_count(h)
        self.settings = L.Settings()
        lib.irt_workload_settings(h, C.byref(self.settings))
        mp = lib.irt_workload_meshes(h)
        self.meshes = np.frombuffer((C.c_uint8 * (self.mesh_count * 128)).from_address(mp),
                                    dtype=L.MESH_DTYPE).copy()
        dims = (C.c_uint32 * 3)()
        ap = lib.irt_workload_atlas(h, dims)
        self.atlas_dims = (dims[0], dims[1], dims[2])
        self.sdf_format = lib.irt_workload_sdf_format(h)
        n = dims[0] * dims[1] * dims[2]
        if self.sdf_format == L.SDF_F16:
            raw = np.frombuffer((C.c_uint16 * n).from_address(ap), dtype=np.uint16)
        else:
            raw = np.frombuffer((C.c_float * n).from_address(ap), dtype=np.float32)
        self.atlas = raw.reshape(dims[2], dims[1], dims[0]).copy()

    def atlas_f32(self) -> np.ndarray:
        """The SDF texels the kernels see, as f32: F16 atlases dequantised
        with each mesh tile's scale (irt_mesh.lo[3])."""
        if self.sdf_format == L.SDF_F32:
            return self.atlas
        if getattr(self, "_atlas_f32", None) is None:
            out = self.atlas.view(np.float16).astype(np.float32)
            for m in self.meshes:
                x, y, z, r = (int(v) for v in m["field"])
                out[z:z + r, y:y + r, x:x + r] *= np.float32(m["lo"][3])
            self._atlas_f32 = out
        return self._atlas_f32

    def close(self):
        if self.handle:
            lib.irt_workload_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- per frame
    def frame(self, index: int, debug: int = 0):
        f = L.Frame()
        objects = np.zeros(self.object_count, L.OBJECT_DTYPE)
        nodes = np.zeros(2 * self.object_count - 1, L.NODE_DTYPE)
        lights = np.zeros(max(self.light_count, 1), L.LIGHT_DTYPE)
        L.check(lib.irt_workload_frame(self.handle, index, debug, C.byref(f), L.ptr(objects), L.ptr(nodes),
                                       L.ptr(lights)), what="workload frame")
        return f, objects, nodes, lights[: self.light_count]

    def gbuffer_cpu(self, f: L.Frame, fmt: int = L.GBUFFER_F32):
        planes = alloc_gbuffer(self.height, self.width, fmt)
        L.check(lib.irt_workload_gbuffer_cpu(self.handle, C.byref(f), None, fmt, L.ptr(planes["depth"]),
                                             L.ptr(planes["normal"]), L.ptr(planes["color"]),
                                             L.ptr(planes["params"]), L.ptr(planes["motion"])), what="gbuffer")
        return planes

    def vpls_cpu(self, f: L.Frame, objects, lights):
        out = np.zeros(f.counts[1], L.VPL_DTYPE)
        lp = L.ptr(lights) if len(lights) else None
        L.check(lib.irt_workload_vpls_cpu(self.handle, C.byref(f), L.ptr(objects), lp, L.ptr(out)), what="vpls")
        return out


def alloc_gbuffer(h: int, w: int, fmt: int):
    if fmt == L.GBUFFER_F32:
        return {"depth": np.zeros((h, w), np.float32), "normal": np.zeros((h, w, 4), np.float32),
                "color": np.zeros((h, w, 4), np.float32), "params": np.zeros((h, w, 2), np.float32),
                "motion": np.zeros((h, w, 2), np.float32)}
    if fmt == L.GBUFFER_F16:
        return {"depth": np.zeros((h, w), np.float32), "normal": np.zeros((h, w, 4), np.uint16),
                "color": np.zeros((h, w, 4), np.uint16), "params": np.zeros((h, w, 2), np.uint16),
                "motion": np.zeros((h, w, 2), np.uint16)}
    if fmt == L.GBUFFER_PACKED:
        return {"depth": np.zeros((h, w), np.float32), "normal": np.zeros((h, w), np.uint32),
                "color": np.zeros((h, w), np.uint32), "params": np.zeros((h, w, 2), np.uint16),
                "motion": np.zeros((h, w, 2), np.uint16)}
    raise ValueError(fmt)


def oct_decode_f32(v: np.ndarray) -> np.ndarray:
    """Octahedral snorm16x2 -> unit vector, the same f32 operations (no
    contraction) as the device decoder."""
    x = np.maximum((v & 0xFFFF).astype(np.uint16).view(np.int16).astype(np.float32) / np.float32(32767),
                   np.float32(-1))
    y = np.maximum((v >> 16).astype(np.uint16).view(np.int16).astype(np.float32) / np.float32(32767),
                   np.float32(-1))
    z = np.float32(1) - np.abs(x) - np.abs(y)
    t = np.maximum(-z, np.float32(0))
    x = np.where(x >= 0, x - t, x + t).astype(np.float32)
    y = np.where(y >= 0, y - t, y + t).astype(np.float32)
    n2 = (x * x + y * y).astype(np.float32) + z * z
    inv = np.float32(1) / np.sqrt(n2.astype(np.float32))
    return np.stack([x * inv, y * inv, z * inv], -1).astype(np.float32)


def gbuffer_as_f32(planes: dict, fmt: int) -> dict:
    """The G-buffer values the kernels see, as F32 planes (for the oracle)."""
    if fmt == L.GBUFFER_F32:
        return planes
    h, w = planes["depth"].shape
    out = alloc_gbuffer(h, w, L.GBUFFER_F32)
    out["depth"][:] = planes["depth"]
    out["params"][:] = planes["params"].view(np.float16).astype(np.float32)
    out["motion"][:] = planes["motion"].view(np.float16).astype(np.float32)
    if fmt == L.GBUFFER_F16:
        out["normal"][:] = planes["normal"].view(np.float16).astype(np.float32)
        out["color"][:] = planes["color"].view(np.float16).astype(np.float32)
    else:
        out["normal"][..., :3] = oct_decode_f32(planes["normal"])
        c = planes["color"]
        for k in range(3):
            out["color"][..., k] = ((c >> (8 * k)) & 255).astype(np.float32) / np.float32(255)
    return out
