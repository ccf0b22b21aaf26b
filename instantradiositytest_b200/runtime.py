"""Device runtime over the C-ABI: context, scene and session handles, and a
frame driver that feeds one workload through the lighting hot path.

torch provides device memory and the stream; every kernel is launched by
libirt.so on torch's current stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from ._lib import lib
from .workload import Workload

_NP_TO_TORCH = {np.float32: torch.float32, np.uint16: torch.int16, np.uint32: torch.int32}


class DeviceView:
    """Zero-copy view of a library-owned device buffer for torch."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def device_tensor(ptr: int, nbytes: int, dtype=torch.float32, shape=None):
    typestr = {torch.float32: "<f4", torch.int32: "<i4", torch.int16: "<i2", torch.uint8: "|u1"}[dtype]
    itemsize = torch.tensor([], dtype=dtype).element_size()
    if shape is None:
        shape = (nbytes // itemsize,)
    return torch.as_tensor(DeviceView(ptr, shape, typestr), device="cuda")


def stream_handle():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class Context:
    def __init__(self, device: int = 0, budget: int = 0):
        cfg = L.Config(device, budget)
        h = C.c_void_p()
        L.check(lib.irt_context_create(C.byref(cfg), C.byref(h)), what="context")
        self.handle = h

    def error(self):
        return lib.irt_last_error(self.handle).decode()

    def bytes_in_use(self):
        return lib.irt_context_bytes_in_use(self.handle)

    def close(self):
        if self.handle:
            lib.irt_context_destroy(self.handle)
            self.handle = None


class Scene:
    def __init__(self, ctx: Context, meshes: np.ndarray, atlas: np.ndarray, sdf_format: int):
        self.ctx = ctx
        dims = (C.c_uint32 * 3)(atlas.shape[2], atlas.shape[1], atlas.shape[0])
        h = C.c_void_p()
        meshes = np.ascontiguousarray(meshes)
        atlas = np.ascontiguousarray(atlas)
        L.check(lib.irt_scene_create(ctx.handle, L.ptr(meshes), len(meshes), L.ptr(atlas), dims, sdf_format,
                                     C.byref(h)), ctx.handle, "scene create")
        self.handle = h

    def update(self, objects, nodes, lights, stream=None):
        lp = L.ptr(lights) if len(lights) else None
        L.check(lib.irt_scene_update(self.handle, L.ptr(objects), len(objects), L.ptr(nodes), len(nodes), lp,
                                     len(lights), stream if stream is not None else stream_handle()),
                self.ctx.handle, "scene update")

    def set_field_filter(self, field_filter: int):
        """L.FIELD_POINT or L.FIELD_LINEAR (the reference's hardware-filtered
        sample_field), from the next update on."""
        L.check(lib.irt_scene_set_field_filter(self.handle, field_filter), self.ctx.handle, "field filter")

    def sample_field(self, mesh: int, q: np.ndarray, field_filter: int = L.FIELD_POINT) -> np.ndarray:
        """sample_field of field mesh `mesh` at grid-space points q [n, 3]
        with the kernels' sampler; returns float32 [n]."""
        qd = torch.from_numpy(np.ascontiguousarray(q, np.float32).reshape(-1)).cuda()
        n = qd.numel() // 3
        out = torch.empty(n, dtype=torch.float32, device="cuda")
        L.check(lib.irt_scene_sample_field(self.handle, field_filter, mesh, C.c_void_p(qd.data_ptr()), n,
                                           C.c_void_p(out.data_ptr()), stream_handle()), self.ctx.handle,
                "sample field")
        return out.cpu().numpy()

    def close(self):
        if self.handle:
            lib.irt_scene_destroy(self.handle)
            self.handle = None


def session_desc(settings: L.Settings, gbuffer_format=L.GBUFFER_F32, radiance_format=L.RADIANCE_F32, fused=True,
                 keep_candidates=False, exact_march=False, moments_format=L.MOMENTS_F32) -> L.SessionDesc:
    return L.SessionDesc(settings, gbuffer_format, radiance_format, moments_format, int(fused), int(keep_candidates),
                         int(exact_march))


class Session:
    def __init__(self, ctx: Context, desc: L.SessionDesc):
        self.ctx = ctx
        self.desc = desc
        self.w, self.h = desc.settings.render_width, desc.settings.render_height
        h = C.c_void_p()
        L.check(lib.irt_session_create(ctx.handle, C.byref(desc), C.byref(h)), ctx.handle, "session create")
        self.handle = h

    def close(self):
        if self.handle:
            lib.irt_session_destroy(self.handle)
            self.handle = None

    def lighting(self, scene, frame, gbuffer: L.GBuffer, cur, prev, stream=None):
        L.check(lib.irt_frame_lighting(self.handle, scene.handle, C.byref(frame), C.byref(gbuffer), cur, prev,
                                       stream if stream is not None else stream_handle()), self.ctx.handle, "lighting")

    def svgf(self, frame, gbuffer: L.GBuffer, stream=None):
        L.check(lib.irt_frame_svgf(self.handle, C.byref(frame), C.byref(gbuffer),
                                   stream if stream is not None else stream_handle()), self.ctx.handle, "svgf")

    def render(self, scene, frame, gbuffer, cur, prev, stream=None):
        L.check(lib.irt_render_frame(self.handle, scene.handle, C.byref(frame), C.byref(gbuffer), cur, prev,
                                     stream if stream is not None else stream_handle()), self.ctx.handle, "frame")

    def render_host(self, scene, frame, host_gbuffer: L.GBuffer, host_vpls, out_host=None, stream=None):
        """irt_render_frame_host: host (pinned) G-buffer planes and VPL pool in,
        the filtered image to out_host (a pinned uint8 tensor) out; pipelined
        with the previous call.  host_vpls / out_host: torch CPU tensors."""
        L.check(lib.irt_render_frame_host(self.handle, scene.handle, C.byref(frame), C.byref(host_gbuffer),
                                          C.c_void_p(host_vpls.data_ptr()),
                                          C.c_void_p(out_host.data_ptr()) if out_host is not None else None,
                                          stream if stream is not None else stream_handle()),
                self.ctx.handle, "render host")

    def host_sync(self, stream=None):
        """Without `stream`: wait for the host copies; with it: order it after them."""
        L.check(lib.irt_session_host_sync(self.handle, stream), self.ctx.handle, "host sync")

    def buffer_ptr(self, which):
        p, n = C.c_void_p(), C.c_uint64()
        L.check(lib.irt_session_buffer(self.handle, which, C.byref(p), C.byref(n)), self.ctx.handle, "buffer")
        return p.value, n.value

    def buffer(self, which, dtype=torch.float32, shape=None):
        p, n = self.buffer_ptr(which)
        return device_tensor(p, n, dtype, shape)

    def reservoirs(self, domain: int, k: int):
        p, n = C.c_void_p(), C.c_uint64()
        L.check(lib.irt_session_reservoirs(self.handle, domain, k, C.byref(p), C.byref(n)), self.ctx.handle,
                "reservoirs")
        return device_tensor(p.value, n.value, torch.uint8)

    def reservoirs_host(self, domain: int, k: int) -> np.ndarray:
        return self.reservoirs(domain, k).cpu().numpy().view(L.RESERVOIR_DTYPE)

    def image_host(self, which) -> np.ndarray:
        """A radiance/moments image as float32 [H, W, 4] on the host."""
        p, n = self.buffer_ptr(which)
        raw = device_tensor(p, n, torch.uint8).cpu().numpy()
        if n == self.w * self.h * 8:
            return raw.view(np.float16).astype(np.float32).reshape(self.h, self.w, 4)
        return raw.view(np.float32).reshape(self.h, self.w, 4)

    def moments_host(self, which=L.BUF_MOMENTS) -> np.ndarray:
        """Moments as the reference's (E[l], E[l^2], age, 0) float32 [H, W, 4],
        whatever the storage format."""
        p, n = self.buffer_ptr(which)
        raw = device_tensor(p, n, torch.uint8).cpu().numpy()
        if n == self.w * self.h * 16:
            return raw.view(np.float32).reshape(self.h, self.w, 4)
        rec = raw.view(np.dtype([("mean", "<f2"), ("dev", "<f2"), ("age", "<f4")])).reshape(self.h, self.w)
        out = np.zeros((self.h, self.w, 4), np.float32)
        mean = rec["mean"].astype(np.float32)
        dev = rec["dev"].astype(np.float32)
        out[..., 0] = mean
        out[..., 1] = dev * dev + mean * mean
        out[..., 2] = rec["age"]
        return out

    def check(self, stream=None):
        return lib.irt_session_check(self.handle, stream if stream is not None else stream_handle())

    def set_profiling(self, on=True):
        L.check(lib.irt_session_set_profiling(self.handle, int(on)), self.ctx.handle, "profiling")

    STAGES = ("archive", "reuse", "spatial", "march", "combine", "svgf_temporal", "svgf_variance", "atrous",
              "history", "total")

    def pass_ms(self, frame_index=None):
        out = (C.c_float * 10)()
        if frame_index is None:
            L.check(lib.irt_session_pass_ms(self.handle, out), self.ctx.handle, "pass ms")
        else:
            L.check(lib.irt_session_pass_ms_at(self.handle, frame_index, out), self.ctx.handle, "pass ms")
        return list(out)


def gbuffer_to_device(planes: dict, fmt: int):
    """Host G-buffer planes -> (device tensors, irt_gbuffer)."""
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).view(torch.uint8).cuda() for k, v in planes.items()}
    return t, gbuffer_struct(t, fmt)


def gbuffer_struct(t: dict, fmt: int) -> L.GBuffer:
    return L.GBuffer(fmt, t["depth"].data_ptr(), t["normal"].data_ptr(), t["color"].data_ptr(),
                     t["params"].data_ptr(), t["motion"].data_ptr())


def gbuffer_device_alloc(h: int, w: int, fmt: int):
    nb = {L.GBUFFER_F32: (16, 16, 8, 8), L.GBUFFER_F16: (8, 8, 4, 4), L.GBUFFER_PACKED: (4, 4, 4, 4)}[fmt]
    t = {"depth": torch.empty(h * w * 4, dtype=torch.uint8, device="cuda")}
    for k, b in zip(("normal", "color", "params", "motion"), nb):
        t[k] = torch.empty(h * w * b, dtype=torch.uint8, device="cuda")
    return t, gbuffer_struct(t, fmt)


def vpls_to_device(v: np.ndarray):
    return torch.from_numpy(np.ascontiguousarray(v).view(np.uint8)).cuda()


class FrameDriver:
    """Runs a workload frame by frame through one session: per frame it packs
    the scene data on the host, produces the G-buffer and VPL pool, uploads
    them and calls the C-ABI (the role of Renderer::encode)."""

    def __init__(self, wl: Workload, ctx: Context | None = None, gbuffer_format=L.GBUFFER_F32,
                 radiance_format=L.RADIANCE_F32, fused=True, keep_candidates=False, gpu_gbuffer=False,
                 exact_march=False, moments_format=L.MOMENTS_F32, gpu_vpls=False):
        self.wl = wl
        self.ctx = ctx or Context()
        self.own_ctx = ctx is None
        self.fmt = gbuffer_format
        self.scene = Scene(self.ctx, wl.meshes, wl.atlas, wl.sdf_format)
        self.session = Session(self.ctx, session_desc(wl.settings, gbuffer_format, radiance_format, fused,
                                                      keep_candidates, exact_march, moments_format))
        self.gpu_gbuffer = gpu_gbuffer
        self.gpu_vpls = gpu_vpls
        self.prev_vpls = None
        self.last = None

    def inputs(self, index: int, debug: int = 0):
        f, objects, nodes, lights = self.wl.frame(index, debug)
        planes = None if self.gpu_gbuffer else self.wl.gbuffer_cpu(f, self.fmt)
        vpls = None if self.gpu_vpls else self.wl.vpls_cpu(f, objects, lights)
        return f, objects, nodes, lights, planes, vpls

    def step(self, index: int, debug: int = 0, inputs=None):
        f, objects, nodes, lights, planes, vpls = inputs or self.inputs(index, debug)
        self.scene.update(objects, nodes, lights)
        if planes is not None:
            gt, gs = gbuffer_to_device(planes, self.fmt)
        else:
            gt, gs = gbuffer_device_alloc(self.wl.height, self.wl.width, self.fmt)
            L.check(lib.irt_gbuffer_render(self.ctx.handle, self.wl.handle, C.byref(f), None, self.fmt,
                                           gs.depth, gs.normal, gs.color, gs.params, gs.motion, stream_handle()),
                    self.ctx.handle, "gbuffer render")
        if vpls is None:
            cur = torch.zeros(f.counts[1] * 48, dtype=torch.uint8, device="cuda")
            L.check(lib.irt_vpl_generate(self.scene.handle, self.wl.handle, C.byref(f), C.c_void_p(cur.data_ptr()),
                                         stream_handle()), self.ctx.handle, "vpl generate")
        else:
            cur = vpls_to_device(vpls)
        prev = self.prev_vpls if self.prev_vpls is not None else torch.zeros_like(cur)
        self.session.render(self.scene, f, gs, C.c_void_p(cur.data_ptr()), C.c_void_p(prev.data_ptr()))
        self.prev_vpls = cur
        self.last = (f, objects, nodes, lights, planes, vpls, gt)
        return self.last

    def close(self):
        self.session.close()
        self.scene.close()
        if self.own_ctx:
            self.ctx.close()
