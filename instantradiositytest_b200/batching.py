"""Batched views over the C-ABI (irt_batch_*): many views of uneven size
rendered with one launch per pass, optionally replayed from a CUDA graph per
frame, with tile shapes from the batch's autotuner."""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L
from ._lib import lib
from .runtime import Context, Scene, Session, gbuffer_device_alloc, stream_handle


class Batch:
    PASSES = ("guides", "archive", "reuse", "spatial", "march", "combine", "temporal", "variance", "atrous",
              "history", "total", "graph")

    def __init__(self, ctx: Context, settings: L.Settings, sizes, gbuffer_format=L.GBUFFER_F32,
                 radiance_format=L.RADIANCE_F32, moments_format=L.MOMENTS_F32, use_graphs=True, vpl_counts=None):
        self.ctx = ctx
        self.n = len(sizes)
        self._w = (C.c_uint32 * self.n)(*[w for w, _ in sizes])
        self._h = (C.c_uint32 * self.n)(*[h for _, h in sizes])
        self._v = (C.c_uint32 * self.n)(*vpl_counts) if vpl_counts is not None else None
        self.desc = L.BatchDesc(settings, gbuffer_format, radiance_format, moments_format, int(use_graphs), self.n,
                                C.cast(self._w, C.POINTER(C.c_uint32)), C.cast(self._h, C.POINTER(C.c_uint32)),
                                C.cast(self._v, C.POINTER(C.c_uint32)) if self._v is not None else None)
        h = C.c_void_p()
        L.check(lib.irt_batch_create(ctx.handle, C.byref(self.desc), C.byref(h)), ctx.handle, "batch create")
        self.handle = h
        self.sizes = list(sizes)

    def view(self, v: int) -> Session:
        """View v's session (buffers, reservoirs); owned by the batch."""
        s = Session.__new__(Session)
        s.ctx = self.ctx
        s.desc = None
        s.w, s.h = self.sizes[v]
        s.handle = C.c_void_p(lib.irt_batch_view(self.handle, v))
        return s

    def render(self, scenes, frames, gbuffers, cur, prev, stream=None):
        n = self.n
        sc = (C.c_void_p * n)(*[s.handle.value for s in scenes])
        fr = (L.Frame * n)(*frames)
        gb = (L.GBuffer * n)(*gbuffers)
        cu = (C.c_void_p * n)(*cur)
        pr = (C.c_void_p * n)(*prev)
        L.check(lib.irt_batch_render(self.handle, sc, fr, gb, cu, pr, stream if stream is not None else stream_handle()),
                self.ctx.handle, "batch render")

    def autotune(self, frames: int):
        L.check(lib.irt_batch_autotune(self.handle, frames), self.ctx.handle, "batch autotune")

    def set_waves(self, budget_px: int):
        L.check(lib.irt_batch_set_waves(self.handle, budget_px), self.ctx.handle, "batch waves")

    def tuning(self) -> str:
        buf = C.create_string_buffer(256)
        L.check(lib.irt_batch_tuning(self.handle, buf, 256), self.ctx.handle, "batch tuning")
        return buf.value.decode()

    def pass_ms(self) -> dict:
        out = (C.c_float * 12)()
        L.check(lib.irt_batch_pass_ms(self.handle, out), self.ctx.handle, "batch pass ms")
        return dict(zip(self.PASSES, list(out)))

    def close(self):
        if self.handle:
            lib.irt_batch_destroy(self.handle)
            self.handle = None


class BatchDriver:
    """Views over workloads (several views may share one workload's scene):
    per frame it updates each distinct scene, renders every view's G-buffer
    and VPL pool on the device into fixed buffers, then calls
    irt_batch_render once."""

    def __init__(self, ctx: Context, views, gbuffer_format=L.GBUFFER_F32, radiance_format=L.RADIANCE_F32,
                 moments_format=L.MOMENTS_F32, use_graphs=True):
        """views: list of (Workload, camera phase offset[, (width, height)]) —
        each view follows its workload's camera path shifted by the offset
        frames, at the workload's frame size or the one given (views of a
        scene share its projection, so any size of the same aspect works)."""
        self.ctx = ctx
        self.sizes = [v[2] if len(v) > 2 else (v[0].width, v[0].height) for v in views]
        views = [(v[0], v[1]) for v in views]
        self.views = views
        self.fmt = gbuffer_format
        wls = []
        for wl, _ in views:
            if all(w is not wl for w in wls):
                wls.append(wl)
        self.wls = wls
        self.scenes = {id(wl): Scene(ctx, wl.meshes, wl.atlas, wl.sdf_format) for wl in wls}
        self.batch = Batch(ctx, wls[0].settings, self.sizes, gbuffer_format, radiance_format, moments_format,
                           use_graphs, [wl.settings.vpl_count for wl, _ in views])
        self.gb = [gbuffer_device_alloc(h, w, gbuffer_format) for w, h in self.sizes]
        self.vpls = [[torch.zeros(wl.settings.vpl_count * 48, dtype=torch.uint8, device="cuda") for _ in range(2)]
                     for wl, _ in views]
        self.zero = [torch.zeros(wl.settings.vpl_count * 48, dtype=torch.uint8, device="cuda") for wl, _ in views]

    def inputs(self, index: int):
        """Per view: frame and scene data of its workload at its path position."""
        return [wl.frame(index + off) for wl, off in self.views]

    def step(self, index: int, data=None):
        data = data or self.inputs(index)
        frames = []
        updated = set()
        sh = stream_handle()
        for v, ((wl, off), (f, obj, nodes, lights)) in enumerate(zip(self.views, data)):
            # every view's frame carries the batch's frame index and history flags
            f.size[0], f.size[1] = self.sizes[v]
            f.size[2] = index
            f.flags[0] = 1 if index > 0 else 0
            f.flags[1] = f.size[3] if index > 0 else 0
            if id(wl) not in updated:
                self.scenes[id(wl)].update(obj, nodes, lights)
                updated.add(id(wl))
            _, gs = self.gb[v]
            L.check(lib.irt_gbuffer_render(self.ctx.handle, wl.handle, C.byref(f), None, self.fmt, gs.depth, gs.normal,
                                           gs.color, gs.params, gs.motion, sh), self.ctx.handle, "gbuffer")
            cur = self.vpls[v][index % 2]
            L.check(lib.irt_vpl_generate(self.scenes[id(wl)].handle, wl.handle, C.byref(f),
                                         C.c_void_p(cur.data_ptr()), sh), self.ctx.handle, "vpls")
            frames.append(f)
        cur = [self.vpls[v][index % 2].data_ptr() for v in range(len(self.views))]
        prev = [(self.vpls[v][(index + 1) % 2] if index > 0 else self.zero[v]).data_ptr()
                for v in range(len(self.views))]
        self.batch.render([self.scenes[id(wl)] for wl, _ in self.views], frames, [g[1] for g in self.gb], cur, prev)
        return frames

    def close(self):
        self.batch.close()
        for s in self.scenes.values():
            s.close()
