"""Render server over the C-ABI (irt_server_*): continuous batching of render
sessions with HBM-byte admission, resident per-session history, sessions
spread over CUDA streams, and latency / throughput statistics."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import lib
from .runtime import Context


class Server:
    def __init__(self, ctx: Context, budget_bytes: int, streams: int = 8, max_sessions: int = 0,
                 frame_rate: float = 60.0, gbuffer_format=L.GBUFFER_F32, radiance_format=L.RADIANCE_F32,
                 moments_format=L.MOMENTS_F32, fused: int = 1):
        self.ctx = ctx
        self.desc = L.ServerDesc(int(budget_bytes), max_sessions, streams, frame_rate, gbuffer_format,
                                 radiance_format, moments_format, fused)
        h = C.c_void_p()
        L.check(lib.irt_server_create(ctx.handle, C.byref(self.desc), C.byref(h)), ctx.handle, "server create")
        self.handle = h
        self._keep = []

    def submit(self, request_id: int, arrival_s: float, frames: int, workload, capture_frame: int | None = None,
               times: np.ndarray | None = None):
        """Queues a render session over `workload`; with capture_frame, returns
        the host array that receives that frame's filtered image.  times: a
        float64 array of 3 that the run fills with the session's admission,
        last-frame-done and retirement times (seconds after the run starts)."""
        out = None
        cap = None
        if capture_frame is not None:
            texel = 8 if self.desc.radiance_format == L.RADIANCE_F16 else 16
            out = np.zeros(workload.width * workload.height * texel, np.uint8)
            cap = C.c_void_p(out.ctypes.data)
        tp = None
        if times is not None:
            assert times.dtype == np.float64 and times.size >= 3 and times.flags["C_CONTIGUOUS"]
            tp = times.ctypes.data_as(C.POINTER(C.c_double))
        r = L.Request(request_id, arrival_s, frames, workload.handle, capture_frame or 0, cap, tp)
        L.check(lib.irt_server_submit(self.handle, C.byref(r)), self.ctx.handle, "server submit")
        self._keep.append((workload, out, times))
        return out

    def request_bytes(self, workload, frames: int = 1) -> int:
        r = L.Request(0, 0.0, frames, workload.handle, 0, None, None)
        return int(lib.irt_server_request_bytes(self.handle, C.byref(r)))

    def run(self) -> dict:
        st = L.ServerStats()
        L.check(lib.irt_server_run(self.handle, C.byref(st)), self.ctx.handle, "server run")
        self._keep.clear()
        return st.as_dict()

    def close(self):
        if self.handle:
            lib.irt_server_destroy(self.handle)
            self.handle = None
