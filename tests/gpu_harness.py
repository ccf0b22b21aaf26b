"""Shared GPU-test harness: runs the CUDA path and the CPU oracle on the same
inputs, frame by frame, and measures the agreement the parity bar asks for.

Agreement metrics
  * selection: fraction of pixels whose reservoir (id, source, count, age)
    is bit-identical — the bar is >= 99.9 %;
  * radiance: mean relative error sum|a - b| / sum|b| over all pixels and
    channels (relative L1) — the bar is <= 1e-3.
"""
from __future__ import annotations

import numpy as np
import torch

from instantradiositytest_b200 import _lib as L
from instantradiositytest_b200.runtime import FrameDriver
from instantradiositytest_b200.workload import Workload, alloc_gbuffer, gbuffer_as_f32
from oracle import Oracle, OracleScene
from oracle import binding as ob

SELECT_BAR = 0.999
RADIANCE_BAR = 1e-3


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.abs(b).sum()
    return float(np.abs(a - b).sum() / den) if den > 0 else float(np.abs(a - b).sum())


def selection_match(a, b):
    keys = ("id", "source", "count", "age")
    same = np.ones(len(a), bool)
    for k in keys:
        same &= a[k] == b[k]
    return float(same.mean())


def sync_history(orc: Oracle, drv: FrameDriver, prev_index: int):
    """Copy the GPU session's history (the state the next frame reads) into
    the oracle so a frame can be compared without accumulated drift."""
    s = drv.session
    for dom, key in ((0, "d"), (1, "i")):
        orc.reservoirs(key, 2, L.RESERVOIR_DTYPE)[:] = s.reservoirs_host(dom, 2)
    arch_ptr, arch_bytes = s.buffer_ptr(L.BUF_VPL_ARCHIVE)
    orc.buffer(ob.ARCHIVE, np.uint8)[:] = s.buffer(L.BUF_VPL_ARCHIVE, torch.uint8).cpu().numpy()
    orc.buffer(ob.PREV_DEPTH)[:] = s.buffer(L.BUF_PREV_DEPTH).cpu().numpy()
    pn = s.buffer(L.BUF_PREV_NORMAL, torch.uint8).cpu().numpy()
    if drv.fmt == L.GBUFFER_F32:
        pn = pn.view(np.float32)
    elif drv.fmt == L.GBUFFER_F16:
        pn = pn.view(np.float16).astype(np.float32)
    else:
        from instantradiositytest_b200.workload import oct_decode_f32

        n3 = oct_decode_f32(pn.view(np.uint32))
        pn = np.concatenate([n3, np.zeros(n3.shape[:-1] + (1,), np.float32)], -1).reshape(-1)
    orc.buffer(ob.PREV_NORMAL)[:] = pn.reshape(-1)
    k = prev_index % 2
    orc.buffer(ob.MOMENTS[k])[:] = s.moments_host(L.BUF_MOMENTS).reshape(-1)
    orc.buffer(ob.FEEDBACK[k])[:] = s.image_host(L.BUF_FEEDBACK).reshape(-1)


def outputs(o: Oracle, index: int):
    d = o.image(ob.DIRECT)[..., :3]
    n = o.image(ob.LIGHTING)[..., :3]
    return {"direct": d, "noisy": n, "indirect": n - d, "filtered": o.image(ob.HISTORIES[index % 2])[..., :3],
            "moments": o.image(ob.MOMENTS[index % 2])[..., :3]}


def download_gbuffer(gt: dict, h: int, w: int, fmt: int) -> dict:
    """Device G-buffer planes (uint8 tensors, as FrameDriver keeps them) ->
    host planes of `fmt` with the shapes and dtypes of alloc_gbuffer."""
    out = alloc_gbuffer(h, w, fmt)
    for k, v in out.items():
        v.reshape(-1).view(np.uint8)[:] = gt[k].cpu().numpy()
    return out


class Lockstep:
    def __init__(self, wl: Workload, gbuffer_format=L.GBUFFER_F32, radiance_format=L.RADIANCE_F32, fused=1,
                 precision=0, moments_format=L.MOMENTS_F32, oracle_f16_storage=None, f64_witness=False,
                 gpu_gbuffer=False, field_filter=L.FIELD_POINT, gpu_vpls=False, filter_witness=False):
        """precision 0: the oracle in f32 (the reference's arithmetic), 1: in
        f64.  oracle_f16_storage: round the oracle's radiance history to f16
        as the reference's Rgba16Float does (default: when the radiance
        format is F16).  f64_witness: also run an f64 oracle without f16
        storage from the same synced history, and report the error of the
        CUDA outputs (`f64_<output>`) and of the primary oracle
        (`floor_<output>`, the f32 arithmetic's own distance from f64)
        against it.  gpu_gbuffer: the G-buffer comes from the CUDA producer
        (irt_gbuffer_render, as in the benchmark) and the oracle is given
        the planes the device rendered; otherwise both get the CPU one.
        field_filter: the SDF sampler of both sides (L.FIELD_LINEAR: the
        reference's hardware-filtered sample_field, emulated by the oracle).
        gpu_vpls: the VPL pools come from the CUDA generator
        (irt_vpl_generate) and the oracle is given the pools it wrote.
        filter_witness (with the filtered field sampler): also run an f32
        oracle whose filter truncates its 8-bit weights instead of rounding
        them, and report the CUDA outputs' error against it (`alt_<output>`)
        and the primary oracle's (`filterfloor_<output>`): how far apart two
        readings of the documented filter put the images."""
        self.wl = wl
        self.drv = FrameDriver(wl, gbuffer_format=gbuffer_format, radiance_format=radiance_format, fused=fused,
                               keep_candidates=True, moments_format=moments_format, gpu_gbuffer=gpu_gbuffer,
                               gpu_vpls=gpu_vpls)
        if oracle_f16_storage is None:
            oracle_f16_storage = radiance_format == L.RADIANCE_F16
        args = (wl.width, wl.height, wl.settings.vpl_count, wl.settings.restir_max_history)
        self.orc = Oracle(*args, precision, oracle_f16_storage)
        self.witness = Oracle(*args, 1, False) if f64_witness else None
        self.filter_witness = Oracle(*args, precision, oracle_f16_storage) if filter_witness else None
        self.drv.scene.set_field_filter(field_filter)
        for o in (self.orc, self.witness):
            if o is not None:
                o.set_field_filter(field_filter)
        if self.filter_witness is not None:
            self.filter_witness.set_field_filter(2)
        self.fmt = gbuffer_format
        self.prev_vpls = None
        self.atlas = atlas_f32(wl)

    def frame(self, index: int, sync=True, debug=0):
        inputs = self.drv.inputs(index, debug)
        f, obj, nodes, lights, planes, vpls = inputs
        orcs = [o for o in (self.orc, self.witness, self.filter_witness) if o is not None]
        if sync and index > 0:
            for o in orcs:
                sync_history(o, self.drv, index - 1)
        self.drv.step(index, debug, inputs=inputs)
        torch.cuda.synchronize()
        if planes is None:  # the CUDA producer's planes, as the kernels read them
            planes = download_gbuffer(self.drv.last[6], self.wl.height, self.wl.width, self.fmt)
        if vpls is None:  # the CUDA generator's pool of this frame
            vpls = self.drv.prev_vpls.cpu().numpy().view(L.VPL_DTYPE).copy()
        prev = self.prev_vpls if self.prev_vpls is not None else np.zeros_like(vpls)
        sc = OracleScene(obj, self.wl.meshes, nodes, lights, self.atlas)
        g = gbuffer_as_f32(planes, self.fmt)
        for o in orcs:
            o.frame(f, sc, g, vpls, prev, self.wl.settings.svgf_iterations)
        self.prev_vpls = vpls
        return self.compare(index)

    def compare(self, index: int):
        s, o = self.drv.session, self.orc
        out = {}
        for dom, key in ((0, "d"), (1, "i")):
            for k in (0, 1, 2):
                out[f"select_{key}{k}"] = selection_match(s.reservoirs_host(dom, k),
                                                          o.reservoirs(key, k, L.RESERVOIR_DTYPE))
        direct = s.image_host(L.BUF_DIRECT)[..., :3]
        noisy = s.image_host(L.BUF_NOISY)[..., :3]
        ours = {"direct": direct, "noisy": noisy, "indirect": noisy - direct,
                "filtered": s.image_host(L.BUF_FILTERED)[..., :3], "moments": s.moments_host(L.BUF_MOMENTS)[..., :3]}
        ref = outputs(o, index)
        for k in ours:
            out[k] = rel_l1(ours[k], ref[k])
        if self.witness is not None:
            w = outputs(self.witness, index)
            for k in ours:
                out[f"f64_{k}"] = rel_l1(ours[k], w[k])
                out[f"floor_{k}"] = rel_l1(ref[k], w[k])
        if self.filter_witness is not None:
            w = outputs(self.filter_witness, index)
            for k in ours:
                out[f"alt_{k}"] = rel_l1(ours[k], w[k])
                out[f"filterfloor_{k}"] = rel_l1(ref[k], w[k])
        return out

    def close(self):
        self.drv.close()
        self.orc.close()
        for o in (self.witness, self.filter_witness):
            if o is not None:
                o.close()


def atlas_f32(wl: Workload) -> np.ndarray:
    """The SDF texels the kernels see, dequantised (f16 x per-mesh scale)."""
    return wl.atlas_f32()
