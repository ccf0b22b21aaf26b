"""Validation at the boundary (the reference validates on the host before it
encodes, src/renderer.rs:713-807, src/settings.rs:42-105): admission by HBM
bytes, malformed scene data and out-of-range frames are refused with a status
and a message, and nothing is launched for them."""
import ctypes as C

import numpy as np
import pytest
import torch

from instantradiositytest_b200 import _lib as L
from instantradiositytest_b200.runtime import Context, FrameDriver, Scene, Session, session_desc
from instantradiositytest_b200.workload import Workload


def test_context_without_device_is_refused():
    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    cfg, h = L.Config(0, 0), C.c_void_p()
    assert L.lib.irt_context_create(C.byref(cfg), C.byref(h)) == L.IRT_E_NODEVICE


@pytest.mark.gpu
def test_admission_by_hbm_budget(cuda):
    wl = Workload(0)
    st = L.Settings.from_buffer_copy(wl.settings)
    st.render_width, st.render_height = 1920, 1200
    big = session_desc(st)
    need = L.lib.irt_session_bytes(C.byref(big))
    ctx = Context(0, budget=need // 2)
    h = C.c_void_p()
    assert L.lib.irt_session_create(ctx.handle, C.byref(big), C.byref(h)) == L.IRT_E_ADMISSION
    assert "budget" in ctx.error()
    assert ctx.bytes_in_use() == 0
    small = Session(ctx, session_desc(wl.settings))  # 256x160 fits
    assert 0 < ctx.bytes_in_use() <= need // 2
    small.close()
    assert ctx.bytes_in_use() == 0
    ctx.close()


@pytest.mark.gpu
def test_malformed_scene_data_is_refused(cuda):
    wl = Workload(0)
    ctx = Context()
    scene = Scene(ctx, wl.meshes, wl.atlas, wl.sdf_format)
    f, obj, nodes, lights = wl.frame(0)
    bad = nodes.copy()
    bad["info"][0, 3] = 0  # an escape link that does not advance
    with pytest.raises(L.IrtError, match="malformed BVH"):
        scene.update(obj, bad, lights)
    bad = obj.copy()
    bad["info"][0, 0] = len(wl.meshes)  # a mesh outside the scene
    with pytest.raises(L.IrtError, match="mesh outside"):
        scene.update(bad, nodes, lights)
    with pytest.raises(L.IrtError, match="2N-1"):
        scene.update(obj, nodes[:-1], lights)
    scene.update(obj, nodes, lights)  # the valid data is accepted
    scene.close()
    ctx.close()


@pytest.mark.gpu
def test_out_of_range_frames_are_refused(cuda):
    wl = Workload(0)
    d = FrameDriver(wl)
    d.step(0)
    f, obj, nodes, lights, planes, vpls = d.inputs(1)
    _, _, _, _, _, _, gt = d.last
    from instantradiositytest_b200.runtime import gbuffer_to_device, vpls_to_device

    gt, gs = gbuffer_to_device(planes, d.fmt)
    cur = vpls_to_device(vpls)
    vp = C.c_void_p(cur.data_ptr())
    for field, idx, value, msg in (("size", 0, 17, "frame size"), ("restir", 0, 0, "ReSTIR/SDF"),
                                   ("restir", 1, 999, "ReSTIR/SDF"), ("counts", 1, 7, "counts")):
        g = L.Frame.from_buffer_copy(f)
        getattr(g, field)[idx] = value
        with pytest.raises(L.IrtError, match=msg):
            d.session.render(d.scene, g, gs, vp, vp)
    g = L.Frame.from_buffer_copy(f)
    g.sdf[0] = 5000.0  # more march steps than validation admits
    with pytest.raises(L.IrtError, match="ReSTIR/SDF"):
        d.session.render(d.scene, g, gs, vp, vp)
    with pytest.raises(L.IrtError, match="VPL pools"):
        d.session.render(d.scene, f, gs, C.c_void_p(0), vp)
    torch.cuda.synchronize()
    assert d.session.check() == L.IRT_OK
    d.close()
