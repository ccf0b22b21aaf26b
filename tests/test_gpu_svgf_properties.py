"""Property tests of the CUDA SVGF and lighting passes, the checks the
reference runs on its own GPU path (src/gpu_tests.rs:79-181 SVGF noise,
edges, disocclusion and HDR range; :183-252 history, lights off and debug
invalidation), on the procedural room and, where IRT_TEST_SCENE names the
shipped assets/test_scene/scene.json, on the scene those tests load, at
their 160x100 and settings.json's 100 VPL paths.

As Renderer::test_svgf_signal (src/renderer.rs:557-640) does, a known signal
replaces the noisy lighting image of a frame before the SVGF passes run.
"""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from instantradiositytest_b200 import _lib as L
from instantradiositytest_b200.runtime import FrameDriver, gbuffer_to_device, vpls_to_device
from instantradiositytest_b200.workload import Workload

pytestmark = pytest.mark.gpu

W, H = 160, 100
SHIPPED = os.environ.get("IRT_TEST_SCENE", "")
SCENES = ["room"] + (["test_scene"] if SHIPPED and os.path.exists(SHIPPED) else [])


@pytest.fixture(params=SCENES)
def scene(request):
    return request.param


def make_workload(scene):
    if scene == "room":
        return Workload(0, width=W, height=H)
    return Workload.load(SHIPPED, width=W, height=H, vpl_count=100)


def xorshift_signal(state, n):
    """The reference's binary noise: xorshift32, 0 or 2 per pixel."""
    out = np.empty(n, np.float32)
    s = state
    for i in range(n):
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
        out[i] = 0.0 if s & 1 == 0 else 2.0
    return s, out


class Rig:
    """One session over the 160x100 room; each frame runs the lighting
    passes, optionally overwrites the noisy image, then the SVGF passes."""

    def __init__(self, moments_format=L.MOMENTS_F32, radiance_format=L.RADIANCE_F32, scene="room"):
        self.wl = make_workload(scene)
        self.drv = FrameDriver(self.wl, radiance_format=radiance_format, moments_format=moments_format)
        self.generation = 1
        self.prev_generation = 0
        self.index = 0

    def frame(self, signal=None, edit_planes=None, edit=None, history=True):
        d = self.drv
        f, obj, nodes, lights, planes, vpls = d.inputs(self.index)
        # scene.changed() bumps the generation (src/scene.rs); the frame
        # carries the current one in size.w and the previous in flags.y.
        f.size[3] = self.generation
        f.flags[1] = self.prev_generation
        if not history:
            f.flags[0] = 0
        if edit is not None:
            edit(f, lights)
            vpls = self.wl.vpls_cpu(f, obj, lights)
        d.scene.update(obj, nodes, lights)
        if edit_planes is not None:
            edit_planes(planes)
        gt, gs = gbuffer_to_device(planes, d.fmt)
        cur = vpls_to_device(vpls)
        prev = d.prev_vpls if d.prev_vpls is not None else torch.zeros_like(cur)
        s = d.session
        s.lighting(d.scene, f, gs, C.c_void_p(cur.data_ptr()), C.c_void_p(prev.data_ptr()))
        if signal is not None:
            noisy = s.buffer(L.BUF_NOISY, torch.uint8)
            rgba = np.repeat(signal.astype(np.float32)[:, None], 4, 1)
            rgba[:, 3] = 1.0
            if noisy.numel() == W * H * 8:
                src = torch.from_numpy(rgba.astype(np.float16).view(np.uint8).reshape(-1))
            else:
                src = torch.from_numpy(rgba.view(np.uint8).reshape(-1))
            noisy.copy_(src.cuda())
        s.svgf(f, gs)
        torch.cuda.synchronize()
        assert s.check() == L.IRT_OK
        d.prev_vpls = cur
        self.prev_generation = self.generation
        self.index += 1
        return planes

    def changed(self):
        self.generation += 1

    def close(self):
        self.drv.close()


@pytest.mark.parametrize("moments_format", [L.MOMENTS_F32, L.MOMENTS_F16])
def test_binary_noise_removed_mean_preserved(cuda, moments_format, scene):
    rig = Rig(moments_format, scene=scene)
    state = 123456789
    for _ in range(12):
        state, sig = xorshift_signal(state, W * H)
        planes = rig.frame(signal=sig)
    s = rig.drv.session
    filt = s.image_host(L.BUF_FILTERED)
    mom = s.moments_host()
    valid = planes["depth"] < 1.0
    v = filt[..., 0][valid]
    assert np.all(np.isfinite(filt[valid])) and np.all(np.isfinite(mom[valid]))
    assert np.all(mom[..., 1][valid] >= 0)
    mse = float(np.mean((v - 1.0) ** 2))
    mean = float(np.mean(v))
    print("binary noise: MSE", mse, "mean", mean)
    assert mse < 0.1, "SVGF must remove at least 90% of the unit input MSE"
    assert abs(mean - 1.0) < 0.04, "SVGF must preserve mean radiance"
    rig.close()


def test_material_edge_is_preserved(cuda, scene):
    rig = Rig(scene=scene)
    for _ in range(3):
        rig.frame()
    # scene.changed(): the signal frame is the first of a new generation, so
    # its SVGF history is invalid and the spatial passes alone shape it.
    rig.changed()
    x = np.arange(W * H) % W
    sig = np.where(x < 80, 0.5, 2.0).astype(np.float32)

    def edge_colors(planes):
        c = planes["color"]
        c[:, : W // 2, :] = (1.0, 0.0, 0.0, 1.0)
        c[:, W // 2:, :] = (0.0, 1.0, 0.0, 1.0)

    planes = rig.frame(signal=sig, edit_planes=edge_colors)
    filt = rig.drv.session.image_host(L.BUF_FILTERED)[..., 0].reshape(-1)
    valid = planes["depth"].reshape(-1) < 1.0
    band = valid & (x >= 78) & (x <= 81)
    err = np.abs(filt[band] - sig[band])
    print("edge pixels", int(band.sum()), "max error", float(err.max()))
    assert band.sum() > 20
    assert np.all(err < 0.02), "material edge bled"
    rig.close()


def test_out_of_bounds_reprojection_restarts_history(cuda, scene):
    rig = Rig(scene=scene)
    for _ in range(4):
        rig.frame()

    def disocclude(planes):
        planes["motion"][:] = 2.0

    planes = rig.frame(edit_planes=disocclude)
    mom = rig.drv.session.moments_host()
    valid = planes["depth"] < 1.0
    assert valid.sum() > 0
    assert np.all(mom[..., 2][valid] == 1.0)
    rig.close()


@pytest.mark.parametrize("moments_format", [L.MOMENTS_F32, L.MOMENTS_F16])
def test_hdr_signal_stays_finite(cuda, moments_format, scene):
    rig = Rig(moments_format, scene=scene)
    for _ in range(2):
        rig.frame()
    rig.changed()
    sig = np.where(np.arange(W * H) % 2 == 0, 0.0, 60000.0).astype(np.float32)
    rig.frame(signal=sig)
    s = rig.drv.session
    filt = s.image_host(L.BUF_FILTERED)
    assert np.all(np.isfinite(filt)), "HDR wavelet radiance/variance must stay finite"
    p, n = s.buffer_ptr(L.BUF_MOMENTS)
    raw = s.buffer(L.BUF_MOMENTS, torch.uint8).cpu().numpy()
    stored = raw.view(np.float32) if n == W * H * 16 else raw.view(np.float16).astype(np.float32)
    assert np.all(np.isfinite(stored)), "stored moments must not overflow"
    mom = s.moments_host()
    assert np.any(mom[..., 1] > 65504.0), "E[l^2] exceeds the f16 range on this signal"
    rig.close()


def test_history_matures_on_static_room(cuda, scene):
    rig = Rig(scene=scene)
    for _ in range(40):
        rig.frame()
    s = rig.drv.session
    age = s.moments_host()[..., 2]
    valid = age > 0
    print("SVGF history: max", float(age.max()), "mature fraction", float((age[valid] >= 16).mean()))
    assert age.max() >= 16
    assert (age[valid] >= 16).mean() > 0.25
    st = rig.wl.settings
    for dom, cand in ((0, st.restir_direct_candidates), (1, st.restir_vpl_candidates)):
        r = s.reservoirs_host(dom, 2)
        assert r["count"].max() >= st.restir_max_history * cand
        assert 1 <= r["age"].max() <= st.restir_max_history
        assert (r["age"] >= 1).mean() > 0.1
    rig.close()


def test_lights_off_is_black_immediately(cuda, scene):
    rig = Rig(scene=scene)
    for _ in range(6):
        rig.frame()
    assert rig.drv.session.image_host(L.BUF_FILTERED)[..., :3].max() > 0

    def lights_off(f, lights):
        lights["position_strength"][:, 3] = 0.0

    rig.changed()
    rig.frame(edit=lights_off)
    s = rig.drv.session
    for which in (L.BUF_DIRECT, L.BUF_NOISY, L.BUF_FILTERED):
        assert np.all(s.image_host(which)[..., :3] == 0.0), which
    rig.close()


def test_history_flag_cleared_restarts_svgf(cuda, scene):
    # flags.x = 0 when the debug mode changes (src/renderer.rs:1729)
    rig = Rig(scene=scene)
    for _ in range(6):
        rig.frame()
    assert rig.drv.session.moments_host()[..., 2].max() > 1
    rig.frame(history=False)
    assert rig.drv.session.moments_host()[..., 2].max() == 1.0
    rig.close()
