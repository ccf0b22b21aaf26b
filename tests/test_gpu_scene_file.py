"""Loaded scene files on the device: the CUDA G-buffer producer and VPL
generator against their CPU counterparts on triangle meshes, and lockstep
parity of the hot path with the oracle on a loaded scene (a scene written by
instantradiositytest_b200.scene_file; the shipped test scene too when
IRT_TEST_SCENE names its scene.json)."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from instantradiositytest_b200 import _lib as L
from instantradiositytest_b200 import scene_file as sf
from instantradiositytest_b200.runtime import Context, Scene, gbuffer_device_alloc, stream_handle
from instantradiositytest_b200.workload import Workload, gbuffer_as_f32

from gpu_harness import RADIANCE_BAR, SELECT_BAR, Lockstep

pytestmark = pytest.mark.gpu

SHIPPED = os.environ.get("IRT_TEST_SCENE", "")


@pytest.fixture(scope="module")
def demo(tmp_path_factory):
    return sf.write_scene(str(tmp_path_factory.mktemp("demo")), sf.demo_scene(resolution=24))


def gpu_gbuffer(ctx, wl, f):
    gt, gs = gbuffer_device_alloc(wl.height, wl.width, L.GBUFFER_F32)
    L.check(L.lib.irt_gbuffer_render(ctx.handle, wl.handle, C.byref(f), None, L.GBUFFER_F32, gs.depth, gs.normal,
                                     gs.color, gs.params, gs.motion, stream_handle()), ctx.handle, "gbuffer")
    torch.cuda.synchronize()
    H, W = wl.height, wl.width
    return {"depth": gt["depth"].cpu().numpy().view(np.float32).reshape(H, W),
            "normal": gt["normal"].cpu().numpy().view(np.float32).reshape(H, W, 4),
            "color": gt["color"].cpu().numpy().view(np.float32).reshape(H, W, 4)}


def gpu_vpls(ctx, scene, wl, f, obj, nodes, lights):
    scene.update(obj, nodes, lights)
    out = torch.zeros(f.counts[1] * 48, dtype=torch.uint8, device="cuda")
    L.check(L.lib.irt_vpl_generate(scene.handle, wl.handle, C.byref(f), C.c_void_p(out.data_ptr()), stream_handle()),
            ctx.handle, "vpl generate")
    torch.cuda.synchronize()
    return out.cpu().numpy().view(L.VPL_DTYPE)


def producers_agree(path, width, height, vpls):
    wl = Workload.load(path, width=width, height=height, vpl_count=vpls)
    ctx = Context()
    scene = Scene(ctx, wl.meshes, wl.atlas, wl.sdf_format)
    f, obj, nodes, lights = wl.frame(0)
    c = wl.gbuffer_cpu(f)
    g = gpu_gbuffer(ctx, wl, f)
    same_hit = (c["depth"] < 1) == (g["depth"] < 1)
    both = (c["depth"] < 1) & (g["depth"] < 1)
    near = np.abs(c["depth"] - g["depth"]) < 1e-4
    nrm = np.abs(c["normal"][..., :3] - g["normal"][..., :3]).max(-1) < 1e-3
    col = (c["color"] == g["color"]).all(-1)
    agree = same_hit & (~both | (near & nrm & col))
    print(f"{os.path.basename(os.path.dirname(path))}: G-buffer agreement {agree.mean():.5f}")
    assert agree.mean() >= 0.995  # f32 vs f64 triangle tests differ on silhouette edges only
    gv = gpu_vpls(ctx, scene, wl, f, obj, nodes, lights)
    cv = wl.vpls_cpu(f, obj, lights)
    dp = np.abs(gv["position"][:, :3] - cv["position"][:, :3]).max(1)
    dn = np.abs(gv["normal"][:, :3] - cv["normal"][:, :3]).max(1)
    fc = np.abs(cv["flux"][:, :3]).max(1)
    df = np.abs(gv["flux"][:, :3] - cv["flux"][:, :3]).max(1) / np.maximum(fc, 1e-12)
    same = (dp < 1e-3) & (dn < 1e-3) & ((df < 1e-3) | ((fc == 0) & (np.abs(gv["flux"][:, :3]).max(1) == 0)))
    print(f"VPL paths agreeing {same.mean():.4f}; contributing {(fc > 0).mean():.3f}")
    assert same.mean() >= 0.98
    assert (fc > 0).mean() > 0.1
    scene.close()
    ctx.close()


def lockstep(path, width, height, vpls, frames, sdf_format=L.SDF_F32, **formats):
    wl = Workload.load(path, width=width, height=height, vpl_count=vpls, sdf_format=sdf_format)
    ls = Lockstep(wl, **formats)
    rows = [ls.frame(i) for i in range(frames)]
    ls.close()
    worst = {k: (min(r[k] for r in rows) if k.startswith("select") else max(r[k] for r in rows)) for k in rows[0]}
    print(f"{os.path.basename(os.path.dirname(path))} lockstep", worst)
    for k, v in worst.items():
        if k.startswith("select"):
            assert v >= SELECT_BAR, (k, v)
        elif k in ("direct", "noisy", "filtered", "moments"):
            assert v <= RADIANCE_BAR, (k, v)


def test_cuda_producers_match_cpu_on_a_loaded_scene(cuda, demo):
    producers_agree(demo, 256, 160, 512)


def test_loaded_scene_lockstep_parity(cuda, demo):
    lockstep(demo, 192, 120, 256, 8)


def test_loaded_scene_mixed_precision_lockstep(cuda, demo):
    """The loaded scene with the mixed-precision storage: f16 SDF corner
    records, packed G-buffer, f16 radiance and moments; the oracle sees the
    same quantised inputs and the reference's f16 storage points."""
    lockstep(demo, 192, 120, 256, 6, sdf_format=L.SDF_F16, gbuffer_format=L.GBUFFER_PACKED,
             radiance_format=L.RADIANCE_F16, moments_format=L.MOMENTS_F16)


@pytest.mark.parametrize("schedule", [0, 2])
def test_loaded_scene_other_schedules_lockstep(cuda, demo, schedule):
    """The one-kernel-per-entry-point (0) and fused-inline (2) schedules on a
    loaded scene, with the reference's own Rgba16Float G-buffer targets."""
    lockstep(demo, 160, 100, 256, 5, gbuffer_format=L.GBUFFER_F16, fused=schedule)


def test_batched_views_of_a_loaded_scene_equal_alone(cuda, demo):
    """A batch over a loaded scene and a procedural room (views of uneven
    size, two views of the loaded scene): every view's outputs equal
    rendering it alone, bit for bit."""
    from instantradiositytest_b200.batching import BatchDriver
    from test_gpu_batch import BUFS, render_alone, workload

    a = Workload.load(demo, width=160, height=100, vpl_count=128)
    b = workload(31, 10, 128, 80)
    views = [(a, 0), (b, 0), (a, 5, (96, 60))]
    ctx = Context()
    drv = BatchDriver(ctx, views, use_graphs=True)
    per_view = [[] for _ in views]
    for i in range(8):
        data = drv.inputs(i)
        frames = drv.step(i, data)
        for v, (f, (_, obj, nodes, lights)) in enumerate(zip(frames, data)):
            per_view[v].append((L.Frame.from_buffer_copy(f), obj, nodes, lights))
    torch.cuda.synchronize()
    for v, view in enumerate(views):
        wl = view[0]
        if len(view) > 2:  # the alone render runs at the view's own size
            continue
        s = drv.batch.view(v)
        got = {w: s.buffer(w, torch.uint8).cpu().numpy() for w in BUFS}
        ref = render_alone(ctx, wl, per_view[v], L.GBUFFER_F32, L.RADIANCE_F32, L.MOMENTS_F32)
        for w in BUFS:
            assert np.array_equal(got[w], ref[w]), (v, w)
    assert np.isfinite(drv.batch.view(2).image_host(L.BUF_FILTERED)).all()
    drv.close()
    ctx.close()


@pytest.mark.skipif(not (SHIPPED and os.path.exists(SHIPPED)), reason="IRT_TEST_SCENE not set")
def test_shipped_test_scene_producers_and_parity(cuda):
    producers_agree(SHIPPED, 320, 200, 1024)
    lockstep(SHIPPED, 320, 200, 1024, 6)
