"""The CUDA VPL generator (irt_vpl_generate, vpl.wgsl:1-47) against the CPU
generator on the same frames, and the path-budget / source-power invariants
of src/gpu_tests.rs:354-407 on the device."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from instantradiositytest_b200 import _lib as L
from instantradiositytest_b200.runtime import Context, Scene, stream_handle
from instantradiositytest_b200.workload import Workload

pytestmark = pytest.mark.gpu


def gpu_vpls(ctx, scene, wl, f, obj, nodes, lights):
    scene.update(obj, nodes, lights)
    out = torch.zeros(f.counts[1] * 48, dtype=torch.uint8, device="cuda")
    L.check(L.lib.irt_vpl_generate(scene.handle, wl.handle, C.byref(f), C.c_void_p(out.data_ptr()), stream_handle()),
            ctx.handle, "vpl generate")
    torch.cuda.synchronize()
    return out.cpu().numpy().view(L.VPL_DTYPE)


@pytest.mark.parametrize("preset,frames", [(0, (0, 1, 7)), (1, (0, 5))])
def test_cuda_vpls_match_cpu_generator(cuda, preset, frames):
    wl = Workload(preset, width=64, height=40)
    ctx = Context()
    scene = Scene(ctx, wl.meshes, wl.atlas, wl.sdf_format)
    for i in frames:
        f, obj, nodes, lights = wl.frame(i)
        g = gpu_vpls(ctx, scene, wl, f, obj, nodes, lights)
        c = wl.vpls_cpu(f, obj, lights)
        dp = np.abs(g["position"][:, :3] - c["position"][:, :3]).max(1)
        dn = np.abs(g["normal"][:, :3] - c["normal"][:, :3]).max(1)
        fl_c = c["flux"][:, :3]
        dflux = np.abs(g["flux"][:, :3] - fl_c).max(1) / np.maximum(np.abs(fl_c).max(1), 1e-12)
        same = (dp < 1e-3) & (dn < 1e-4) & ((dflux < 1e-3) | (np.abs(fl_c).max(1) == 0) & (np.abs(g["flux"][:, :3]).max(1) == 0))
        tot_g, tot_c = g["flux"][:, :3].sum(), c["flux"][:, :3].sum()
        print(f"preset {preset} frame {i}: {same.mean():.4f} of {len(c)} paths agree; total flux {tot_g} vs {tot_c}")
        assert same.mean() >= 0.99
        assert abs(tot_g - tot_c) <= 2e-2 * abs(tot_c)
        assert (np.abs(c["flux"][:, :3]).max(1) > 0).mean() > 0.5  # contributing VPLs exist
    scene.close()
    ctx.close()


SHIPPED = os.environ.get("IRT_TEST_SCENE", "")


@pytest.mark.parametrize("scene", ["room"] + (["test_scene"] if SHIPPED and os.path.exists(SHIPPED) else []))
def test_cuda_vpl_budget_and_power_normalization(cuda, scene):
    """src/gpu_tests.rs:354-407 — on the procedural room, and on the shipped
    test scene it was written for (16x16, settings.json's 100 paths) where
    IRT_TEST_SCENE names it."""
    if scene == "room":
        wl = Workload(0, width=64, height=40)
    else:
        wl = Workload.load(SHIPPED, width=16, height=16, vpl_count=100)
    ctx = Context()
    scene = Scene(ctx, wl.meshes, wl.atlas, wl.sdf_format)
    f, obj, nodes, lights = wl.frame(0)
    base = gpu_vpls(ctx, scene, wl, f, obj, nodes, lights)
    f2 = L.Frame.from_buffer_copy(f)
    f2.counts[1] = f.counts[1] * 2
    doubled = gpu_vpls(ctx, scene, wl, f2, obj, nodes, lights)
    n = f.counts[1]
    # same emission and roulette decisions for the shared paths, half flux
    assert np.array_equal(base["position"], doubled["position"][:n])
    assert np.array_equal(base["normal"], doubled["normal"][:n])
    assert np.all(np.abs(base["flux"][:, :3] - 2 * doubled["flux"][:n, :3]) < 1e-6)
    l2 = lights.copy()
    l2["position_strength"][:, 3] *= 2
    power = gpu_vpls(ctx, scene, wl, f, obj, nodes, l2)
    assert np.array_equal(base["position"], power["position"])
    assert np.all(np.abs(2 * base["flux"][:, :3] - power["flux"][:, :3]) < 1e-6)
    assert np.any(base["flux"][:, :3] > 0)
    scene.close()
    ctx.close()
