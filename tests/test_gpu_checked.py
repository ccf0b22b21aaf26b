"""The checked build (libirt_checked.so) against the default one.

The checked build's kernels test every index they take from data before
following it and report a bad one through the session's error word instead
of faulting; compute-sanitizer's role on a pool where it is closed.  Here
both builds render the same frames (the ray-queue and per-entry-point
schedules, f32 and mixed-precision storage, batched views): the checked build
must report no bad index and give the same bytes in every output buffer.
The checked build runs in a child process (IRT_LIBRARY=checked), since one
process loads one build.
"""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

from instantradiositytest_b200 import _lib as L

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUFS = (L.BUF_DIRECT, L.BUF_NOISY, L.BUF_FILTERED, L.BUF_MOMENTS, L.BUF_FEEDBACK)
CASES = {
    "f32_queue": dict(preset=0, size=(256, 160), fused=1, formats=(0, 0, 0)),
    "f32_plain": dict(preset=0, size=(160, 100), fused=0, formats=(0, 0, 0)),
    "mixed_queue": dict(preset=2, size=(240, 150), fused=1, formats=(2, 1, 1)),
}
FRAMES = 6


def render_all(out_path):
    """Renders every case with the loaded build and saves the output buffers,
    reservoirs and error-word status."""
    from instantradiositytest_b200 import _lib as LL
    from instantradiositytest_b200.batching import BatchDriver
    from instantradiositytest_b200.runtime import Context, FrameDriver
    from instantradiositytest_b200.workload import Workload

    saved = {"flavour": np.array(LL.lib.irt_build_flavour().decode())}
    for name, c in CASES.items():
        wl = Workload(c["preset"], width=c["size"][0], height=c["size"][1])
        g, r, m = c["formats"]
        d = FrameDriver(wl, gbuffer_format=g, radiance_format=r, moments_format=m, fused=c["fused"],
                        gpu_gbuffer=True, gpu_vpls=True)
        for i in range(FRAMES):
            d.step(i)
        torch.cuda.synchronize()
        saved[f"{name}_status"] = np.array(d.session.check())
        for b in BUFS:
            saved[f"{name}_{b}"] = d.session.buffer(b, torch.uint8).cpu().numpy()
        for dom in (0, 1):
            saved[f"{name}_res{dom}"] = d.session.reservoirs_host(dom, 2).view(np.uint8)
        d.close()
        wl.close()
    ctx = Context()
    a = Workload(0, width=160, height=100)
    b = Workload(2, width=192, height=120)
    drv = BatchDriver(ctx, [(a, 0), (b, 0), (a, 5)], 2, 1, 1, use_graphs=True)
    for i in range(FRAMES):
        drv.step(i)
    torch.cuda.synchronize()
    for v in range(3):
        s = drv.batch.view(v)
        saved[f"batch{v}_status"] = np.array(s.check())
        saved[f"batch{v}_filtered"] = s.buffer(LL.BUF_FILTERED, torch.uint8).cpu().numpy()
    drv.close()
    ctx.close()
    np.savez(out_path, **saved)


def test_checked_build_reports_no_bad_index_and_matches_default(cuda, tmp_path):
    assert os.path.exists(L.CHECKED_LIB_PATH), "build libirt_checked.so (make -C instantradiositytest_b200)"
    checked = tmp_path / "checked.npz"
    env = dict(os.environ, IRT_LIBRARY="checked", PYTHONPATH=os.pathsep.join([ROOT, os.path.join(ROOT, "tests")]))
    code = f"import test_gpu_checked as t; t.render_all({str(checked)!r})"
    r = subprocess.run([sys.executable, "-c", code], env=env, cwd=ROOT, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    default = tmp_path / "default.npz"
    render_all(str(default))
    a, b = np.load(checked), np.load(default)
    assert str(a["flavour"]) == "checked" and str(b["flavour"]) == "default"
    for k in a.files:
        if k.endswith("_status"):
            assert int(a[k]) == L.IRT_OK, f"checked build reported a bad index: {k}"
    for k in a.files:
        if k != "flavour":
            assert np.array_equal(a[k], b[k]), k
    print("checked build: no bad index;", len(a.files) - 1, "buffers identical to the default build")
