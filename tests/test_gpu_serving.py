"""The render server (irt_server_*): a session's results are the same alone,
in a mix of concurrent sessions, and on the plain per-session path; admission
by HBM bytes; pacing."""
import time

import numpy as np
import pytest
import torch

from instantradiositytest_b200 import _lib as L
from instantradiositytest_b200.runtime import Context, FrameDriver
from instantradiositytest_b200.serving import Server
from instantradiositytest_b200.workload import Workload, preset_spec

pytestmark = pytest.mark.gpu


def workload(seed, meshes, w, h):
    spec = preset_spec(2, seed=seed, width=w, height=h, n_boxes=(meshes - 1) * 6 // 10,
                       n_spheres=(meshes - 1) - (meshes - 1) * 6 // 10)
    return Workload(spec)


@pytest.fixture(scope="module")
def scenes():
    return [workload(11, 8, 160, 100), workload(12, 16, 192, 120), workload(13, 12, 128, 80)]


def test_session_same_alone_in_mix_and_plain(cuda, scenes):
    frames = 6
    ctx = Context()
    # alone
    srv = Server(ctx, 8 << 30, streams=1, frame_rate=0)
    alone = srv.submit(0, 0.0, frames, scenes[0], capture_frame=frames - 1)
    st_alone = srv.run()
    srv.close()
    # in a mix of three concurrent sessions on three streams
    srv = Server(ctx, 8 << 30, streams=3, frame_rate=0)
    caps = [srv.submit(i, 0.0, frames + i, wl, capture_frame=frames - 1) for i, wl in enumerate(scenes)]
    st_mix = srv.run()
    srv.close()
    print("alone", st_alone, "mix", st_mix)
    assert st_mix["sessions"] == 3 and st_mix["frames"] == 3 * frames + 3
    assert st_mix["peak_active"] == 3
    assert np.array_equal(alone, caps[0])
    assert np.abs(alone.view(np.float32)).max() > 0
    # the plain per-session path with the same device-produced inputs
    d = FrameDriver(scenes[0], ctx=ctx, gpu_gbuffer=True, gpu_vpls=True)
    for i in range(frames):
        d.step(i)
    torch.cuda.synchronize()
    plain = d.session.buffer(L.BUF_FILTERED, torch.uint8).cpu().numpy()
    d.close()
    assert np.array_equal(alone, plain)
    ctx.close()


def test_admission_by_bytes_and_rejection(cuda, scenes):
    ctx = Context()
    probe = Server(ctx, 1 << 40)
    need = [probe.request_bytes(wl) for wl in scenes[:2]]
    probe.close()
    # room for the larger of the two, not both: sessions run one at a time
    srv = Server(ctx, max(need) + min(need) // 2, streams=2, frame_rate=0)
    srv.submit(0, 0.0, 4, scenes[0])
    srv.submit(1, 0.0, 4, scenes[1])
    big = workload(14, 8, 2560, 1600)
    srv.submit(2, 0.0, 4, big)  # larger than the whole budget
    st = srv.run()
    srv.close()
    print(st)
    assert st["sessions"] == 2 and st["rejected"] == 1 and st["frames"] == 8
    assert st["peak_active"] == 1
    assert st["peak_bytes"] <= max(need) + min(need) // 2
    assert ctx.bytes_in_use() == 0
    ctx.close()


def test_frame_pacing(cuda, scenes):
    ctx = Context()
    srv = Server(ctx, 8 << 30, streams=1, frame_rate=60.0)
    srv.submit(0, 0.0, 12, scenes[2])
    t = time.perf_counter()
    st = srv.run()
    wall = time.perf_counter() - t
    srv.close()
    ctx.close()
    print(st, wall)
    assert st["frames"] == 12
    assert wall >= 11 / 60.0  # frame k is not started before k / 60 s
    assert st["p99_latency_ms"] < 1000.0
