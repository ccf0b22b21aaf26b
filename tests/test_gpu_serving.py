"""The render server (irt_server_*): a session's results are the same alone,
in a mix of concurrent sessions, and on the plain per-session path, and
match the oracle; admission by HBM bytes, also of requests that arrive while
others render; pacing."""
import time

import numpy as np
import pytest
import torch

from instantradiositytest_b200 import _lib as L
from instantradiositytest_b200.runtime import Context, FrameDriver
from instantradiositytest_b200.serving import Server
from instantradiositytest_b200.workload import Workload, preset_spec

from gpu_harness import RADIANCE_BAR, SELECT_BAR, Lockstep, outputs, rel_l1

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


def test_served_session_against_the_oracle(cuda, scenes):
    """A served session's captured frame against the oracle: the same
    workload runs in lockstep with the oracle on the device-produced
    G-buffer and VPL pools the server uses (per frame the oracle starts from
    the session's history), and the served capture equals that session's
    image bit for bit and the oracle's within the radiance bar."""
    frames = 6
    wl = scenes[1]
    ctx = Context()
    srv = Server(ctx, 8 << 30, streams=2, frame_rate=0)
    served = srv.submit(0, 0.0, frames, wl, capture_frame=frames - 1)
    srv.submit(1, 0.0, frames + 3, scenes[2])  # company on the other stream
    srv.run()
    srv.close()
    ctx.close()
    ls = Lockstep(wl, gpu_gbuffer=True, gpu_vpls=True)
    rows = [ls.frame(i) for i in range(frames)]
    mine = ls.drv.session.buffer(L.BUF_FILTERED, torch.uint8).cpu().numpy()
    ref = outputs(ls.orc, frames - 1)["filtered"].copy()  # a view of the oracle's buffer until close()
    ls.close()
    worst = {k: (min(r[k] for r in rows) if k.startswith("select") else max(r[k] for r in rows)) for k in rows[0]}
    print("served session lockstep", worst)
    for k, v in worst.items():
        if k.startswith("select"):
            assert v >= SELECT_BAR, (k, v)
        elif k in ("direct", "noisy", "filtered"):
            assert v <= RADIANCE_BAR, (k, v)
    assert np.array_equal(served, mine)
    img = served.view(np.float32).reshape(wl.height, wl.width, 4)[..., :3]
    assert rel_l1(img, ref) <= RADIANCE_BAR


def test_late_arrivals_wait_for_retirements_and_match_alone(cuda, scenes):
    """Continuous batching: C arrives while A and B are on the GPU and the
    budget holds two sessions, so C waits; it is admitted when B retires,
    while A is still rendering, and runs alongside A.  Each session's
    captured frame equals rendering it alone."""
    ctx = Context()
    plan = [(0, 0.0, 40, scenes[0]), (1, 0.0, 6, scenes[1]), (2, 0.03, 10, scenes[2])]  # id, arrival, frames
    probe = Server(ctx, 1 << 40)
    need = [probe.request_bytes(wl) for _, _, _, wl in plan]
    probe.close()
    # A and B fit together, C does not fit beside both, but fits beside A
    budget = need[0] + max(need[1], need[2]) + need[2] // 2
    srv = Server(ctx, budget, streams=2, frame_rate=60.0)
    times = [np.zeros(3, np.float64) for _ in plan]
    caps = [srv.submit(i, t, n, wl, capture_frame=n - 1, times=times[i]) for i, t, n, wl in plan]
    st = srv.run()
    srv.close()
    (a_adm, a_done, a_ret), (b_adm, b_done, b_ret), (c_adm, c_done, c_ret) = (tuple(t) for t in times)
    print("stats", st)
    print("timeline A", times[0], "B", times[1], "C", times[2])
    assert st["sessions"] == 3 and st["frames"] == 56 and st["peak_active"] == 2
    assert c_adm >= b_ret  # C waited for B's bytes
    assert c_adm > plan[2][1]  # ... after it arrived
    assert c_adm < a_done  # while A was still rendering
    assert c_done < a_done  # and its frames ran alongside A's
    for (i, _, n, wl), cap in zip(plan, caps):
        solo = Server(ctx, 8 << 30, streams=1, frame_rate=0)
        alone = solo.submit(i, 0.0, n, wl, capture_frame=n - 1)
        solo.run()
        solo.close()
        assert np.array_equal(alone, cap), i
        assert np.abs(cap.view(np.float32)).max() > 0
    ctx.close()
