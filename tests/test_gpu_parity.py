"""Parity of the CUDA lighting path (through the C-ABI) with the CPU oracle.

Per frame the oracle starts from the GPU's history (reservoirs [2], VPL
archive, SVGF moments/feedback, previous depth/normal), so every frame is an
independent parity case of all 11 reference passes; a free-running run then
checks that the accumulated images stay within the radiance bar.
"""
import numpy as np
import pytest
import torch

from instantradiositytest_b200 import _lib as L
from instantradiositytest_b200.runtime import FrameDriver
from instantradiositytest_b200.workload import Workload

from gpu_harness import RADIANCE_BAR, SELECT_BAR, Lockstep, rel_l1

pytestmark = pytest.mark.gpu


def summarize(rows):
    keys = rows[0].keys()
    return {k: (min(r[k] for r in rows) if k.startswith("select") else max(r[k] for r in rows)) for k in keys}


def check(stats, label, radiance_keys=("direct", "noisy", "filtered", "moments")):
    for k, v in stats.items():
        if k.startswith("select"):
            assert v >= SELECT_BAR, f"{label}: {k} = {v}"
        elif k in radiance_keys:
            assert v <= RADIANCE_BAR, f"{label}: {k} = {v}"


@pytest.mark.parametrize("schedule", [1, 0])
def test_small_room_lockstep_parity(cuda, schedule):
    """256x160 room of 12 meshes, 16 frames, f32 G-buffer and radiance;
    schedule 1 = ray-queue march, 0 = one kernel per reference entry point."""
    wl = Workload(0)
    ls = Lockstep(wl, fused=schedule)
    rows = [ls.frame(i) for i in range(16)]
    ls.close()
    stats = summarize(rows)
    print("lockstep schedule", schedule, stats)
    check(stats, "lockstep")


def test_reference_formats_lockstep_parity(cuda):
    """The reference's own storage formats: Rgba16Float G-buffer, noisy and
    SVGF radiance, Rgba32Float moments."""
    wl = Workload(0, width=160, height=100)
    ls = Lockstep(wl, gbuffer_format=L.GBUFFER_F16, radiance_format=L.RADIANCE_F16)
    rows = [ls.frame(i) for i in range(10)]
    ls.close()
    stats = summarize(rows)
    print("f16 formats", stats)
    check(stats, "f16")


def test_mixed_precision_storage(cuda):
    """The mixed-precision storage of the 1920x1200 room at 240x150: packed
    G-buffer (octahedral 2x16-bit normals, RGBA8 albedo), f16 SDF grids with
    per-mesh scale, f16 radiance history and f16 (mean, deviation) moments;
    reservoirs and all accumulation f32.

    Bar: against the f32 oracle with the reference's own f16 storage points
    (Rgba16Float radiance, Rgba32Float moments) on the same quantised inputs,
    selection >= 99.9 % and direct/noisy/filtered within 1e-3.
    Stated: the error of each output (direct, indirect, combined noisy and
    filtered) against an f64 oracle without f16 storage, next to the f32
    oracle's own error against it (the floor f32 arithmetic sets: grazing
    soft-shadow penumbrae amplify f32 rounding); the CUDA outputs may not be
    further from f64 than 1.5x that floor or 1e-3, whichever is larger."""
    wl = Workload(2, width=240, height=150)
    ls = Lockstep(wl, gbuffer_format=L.GBUFFER_PACKED, radiance_format=L.RADIANCE_F16,
                  moments_format=L.MOMENTS_F16, f64_witness=True)
    rows = [ls.frame(i) for i in range(8)]
    ls.close()
    stats = summarize(rows)
    print("mixed precision", {k: v for k, v in stats.items() if not k.startswith(("f64", "floor"))})
    print("against f64:", {k: (stats[f"f64_{k}"], stats[f"floor_{k}"])
                           for k in ("direct", "indirect", "noisy", "filtered")})
    check({k: v for k, v in stats.items() if not k.startswith(("f64", "floor"))}, "mixed precision",
          radiance_keys=("direct", "noisy", "filtered"))
    assert stats["direct"] > 0 or stats["f64_direct"] > 0  # the scene is lit
    for k in ("direct", "noisy", "filtered"):
        assert stats[f"f64_{k}"] <= max(RADIANCE_BAR, 1.5 * stats[f"floor_{k}"]), k


@pytest.mark.parametrize("debug", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("schedule", [1, 0])
def test_debug_views_lockstep_parity(cuda, debug, schedule):
    """The renderer's debug views (lighting.wgsl:106-134 gates: 1 direct only,
    2 indirect only, 3 albedo, 4 normals, 5 motion; src/svgf.rs:154-161
    bypasses SVGF from 3 on) against the oracle."""
    wl = Workload(0, width=96, height=64)
    ls = Lockstep(wl, fused=schedule)
    rows = [ls.frame(i, debug=debug) for i in range(4)]
    ls.close()
    stats = summarize(rows)
    print("debug", debug, "schedule", schedule, stats)
    check(stats, f"debug {debug}")


def test_free_running_images_stay_within_bar(cuda):
    wl = Workload(0)
    ls = Lockstep(wl)
    for i in range(16):
        r = ls.frame(i, sync=False)
    ls.close()
    print("free running, frame 15", r)
    assert r["noisy"] <= 5 * RADIANCE_BAR  # drift allowance over 16 frames without re-sync
    assert r["filtered"] <= 5 * RADIANCE_BAR


@pytest.mark.parametrize("schedule,size", [(1, (128, 96)), (2, (128, 96)), (1, (640, 480))])
def test_fused_and_plain_schedules_are_bit_identical(cuda, schedule, size):
    # With IEEE division and square root in the march, the ray-queue march
    # over the leaf-order cache reproduces the per-pixel BVH walk bit for bit.
    # At 640x480 the queue (about 600 000 rays) is long enough that the
    # march's warps reserve it in chunks before taking its last entries one
    # by one; at 128x96 they take every entry as their lanes go idle.
    wl = Workload(0, width=size[0], height=size[1])
    a = FrameDriver(wl, fused=schedule, keep_candidates=True, exact_march=True)
    b = FrameDriver(wl, fused=0)
    for i in range(6):
        inputs = a.inputs(i)
        a.step(i, inputs=inputs)
        b.step(i, inputs=inputs)
    torch.cuda.synchronize()
    for dom in (0, 1):
        for k in (0, 1, 2):
            assert np.array_equal(a.session.reservoirs_host(dom, k).view(np.uint8),
                                  b.session.reservoirs_host(dom, k).view(np.uint8)), (dom, k)
    for which in (L.BUF_DIRECT, L.BUF_NOISY, L.BUF_FILTERED, L.BUF_MOMENTS, L.BUF_FEEDBACK):
        assert np.array_equal(a.session.image_host(which), b.session.image_host(which)), which
    a.close()
    b.close()


def test_two_runs_are_bit_identical(cuda):
    # tools/verify.py:61-67 demands identical captures at tolerance 0.
    wl = Workload(0, width=96, height=64)
    outs = []
    for _ in range(2):
        d = FrameDriver(wl)
        for i in range(5):
            d.step(i)
        torch.cuda.synchronize()
        outs.append((d.session.image_host(L.BUF_FILTERED), d.session.reservoirs_host(1, 2).view(np.uint8)))
        d.close()
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_outputs_finite_capped_and_error_word_clear(cuda):
    wl = Workload(0)
    d = FrameDriver(wl)
    for i in range(8):
        d.step(i)
    torch.cuda.synchronize()
    assert d.session.check() == L.IRT_OK
    for which in (L.BUF_DIRECT, L.BUF_NOISY, L.BUF_FILTERED):
        img = d.session.image_host(which)
        assert np.all(np.isfinite(img)) and np.all(img[..., :3] >= 0)
    s = d.settings if hasattr(d, "settings") else wl.settings
    for dom, cand in ((0, s.restir_direct_candidates), (1, s.restir_vpl_candidates)):
        r = d.session.reservoirs_host(dom, 2)
        assert r["count"].max() <= s.restir_max_history * cand * 8
        assert r["count"].max() >= s.restir_max_history * cand  # temporal reuse retained
        assert r["age"].max() <= s.restir_max_history
    m = d.session.image_host(L.BUF_MOMENTS)
    assert m[..., 2].max() >= 6  # SVGF history accumulates on the static room
    d.close()
