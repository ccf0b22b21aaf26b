"""Pins of the CPU oracle: the reference's CPU known-answer tests
(src/math.rs:77-200), binary16 conversion (half 2.7.1, round to nearest
even) and the RNG restated in plain Python integers, checked against the
committed golden vectors in tests/golden/."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from instantradiositytest_b200 import _lib as L
from oracle import binding as ob

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
F3 = C.c_float * 3


def res():
    return np.zeros(1, L.RESERVOIR_DTYPE)


def add(r, id_, target, weight, count, u):
    return ob.lib().oracle_res_add_u(r.ctypes.data, id_, 0, target, 0.0, weight, count, 0, u)


def norm(r):
    return ob.lib().oracle_normalization(r.ctypes.data)


def test_constant_target_reservoir_recovers_light_sum():
    # src/math.rs:109-116: 8 inserts of target 2 at pdf 1/4.
    r = res()
    for i in range(8):
        add(r, i, 2.0, 2.0 / 0.25, 1, 0.1)
    assert r["count"][0] == 8
    assert abs(2 * norm(r) - 8) < 1e-6


def test_reuse_reweights_target():
    # src/math.rs:118-130
    src = res()
    add(src, 0, 2.0, 2.0 / 0.25, 1, 0.0)
    r = res()
    add(r, src["id"][0], 4.0, 4.0 * norm(src) * src["count"][0], src["count"][0], 0.0)
    assert abs(norm(r) - 4) < 1e-6


def test_rejected_weights_do_not_select():
    r = res()
    assert add(r, 3, 1.0, 0.0, 1, 0.0) == 0
    assert add(r, 3, 1.0, 2e30, 1, 0.0) == 0
    assert r["count"][0] == 2 and r["sum"][0] == 0 and norm(r) == 0


def test_second_shadow_method_is_finite_and_monotonic():
    # src/math.rs:158-163, with the march's first `previous` of 1e20.
    q = ob.lib().oracle_quilez_step
    a = q(1.0, 0.1, 1e20, 2.0, 16.0)
    assert abs(a - 0.8) < 1e-5
    b = q(a, 0.01, 0.1, 2.1, 16.0)
    assert 0 <= b <= a


def sbd(p, lo=(-1, -1, -1), hi=(1, 1, 1)):
    return ob.lib().oracle_signed_box_distance(F3(*p), F3(*lo), F3(*hi))


def test_enclosing_box_and_sphere_are_signed_lower_bounds():
    # src/math.rs:81-107
    assert sbd((0, 0, 0)) == -1
    assert sbd((2, 0, 0)) == 1
    assert abs(sbd((2, 2, 2)) - np.sqrt(3)) < 1e-6
    assert abs(sbd((1, 0, 0))) < 1e-6
    g = np.arange(-15, 16, 3) / 10
    for x in g:
        for y in g:
            for z in g:
                p = np.array([x, y, z], np.float32)
                bound = max(sbd(p), float(np.linalg.norm(p)) - 1)
                sphere = float(np.linalg.norm(p)) - 1
                torus = float(np.hypot(np.hypot(p[0], p[1]) - 0.7, p[2])) - 0.3
                assert bound <= sphere + 1e-6
                assert bound <= torus + 1e-6


def sphere_mesh_and_atlas(res_=16, radius=0.6):
    lo = np.float32(-1.0)
    spacing = np.float32(2.0) / np.float32(res_ - 1)
    i = np.arange(res_, dtype=np.float32)
    z, y, x = np.meshgrid(i, i, i, indexing="ij")
    p = np.stack([x, y, z], -1) * spacing + lo
    field = (np.sqrt((p * p).sum(-1)) - radius).astype(np.float32)
    m = np.zeros(1, L.MESH_DTYPE)
    m["lo"][0, :3] = lo
    m["hi"][0, :3] = 1.0
    m["field"][0] = [0, 0, 0, res_]
    m["grid"][0] = [1 / spacing, 1 / spacing, 1 / spacing, np.sqrt(3) * spacing]
    m["geometry_lo"][0] = [-radius, -radius, -radius, 0]
    s = np.ascontiguousarray(field.reshape(-1))
    bound = ob.lib  # noqa: F841
    lip = L.lib.irt_field_lipschitz_bound(L.ptr(s), res_, F3(spacing, spacing, spacing))
    m["geometry_hi"][0] = [radius, radius, radius, 1 / lip]
    m["enclosing_sphere"][0] = [0, 0, 0, radius * 1.000001 + 1e-6]
    return m, np.ascontiguousarray(field)


def mesh_distance(m, atlas, p):
    dims = (C.c_uint32 * 3)(atlas.shape[2], atlas.shape[1], atlas.shape[0])
    return ob.lib().oracle_mesh_distance(m.ctypes.data, atlas.ctypes.data, dims, F3(*p))


def test_field_bound_never_oversteps_and_is_continuous():
    # src/math.rs:165-199 for the field path of mesh_distance (sdf.wgsl:5-33):
    # the bound stays below the exact sphere distance everywhere, inside and
    # outside the padded grid, and does not jump across cell faces.
    m, atlas = sphere_mesh_and_atlas()
    rng = np.random.default_rng(7)
    pts = rng.uniform(-2.5, 2.5, (3000, 3)).astype(np.float32)
    for p in pts:
        d = mesh_distance(m, atlas, p)
        exact = float(np.linalg.norm(p)) - 0.6
        assert d <= exact + 1e-5, (p, d, exact)
    spacing = 2.0 / 15
    face = -1.0 + 7 * spacing
    a = mesh_distance(m, atlas, (face - 1e-6, 0.31, 0.17))
    b = mesh_distance(m, atlas, (face + 1e-6, 0.31, 0.17))
    assert abs(a - b) < 1e-4


def test_f16_conversion_matches_numpy_round_to_nearest_even():
    rng = np.random.default_rng(3)
    vals = np.concatenate([
        rng.standard_normal(4000).astype(np.float32) * np.float32(100),
        rng.uniform(0, 1e-4, 500).astype(np.float32),  # subnormal range of f16
        np.array([65504, 65519.9, 65520, 1e6, -1e6, 0.0, -0.0, 6.1e-5, 5.96e-8, 2.98e-8], np.float32),
    ])
    for v in vals:
        assert ob.f16_bits(v) == int(np.float32(v).astype(np.float16).view(np.uint16)), v
        h = int(np.float32(v).astype(np.float16).view(np.uint16))
        assert ob.f16_from_bits(h) == float(np.uint16(h).view(np.float16).astype(np.float32))


def py_random_stream(i, salt, frame, n):
    """common.wgsl:39-44 in Python integers (independent of the C++)."""
    m = 0xFFFFFFFF
    s = (i * 1973 + frame * 9277 + salt * 26699 + 89173) & m
    out = []
    for _ in range(n):
        s = (s * 747796405 + 2891336453) & m
        w = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & m
        out.append((s, np.float32((w >> 22) ^ w) * np.float32(1.0 / 4294967296.0)))
    return out


def oracle_stream(i, salt, frame, n):
    vals = np.zeros(n, np.float32)
    states = np.zeros(n, np.uint32)
    ob.lib().oracle_random_stream(i, salt, frame, n, vals.ctypes.data, states.ctypes.data)
    return states, vals


def test_rng_matches_integer_restatement_and_golden():
    with open(os.path.join(GOLDEN, "rng_streams.json")) as fh:
        golden = json.load(fh)
    for case in golden["cases"]:
        st, vals = oracle_stream(case["i"], case["salt"], case["frame"], len(case["states"]))
        assert st.tolist() == case["states"]
        assert vals.view(np.uint32).tolist() == case["value_bits"]
        py = py_random_stream(case["i"], case["salt"], case["frame"], len(case["states"]))
        assert [s for s, _ in py] == case["states"]
        assert [int(np.float32(v).view(np.uint32)) for _, v in py] == case["value_bits"]


def test_random_can_return_one():
    # f32((w>>22)^w) rounds to 2^32 for the largest outputs; callers clamp.
    assert np.float32(0xFFFFFFFF) * np.float32(1.0 / 4294967296.0) == np.float32(1.0)


@pytest.mark.parametrize("precision", [0, 1])
def test_oracle_small_frames_run_in_both_precisions(precision):
    from instantradiositytest_b200.workload import Workload
    from oracle import Oracle, OracleScene

    wl = Workload(0, width=48, height=32)
    orc = Oracle(48, 32, wl.settings.vpl_count, 4, precision)
    prev = None
    for fi in range(3):
        f, obj, nodes, lights = wl.frame(fi)
        g = wl.gbuffer_cpu(f)
        v = wl.vpls_cpu(f, obj, lights)
        prev = np.zeros_like(v) if prev is None else prev
        orc.frame(f, OracleScene(obj, wl.meshes, nodes, lights, wl.atlas), g, v, prev)
        prev = v
    out = orc.image(ob.HISTORIES[2 % 2])
    assert np.all(np.isfinite(out)) and out[..., :3].mean() > 0
    r = orc.reservoirs("d", 2, L.RESERVOIR_DTYPE)
    assert r["count"].max() >= 8
    orc.close()
    wl.close()


def test_filtered_field_emulation_weights_and_texel_centres():
    """The oracle's restatement of the reference's filtered sample_field
    (src/renderer.rs:277-286): on an atlas whose texels hold their x index,
    the value is the base texel plus an 8-bit fixed-point weight; at texel
    centres of a random atlas it equals the point-sampled form; and it never
    leaves the point-sampled value by more than the voxel/128 allowance the
    mesh bound carries for fixed-point hardware weights (sdf.wgsl:16-17)."""
    mesh = np.zeros(1, L.MESH_DTYPE)[0]
    res = 8
    mesh["field"] = (4, 0, 0, res)
    mesh["grid"] = (1.0, 1.0, 1.0, np.sqrt(3.0))
    dims = (res, res, 16)  # z, y, x
    ramp = np.broadcast_to(np.arange(dims[2], dtype=np.float32), dims).copy()
    for fx in np.linspace(0.0, 0.999, 37, dtype=np.float32):
        v = ob.sample_field(mesh, ramp, (2.0 + fx, 1.5, 3.25), 1)
        base = 4 + 2
        assert v - base == pytest.approx(np.floor(float(fx) * 256 + 0.5) / 256, abs=1e-6)
    rng = np.random.default_rng(3)
    atlas = rng.uniform(-1, 1, size=dims).astype(np.float32)
    for _ in range(64):
        c = rng.integers(0, res, size=3).astype(np.float32)
        assert ob.sample_field(mesh, atlas, c, 1) == pytest.approx(ob.sample_field(mesh, atlas, c, 0), abs=1e-6)
    smooth = (np.arange(dims[2], dtype=np.float32)[None, None, :] * 0.3
              + np.arange(dims[1], dtype=np.float32)[None, :, None] * 0.2
              + np.arange(dims[0], dtype=np.float32)[:, None, None] * 0.1).astype(np.float32)
    worst = 0.0
    for _ in range(256):
        q = rng.uniform(0, res - 1, size=3).astype(np.float32)
        worst = max(worst, abs(ob.sample_field(mesh, smooth, q, 1) - ob.sample_field(mesh, smooth, q, 0)))
    assert worst <= np.sqrt(3.0) / 128
