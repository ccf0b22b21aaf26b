"""Known-answer tests of the host logic (C++ in libirt.so) restated from the
reference's unit tests: src/renderer.rs:2169-2230 and the hierarchy/atlas/
object packing rules of src/renderer.rs:359-455 and :778-817."""
import ctypes as C
import struct

import numpy as np
import pytest

from instantradiositytest_b200 import _lib as L
from instantradiositytest_b200.workload import Workload

lib = L.lib
F3 = C.c_float * 3


def cube_vertices(perturb=False):
    v = np.zeros(8, L.VERTEX_DTYPE)
    for i in range(8):
        v["position"][i] = [1 if i & 1 else -1, 1 if i & 2 else -1, 1 if i & 4 else -1, 1]
    if perturb:
        v["position"][0, 0] += np.float32(0.001)
    return v


CUBE = [0, 2, 6, 0, 6, 4, 1, 5, 7, 1, 7, 3, 0, 4, 5, 0, 5, 1, 2, 3, 7, 2, 7, 6, 0, 1, 3, 0, 3, 2, 4, 6, 7, 4, 7, 5]


def is_box(v, idx):
    idx = np.asarray(idx, np.uint32)
    return lib.irt_is_box_geometry(L.ptr(v), len(v), L.ptr(idx), len(idx), F3(-1, -1, -1), F3(1, 1, 1))


def test_box_certification_rejects_holes_overlap_and_other_geometry():
    # src/renderer.rs:2196-2230
    v = cube_vertices()
    assert is_box(v, CUBE) == 1
    assert is_box(v, CUBE[:33]) == 0
    overlap = list(CUBE)
    overlap[3:6] = CUBE[:3]
    assert is_box(v, overlap) == 0
    hole = list(CUBE)
    hole[3:6] = [0, 2, 4]
    assert is_box(v, hole) == 0
    nonface = list(CUBE)
    nonface[:3] = [0, 3, 7]
    assert is_box(v, nonface) == 0
    assert is_box(cube_vertices(perturb=True), CUBE) == 0


def lipschitz(samples, n, spacing):
    s = np.ascontiguousarray(samples, np.float32)
    return lib.irt_field_lipschitz_bound(L.ptr(s), n, F3(*spacing))


def test_trilinear_gradient_bound_covers_simultaneous_axis_slopes():
    # src/renderer.rs:2169-2195
    spacing = np.array([0.25, 0.5, 1.0], np.float32)
    samples = []
    for i in range(8):
        p = np.array([i & 1, (i >> 1) & 1, i >> 2], np.float32) * spacing
        samples.append(np.float32(10) + np.float32(p @ np.array([1, 2, 3], np.float32)))
    b = lipschitz(samples, 2, spacing)
    assert b >= np.sqrt(np.float32(14))
    assert b < np.sqrt(np.float32(14)) * 1.001
    assert lipschitz(np.zeros(8), 2, spacing) >= 1
    assert lipschitz(np.full(8, -100.0), 2, spacing) >= 1
    n = 16
    i = np.arange(n ** 3)
    p = np.stack([i % n, (i // n) % n, i // (n * n)], -1).astype(np.float32) * np.float32(0.2) - np.float32(1.5)
    sphere = np.sqrt((p * p).sum(-1)) - 1
    sb = lipschitz(sphere, n, (0.2, 0.2, 0.2))
    assert 1.0 <= sb < 1.2, sb


def test_atlas_layout_matches_reference_tiling():
    # src/renderer.rs:778-795: gx^3 >= count, gx*gy^2 >= count, gz = ceil.
    for count in range(1, 70):
        g = (C.c_uint32 * 3)()
        e = (C.c_uint32 * 3)()
        lib.irt_atlas_layout(count, 48, g, e)
        gx = 1
        while gx ** 3 < count:
            gx += 1
        gy = 1
        while gx * gy * gy < count:
            gy += 1
        gz = -(-count // (gx * gy))
        assert tuple(g) == (gx, gy, gz)
        assert tuple(e) == (48 * gx, 48 * gy, 48 * gz)


def build_bvh(lo, hi):
    lo = np.ascontiguousarray(lo, np.float32)
    hi = np.ascontiguousarray(hi, np.float32)
    n = len(lo)
    nodes = np.zeros(2 * n - 1, L.NODE_DTYPE)
    assert lib.irt_build_hierarchy(L.ptr(lo), L.ptr(hi), n, L.ptr(nodes)) == 0
    return nodes


def reference_hierarchy(bounds):
    """Pure-Python restatement of hierarchy()'s build (src/renderer.rs:404-450)."""
    nodes = []

    def build(b):
        index = len(nodes)
        nodes.append(None)
        lo = np.min([x[1] for x in b], 0)
        hi = np.max([x[2] for x in b], 0)
        if len(b) == 1:
            meta = [b[0][0], 0, 1, 0]
        else:
            e = hi - lo
            axis = 0 if (e[0] > e[1] and e[0] > e[2]) else (1 if e[1] > e[2] else 2)
            b = sorted(b, key=lambda x: np.float32(x[1][axis] + x[2][axis]))  # stable
            m = len(b) // 2
            meta = [build(b[:m]), build(b[m:]), 0, 0]
        meta[3] = len(nodes)
        nodes[index] = (lo, hi, meta)
        return index

    build(bounds)
    return nodes


@pytest.mark.parametrize("n", [1, 2, 3, 7, 12, 24, 64])
def test_hierarchy_matches_restatement_and_escape_links(n):
    rng = np.random.default_rng(n)
    c = rng.uniform(-5, 5, (n, 3)).astype(np.float32)
    h = rng.uniform(0.1, 1, (n, 3)).astype(np.float32)
    lo, hi = c - h, c + h
    nodes = build_bvh(lo, hi)
    ref = reference_hierarchy([(i, lo[i], hi[i]) for i in range(n)])
    assert len(nodes) == 2 * n - 1 == len(ref)
    for k, (rlo, rhi, meta) in enumerate(ref):
        np.testing.assert_array_equal(nodes["lo"][k, :3], rlo)
        np.testing.assert_array_equal(nodes["hi"][k, :3], rhi)
        assert list(nodes["info"][k]) == meta
        assert meta[3] > k  # escape strictly after the node: the walk terminates
    leaves = sorted(nodes["info"][nodes["info"][:, 2] == 1][:, 0].tolist())
    assert leaves == list(range(n))


def test_pack_object_scale_and_spacing_bits():
    # objects() (src/renderer.rs:359-384): inverse, scale = |x axis|,
    # info.w = |spacing| * scale with spacing = (max - min) / (res - 1).
    m = L.Mat4()
    s, t = 1.5, (1.0, -2.0, 3.0)
    vals = [s, 0, 0, 0, 0, s, 0, 0, 0, 0, s, 0, t[0], t[1], t[2], 1]
    for i, v in enumerate(vals):
        m.m[i] = v
    out = np.zeros(1, L.OBJECT_DTYPE)
    lib.irt_pack_object(C.byref(m), C.byref(m), 3, 5, F3(-1, -1, -1), F3(1, 1, 1), 65, L.ptr(out))
    info = out["info"][0]
    assert info[0] == 3 and info[1] == 5
    assert struct.unpack("<f", struct.pack("<I", int(info[2])))[0] == np.float32(1.5)
    spacing = np.float32(2) / np.float32(64)
    expect = np.float32(np.sqrt(np.float32(3) * spacing * spacing)) * np.float32(1.5)
    assert struct.unpack("<f", struct.pack("<I", int(info[3])))[0] == pytest.approx(expect, rel=1e-6)
    inv = out["inverse"][0].reshape(4, 4)  # column-major
    model = np.array(vals, np.float64).reshape(4, 4)
    np.testing.assert_allclose(inv.T @ model.T, np.eye(4), atol=1e-6)


def test_workload_meshes_certify_boxes_and_bound_fields():
    wl = Workload(0)
    m = wl.meshes
    # 6 walls + 4 boxes certify as boxes; the 2 spheres use the field path.
    assert (m["geometry_lo"][:, 3] == 1).sum() == 10
    assert (m["geometry_lo"][:, 3] == 0).sum() == 2
    assert np.all(m["geometry_hi"][:, 3] > 0) and np.all(m["geometry_hi"][:, 3] <= 1.0)
    # exporter padding: bounds extend the vertex box by 2 voxels of its diagonal
    res = m["field"][:, 3]
    gdiag = np.linalg.norm(m["geometry_hi"][:, :3] - m["geometry_lo"][:, :3], axis=1)
    pad = gdiag / (res - 1) * 2
    np.testing.assert_allclose(m["geometry_lo"][:, :3] - m["lo"][:, :3], np.repeat(pad[:, None], 3, 1), rtol=1e-4)
    # every field tile lies inside the atlas
    dims = wl.atlas_dims
    assert np.all(m["field"][:, :3] + res[:, None] <= np.array(dims))
    wl.close()


def test_workload_frame_packing():
    wl = Workload(0)
    f0, obj, nodes, lights = wl.frame(0)
    f1, _, _, _ = wl.frame(1)
    assert tuple(f0.size) == (256, 160, 0, 1) and tuple(f1.size) == (256, 160, 1, 1)
    assert tuple(f0.counts) == (1, 100, 3, 12)
    assert tuple(f0.restir) == (8, 8, 4, 12)
    assert list(f0.flags)[:3] == [0, 0, 0] and list(f1.flags)[:3] == [1, 1, 0]
    assert tuple(f0.sdf)[:3] == (96.0, np.float32(0.001), 16.0)
    assert f0.rr[2] == 4.0 and f0.temporal[3] == 32.0
    # previous_vp of frame 1 is frame 0's vp
    assert list(f1.previous_vp.m) == list(f0.vp.m)
    assert len(nodes) == 2 * len(obj) - 1
    assert np.all(nodes["info"][:, 3] > np.arange(len(nodes)))
    assert lights["position_strength"][0, 3] == pytest.approx(5.0)  # radiance 20 x 0.5^2
    wl.close()


def test_cpu_gbuffer_and_vpls_are_sane():
    wl = Workload(0)
    f, obj, nodes, lights = wl.frame(2)
    g = wl.gbuffer_cpu(f)
    assert np.all(g["depth"] < 1) and np.all(g["depth"] > 0)  # closed room
    n = g["normal"][..., :3]
    np.testing.assert_allclose(np.linalg.norm(n, axis=-1), 1, atol=1e-5)
    assert np.all(g["params"][..., 0] == 1) and np.all(g["params"][..., 1] == 0)
    assert np.abs(g["motion"]).max() < 0.05
    v = wl.vpls_cpu(f, obj, lights)
    assert len(v) == 100
    assert np.all(np.isfinite(v["flux"]))
    alive = v["flux"][:, :3].sum(1) > 0
    assert alive.mean() > 0.3
    np.testing.assert_allclose(np.linalg.norm(v["normal"][alive, :3], axis=1), 1, atol=1e-5)
    wl.close()


def test_vpl_budget_and_power_normalization():
    # gpu_integration_vpl_budget_and_power_normalization (src/gpu_tests.rs:354-407)
    # restated for the CPU VPL generator: doubling the path budget keeps each
    # shared path and halves its flux; doubling power doubles flux.
    wl = Workload(0)
    f, obj, nodes, lights = wl.frame(0)
    base = wl.vpls_cpu(f, obj, lights)
    f.counts[1] = 200
    doubled = wl.vpls_cpu(f, obj, lights)[:100]
    np.testing.assert_array_equal(base["position"], doubled["position"])
    np.testing.assert_array_equal(base["normal"], doubled["normal"])
    np.testing.assert_allclose(base["flux"][:, :3], 2 * doubled["flux"][:, :3], atol=1e-6)
    f.counts[1] = 100
    lights2 = lights.copy()
    lights2["position_strength"][:, 3] *= 2
    power = wl.vpls_cpu(f, obj, lights2)
    np.testing.assert_array_equal(base["position"], power["position"])
    np.testing.assert_allclose(2 * base["flux"][:, :3], power["flux"][:, :3], atol=1e-6)
    assert (base["flux"][:, :3] > 0).any()
    wl.close()
