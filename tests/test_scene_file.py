"""Scene-format loader (Workload.load -> irt_workload_load): Scene::load and
Scene::validate of src/scene.rs:157-382, restating the reference's unit tests
(src/scene.rs:392-493: scalar-scale transforms, binary ranges, camera depth
round trip, validation diagnostics) on scene files written by
instantradiositytest_b200.scene_file, plus the loaded workload's host data
(mesh rows, atlas tiles, objects, lights, camera) and its CPU producers."""
import copy
import json
import math
import os
import shutil

import numpy as np
import pytest

from instantradiositytest_b200 import _lib as L
from instantradiositytest_b200 import scene_file as sf
from instantradiositytest_b200.workload import SceneLoadError, Workload

# The reference's shipped assets/test_scene/scene.json, where a copy is at hand.
SHIPPED = os.environ.get("IRT_TEST_SCENE", "")


@pytest.fixture(scope="module")
def demo(tmp_path_factory):
    d = tmp_path_factory.mktemp("demo")
    return sf.write_scene(str(d), sf.demo_scene(resolution=16))


def load(path, **kw):
    kw.setdefault("width", 96)
    kw.setdefault("height", 64)
    kw.setdefault("vpl_count", 64)
    return Workload.load(path, **kw)


def mutated(tmp_path, manifest_path, edit):
    """Copy of the scene with its manifest edited by `edit(doc)`."""
    src = os.path.dirname(manifest_path)
    dst = tmp_path / "scene"
    shutil.copytree(src, dst)
    doc = json.load(open(manifest_path))
    edit(doc)
    with open(dst / "scene.json", "w") as f:
        json.dump(doc, f)
    return str(dst / "scene.json")


def error_of(path):
    with pytest.raises(SceneLoadError) as e:
        load(path)
    return str(e.value)


# ------------------------------------------------------------------ writer
def test_writer_meshes_face_outward():
    for m in (sf.box("b", (-1, -2, -3), (1, 2, 3)), sf.uv_sphere("s", 0.7), sf.torus("t", 0.6, 0.2)):
        v = m.vertices[:, :3].astype(np.float64)
        n = m.vertices[:, 4:7].astype(np.float64)
        tri = m.indices.reshape(-1, 3)
        g = np.cross(v[tri[:, 1]] - v[tri[:, 0]], v[tri[:, 2]] - v[tri[:, 0]])
        area = np.linalg.norm(g, axis=1)
        ok = area > 1e-9
        assert ok.mean() > 0.9
        assert (np.einsum("ij,ij->i", g[ok], n[tri[ok, 0]]) > 0).all(), m.id


# ------------------------------------------------------------------ load
def test_load_round_trips_meshes_atlas_objects_lights_camera(demo):
    doc = json.load(open(demo))
    wl = load(demo)
    assert (wl.mesh_count, wl.object_count, wl.light_count) == (5, 6, 2)
    # atlas tiles of the largest resolution (src/renderer.rs:778-795)
    assert wl.atlas_dims == (32, 32, 32)
    fields = np.fromfile(os.path.join(os.path.dirname(demo), doc["meshes"][0]["sdf"]["path"]), "<f4")
    for i, m in enumerate(doc["meshes"]):
        r = m["sdf"]["resolution"]
        x, y, z, res = (int(v) for v in wl.meshes[i]["field"])
        assert res == r
        tile = wl.atlas[z:z + r, y:y + r, x:x + r].reshape(-1)
        want = fields[m["sdf"]["offset"] // 4:m["sdf"]["offset"] // 4 + r ** 3]
        np.testing.assert_array_equal(tile, want)
        np.testing.assert_array_equal(wl.meshes[i]["lo"][:3], np.float32(m["sdf"]["bounds_min"]))
        np.testing.assert_array_equal(wl.meshes[i]["hi"][:3], np.float32(m["sdf"]["bounds_max"]))
    # the three box meshes are certified boxes, the curved ones are not
    assert [float(m["geometry_lo"][3]) for m in wl.meshes] == [1.0, 1.0, 1.0, 0.0, 0.0]
    f, objects, nodes, lights = wl.frame(0)
    # objects in manifest order with their mesh and material indices
    mesh_ix = {m["id"]: i for i, m in enumerate(doc["meshes"])}
    mat_ix = {m["id"]: i for i, m in enumerate(doc["materials"])}
    for i, o in enumerate(doc["objects"]):
        assert objects["info"][i][0] == mesh_ix[o["mesh"]]
        assert objects["info"][i][1] == mat_ix[o["material"]]
        model = objects["model"][i].reshape(4, 4)  # column-major rows = columns
        np.testing.assert_allclose(model[3, :3], o["transform"]["position"], atol=1e-6)
        s = o["transform"]["scale"]
        np.testing.assert_allclose(np.linalg.norm(model[:3, :3], axis=1), [s] * 3, rtol=1e-6)
    # lights (src/renderer.rs:1747-1755)
    spot = doc["lights"][1]
    np.testing.assert_array_equal(lights["position_strength"][1], np.float32(spot["position"] + [spot["strength"]]))
    np.testing.assert_array_equal(lights["direction_angle"][1],
                                  np.float32(spot["direction"] + [spot["angle_radians"]]))
    assert lights["color_type"][1][3] == 1.0 and lights["color_type"][0][3] == 0.0
    np.testing.assert_array_equal(lights["direction_angle"][0], np.zeros(4, np.float32))
    # fixed camera
    np.testing.assert_allclose(np.float32(f.camera[:3]), doc["camera"]["position"], atol=1e-6)
    f1 = wl.frame(5)[0]
    assert list(f1.vp.m) == list(f.vp.m) and list(f1.previous_vp.m) == list(f.vp.m)
    assert (f.counts[0], f.counts[1], f.counts[3]) == (2, 64, 6)


def test_camera_depth_reconstruction_round_trip(demo):
    # src/scene.rs:429-444: a point in front of the camera projects and
    # unprojects to itself through the frame's vp / inv_vp.
    doc = json.load(open(demo))
    wl = load(demo, width=160, height=100)
    f = wl.frame(0)[0]
    vp = np.array(f.vp.m, np.float64).reshape(4, 4).T
    inv = np.array(f.inv_vp.m, np.float64).reshape(4, 4).T
    c = doc["camera"]
    x, y, z, w = c["rotation"]
    R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                  [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                  [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
    p = np.array(c["position"]) + R @ np.array([0.2, 0.1, -4.0])
    h = vp @ np.append(p, 1.0)
    ndc = h / h[3]
    assert 0 < ndc[2] < 1 and abs(ndc[0]) < 1 and abs(ndc[1]) < 1
    back = inv @ ndc
    assert np.linalg.norm(back[:3] / back[3] - p) < 1e-4


def test_cpu_gbuffer_and_vpls_of_a_loaded_scene(demo):
    doc = json.load(open(demo))
    wl = load(demo, width=160, height=100, vpl_count=256)
    f, objects, nodes, lights = wl.frame(0)
    g = wl.gbuffer_cpu(f)
    hit = g["depth"] < 1
    assert hit.mean() > 0.5
    n = g["normal"][..., :3][hit]
    np.testing.assert_allclose(np.linalg.norm(n, axis=-1), 1.0, atol=1e-5)
    colors = {tuple(np.float32(m["base_color"][:3])) for m in doc["materials"]}
    seen = {tuple(c) for c in np.unique(g["color"][..., :3][hit], axis=0)}
    assert seen <= colors and len(seen) >= 4
    # back faces are culled: every visible normal faces the camera
    cam = np.array(f.camera[:3], np.float64)
    H, W = g["depth"].shape
    ys, xs = np.nonzero(hit)
    inv = np.array(f.inv_vp.m, np.float64).reshape(4, 4).T
    ndc = np.stack([(xs + .5) / W * 2 - 1, 1 - (ys + .5) / H * 2, g["depth"][hit], np.ones(len(xs))], 0)
    wp = inv @ ndc
    wp = (wp[:3] / wp[3]).T
    assert (np.einsum("ij,ij->i", n, cam - wp) > 0).mean() > 0.999
    v = wl.vpls_cpu(f, objects, lights)
    alive = np.abs(v["flux"][:, :3]).sum(1) > 0
    assert 0.2 < alive.mean() <= 1.0
    np.testing.assert_allclose(np.linalg.norm(v["normal"][alive, :3], axis=1), 1.0, atol=1e-4)


def test_f16_atlas_of_a_loaded_scene(demo):
    a = load(demo)
    b = load(demo, sdf_format=L.SDF_F16)
    da = a.atlas_f32()
    db = b.atlas_f32()
    assert (db <= da).all()
    for m in b.meshes:
        assert m["lo"][3] == m["grid"][3]
    # rounded down by less than one f16 ulp of value / scale
    assert (da - db <= np.abs(da) * 2.0 ** -10 + 1e-6).all()


# ------------------------------------------------------------------ diagnostics
def test_transform_scalar_scale_validates(tmp_path, demo):
    # src/scene.rs:395-420
    p = mutated(tmp_path, demo, lambda d: d["objects"][0]["transform"].update(scale=-1.0))
    assert "object floor: scale must be a positive finite uniform scalar" in error_of(p)


def test_transform_rejects_vector_scale_and_unknown_fields(tmp_path, demo):
    p = mutated(tmp_path, demo, lambda d: d["objects"][0]["transform"].update(scale=[1, 2, 1]))
    assert error_of(p).startswith("parsing ")
    shutil.rmtree(tmp_path / "scene")
    p = mutated(tmp_path, demo, lambda d: d["objects"][0]["transform"].update(shear=1.0))
    assert "unknown field `shear`" in error_of(p)


def _geometry(d, **kw):
    d["meshes"][0]["geometry"].update(kw)


@pytest.mark.parametrize("edit,needle", [
    (lambda d: _geometry(d, vertex_offset=10 ** 9), "binary range ["),
    (lambda d: _geometry(d, vertex_offset=2 ** 64 - 1), "binary range overflow"),
    (lambda d: _geometry(d, index_count=35), "geometry must have triangles"),
    (lambda d: d["meshes"][0]["sdf"].update(offset=10 ** 8), "exceeds"),
])
def test_binary_ranges_reject_overflow_and_oob(tmp_path, demo, edit, needle):
    # src/scene.rs:421-428 through the per-mesh loads
    msg = error_of(mutated(tmp_path, demo, edit))
    assert msg.startswith("mesh floor_box: ") and needle in msg


def _obj(i, **kw):
    return lambda d: d["objects"][i].update(kw)


@pytest.mark.parametrize("edit,needle", [
    (lambda d: d.update(version=2), "unsupported scene version 2"),
    (lambda d: d["meshes"][1].update(id="floor_box"), "duplicate/empty mesh ID: floor_box"),
    (lambda d: d["materials"][1].update(id=""), "duplicate/empty material ID"),
    (lambda d: d["objects"][1].update(id=d["objects"][0]["id"]), "duplicate/empty object/light ID: floor"),
    (lambda d: d["lights"][0].update(id="floor"), "duplicate/empty object/light ID: floor"),
    (lambda d: d.update(objects=[]), "scene has no objects"),
    (lambda d: d["meshes"][0]["sdf"].update(resolution=3), "mesh floor_box: invalid SDF bounds/resolution"),
    (lambda d: d["meshes"][0]["sdf"].update(bounds_max=d["meshes"][0]["sdf"]["bounds_min"]),
     "invalid SDF bounds/resolution"),
    (lambda d: d["meshes"][0]["sdf"].update(conservative=False), "conservative"),
    (lambda d: d["meshes"][0]["sdf"].update(query="nearest"), "SDF must be conservative with trilinear_bound query"),
    (lambda d: d["meshes"][0]["sdf"].update(error_bound=-1.0), "trilinear_bound"),
    (lambda d: d["materials"][0].update(roughness=1e39), "material white: invalid PBR values"),
    (lambda d: d["materials"][0].update(metallic=1.5), "material white: invalid PBR values"),
    (lambda d: d["materials"][0].update(base_color=[1, -0.5, 0, 1]), "invalid PBR values"),
    (lambda d: d["materials"][0].update(texture_channels=[0, 4, 0, 0]), "material white: invalid texture settings"),
    (lambda d: d["materials"][0].update(normal_strength=-1.0), "invalid texture settings"),
    (lambda d: d["materials"][0].update(base_color_texture="missing.png"), "material white: missing texture missing.png"),
    (_obj(0, mesh="missing_mesh"), "object floor: missing mesh missing_mesh"),
    (_obj(0, material="nope"), "object floor: missing material nope"),
    (lambda d: d["objects"][0]["transform"].update(rotation=[0, 0, 0, 0]), "object floor: invalid position/quaternion"),
    (lambda d: d["lights"][0].update(strength=-1.0), "light lamp: invalid values"),
    (lambda d: d["lights"][0].update(color=[1, -1, 1]), "light lamp: invalid values"),
    (lambda d: d["lights"][0].update(type="area"), "light lamp: unsupported type area"),
    (lambda d: d["lights"][0].update(type="spot", direction=[0, 0, 0]), "spot"),
    (lambda d: d["lights"][1].update(angle_radians=3.2), "light spot: invalid spot cone/direction"),
    (lambda d: d["camera"].update(fov_y_radians=3.2), "invalid camera"),
    (lambda d: d["camera"].update(far=0.05), "invalid camera"),
    (lambda d: d["camera"].update(rotation=[3.4e38] * 4), "invalid camera"),
])
def test_validation_rejects_invalid_entities_with_diagnostics(tmp_path, demo, edit, needle):
    # src/scene.rs:445-493 and the remaining ensure! rules of Scene::validate
    msg = error_of(mutated(tmp_path, demo, edit))
    assert msg.startswith("scene ") and needle in msg, msg


def test_missing_fields_types_and_syntax(tmp_path, demo):
    p = mutated(tmp_path, demo, lambda d: d["meshes"][0]["sdf"].pop("resolution"))
    assert "missing field `resolution`" in error_of(p) and error_of(p).startswith("parsing ")
    shutil.rmtree(tmp_path / "scene")
    p = mutated(tmp_path, demo, lambda d: d["meshes"][0]["geometry"].update(vertex_count=-4))
    assert error_of(p).startswith("parsing ")
    with open(p, "a") as f:
        f.write("}")
    assert "trailing characters" in error_of(p)
    assert error_of(str(tmp_path / "none.json")).startswith("reading ")


def test_json_strings_duplicates_and_nesting(tmp_path, demo):
    # \u escapes (json.dump writes the e-acute as one) decode to the id the
    # diagnostics print, and an escaped backslash stays one backslash
    p = mutated(tmp_path, demo, lambda d: d["objects"][0].update(mesh="caf\u00e9\\x"))
    assert "\\u00e9" in open(p).read()
    assert "missing mesh caf\u00e9\\x" in error_of(p)
    # a key given twice and nesting deeper than serde_json's 128 levels are syntax errors
    txt = open(demo).read()
    dup = tmp_path / "dup.json"
    dup.write_text(txt.replace('"version": 1,', '"version": 1, "version": 1,', 1))
    assert "duplicate field `version`" in error_of(str(dup))
    deep = tmp_path / "deep.json"
    deep.write_text(txt.replace('"version": 1,', '"version": 1, "x": ' + "[" * 200 + "]" * 200 + ",", 1))
    assert "recursion limit" in error_of(str(deep))


def test_defaults_and_unknown_fields_are_accepted(tmp_path, demo):
    def edit(d):
        for m in d["materials"]:
            for k in ("base_color_srgb", "normal_strength", "texture_channels"):
                m.pop(k, None)
            m["base_color_texture"] = None
        d["lights"][0].pop("direction", None)
        d["extra"] = {"note": "ignored"}
        d["meshes"][0]["comment"] = "ignored"
    wl = load(mutated(tmp_path, demo, edit))
    assert wl.object_count == 6


def test_bad_binary_contents(tmp_path, demo):
    doc = json.load(open(demo))
    g = doc["meshes"][0]["geometry"]
    geo_path = os.path.join(os.path.dirname(demo), g["path"])

    def corrupt(offset, raw):
        d = tmp_path / f"c{offset}"
        shutil.copytree(os.path.dirname(demo), d)
        b = bytearray(open(geo_path, "rb").read())
        b[offset:offset + len(raw)] = raw
        open(d / g["path"], "wb").write(bytes(b))
        return error_of(str(d / "scene.json"))

    assert "mesh floor_box: index outside vertex range" in corrupt(g["index_offset"], np.uint32(10 ** 6).tobytes())
    assert "mesh floor_box: nonfinite vertex" in corrupt(g["vertex_offset"] + 8, np.float32(np.nan).tobytes())
    s = doc["meshes"][0]["sdf"]
    d = tmp_path / "sdf"
    shutil.copytree(os.path.dirname(demo), d)
    b = bytearray(open(os.path.join(os.path.dirname(demo), s["path"]), "rb").read())
    b[s["offset"]:s["offset"] + 4] = np.float32(np.inf).tobytes()
    open(d / s["path"], "wb").write(bytes(b))
    assert "mesh floor_box: nonfinite SDF" in error_of(str(d / "scene.json"))


def test_textured_materials_are_refused_after_validation(tmp_path, demo):
    def edit(d):
        d["materials"][0]["roughness_texture"] = "rough.png"
    p = mutated(tmp_path, demo, edit)
    open(os.path.join(os.path.dirname(p), "rough.png"), "wb").write(b"\x89PNG")
    assert "textures are not supported" in error_of(p)


# ------------------------------------------------------------------ shipped scene
@pytest.mark.skipif(not (SHIPPED and os.path.exists(SHIPPED)), reason="IRT_TEST_SCENE not set")
def test_shipped_test_scene_loads():
    wl = load(SHIPPED, width=160, height=100, vpl_count=256)
    assert (wl.mesh_count, wl.object_count, wl.light_count) == (7, 7, 2)
    assert all(int(m["field"][3]) == 48 for m in wl.meshes)
    # is_box_geometry compares corners exactly (src/renderer.rs:287-329):
    # Cube.001 and Cube.002 are certified boxes; Cube.003 has one z of
    # -0.27145106 against -0.27145088 elsewhere and stays a field mesh.
    assert [float(m["geometry_lo"][3]) for m in wl.meshes] == [0.0] * 4 + [1.0, 1.0, 0.0]
    f, objects, nodes, lights = wl.frame(0)
    g = wl.gbuffer_cpu(f)
    assert (g["depth"] < 1).mean() > 0.9
    v = wl.vpls_cpu(f, objects, lights)
    assert (np.abs(v["flux"][:, :3]).sum(1) > 0).mean() > 0.1
