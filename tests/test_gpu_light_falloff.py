"""Direct lighting falloff, the spot cone and a moving occluder
(src/gpu_tests.rs:281-352) on the reference's exported cube fixture,
recreated as a scene file, and on the procedural room: a point light on the
normal of the surface seen at the image centre, at 1 and at 2.5 units (the
reference's 2 and 5 would leave the room), gives radiance in the ratio 25/4; a spot of half-angle 0.2 rad aimed at the point
gives the point light's radiance, aimed away gives zero."""
import ctypes as C

import numpy as np
import pytest
import torch

from instantradiositytest_b200 import _lib as L
from instantradiositytest_b200.runtime import Context, Scene, Session, gbuffer_to_device, session_desc, vpls_to_device
from instantradiositytest_b200.workload import Workload

pytestmark = pytest.mark.gpu


def centre_radiance(ctx, wl, f, obj, nodes, light, planes):
    """A fresh session renders one frame with only `light`, debug view 1
    (direct light), and returns the direct radiance at the centre pixel."""
    f = L.Frame.from_buffer_copy(f)
    f.counts[0] = 1
    f.flags[2] = 1
    lights = np.zeros(1, L.LIGHT_DTYPE)
    lights[0] = light
    scene = Scene(ctx, wl.meshes, wl.atlas, wl.sdf_format)
    scene.update(obj, nodes, lights)
    sess = Session(ctx, session_desc(wl.settings))
    gt, gs = gbuffer_to_device(planes, L.GBUFFER_F32)
    v = vpls_to_device(wl.vpls_cpu(f, obj, lights))
    sess.render(scene, f, gs, C.c_void_p(v.data_ptr()), C.c_void_p(v.data_ptr()))
    torch.cuda.synchronize()
    img = sess.image_host(L.BUF_DIRECT)
    sess.close()
    scene.close()
    h, w = img.shape[:2]
    return float(img[h // 2, w // 2, :3].mean())


def test_inverse_square_and_spot_cone(cuda):
    wl = Workload(0, width=64, height=64)
    ctx = Context()
    f, obj, nodes, lights = wl.frame(0)
    planes = wl.gbuffer_cpu(f, L.GBUFFER_F32)
    c = planes["depth"].shape[0] // 2, planes["depth"].shape[1] // 2
    assert planes["depth"][c] < 1.0
    # world position of the centre pixel from depth (the kernels' world())
    inv = np.array(f.inv_vp.m, np.float64).reshape(4, 4).T
    u, v = (c[1] + 0.5) / 64, (c[0] + 0.5) / 64
    hp = inv @ np.array([u * 2 - 1, 1 - v * 2, planes["depth"][c], 1.0])
    p = hp[:3] / hp[3]
    n = planes["normal"][c][:3].astype(np.float64)
    n /= np.linalg.norm(n)

    def light(dist, spot=False, toward=True, strength=5.0):
        rec = np.zeros((), L.LIGHT_DTYPE)
        pos = p + n * dist
        rec["position_strength"] = (*pos, strength)
        d = -n if toward else n
        rec["direction_angle"] = (*d, 0.4)
        rec["color_type"] = (1.0, 1.0, 1.0, 1.0 if spot else 0.0)
        return rec

    near = centre_radiance(ctx, wl, f, obj, nodes, light(1.0), planes)
    far = centre_radiance(ctx, wl, f, obj, nodes, light(2.5), planes)
    print("near", near, "far", far, "ratio", near / far)
    assert near > 0
    assert abs(near / far - 6.25) < 0.05
    spot_in = centre_radiance(ctx, wl, f, obj, nodes, light(2.5, spot=True), planes)
    assert abs(spot_in - far) < 0.002 * max(1.0, far)
    spot_out = centre_radiance(ctx, wl, f, obj, nodes, light(2.5, spot=True, toward=False), planes)
    assert spot_out == 0.0
    ctx.close()


def test_inverse_square_and_spot_cone_on_the_cube_fixture(cuda, tmp_path):
    """src/gpu_tests.rs:281-317 on its own fixture, recreated as a scene file
    and loaded through Workload.load: the exporter's cube (a 2 m box at the
    origin, tools/test_export.py), camera at (0, 0, 5) looking down -z, a
    point light at (0, 0, 3) then (0, 0, 6) — 2 and 5 m from the lit face —
    then a spot of angle 0.4 aimed down, then up; 64x64, direct light."""
    from instantradiositytest_b200 import scene_file as sf

    sc = sf.Scene()
    sc.meshes = [sf.box("Cube", (-1, -1, -1), (1, 1, 1), resolution=16)]
    sc.materials = [sf.material("Material", (0.8, 0.8, 0.8), 0.5, 0.0)]
    sc.objects = [sf.obj("Cube", "Cube", "Material")]
    sc.lights = [sf.point_light("Light", (0, 0, 3), (1, 1, 1), 10.0)]
    sc.camera = {"position": [0.0, 0.0, 5.0], "rotation": [0.0, 0.0, 0.0, 1.0], "fov_y_radians": 0.6911,
                 "near": 0.1, "far": 100.0}
    wl = Workload.load(sf.write_scene(str(tmp_path), sc), width=64, height=64, vpl_count=100)
    ctx = Context()
    f, obj, nodes, lights = wl.frame(0)
    planes = wl.gbuffer_cpu(f, L.GBUFFER_F32)
    assert planes["depth"][32, 32] < 1.0 and planes["normal"][32, 32][2] > 0.99  # the top face

    def light(z, spot=False, down=True):
        rec = np.zeros((), L.LIGHT_DTYPE)
        rec[...] = lights[0]
        rec["position_strength"] = (0.0, 0.0, z, float(lights[0]["position_strength"][3]))
        if spot:
            rec["direction_angle"] = (0.0, 0.0, -1.0 if down else 1.0, 0.4)
            rec["color_type"][3] = 1.0
        return rec

    near = centre_radiance(ctx, wl, f, obj, nodes, light(3.0), planes)
    far = centre_radiance(ctx, wl, f, obj, nodes, light(6.0), planes)
    print("cube fixture: near", near, "far", far, "ratio", near / far)
    assert near > 0
    assert abs(near / far - 6.25) < 0.05, "distance 2 versus 5 must attenuate by 25/4"
    assert abs(centre_radiance(ctx, wl, f, obj, nodes, light(6.0, spot=True), planes) - far) < 0.002
    assert centre_radiance(ctx, wl, f, obj, nodes, light(6.0, spot=True, down=False), planes) == 0.0
    ctx.close()


def _world_aabb(model16, lo, hi):
    """World AABB of the SDF-bounds corners under a column-major model (f32,
    the arithmetic of Workload::frame_data / src/renderer.rs:388-400)."""
    m = np.asarray(model16, np.float32)
    pts = []
    for c in range(8):
        p = [hi[0] if c & 1 else lo[0], hi[1] if c & 2 else lo[1], hi[2] if c & 4 else lo[2]]
        pts.append([np.float32(m[a] * np.float32(p[0]) + m[4 + a] * np.float32(p[1]) + m[8 + a] * np.float32(p[2]) +
                               m[12 + a]) for a in range(3)])
    pts = np.array(pts, np.float32)
    return pts.min(0), pts.max(0)


def _moved(wl, obj, k, scale, pos):
    """The objects with object k placed at `pos` with uniform `scale` (no
    rotation), packed as objects() does, and the rebuilt hierarchy."""
    mesh, material = int(obj["info"][k, 0]), int(obj["info"][k, 1])
    lo, hi = wl.meshes[mesh]["lo"][:3].copy(), wl.meshes[mesh]["hi"][:3].copy()
    model = L.Mat4()
    vals = [scale, 0, 0, 0, 0, scale, 0, 0, 0, 0, scale, 0, pos[0], pos[1], pos[2], 1.0]
    for i, x in enumerate(vals):
        model.m[i] = x
    moved = obj.copy()
    rec = np.zeros(1, L.OBJECT_DTYPE)
    L.lib.irt_pack_object(C.byref(model), C.byref(model), mesh, material, (C.c_float * 3)(*lo), (C.c_float * 3)(*hi),
                          int(wl.meshes[mesh]["field"][3]), L.ptr(rec))
    moved[k] = rec[0]
    los, his = [], []
    for i in range(len(moved)):
        mi = int(moved["info"][i, 0])
        a, b = _world_aabb(moved["model"][i], wl.meshes[mi]["lo"][:3], wl.meshes[mi]["hi"][:3])
        los.append(a)
        his.append(b)
    los = np.ascontiguousarray(np.array(los, np.float32))
    his = np.ascontiguousarray(np.array(his, np.float32))
    new_nodes = np.zeros(2 * len(moved) - 1, L.NODE_DTYPE)
    assert L.lib.irt_build_hierarchy(L.ptr(los), L.ptr(his), len(moved), L.ptr(new_nodes)) == L.IRT_OK
    return moved, new_nodes


def test_moving_occluder_on_the_cube_fixture(cuda, tmp_path):
    """src/gpu_tests.rs:319-352 on its fixture, recreated as a scene file: a
    copy of the cube scaled by 0.25 at (20, 0, 2), the point light at
    (3, 0, 3); moving the copy to (1.5, 0, 2), into the light ray of the
    centre pixel, makes it dark."""
    from instantradiositytest_b200 import scene_file as sf

    sc = sf.Scene()
    sc.meshes = [sf.box("Cube", (-1, -1, -1), (1, 1, 1), resolution=16)]
    sc.materials = [sf.material("Material", (0.8, 0.8, 0.8), 0.5, 0.0)]
    sc.objects = [sf.obj("Cube", "Cube", "Material"),
                  sf.obj("moving_occluder", "Cube", "Material", (20.0, 0.0, 2.0), scale=0.25)]
    sc.lights = [sf.point_light("Light", (3, 0, 3), (1, 1, 1), 10.0)]
    sc.camera = {"position": [0.0, 0.0, 5.0], "rotation": [0.0, 0.0, 0.0, 1.0], "fov_y_radians": 0.6911,
                 "near": 0.1, "far": 100.0}
    wl = Workload.load(sf.write_scene(str(tmp_path), sc), width=64, height=64, vpl_count=100, vpl_bounces=1)
    ctx = Context()
    f, obj, nodes, lights = wl.frame(0)
    planes = wl.gbuffer_cpu(f, L.GBUFFER_F32)
    lit = centre_radiance(ctx, wl, f, obj, nodes, lights[0], planes)
    assert lit > 0.001
    moved, new_nodes = _moved(wl, obj, 1, 0.25, (1.5, 0.0, 2.0))
    dark = centre_radiance(ctx, wl, f, moved, new_nodes, lights[0], planes)
    print("cube fixture: lit", lit, "occluded", dark)
    assert dark == 0.0, "moving a uniformly scaled occluder into the light ray must update the SDF hierarchy"
    ctx.close()


def test_moving_occluder_updates_the_hierarchy(cuda):
    """src/gpu_tests.rs:319-352: moving a uniformly scaled object into the
    light ray darkens the point — the BVH, the march records and the
    leaf-order cache follow the objects."""
    wl = Workload(0, width=64, height=64)
    ctx = Context()
    f, obj, nodes, lights = wl.frame(0)
    planes = wl.gbuffer_cpu(f, L.GBUFFER_F32)
    inv = np.array(f.inv_vp.m, np.float64).reshape(4, 4).T
    hp = inv @ np.array([(32 + 0.5) / 64 * 2 - 1, 1 - (32 + 0.5) / 64 * 2, planes["depth"][32, 32], 1.0])
    p = hp[:3] / hp[3]
    n = planes["normal"][32, 32][:3].astype(np.float64)
    n /= np.linalg.norm(n)
    light = np.zeros((), L.LIGHT_DTYPE)
    light["position_strength"] = (*(p + n * 2.5), 5.0)
    light["color_type"] = (1.0, 1.0, 1.0, 0.0)
    lit = centre_radiance(ctx, wl, f, obj, nodes, light, planes)
    assert lit > 0
    # move the last object (a sphere) to the middle of the ray, scaled by 0.25
    moved, new_nodes = _moved(wl, obj, len(obj) - 1, 0.25, p + n * 1.25)
    dark = centre_radiance(ctx, wl, f, moved, new_nodes, light, planes)
    print("lit", lit, "occluded", dark)
    assert dark == 0.0
    ctx.close()
