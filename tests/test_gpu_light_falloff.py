"""Direct lighting falloff and the spot cone (src/gpu_tests.rs:281-317 on the
exported analytic cube, here on the procedural room): a point light on the
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
