"""irt_render_frame_host (host G-buffer and VPL pool in, filtered image out,
copies pipelined with rendering) gives exactly the results of
irt_render_frame on the same inputs placed on the device."""
import numpy as np
import pytest
import torch

from instantradiositytest_b200 import _lib as L
from instantradiositytest_b200.runtime import Context, FrameDriver, Scene, Session, session_desc
from instantradiositytest_b200.workload import Workload

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("gfmt", [L.GBUFFER_F32, L.GBUFFER_PACKED])
def test_host_inputs_equal_device_inputs(cuda, gfmt):
    wl = Workload(0, width=160, height=100)
    ctx = Context()
    ref = FrameDriver(wl, ctx=ctx, gbuffer_format=gfmt)
    scene = Scene(ctx, wl.meshes, wl.atlas, wl.sdf_format)
    sess = Session(ctx, session_desc(wl.settings, gfmt))
    outs = []
    keep = []
    for i in range(7):
        inputs = ref.inputs(i)
        f, obj, nodes, lights, planes, vpls = inputs
        ref.step(i, inputs=inputs)
        g = {k: torch.from_numpy(np.ascontiguousarray(v).view(np.uint8).reshape(-1)).pin_memory()
             for k, v in planes.items()}
        hg = L.GBuffer(gfmt, g["depth"].data_ptr(), g["normal"].data_ptr(), g["color"].data_ptr(),
                       g["params"].data_ptr(), g["motion"].data_ptr())
        hv = torch.from_numpy(vpls.view(np.uint8)).pin_memory()
        out = torch.zeros(sess.buffer_ptr(L.BUF_FILTERED)[1], dtype=torch.uint8).pin_memory()
        scene.update(obj, nodes, lights)
        sess.render_host(scene, f, hg, hv, out)
        keep.append((g, hv))  # host inputs must outlive their copies
        outs.append(out)
    sess.host_sync()
    torch.cuda.synchronize()
    want = ref.session.buffer(L.BUF_FILTERED, torch.uint8).cpu().numpy()
    assert np.array_equal(outs[-1].numpy(), want)
    assert np.array_equal(sess.buffer(L.BUF_FILTERED, torch.uint8).cpu().numpy(), want)
    for d in (0, 1):
        assert np.array_equal(sess.reservoirs_host(d, 2).view(np.uint8), ref.session.reservoirs_host(d, 2).view(np.uint8))
    assert np.abs(outs[-1].numpy().view(np.float32)).max() > 0
    sess.close()
    scene.close()
    ref.close()
    ctx.close()
