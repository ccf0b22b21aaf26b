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
    wants = []
    keep = []

    def frame(i):
        inputs = ref.inputs(i)
        f, obj, nodes, lights, planes, vpls = inputs
        ref.step(i, inputs=inputs)
        wants.append(ref.session.buffer(L.BUF_FILTERED, torch.uint8).cpu().numpy())
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

    for i in range(7):
        frame(i)
    sess.host_sync()
    torch.cuda.synchronize()
    want = wants[-1]
    # Every call's image reaches its host buffer (each is copied after the
    # next call's march, the last at irt_session_host_sync).
    for i in range(7):
        assert np.array_equal(outs[i].numpy(), wants[i]), i
    assert np.array_equal(sess.buffer(L.BUF_FILTERED, torch.uint8).cpu().numpy(), want)
    for d in (0, 1):
        assert np.array_equal(sess.reservoirs_host(d, 2).view(np.uint8), ref.session.reservoirs_host(d, 2).view(np.uint8))
    assert np.abs(outs[-1].numpy().view(np.float32)).max() > 0
    # One more call, then the session closed without irt_session_host_sync:
    # its image still arrives.
    frame(7)
    sess.close()
    assert np.array_equal(outs[7].numpy(), wants[7])
    scene.close()
    ref.close()
    ctx.close()
