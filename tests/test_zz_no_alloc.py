"""The allocation-free SVGF entry point against the session path.

Some callers cannot let a library allocate device memory (a frame thread that
must not stall on an allocation, a host that owns all device memory through
its own allocator).  irt_svgf_spatial_noalloc gives them the SVGF spatial
stages with the filter's scratch images in a fixed device array instead of a
session.  This test renders a few frames through a normal session, then feeds
that session's temporal radiance and moments to the allocation-free entry
point twice in a row and checks that the filtered and feedback images equal
the session's, within the radiance bar of the parity tests.

It lives in its own file named to be collected last, so a run that stops at
the first failure has run every other test first; it also passes alone.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from instantradiositytest_b200 import _lib as L
from instantradiositytest_b200.runtime import FrameDriver, stream_handle
from instantradiositytest_b200.workload import Workload

pytestmark = pytest.mark.gpu

RADIANCE_BAR = 1e-3  # relative L1 error, as in the parity tests


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-30))


def host_image(t: torch.Tensor, h, w, f16):
    raw = t.cpu().numpy()
    return (raw.view(np.float16).astype(np.float32) if f16 else raw.view(np.float32)).reshape(h, w, 4)


@pytest.mark.parametrize("radiance_format", [L.RADIANCE_F32, L.RADIANCE_F16])
def test_noalloc_svgf_matches_session_on_two_calls(cuda, radiance_format):
    wl = Workload(0)  # 256x160, under the 512x512 limit
    drv = FrameDriver(wl, radiance_format=radiance_format)
    for i in range(4):
        drv.step(i)
    torch.cuda.synchronize()
    s = drv.session
    f, _, _, _, _, _, gt = drv.last
    g = L.GBuffer(L.GBUFFER_F32, gt["depth"].data_ptr(), gt["normal"].data_ptr(), gt["color"].data_ptr(),
                  gt["params"].data_ptr(), gt["motion"].data_ptr())
    f16 = radiance_format == L.RADIANCE_F16
    h, w = wl.height, wl.width
    temporal_ptr, nbytes = s.buffer_ptr(L.BUF_TEMPORAL)
    moments_ptr, _ = s.buffer_ptr(L.BUF_MOMENTS)
    want_filtered = s.image_host(L.BUF_FILTERED)
    want_feedback = s.image_host(L.BUF_FEEDBACK)
    for call in range(2):
        filtered = torch.full((nbytes,), 0x7F, dtype=torch.uint8, device="cuda")
        feedback = torch.full((nbytes,), 0x7F, dtype=torch.uint8, device="cuda")
        err = C.create_string_buffer(256)
        st = L.lib.irt_svgf_spatial_noalloc(C.byref(f), C.byref(g), radiance_format,
                                            wl.settings.svgf_iterations, temporal_ptr, moments_ptr,
                                            filtered.data_ptr(), feedback.data_ptr(), stream_handle(), err, 256)
        assert st == L.IRT_OK, err.value.decode()
        torch.cuda.synchronize()
        got_f = host_image(filtered, h, w, f16)
        got_b = host_image(feedback, h, w, f16)
        assert np.all(np.isfinite(got_f))
        assert rel_l1(got_f[..., :3], want_filtered[..., :3]) <= RADIANCE_BAR, call
        assert rel_l1(got_b[..., :3], want_feedback[..., :3]) <= RADIANCE_BAR, call
        assert rel_l1(got_f[..., 3], want_filtered[..., 3]) <= RADIANCE_BAR, call
    drv.close()


def test_noalloc_rejects_frames_above_its_limit(cuda):
    f = L.Frame()
    f.size[0], f.size[1] = 1024, 1024
    dummy = torch.zeros(16, dtype=torch.uint8, device="cuda")
    p = dummy.data_ptr()
    g = L.GBuffer(L.GBUFFER_F32, p, p, p, p, p)
    err = C.create_string_buffer(256)
    st = L.lib.irt_svgf_spatial_noalloc(C.byref(f), C.byref(g), L.RADIANCE_F32, 4, p, p, p, p, stream_handle(),
                                        err, 256)
    assert st == L.IRT_E_INVALID
    assert "262144" in err.value.decode()
