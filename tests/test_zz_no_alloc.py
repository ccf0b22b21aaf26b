"""The allocation-free SVGF entry point against the session path.

Some callers cannot let a library allocate device memory (a frame thread that
must not stall on an allocation, a host that owns all device memory through
its own allocator).  irt_svgf_spatial_noalloc gives them the SVGF spatial
stages with the filter's working images in a fixed device array instead of a
session.  This test renders a few frames through a normal session, then feeds
that session's temporal radiance and moments — in the session's own radiance,
moments and G-buffer formats — to the allocation-free entry point several
times in a row and checks that the filtered and feedback images equal the
session's bit for bit (the same kernels on the same inputs), also with one or
four a-trous passes and without a feedback image.

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

# (G-buffer, radiance, moments, a-trous passes): the f32 formats, the
# reference's own formats, the mixed-precision storage, and single-pass
# filters (the first pass writes the filtered and feedback images at once).
CASES = [
    (L.GBUFFER_F32, L.RADIANCE_F32, L.MOMENTS_F32, 4),
    (L.GBUFFER_F16, L.RADIANCE_F16, L.MOMENTS_F32, 4),
    (L.GBUFFER_PACKED, L.RADIANCE_F16, L.MOMENTS_F16, 4),
    (L.GBUFFER_PACKED, L.RADIANCE_F32, L.MOMENTS_F16, 1),
    (L.GBUFFER_F32, L.RADIANCE_F16, L.MOMENTS_F16, 1),
]


def call(f, g, rfmt, mfmt, iters, temporal, moments, filtered, feedback):
    err = C.create_string_buffer(256)
    st = L.lib.irt_svgf_spatial_noalloc(C.byref(f), C.byref(g), rfmt, mfmt, iters, temporal, moments, filtered,
                                        feedback, stream_handle(), err, 256)
    return st, err.value.decode()


@pytest.mark.parametrize("gfmt,rfmt,mfmt,iters", CASES)
def test_noalloc_svgf_equals_session_on_calls_in_a_row(cuda, gfmt, rfmt, mfmt, iters):
    wl = Workload(0)  # 256x160, under the 512x512 limit
    wl.settings.svgf_iterations = iters
    drv = FrameDriver(wl, gbuffer_format=gfmt, radiance_format=rfmt, moments_format=mfmt)
    for i in range(4):
        drv.step(i)
    torch.cuda.synchronize()
    s = drv.session
    f, _, _, _, _, _, gt = drv.last
    g = L.GBuffer(gfmt, gt["depth"].data_ptr(), gt["normal"].data_ptr(), gt["color"].data_ptr(),
                  gt["params"].data_ptr(), gt["motion"].data_ptr())
    temporal_ptr, nbytes = s.buffer_ptr(L.BUF_TEMPORAL)
    moments_ptr, mbytes = s.buffer_ptr(L.BUF_MOMENTS)
    assert mbytes == wl.width * wl.height * (8 if mfmt == L.MOMENTS_F16 else 16)
    want_filtered = s.buffer(L.BUF_FILTERED, torch.uint8).cpu().numpy()
    want_feedback = s.buffer(L.BUF_FEEDBACK, torch.uint8).cpu().numpy()
    for k in range(3):
        filtered = torch.full((nbytes,), 0x7F, dtype=torch.uint8, device="cuda")
        feedback = torch.full((nbytes,), 0x7F, dtype=torch.uint8, device="cuda")
        with_feedback = k < 2  # the third call passes no feedback image
        st, msg = call(f, g, rfmt, mfmt, iters, temporal_ptr, moments_ptr, filtered.data_ptr(),
                       feedback.data_ptr() if with_feedback else None)
        assert st == L.IRT_OK, msg
        torch.cuda.synchronize()
        assert np.array_equal(filtered.cpu().numpy(), want_filtered), k
        if with_feedback:
            assert np.array_equal(feedback.cpu().numpy(), want_feedback), k
        else:
            assert np.all(feedback.cpu().numpy() == 0x7F)
    drv.close()
    wl.close()


def test_noalloc_rejects_frames_above_its_limit_and_bad_formats(cuda):
    f = L.Frame()
    f.size[0], f.size[1] = 1024, 1024
    dummy = torch.zeros(16, dtype=torch.uint8, device="cuda")
    p = dummy.data_ptr()
    g = L.GBuffer(L.GBUFFER_F32, p, p, p, p, p)
    st, msg = call(f, g, L.RADIANCE_F32, L.MOMENTS_F32, 4, p, p, p, p)
    assert st == L.IRT_E_INVALID and "262144" in msg
    f.size[0], f.size[1] = 64, 40
    st, msg = call(f, g, L.RADIANCE_F32, 7, 4, p, p, p, p)
    assert st == L.IRT_E_INVALID and "moments format" in msg
    st, msg = call(f, g, 5, L.MOMENTS_F32, 4, p, p, p, p)
    assert st == L.IRT_E_INVALID and "radiance format" in msg
    st, msg = call(f, g, L.RADIANCE_F32, L.MOMENTS_F32, 0, p, p, p, p)
    assert st == L.IRT_E_INVALID and "iterations" in msg
