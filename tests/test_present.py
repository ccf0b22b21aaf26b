"""Presentation (irt_present) and PNG capture: the CUDA pass against the
float64 sRGB encoding of the same radiance, and the PNG writer's round trip
(src/renderer.rs:2109-2163 writes the display target as an RGBA8 PNG)."""
import numpy as np
import pytest
import torch

from instantradiositytest_b200 import _lib as L
from instantradiositytest_b200.present import png_bytes, present, read_png, srgb8_reference, write_png


def test_srgb_reference_values():
    v = srgb8_reference(np.array([0.0, 1.0, 0.5, 0.0031308, -2.0, 7.0, np.nan]))
    assert list(v) == [0, 255, 188, 10, 0, 255, 0]


def test_png_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    img = rng.integers(0, 256, (37, 53, 4), dtype=np.uint8)
    path = str(tmp_path / "sub" / "frame.png")
    write_png(path, img)
    assert np.array_equal(read_png(path), img)
    assert png_bytes(img)[:8] == b"\x89PNG\r\n\x1a\n"


@pytest.mark.gpu
@pytest.mark.parametrize("radiance_format", [L.RADIANCE_F32, L.RADIANCE_F16])
def test_present_matches_srgb_encoding(cuda, tmp_path, radiance_format):
    from instantradiositytest_b200.runtime import FrameDriver
    from instantradiositytest_b200.workload import Workload

    d = FrameDriver(Workload(0, width=160, height=100), radiance_format=radiance_format)
    for i in range(6):
        d.step(i)
    torch.cuda.synchronize()
    img = present(d.session)
    filt = d.session.image_host(L.BUF_FILTERED)
    ref = srgb8_reference(filt[..., :3])
    diff = np.abs(img[..., :3].astype(int) - ref.astype(int))
    print("present: exact", float((diff == 0).mean()), "max", int(diff.max()), "mean value", float(img[..., :3].mean()))
    assert diff.max() <= 1 and (diff == 0).mean() >= 0.999
    assert np.all(img[..., 3] == 255) and img[..., :3].max() > 0
    path = str(tmp_path / "capture.png")
    write_png(path, img)
    assert np.array_equal(read_png(path), img)
    d.close()
