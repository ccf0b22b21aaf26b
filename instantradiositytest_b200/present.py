"""Presentation and PNG capture: the display image of a session
(irt_present: sRGB-encoded 8-bit RGBA of the filtered radiance) and a PNG
writer for it, as Renderer::capture does (src/renderer.rs:2109-2163)."""
from __future__ import annotations

import ctypes as C
import os
import struct
import zlib

import numpy as np
import torch

from . import _lib as L
from ._lib import lib
from .runtime import Session, stream_handle


def present(session: Session, which: int = L.BUF_FILTERED) -> np.ndarray:
    """The display image of a session's radiance buffer as uint8 [H, W, 4]."""
    p, n = session.buffer_ptr(which)
    fmt = L.RADIANCE_F16 if n == session.w * session.h * 8 else L.RADIANCE_F32
    out = torch.empty(session.w * session.h * 4, dtype=torch.uint8, device="cuda")
    L.check(lib.irt_present(C.c_void_p(p), fmt, session.w, session.h, C.c_void_p(out.data_ptr()), stream_handle()),
            session.ctx.handle, "present")
    return out.cpu().numpy().reshape(session.h, session.w, 4)


def _chunk(tag: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)


def png_bytes(rgba: np.ndarray) -> bytes:
    """8-bit RGBA PNG (colour type 6), one filter byte 0 per row."""
    rgba = np.ascontiguousarray(rgba, dtype=np.uint8)
    h, w, c = rgba.shape
    assert c == 4
    raw = np.concatenate([np.zeros((h, 1), np.uint8), rgba.reshape(h, w * 4)], axis=1).tobytes()
    return (b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)) +
            _chunk(b"IDAT", zlib.compress(raw, 6)) + _chunk(b"IEND", b""))


def write_png(path: str, rgba: np.ndarray):
    parent = os.path.dirname(path)
    if parent:
        os.makedirs(parent, exist_ok=True)
    with open(path, "wb") as fh:
        fh.write(png_bytes(rgba))


def read_png(path: str) -> np.ndarray:
    """Reads back an 8-bit RGBA PNG written by write_png (filter type 0)."""
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w, h = 8, b"", None, None
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        tag, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        if zlib.crc32(tag + body) & 0xFFFFFFFF != struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]:
            raise ValueError("PNG chunk CRC mismatch")
        if tag == b"IHDR":
            w, h = struct.unpack(">II", body[:8])
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, w * 4 + 1)
    assert np.all(raw[:, 0] == 0)
    return raw[:, 1:].reshape(h, w, 4)


def srgb8_reference(rgb: np.ndarray) -> np.ndarray:
    """sRGB encoding of linear values (IEC 61966-2-1), clamped to [0, 1] and
    rounded to 8 bits, in float64 — the checker for irt_present."""
    v = np.clip(np.nan_to_num(np.asarray(rgb, np.float64), nan=0.0), 0.0, 1.0)
    e = np.where(v <= 0.0031308, v * 12.92, 1.055 * np.power(v, 1.0 / 2.4) - 0.055)
    return np.rint(e * 255.0).astype(np.uint8)
