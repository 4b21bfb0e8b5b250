"""Image output: framebuffer::ToImage semantics (src/renderbuffer.hxx:99-137) and headless
writers.  The reference saves through CImg; here a linear float buffer is written as PFM
(HDR) or an 8-bit PNG produced with zlib.
"""
from __future__ import annotations

import struct
import zlib
from pathlib import Path

import numpy as np


def linear_to_srgb(x: np.ndarray) -> np.ndarray:
    """Color::LinearToSRGB (spectral.hxx:146-152)."""
    return np.where(x <= 0.0031308, 12.92 * x, 1.055 * np.power(np.maximum(x, 0.0), 1.0 / 2.4) - 0.055)


def to_image(rgb_linear: np.ndarray, xres: int, yres: int, linear_output: bool = False) -> np.ndarray:
    """(yres, xres, 3) uint8 with row 0 at the TOP.  Input is in unit order (row 0 at the
    bottom).  Clamp to [0,1], sRGB unless linear_output, scale by 255.999, truncate."""
    a = np.asarray(rgb_linear, dtype=np.float64).reshape(yres, xres, 3)
    a = np.clip(a, 0.0, 1.0)
    if not linear_output:
        a = linear_to_srgb(a)
    out = (a * 255.999).astype(np.uint8)
    return out[::-1].copy()


def write_png(path, img: np.ndarray) -> None:
    img = np.ascontiguousarray(img, dtype=np.uint8)
    h, w, c = img.shape
    raw = b"".join(b"\x00" + img[y].tobytes() for y in range(h))

    def chunk(tag, data):
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    png = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0))
    png += chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b"")
    Path(path).write_bytes(png)


def write_pfm(path, rgb_linear: np.ndarray, xres: int, yres: int) -> None:
    """PFM stores rows bottom to top, which is the unit order already."""
    a = np.asarray(rgb_linear, dtype="<f4").reshape(yres, xres, 3)
    with open(path, "wb") as f:
        f.write(f"PF\n{xres} {yres}\n-1.0\n".encode())
        f.write(a.tobytes())
