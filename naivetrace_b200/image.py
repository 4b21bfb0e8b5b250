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


def write_exr(path, rgb_linear: np.ndarray, xres: int, yres: int) -> None:
    """OpenEXR, single-part scanline image, uncompressed, channels B, G, R as 32-bit floats
    (the file layout of the OpenEXR specification: magic and version, header attributes,
    one offset per scanline, then per line its y, byte count and the channels in name
    order).  Input in unit order (row 0 at the bottom); EXR's first line is the top."""
    a = np.asarray(rgb_linear, dtype="<f4").reshape(yres, xres, 3)[::-1]

    def attr(name, typ, data):
        return name.encode() + b"\0" + typ.encode() + b"\0" + struct.pack("<i", len(data)) + data

    chlist = b"".join(c.encode() + b"\0" + struct.pack("<iB3xii", 2, 0, 1, 1) for c in "BGR") + b"\0"
    box = struct.pack("<iiii", 0, 0, xres - 1, yres - 1)
    header = (attr("channels", "chlist", chlist) + attr("compression", "compression", b"\0") +
              attr("dataWindow", "box2i", box) + attr("displayWindow", "box2i", box) +
              attr("lineOrder", "lineOrder", b"\0") + attr("pixelAspectRatio", "float", struct.pack("<f", 1.0)) +
              attr("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0)) +
              attr("screenWindowWidth", "float", struct.pack("<f", 1.0)) + b"\0")
    head = struct.pack("<ii", 20000630, 2) + header
    line_bytes = 3 * 4 * xres
    first = len(head) + 8 * yres
    offsets = struct.pack(f"<{yres}Q", *[first + y * (8 + line_bytes) for y in range(yres)])
    body = b"".join(struct.pack("<ii", y, line_bytes) + a[y, :, 2].tobytes() + a[y, :, 1].tobytes() +
                    a[y, :, 0].tobytes() for y in range(yres))
    Path(path).write_bytes(head + offsets + body)


def read_exr(path) -> np.ndarray:
    """Reads the uncompressed single-part FLOAT R, G, B images write_exr produces; returns
    (height, width, 3) with row 0 at the top."""
    data = Path(path).read_bytes()
    magic, version = struct.unpack_from("<ii", data, 0)
    if magic != 20000630:
        raise ValueError("not an OpenEXR file")
    pos = 8
    attrs = {}
    while data[pos] != 0:
        end = data.index(b"\0", pos)
        name = data[pos:end].decode()
        tend = data.index(b"\0", end + 1)
        size = struct.unpack_from("<i", data, tend + 1)[0]
        attrs[name] = data[tend + 5:tend + 5 + size]
        pos = tend + 5 + size
    pos += 1
    if attrs["compression"] != b"\0":
        raise ValueError("only uncompressed EXR files are read here")
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    names, p, cl = [], 0, attrs["channels"]
    while cl[p] != 0:
        e = cl.index(b"\0", p)
        names.append(cl[p:e].decode())
        p = e + 1 + 16
    offsets = struct.unpack_from(f"<{h}Q", data, pos)
    img = np.zeros((h, w, 3), np.float32)
    for off in offsets:
        y, size = struct.unpack_from("<ii", data, off)
        row = np.frombuffer(data, "<f4", count=len(names) * w, offset=off + 8).reshape(len(names), w)
        for c, name in enumerate(names):
            if name in "RGB":
                img[y - y0, :, "RGB".index(name)] = row[c]
    return img
