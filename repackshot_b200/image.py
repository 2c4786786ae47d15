"""Image files of rendered films: PNG, 8- or 16-bit RGB, written with the standard library.

The pixels come from Film.srgb (rtg_film_srgb8 / rtg_film_srgb16: the reference's resolve,
exposure, tone curve and sRGB quantisation). PNG stores 16-bit samples big-endian.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np


def _chunk(tag: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)


def png_bytes(image: np.ndarray) -> bytes:
    """PNG file bytes of an (h, w, 3) uint8 or uint16 image (no filtering, zlib level 6)."""
    img = np.ascontiguousarray(image)
    if img.ndim != 3 or img.shape[2] != 3 or img.dtype not in (np.uint8, np.uint16):
        raise ValueError("expected an (h, w, 3) uint8 or uint16 array")
    h, w, _ = img.shape
    depth = 8 if img.dtype == np.uint8 else 16
    rows = img.astype(">u2") if depth == 16 else img
    raw = b"".join(b"\x00" + rows[y].tobytes() for y in range(h))
    header = struct.pack(">IIBBBBB", w, h, depth, 2, 0, 0, 0)
    return b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", header) + _chunk(b"IDAT", zlib.compress(raw, 6)) + _chunk(b"IEND", b"")


def write_png(path, image: np.ndarray) -> None:
    with open(path, "wb") as f:
        f.write(png_bytes(image))


def read_png(data: bytes) -> np.ndarray:
    """Decodes the PNGs png_bytes writes (unfiltered RGB, 8 or 16 bits): for round trips."""
    pos, idat, w = 8, b"", 0
    while pos < len(data):
        n, tag = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        if tag == b"IHDR":
            w, h, depth, colour = struct.unpack(">IIBB", body[:10])
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    bpp = 3 * (depth // 8)
    raw = zlib.decompress(idat)
    rows = [raw[y * (1 + w * bpp) + 1:(y + 1) * (1 + w * bpp)] for y in range(h)]
    dtype = np.uint8 if depth == 8 else ">u2"
    return np.frombuffer(b"".join(rows), dtype).reshape(h, w, 3).astype(np.uint8 if depth == 8 else np.uint16)
