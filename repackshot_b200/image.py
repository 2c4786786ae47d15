"""Image files of rendered films, byte for byte as the reference's command line writes them: PNG
(8-bit sRGB), uncompressed TIFF (8 or 16 bit sRGB, or 32-bit float linear light, RGB or RGBA) and
linear raw DNG (32-bit float). Standard library and numpy only.

The pixels come from Film.srgb (rtg_film_srgb8 / rtg_film_srgb16: the reference's resolve,
exposure, tone curve and sRGB quantisation) and Film.linear (rtg_film_linear: resolve times 2^ev).

* PNG (rt-core/src/png.rs): signature, IHDR, one IDAT, IEND. The scanlines are unfiltered (filter
  byte 0) and the zlib stream (RFC 1950) holds stored deflate blocks (RFC 1951 section 3.2.4) of at
  most 65,535 bytes, not compressed ones. 16-bit samples are big-endian; the command line writes 8.
* TIFF (rt-core/src/tiff.rs, from TIFF 6.0): little-endian, one directory at offset 8 with its
  fields sorted by tag, values longer than 4 bytes after it in field order (each at an even
  offset), then the pixels in contiguous strips of about 8 KiB.
* DNG (rt-core/src/dng.rs, from DNG 1.4): the TIFF layout with a LinearRaw float image and the DNG
  fields a raw developer needs.
"""
from __future__ import annotations

import struct
import zlib
from fractions import Fraction

import numpy as np

PNG_SIGNATURE = b"\x89PNG\r\n\x1a\n"
MAX_STORED_BLOCK = 65_535  # the largest LEN of a stored deflate block


def _chunk(tag: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)


def zlib_stored(raw: bytes) -> bytes:
    """A zlib stream of stored deflate blocks: header 0x78 0x01 (deflate, 32 KiB window, no
    dictionary; a multiple of 31), blocks of at most 65,535 bytes, each BFINAL/BTYPE byte, LEN and
    its complement little-endian then the bytes, and the Adler-32 of `raw` big-endian
    (png.rs:64-86). An empty input is one empty final block."""
    out = bytearray(b"\x78\x01")
    if not raw:
        out += b"\x01\x00\x00\xff\xff"
    for start in range(0, len(raw), MAX_STORED_BLOCK):
        block = raw[start:start + MAX_STORED_BLOCK]
        final = start + MAX_STORED_BLOCK >= len(raw)
        out += struct.pack("<BHH", int(final), len(block), len(block) ^ 0xFFFF) + block
    out += struct.pack(">I", zlib.adler32(raw) & 0xFFFFFFFF)
    return bytes(out)


def png_bytes(image: np.ndarray) -> bytes:
    """PNG file bytes of an (h, w, 3) uint8 or uint16 image: unfiltered scanlines in stored deflate
    blocks (png.rs:102-131 for 8 bits; 16-bit samples big-endian, as PNG stores them)."""
    img = np.ascontiguousarray(image)
    if img.ndim != 3 or img.shape[2] != 3 or img.dtype not in (np.uint8, np.uint16):
        raise ValueError("expected an (h, w, 3) uint8 or uint16 array")
    h, w, _ = img.shape
    if w == 0 or h == 0:
        raise ValueError("PNG dimensions must be non-zero")
    depth = 8 if img.dtype == np.uint8 else 16
    rows = img.astype(">u2") if depth == 16 else img
    raw = b"".join(b"\x00" + rows[y].tobytes() for y in range(h))
    header = struct.pack(">IIBBBBB", w, h, depth, 2, 0, 0, 0)
    return PNG_SIGNATURE + _chunk(b"IHDR", header) + _chunk(b"IDAT", zlib_stored(raw)) + _chunk(b"IEND", b"")


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


# ---- TIFF 6.0 ------------------------------------------------------------------------------------

# Field types (TIFF 6.0 section 2) and the struct code of one number of each (a RATIONAL or
# SRATIONAL value is two of them: numerator, denominator).
BYTE, ASCII, SHORT, LONG, RATIONAL, SRATIONAL = 1, 2, 3, 4, 5, 10
_PACK = {BYTE: "B", SHORT: "H", LONG: "I", RATIONAL: "I", SRATIONAL: "i"}

# Tags of the baseline fields (TIFF 6.0 section 8) and the floating point extension (section 19).
NEW_SUBFILE_TYPE, IMAGE_WIDTH, IMAGE_LENGTH, BITS_PER_SAMPLE, COMPRESSION = 254, 256, 257, 258, 259
PHOTOMETRIC, MAKE, MODEL, STRIP_OFFSETS, SAMPLES_PER_PIXEL = 262, 271, 272, 273, 277
ROWS_PER_STRIP, STRIP_BYTE_COUNTS, X_RESOLUTION, Y_RESOLUTION = 278, 279, 282, 283
PLANAR_CONFIGURATION, RESOLUTION_UNIT, EXTRA_SAMPLES, SAMPLE_FORMAT = 284, 296, 338, 339

STRIP_TARGET = 8192  # bytes a strip aims at: "about 8K bytes" (TIFF 6.0 section 7)
TIFF_DPI = 72        # the resolution the command line writes (rt-cli/src/lib.rs:662)


def field(tag: int, kind: int, values) -> tuple[int, int, int, bytes]:
    """A directory entry as (tag, type, count, little-endian value bytes). ASCII takes a str and
    stores it with its terminating NUL (counted); RATIONAL and SRATIONAL take (numerator,
    denominator) pairs."""
    if kind == ASCII:
        data = values.encode("ascii") + b"\x00"
        return tag, kind, len(data), data
    values = list(values)
    flat = [v for pair in values for v in pair] if kind in (RATIONAL, SRATIONAL) else values
    return tag, kind, len(values), struct.pack("<" + _PACK[kind] * len(flat), *flat)


class Raster:
    """An (h, w, 3 or 4) image of uint8, uint16 or float32 samples (tiff.rs:168-262): its strips and
    the fields every TIFF of it has."""

    def __init__(self, image: np.ndarray):
        img = np.asarray(image)
        if img.ndim != 3 or img.shape[2] not in (3, 4):
            raise ValueError("TIFF is written as RGB or RGBA: expected an (h, w, 3) or (h, w, 4) array")
        if img.dtype not in (np.uint8, np.uint16, np.float32):
            raise ValueError("TIFF samples are uint8, uint16 or float32")
        self.height, self.width, self.channels = img.shape
        if self.width == 0 or self.height == 0:
            raise ValueError("TIFF dimensions must be non-zero")
        self.bits = 8 * img.dtype.itemsize
        self.is_float = img.dtype == np.float32
        self.pixels = np.ascontiguousarray(img, img.dtype.newbyteorder("<")).tobytes()
        row_bytes = self.width * self.channels * img.dtype.itemsize
        self.rows_per_strip = min(max(STRIP_TARGET // row_bytes, 1), self.height)
        strips = -(-self.height // self.rows_per_strip)
        self.strip_bytes = [min(self.rows_per_strip, self.height - i * self.rows_per_strip) * row_bytes
                            for i in range(strips)]

    def fields(self) -> list:
        """Width, length, bits, compression 1, strip offsets (zeros until assemble), samples per
        pixel, rows per strip, strip byte counts, planar configuration 1 (chunky); ExtraSamples 2
        (unassociated alpha) for RGBA and SampleFormat 3 (IEEE float) for floats."""
        c = self.channels
        out = [
            field(IMAGE_WIDTH, LONG, [self.width]),
            field(IMAGE_LENGTH, LONG, [self.height]),
            field(BITS_PER_SAMPLE, SHORT, [self.bits] * c),
            field(COMPRESSION, SHORT, [1]),
            field(STRIP_OFFSETS, LONG, [0] * len(self.strip_bytes)),
            field(SAMPLES_PER_PIXEL, SHORT, [c]),
            field(ROWS_PER_STRIP, LONG, [self.rows_per_strip]),
            field(STRIP_BYTE_COUNTS, LONG, self.strip_bytes),
            field(PLANAR_CONFIGURATION, SHORT, [1]),
        ]
        if c == 4:
            out.append(field(EXTRA_SAMPLES, SHORT, [2]))
        if self.is_float:
            out.append(field(SAMPLE_FORMAT, SHORT, [3] * c))
        return out


def assemble(fields: list, raster: Raster) -> bytes:
    """The file (tiff.rs:264-332): header "II" 42 with the directory at 8; the entry count, the
    entries sorted by tag (12 bytes: tag, type, count, then the value left-justified when it fits
    in 4 bytes, else its offset) and a zero next-directory offset; the longer values in entry order,
    each padded to an even length; then the strips back to back, whose offsets replace the
    StripOffsets placeholder."""
    fields = sorted(fields, key=lambda f: f[0])
    directory = 2 + 12 * len(fields) + 4
    first_pixel = 8 + directory + sum(len(d) + (len(d) & 1) for _, _, _, d in fields if len(d) > 4)
    if first_pixel + len(raster.pixels) > 0xFFFFFFFF:
        raise ValueError("the image is too large for a TIFF")
    offsets = list(np.cumsum([first_pixel] + raster.strip_bytes[:-1]))
    fields = [(t, k, n, struct.pack(f"<{n}I", *offsets)) if t == STRIP_OFFSETS else (t, k, n, d) for t, k, n, d in fields]
    out = bytearray(b"II*\x00" + struct.pack("<IH", 8, len(fields)))
    extra, at = bytearray(), 8 + directory
    for tag, kind, count, data in fields:
        out += struct.pack("<HHI", tag, kind, count)
        if len(data) <= 4:
            out += data.ljust(4, b"\x00")
        else:
            out += struct.pack("<I", at + len(extra))
            extra += data + b"\x00" * (len(data) & 1)
    out += struct.pack("<I", 0) + extra
    assert len(out) == first_pixel
    return bytes(out) + raster.pixels


def tiff_bytes(image: np.ndarray, dpi: int = TIFF_DPI) -> bytes:
    """An uncompressed RGB or RGBA TIFF of an (h, w, 3 | 4) uint8, uint16 or float32 image
    (tiff.rs:334-352): the raster's fields, photometric 2 (RGB), `dpi` (0 written as 1) as the
    resolution both ways over resolution unit 2 (inches). 8 and 16 bit samples are sRGB by
    convention; floats are linear light."""
    raster = Raster(image)
    dpi = max(int(dpi), 1)
    fields = raster.fields() + [
        field(PHOTOMETRIC, SHORT, [2]),
        field(X_RESOLUTION, RATIONAL, [(dpi, 1)]),
        field(Y_RESOLUTION, RATIONAL, [(dpi, 1)]),
        field(RESOLUTION_UNIT, SHORT, [2]),
    ]
    return assemble(fields, raster)


# ---- DNG 1.4 -------------------------------------------------------------------------------------

# DNG tags (DNG 1.4 chapter 4).
DNG_VERSION, DNG_BACKWARD_VERSION, UNIQUE_CAMERA_MODEL, WHITE_LEVEL = 50706, 50707, 50708, 50717
COLOR_MATRIX_1, AS_SHOT_NEUTRAL, BASELINE_EXPOSURE, CALIBRATION_ILLUMINANT_1 = 50721, 50728, 50730, 50778

PHOTOMETRIC_LINEAR_RAW = 34892
ILLUMINANT_D65 = 21          # CalibrationIlluminant1 for D65 (the Exif LightSource value)
DNG_FILE_VERSION = (1, 4, 0, 0)  # floating point samples need DNG 1.4
CAMERA = "Repackshot"        # UniqueCameraModel, Make and Model (dng.rs:52)
MATRIX_DENOMINATOR = 10_000_000


def xyz_to_linear_srgb() -> list[int]:
    """ColorMatrix1, row by row, as numerators over 10^7 (dng.rs:55-68): the inverse of the linear
    sRGB to CIE XYZ matrix of the primaries (0.64, 0.33), (0.30, 0.60), (0.15, 0.06) and the D65
    white (0.3127, 0.3290), in exact rational arithmetic, rounded to seven decimals."""
    def xyz(x, y):
        x, y = Fraction(x), Fraction(y)
        return [x / y, Fraction(1), (1 - x - y) / y]

    primaries = [xyz("0.64", "0.33"), xyz("0.30", "0.60"), xyz("0.15", "0.06")]
    white = xyz("0.3127", "0.3290")
    # Columns are the primaries' XYZ scaled so that equal RGB maps to the white: solve P s = white.
    p = [[primaries[col][row] for col in range(3)] for row in range(3)]
    scale = _solve3(p, white)
    m = [[p[row][col] * scale[col] for col in range(3)] for row in range(3)]
    inverse = _inverse3(m)
    return [round(inverse[row][col] * MATRIX_DENOMINATOR) for row in range(3) for col in range(3)]


def _det3(a) -> Fraction:
    return (a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0])
            + a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]))


def _solve3(a, b) -> list:
    """Cramer's rule."""
    d = _det3(a)
    return [_det3([[b[r] if c == k else a[r][c] for c in range(3)] for r in range(3)]) / d for k in range(3)]


def _inverse3(a) -> list:
    """The inverse by cofactors: entry (r, c) is the (c, r) cofactor over the determinant."""
    d = _det3(a)

    def minor(r, c):
        rows = [i for i in range(3) if i != r]
        cols = [j for j in range(3) if j != c]
        return a[rows[0]][cols[0]] * a[rows[1]][cols[1]] - a[rows[0]][cols[1]] * a[rows[1]][cols[0]]

    return [[(-1) ** (r + c) * minor(c, r) / d for c in range(3)] for r in range(3)]


def dng_bytes(rgb: np.ndarray) -> bytes:
    """A linear raw DNG of an (h, w, 3) float32 image of scene-linear light (dng.rs:70-98): the
    float RGB raster's TIFF fields plus NewSubfileType 0, photometric LinearRaw, Make and Model,
    DNGVersion and DNGBackwardVersion 1.4.0.0, UniqueCameraModel, WhiteLevel 1 (the render's white;
    values above it are kept), ColorMatrix1 (XYZ to linear sRGB, D65 by CalibrationIlluminant1),
    AsShotNeutral 1 1 1 and BaselineExposure 0."""
    img = np.asarray(rgb)
    if img.ndim != 3 or img.shape[2] != 3 or img.dtype != np.float32:
        raise ValueError("a DNG is written from an (h, w, 3) float32 image")
    raster = Raster(img)
    fields = raster.fields() + [
        field(NEW_SUBFILE_TYPE, LONG, [0]),
        field(PHOTOMETRIC, SHORT, [PHOTOMETRIC_LINEAR_RAW]),
        field(MAKE, ASCII, CAMERA),
        field(MODEL, ASCII, CAMERA),
        field(DNG_VERSION, BYTE, DNG_FILE_VERSION),
        field(DNG_BACKWARD_VERSION, BYTE, DNG_FILE_VERSION),
        field(UNIQUE_CAMERA_MODEL, ASCII, CAMERA),
        field(WHITE_LEVEL, LONG, [1]),
        field(COLOR_MATRIX_1, SRATIONAL, [(n, MATRIX_DENOMINATOR) for n in xyz_to_linear_srgb()]),
        field(AS_SHOT_NEUTRAL, RATIONAL, [(1, 1)] * 3),
        field(BASELINE_EXPOSURE, SRATIONAL, [(0, 1)]),
        field(CALIBRATION_ILLUMINANT_1, SHORT, [ILLUMINANT_D65]),
    ]
    return assemble(fields, raster)
