"""The image files of the command line, on the CPU: the TIFF and DNG writers reproduce the reference's
golden files byte for byte (engine/crates/rt-cli/tests/tiff_golden.rs:48-94, the files copied to
tests/golden/tiff by tests/golden/make_golden.py), the PNG writer keeps the reference's known answers
(engine/crates/rt-core/src/png.rs:192-255: stored deflate blocks of at most 65,535 bytes), and
--format / --bits resolve as OutputSpec::resolve does (rt-cli/src/lib.rs:673-710)."""
import struct
import zlib
from pathlib import Path

import numpy as np
import pytest

from repackshot_b200 import image
from repackshot_b200.__main__ import output_spec

TIFF = Path(__file__).resolve().parent / "golden" / "tiff"


# The inputs tiff_golden.rs:18-45 encodes: sample c of pixel p of a 4 x 4 image, and a 50 x 60 one
# of two strips (54 rows of 150 bytes, then 6).
def u8_image(channels):
    return np.array([[(p * 17 + c * 5) & 255 for c in range(channels)] for p in range(16)], np.uint8).reshape(4, 4, channels)


def u16_image(channels):
    return np.array([[(p * 4099 + c * 1021) & 0xFFFF for c in range(channels)] for p in range(16)], np.uint16).reshape(4, 4, channels)


def f32_image(channels):
    return np.array([[(p * 7 + c * 13) / 64 for c in range(channels)] for p in range(16)], np.float32).reshape(4, 4, channels)


def strips_image():
    return np.array([[[(x * 5 + y * 3 + c * 7) & 255 for c in range(3)] for x in range(50)] for y in range(60)], np.uint8)


GOLDEN = {
    "strips.tif": lambda: image.tiff_bytes(strips_image(), 72),
    "rgb8.tif": lambda: image.tiff_bytes(u8_image(3), 72),
    "rgba8.tif": lambda: image.tiff_bytes(u8_image(4), 72),
    "rgb16.tif": lambda: image.tiff_bytes(u16_image(3), 72),
    "rgba16-300dpi.tif": lambda: image.tiff_bytes(u16_image(4), 300),
    "rgb32.tif": lambda: image.tiff_bytes(f32_image(3), 72),
    "rgba32.tif": lambda: image.tiff_bytes(f32_image(4), 72),
    "linear.dng": lambda: image.dng_bytes(f32_image(3)),
}


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_writers_produce_the_golden_files(name):
    assert GOLDEN[name]() == (TIFF / name).read_bytes()


def read_tiff(data: bytes):
    """The fields (tag -> (type, count, value bytes)) and the strips joined, read as TIFF 6.0 lays
    them out; checks the header, the tag order and that every out-of-line value starts at an even
    offset."""
    assert data[:4] == b"II*\x00"
    ifd = struct.unpack_from("<I", data, 4)[0]
    n = struct.unpack_from("<H", data, ifd)[0]
    unit = {1: 1, 2: 1, 3: 2, 4: 4, 5: 8, 10: 8}
    fields, tags = {}, []
    for i in range(n):
        tag, kind, count, value = struct.unpack_from("<HHII", data, ifd + 2 + 12 * i)
        size = unit[kind] * count
        at = ifd + 2 + 12 * i + 8 if size <= 4 else value
        if size > 4:
            assert at % 2 == 0
        fields[tag] = (kind, count, data[at:at + size])
        tags.append(tag)
    assert tags == sorted(tags)
    assert struct.unpack_from("<I", data, ifd + 2 + 12 * n)[0] == 0
    longs = lambda t: struct.unpack(f"<{fields[t][1]}I", fields[t][2])  # noqa: E731
    pixels = b"".join(data[o:o + c] for o, c in zip(longs(273), longs(279)))
    return fields, pixels


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.float32])
@pytest.mark.parametrize("size", [(1, 1), (3, 7), (61, 50), (200, 13)])
def test_tiff_round_trips_any_size(dtype, size):
    rng = np.random.default_rng(size[0] * 1000 + size[1])
    h, w = size
    img = (rng.random((h, w, 3)) * 60000).astype(dtype)
    fields, pixels = read_tiff(image.tiff_bytes(img))
    assert struct.unpack("<2I", fields[256][2] + fields[257][2]) == (w, h)
    rows = struct.unpack("<I", fields[278][2])[0]
    row_bytes = w * 3 * img.dtype.itemsize
    assert rows == min(max(8192 // row_bytes, 1), h)
    assert fields[279][1] == -(-h // rows)
    assert np.array_equal(np.frombuffer(pixels, img.dtype.newbyteorder("<")).reshape(h, w, 3), img)
    assert (339 in fields) == (dtype == np.float32)
    assert 338 not in fields


def test_tiff_writes_zero_dpi_as_one():
    fields, _ = read_tiff(image.tiff_bytes(u8_image(3), 0))
    assert fields[282][2] == struct.pack("<II", 1, 1) and fields[283][2] == struct.pack("<II", 1, 1)


@pytest.mark.parametrize("bad", [np.zeros((0, 4, 3), np.uint8), np.zeros((4, 4, 2), np.uint8), np.zeros((4, 4, 3), np.int32),
                                 np.zeros((4, 4), np.uint8)])
def test_tiff_refuses_what_it_cannot_write(bad):
    with pytest.raises(ValueError):
        image.tiff_bytes(bad)


def test_dng_is_a_linear_raw_float_tiff():
    fields, pixels = read_tiff(image.dng_bytes(f32_image(3)))
    assert struct.unpack("<H", fields[262][2][:2])[0] == 34892
    assert fields[50706][2] == bytes([1, 4, 0, 0]) and fields[50707][2] == bytes([1, 4, 0, 0])
    for tag in (271, 272, 50708):
        assert fields[tag][2] == b"Repackshot\x00"
    assert 338 not in fields
    assert np.array_equal(np.frombuffer(pixels, "<f4"), f32_image(3).reshape(-1))
    with pytest.raises(ValueError):
        image.dng_bytes(f32_image(4))


def test_dng_colour_matrix_inverts_srgb_to_xyz():
    """ColorMatrix1 over 10^7 times the sRGB to XYZ matrix (from the primaries and D65, in f64) is the
    identity to the rounding of seven decimals, and D65 white maps to equal channels."""
    m = np.array(image.xyz_to_linear_srgb(), np.float64).reshape(3, 3) / 1e7
    xyz = lambda x, y: np.array([x / y, 1.0, (1 - x - y) / y])  # noqa: E731
    p = np.stack([xyz(0.64, 0.33), xyz(0.30, 0.60), xyz(0.15, 0.06)], axis=1)
    white = xyz(0.3127, 0.3290)
    to_xyz = p * np.linalg.solve(p, white)
    assert np.allclose(m @ to_xyz, np.eye(3), atol=5e-7)
    assert np.allclose(m @ white, 1.0, atol=5e-7)


def inflate_stored(z: bytes) -> bytes:
    assert z[0] == 0x78 and ((z[0] << 8) | z[1]) % 31 == 0
    pos, raw = 2, b""
    while True:
        head = z[pos]
        assert head & 0b110 == 0, "only stored blocks"
        n, nn = struct.unpack_from("<HH", z, pos + 1)
        assert n == nn ^ 0xFFFF
        raw += z[pos + 5:pos + 5 + n]
        pos += 5 + n
        if head & 1:
            break
    assert pos + 4 == len(z) and struct.unpack(">I", z[pos:])[0] == zlib.adler32(raw)
    return raw


def png_chunks(data: bytes):
    assert data[:8] == image.PNG_SIGNATURE
    pos, out = 8, []
    while pos < len(data):
        n, tag = struct.unpack_from(">I4s", data, pos)
        body = data[pos + 8:pos + 8 + n]
        assert struct.unpack_from(">I", data, pos + 8 + n)[0] == zlib.crc32(tag + body)
        out.append((tag, body))
        pos += 12 + n
    assert pos == len(data)
    return out


def test_png_one_white_pixel_has_the_fixed_length():  # png.rs one_by_one_white_has_a_fixed_length
    data = image.png_bytes(np.full((1, 1, 3), 255, np.uint8))
    assert len(data) == 72
    chunks = png_chunks(data)
    assert [t for t, _ in chunks] == [b"IHDR", b"IDAT", b"IEND"]
    assert chunks[0][1] == bytes([0, 0, 0, 1, 0, 0, 0, 1, 8, 2, 0, 0, 0])
    assert inflate_stored(chunks[1][1]) == bytes([0, 255, 255, 255])


def test_png_scanlines_round_trip():  # png.rs scanlines_round_trip_through_the_chunks
    w, h = 5, 4
    px = (np.arange(w * h * 3) * 7 % 256).astype(np.uint8).reshape(h, w, 3)
    raw = inflate_stored(png_chunks(image.png_bytes(px))[1][1])
    assert len(raw) == (w * 3 + 1) * h
    for y in range(h):
        line = raw[y * (w * 3 + 1):(y + 1) * (w * 3 + 1)]
        assert line[0] == 0 and line[1:] == px[y].tobytes()
    assert np.array_equal(image.read_png(image.png_bytes(px)), px)


def test_png_large_images_split_into_blocks_of_65535():  # png.rs large_images_are_split_...
    z = png_chunks(image.png_bytes(np.full((200, 200, 3), 9, np.uint8)))[1][1]
    assert z[2] == 0 and struct.unpack_from("<H", z, 3)[0] == 65535
    assert len(inflate_stored(z)) == 120_200


def test_empty_zlib_stream_is_valid():
    assert inflate_stored(image.zlib_stored(b"")) == b""


@pytest.mark.parametrize("fmt,bits,path,want", [
    (None, None, "a.png", ("png", 8)), (None, None, "a.out", ("png", 8)), (None, None, "a", ("png", 8)),
    (None, None, "a.tif", ("tiff", 8)), (None, None, "a.TIFF", ("tiff", 8)), (None, 16, "a.tiff", ("tiff", 16)),
    (None, 32, "a.tif", ("tiff", 32)), (None, None, "a.dng", ("dng", 32)), (None, 32, "a.DNG", ("dng", 32)),
    ("tiff", None, "a.out", ("tiff", 8)), ("png", None, "a.tif", ("png", 8)), ("png", 8, "a.tif", ("png", 8)),
    ("dng", None, "a.png", ("dng", 32)),
])
def test_output_spec_resolves_as_the_reference(fmt, bits, path, want):
    assert output_spec(fmt, bits, path) == want


@pytest.mark.parametrize("fmt,bits,path,message", [
    (None, 16, "a.png", "a PNG is written with 8 bits per channel: use --format tiff for 16 or 32"),
    ("png", 32, "a.tif", "a PNG is written with 8 bits per channel: use --format tiff for 16 or 32"),
    (None, 12, "a.tif", "--bits expects 8, 16 or 32"),
    (None, 8, "a.dng", "a DNG is always 32-bit float: --bits can only be 32"),
    ("exr", None, "a.exr", "--format expects png, tiff or dng, got 'exr'"),
])
def test_output_spec_refuses_as_the_reference(fmt, bits, path, message):
    with pytest.raises(ValueError, match="^" + message.replace("-", r"\-") + "$"):
        output_spec(fmt, bits, path)
