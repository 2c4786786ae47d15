"""Renders an RSB scene on the GPU and writes a PNG, TIFF or DNG: the progressive loop of the
reference's command line (engine/crates/rt-cli/src/lib.rs:239-368, cli.rs:841-843) and its output
files (lib.rs:650-760) on this library.

    python -m repackshot_b200 SCENE.rsb -o OUT [--samples N] [--budget SECONDS] [--ev STOPS]
                              [--tonemap 0..4] [--format png|tiff|dng] [--bits 8|16|32]

Samples go in passes of 1, 2, 4, ... up to 16 sample indices (MAX_PASS_SAMPLES), each pass one
rtg_render_progressive call; with a time budget, rendering stops between passes once it is spent.
The result does not depend on the pass sizes: each pixel's samples are added in index order.
Exposure and tone curve default to the scene's RNDR settings.

The format is --format, else the output's extension (.tif and .tiff: TIFF, .dng: DNG, anything else
PNG). A PNG is 8-bit sRGB; a TIFF is 8 (the default) or 16 bit sRGB, or 32-bit float linear light
with the exposure applied and no tone curve; a DNG is always the 32-bit linear light.
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

MAX_PASS_SAMPLES = 16
FORMATS = ("png", "tiff", "dng")


def render(rsb: bytes, samples: int | None = None, budget: float | None = None):
    """(scene, film, samples rendered) after the progressive loop."""
    from . import Scene
    scene = Scene(rsb)
    film = scene.film()
    total = samples or scene.output()[2] or 16
    start, done, step = time.perf_counter(), 0, 1
    while done < total:
        n = min(step, total - done)
        film.render(done, n)
        done += n
        step = min(step * 2, MAX_PASS_SAMPLES)
        if budget is not None and time.perf_counter() - start >= budget:
            break
    return scene, film, done


def output_spec(fmt: str | None, bits: int | None, path) -> tuple[str, int]:
    """(format, bits) from --format, --bits and the output path (OutputSpec::resolve,
    lib.rs:673-710); raises ValueError with the reference's messages for combinations it refuses."""
    if fmt is None:
        ext = Path(path).suffix.lower()
        fmt = "tiff" if ext in (".tif", ".tiff") else "dng" if ext == ".dng" else "png"
    if fmt not in FORMATS:
        raise ValueError(f"--format expects png, tiff or dng, got '{fmt}'")
    if fmt == "png":
        if bits not in (None, 8):
            raise ValueError("a PNG is written with 8 bits per channel: use --format tiff for 16 or 32")
        return fmt, 8
    if fmt == "tiff":
        if bits not in (None, 8, 16, 32):
            raise ValueError("--bits expects 8, 16 or 32")
        return fmt, bits or 8
    if bits not in (None, 32):
        raise ValueError("a DNG is always 32-bit float: --bits can only be 32")
    return fmt, 32


def encode_film(film, ev: float | None, tonemap: int | None, fmt: str, bits: int) -> bytes:
    """The file bytes (encode_film, lib.rs:737-760): tone-mapped sRGB for the PNG and the 8 and 16
    bit TIFFs, the linear exposed film (no curve, no clamp) for the 32-bit TIFF and the DNG. Colour
    only: the film's coverage is not written."""
    from . import image
    if fmt == "dng":
        return image.dng_bytes(film.linear(ev))
    if fmt == "tiff" and bits == 32:
        return image.tiff_bytes(film.linear(ev))
    px = film.srgb(ev, tonemap, bits)
    return image.png_bytes(px) if fmt == "png" else image.tiff_bytes(px)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m repackshot_b200", description=__doc__.splitlines()[0])
    ap.add_argument("scene", help="an RSB file")
    ap.add_argument("-o", "--output", required=True, help="image file to write (PNG, or TIFF or DNG by --format or extension)")
    ap.add_argument("--samples", type=int, default=None, help="samples per pixel (default: the scene's)")
    ap.add_argument("--budget", type=float, default=None, help="stop between passes after this many seconds")
    ap.add_argument("--ev", type=float, default=None, help="exposure in stops (default: the scene's)")
    ap.add_argument("--tonemap", type=int, default=None, help="0 linear, 1 ACES, 2 filmic, 3 AgX, 4 standard")
    ap.add_argument("--format", default=None, help="png (the default), tiff or dng; without it the output's extension decides")
    ap.add_argument("--bits", type=int, default=None, help="bits per channel: PNG 8; TIFF 8, 16 (sRGB) or 32 (float, linear); DNG 32")
    args = ap.parse_args(argv)
    try:
        fmt, bits = output_spec(args.format, args.bits, args.output)
    except ValueError as e:
        ap.error(str(e))
    with open(args.scene, "rb") as f:
        rsb = f.read()
    t0 = time.perf_counter()
    scene, film, done = render(rsb, args.samples, args.budget)
    data = encode_film(film, args.ev, args.tonemap, fmt, bits)
    out = Path(args.output)
    out.parent.mkdir(parents=True, exist_ok=True)
    out.write_bytes(data)
    dt = time.perf_counter() - t0
    print(f"{scene.width}x{scene.height}, {done} spp, {dt:.3f} s, {scene.width * scene.height * done / dt / 1e6:.1f} Mpaths/s -> "
          f"{args.output} ({fmt}, {bits} bits)", file=sys.stderr)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
