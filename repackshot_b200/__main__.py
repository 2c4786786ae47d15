"""Renders an RSB scene on the GPU and writes a PNG, TIFF or DNG: the reference's command line
renderer `rt` (engine/crates/rt-cli/src/cli.rs, lib.rs) for one scene, on this library.

    python -m repackshot_b200 SCENE.rsb|--example -o OUT [--samples N] [--size WxH]
        [--max-seconds S] [--denoise] [--denoise-strength S] [--keep-noisy] [--adaptive]
        [--noise P] [--pixel-filter none|standard|soft|fine] [--edge-samples K] [--caustics N]
        [--format png|tiff|dng] [--bits 8|16|32] [--ev STOPS] [--tonemap 0..4]

The flags change the scene's RNDR settings before it loads, as Options::apply does
(cli.rs:350-391): image size, denoise bits and strength, adaptive sampling and its noise target,
pixel filter, edge samples, caustic photons (a scene with caustics is refused at load). Samples
default to the scene's, else 16; the time budget to the scene's max_seconds (0: none).

The render follows render_until (lib.rs:239-368, 446-636). Without adaptive sampling, samples go
in passes of 1, 2, 4, ... up to 16 sample indices, each one rtg_render_progressive call; with a
budget, rendering stops between passes once it is spent. The result does not depend on the pass
sizes: each pixel's samples are added in index order. With RNDR.adaptive, rtg_adaptive_run renders
the rounds (the first one in passes of 1, 2, 4, 8, then passes of 16), with the same budget rule.
When the scene asks for denoise, the guide passes are rendered with the film (the albedo of every
sample, or of the adaptive first round) and the image written is the denoised one at the scene's
strength; RNDR.denoise bit 1 (--keep-noisy) also writes the image without denoise beside it, as
<out>-noisy.<ext> (cli.rs:1886-1900).

The format is --format, else the output's extension (.tif and .tiff: TIFF, .dng: DNG, anything else
PNG). A PNG is 8-bit sRGB; a TIFF is 8 (the default) or 16 bit sRGB, or 32-bit float linear light
with the exposure applied and no tone curve; a DNG is always the 32-bit linear light. Exposure and
tone curve default to the scene's RNDR settings (--ev and --tonemap override them).
"""
from __future__ import annotations

import argparse
import struct
import sys
import time
from pathlib import Path

import numpy as np

MAX_PASS_SAMPLES = 16
FORMATS = ("png", "tiff", "dng")
DENOISE_IMAGE, DENOISE_KEEP_NOISY = 1, 2         # RNDR.denoise bits (scene/mod.rs:878-880)
ADAPTIVE_ON = 1                                  # RNDR.adaptive bit 0 (adaptive.rs:45)
ADAPTIVE_WARMUP = 16                             # samples of the adaptive first round (adaptive.rs:49)
PIXEL_FILTERS = {"standard": 0, "none": 1, "soft": 2, "fine": 3}  # pixel_filter.rs:43-49
MAX_EDGE_SAMPLES = 16
MAX_CAUSTIC_PHOTONS = 1 << 22
MAX_DIMENSION = 16384

# The RNDR section: its fields in file order, their types and the values a reader takes for the
# trailing fields a shorter section leaves out (rsb.rs; the loader's RNDR reader).
RNDR_FIELDS = (
    ("width", "I", 640), ("height", "I", 360), ("max_samples", "I", 64), ("seed", "I", 0),
    ("max_seconds", "f", 0.0), ("exposure_ev", "f", 0.0), ("tonemap", "I", 1), ("max_depth", "I", 8),
    ("clamp_indirect", "f", 0.0), ("passes", "I", 0), ("denoise", "I", 0), ("caustic_photons", "I", 0),
    ("caustic_radius", "f", 0.0), ("denoise_strength", "f", 1.0), ("pixel_filter", "I", 0),
    ("edge_supersample", "I", 1), ("adaptive", "I", 0), ("noise_threshold", "f", 0.0),
)


def _sections(rsb: bytes):
    """(tag, start of the section, start of its payload, payload length) of every section."""
    if rsb[:4] != b"RSB1" or len(rsb) < 8:
        raise ValueError("not an RSB file (missing RSB1 magic)")
    pos = 8 + struct.unpack_from("<I", rsb, 4)[0]
    while pos + 8 <= len(rsb):
        n = struct.unpack_from("<I", rsb, pos + 4)[0]
        yield rsb[pos:pos + 4], pos, pos + 8, n
        pos += 8 + n


def render_settings(rsb: bytes) -> dict:
    """The RNDR settings of a file, defaults for the fields (or the section) it leaves out."""
    out = {name: default for name, _, default in RNDR_FIELDS}
    for tag, _, at, n in _sections(rsb):
        if tag == b"RNDR":
            for i, (name, kind, _) in enumerate(RNDR_FIELDS):
                if 4 * i + 4 <= n:
                    out[name] = struct.unpack_from("<" + kind, rsb, at + 4 * i)[0]
    return out


def with_render_settings(rsb: bytes, **changes) -> bytes:
    """The file with its RNDR section rewritten, every field present, `changes` applied (a file
    without one gets one at the end)."""
    for name in changes:
        if name not in dict((f[0], f) for f in RNDR_FIELDS):
            raise KeyError(name)
    settings = render_settings(rsb)
    settings.update(changes)
    payload = b"".join(struct.pack("<" + kind, settings[name]) for name, kind, _ in RNDR_FIELDS)
    section = b"RNDR" + struct.pack("<I", len(payload)) + payload
    for tag, start, at, n in _sections(rsb):
        if tag == b"RNDR":
            return rsb[:start] + section + rsb[at + n:]
    return rsb + section


# ---- options (cli.rs:744-1013, 350-403) ----------------------------------------------------------

def _positive(text: str, flag: str) -> int:
    try:
        n = int(text)
    except ValueError:
        n = 0
    if n <= 0:
        raise ValueError(f"{flag} expects a positive integer, got '{text}'")
    return n


def _seconds(text: str, flag: str) -> float:
    try:
        s = float(np.float32(text))
    except ValueError:
        s = -1.0
    if not (s >= 0.0 and np.isfinite(s)):
        raise ValueError(f"{flag} expects a non-negative number of seconds, got '{text}'")
    return s


def _size(text: str) -> tuple[int, int]:
    bad = f"--size expects WxH such as 1280x720, got '{text}'"
    w, sep, h = text.replace("X", "x").partition("x")
    if not sep or not w.isdigit() or not h.isdigit():
        raise ValueError(bad)
    w, h = int(w), int(h)
    if not (1 <= w <= MAX_DIMENSION and 1 <= h <= MAX_DIMENSION):
        raise ValueError(f"--size must be between 1x1 and {MAX_DIMENSION}x{MAX_DIMENSION}")
    return w, h


def _unit_interval(text: str, flag: str, what: str, top: float = 1.0) -> float:
    try:
        v = float(np.float32(text))
    except ValueError:
        v = float("nan")
    if not (0.0 <= v <= top):
        raise ValueError(f"{flag} expects {what}, got '{text}'")
    return v


def _bounded(text: str, flag: str, lo: int, hi: int, what: str) -> int:
    try:
        n = int(text)
    except ValueError:
        n = lo - 1
    if not (lo <= n <= hi):
        raise ValueError(f"{flag} expects {what}, got '{text}'")
    return n


def parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(prog="python -m repackshot_b200", description=__doc__.splitlines()[0])
    ap.add_argument("scene", nargs="?", help="an RSB file")
    ap.add_argument("--example", action="store_true", help="render the built-in example scene instead of a file")
    ap.add_argument("-o", "--output", required=True, help="image file to write (PNG, or TIFF or DNG by --format or extension)")
    ap.add_argument("--samples", help="samples per pixel (default: the scene's, else 16)")
    ap.add_argument("--size", help="image size WxH, overriding the scene")
    ap.add_argument("--max-seconds", "--budget", dest="max_seconds",
                    help="time budget, overriding RNDR.max_seconds: rendering stops between passes once it is spent (0: none)")
    ap.add_argument("--denoise", action="store_true", help="write the denoised image (RNDR.denoise bit 0)")
    ap.add_argument("--denoise-strength", help="how much of the denoised image, 0 to 1 (RNDR.denoise_strength)")
    ap.add_argument("--keep-noisy", action="store_true", help="with --denoise, also write <out>-noisy.<ext>")
    ap.add_argument("--adaptive", action="store_true", help="sample adaptively (RNDR.adaptive): at most --samples per pixel")
    ap.add_argument("--noise", help="adaptive noise target in percent (RNDR.noise_threshold; implies --adaptive)")
    ap.add_argument("--pixel-filter", help="none, standard (the default), soft or fine (RNDR.pixel_filter)")
    ap.add_argument("--edge-samples", help="samples per sample index of the edge pixels, 1 to 16 (RNDR.edge_supersample)")
    ap.add_argument("--caustics", help="caustic photons per sample (RNDR.caustic_photons; scenes with caustics are refused)")
    ap.add_argument("--threads", help="accepted for the reference's command lines; the GPU render has no thread count")
    ap.add_argument("--format", default=None, help="png (the default), tiff or dng; without it the output's extension decides")
    ap.add_argument("--bits", default=None, help="bits per channel: PNG 8; TIFF 8, 16 (sRGB) or 32 (float, linear); DNG 32")
    ap.add_argument("--ev", type=float, default=None, help="exposure in stops (default: the scene's)")
    ap.add_argument("--tonemap", type=int, default=None, help="0 linear, 1 ACES, 2 filmic, 3 AgX, 4 standard (default: the scene's)")
    return ap


def apply(rsb: bytes, args) -> tuple[bytes, int, float | None]:
    """(the file with the flags' RNDR changes, samples per pixel, time budget or None)."""
    changes = {}
    if args.size is not None:
        changes["width"], changes["height"] = _size(args.size)
    settings = render_settings(rsb)
    denoise = settings["denoise"] | (DENOISE_IMAGE if args.denoise else 0) | (DENOISE_KEEP_NOISY if args.keep_noisy else 0)
    if denoise != settings["denoise"]:
        changes["denoise"] = denoise
    if args.denoise_strength is not None:
        changes["denoise_strength"] = _unit_interval(args.denoise_strength, "--denoise-strength", "a number from 0 to 1")
    if args.caustics is not None:
        changes["caustic_photons"] = _bounded(args.caustics, "--caustics", 0, MAX_CAUSTIC_PHOTONS,
                                              f"a number of photons up to {MAX_CAUSTIC_PHOTONS}")
    if args.pixel_filter is not None:
        if args.pixel_filter not in PIXEL_FILTERS:
            raise ValueError(f"--pixel-filter expects none, standard, soft or fine, got '{args.pixel_filter}'")
        changes["pixel_filter"] = PIXEL_FILTERS[args.pixel_filter]
    if args.edge_samples is not None:
        changes["edge_supersample"] = _bounded(args.edge_samples, "--edge-samples", 1, MAX_EDGE_SAMPLES,
                                               f"a number from 1 to {MAX_EDGE_SAMPLES}")
    target = None
    if args.adaptive:
        target = 0.0
    if args.noise is not None:
        target = _unit_interval(args.noise, "--noise", "a percentage from 0 to 100", 100.0) / 100.0
    if target is not None:
        changes["adaptive"] = settings["adaptive"] | ADAPTIVE_ON
        changes["noise_threshold"] = float(np.float32(target))
    if args.threads is not None:
        _positive(args.threads, "--threads")
    if changes:
        rsb = with_render_settings(rsb, **changes)
        settings = render_settings(rsb)
    samples = _positive(args.samples, "--samples") if args.samples is not None else (settings["max_samples"] or 16)
    seconds = _seconds(args.max_seconds, "--max-seconds") if args.max_seconds is not None else settings["max_seconds"]
    return rsb, samples, (seconds if seconds > 0.0 else None)


def output_spec(fmt: str | None, bits, path) -> tuple[str, int]:
    """(format, bits) from --format, --bits and the output path (OutputSpec::resolve,
    lib.rs:673-710); raises ValueError with the reference's messages for what it refuses."""
    if bits is not None:
        try:
            bits = int(bits)
        except ValueError:
            bits = -1
        if bits not in (8, 16, 32):
            raise ValueError("--bits expects 8, 16 or 32")
    if fmt is None:
        ext = Path(path).suffix.lower()
        fmt = "tiff" if ext in (".tif", ".tiff") else "dng" if ext == ".dng" else "png"
    if fmt.lower() not in FORMATS:
        raise ValueError(f"--format expects png, tiff or dng, got '{fmt}'")
    fmt = fmt.lower()
    if fmt == "png":
        if bits not in (None, 8):
            raise ValueError("a PNG is written with 8 bits per channel: use --format tiff for 16 or 32")
        return fmt, 8
    if fmt == "tiff":
        return fmt, bits or 8
    if bits not in (None, 32):
        raise ValueError("a DNG is always 32-bit float: --bits can only be 32")
    return fmt, 32


class Planes:
    """Film planes held on the host (a denoised film): encoded on the device as a render's film is."""

    def __init__(self, rgb: np.ndarray, weight: np.ndarray, scene):
        self.rgb, self.weight, self.scene = rgb, weight, scene

    def srgb(self, ev=None, tonemap=None, bits=8):
        from . import encode_planes
        sev, stm, _ = self.scene.output()
        return encode_planes(self.rgb, self.weight, sev if ev is None else ev, stm if tonemap is None else tonemap, bits)

    def linear(self, ev=None):
        from . import encode_planes
        return encode_planes(self.rgb, self.weight, self.scene.output()[0] if ev is None else ev, 0, 32)


def encode_film(film, ev: float | None, tonemap: int | None, fmt: str, bits: int) -> bytes:
    """The file bytes (encode_film, lib.rs:716-760): tone-mapped sRGB for the PNG and the 8 and 16
    bit TIFFs, the linear exposed film (no curve, no clamp) for the 32-bit TIFF and the DNG. Colour
    only: the film's coverage is not written. `film` is a Film or Planes."""
    from . import image
    if fmt == "dng":
        return image.dng_bytes(film.linear(ev))
    if fmt == "tiff" and bits == 32:
        return image.tiff_bytes(film.linear(ev))
    px = film.srgb(ev, tonemap, bits)
    return image.png_bytes(px) if fmt == "png" else image.tiff_bytes(px)


def noisy_path(output) -> Path:
    """<out>-noisy.<ext>, where --keep-noisy writes the image without denoise (cli.rs:1375-1386)."""
    p = Path(output)
    stem = p.stem or "out"
    return p.with_name(f"{stem}-noisy{p.suffix}" if p.suffix else f"{stem}-noisy")


# ---- the render (lib.rs:239-368, 446-636) --------------------------------------------------------

class RenderOutput:
    """What a render made: the scene, its film, the samples per pixel (the most of any pixel after
    adaptive sampling), the rays cast by adaptive passes, and the adaptive state (or None)."""

    def __init__(self, scene, film, samples, adaptive=None):
        self.scene, self.film, self.samples, self.adaptive = scene, film, samples, adaptive


def render_until(rsb: bytes, samples: int, budget: float | None = None) -> RenderOutput:
    """Renders `rsb` up to `samples` samples per pixel, progressively, stopping between passes once
    `budget` seconds are spent; adaptively when RNDR.adaptive asks for it, with the denoiser's
    guide passes when RNDR.denoise does."""
    from . import Adaptive, Scene
    settings = render_settings(rsb)
    scene = Scene(rsb)
    film = scene.film()
    denoise = settings["denoise"] & DENOISE_IMAGE != 0
    start = time.perf_counter()
    spent = lambda: budget is not None and time.perf_counter() - start >= budget  # noqa: E731
    if settings["adaptive"] & ADAPTIVE_ON:
        ad = Adaptive(scene, film, samples)
        warmup = min(ADAPTIVE_WARMUP, samples) if samples > 0 else ADAPTIVE_WARMUP
        step = 1
        while True:
            passes, _ = ad.run(step, 1)
            st = ad.state()
            if passes == 0 or st["converged"] or spent():
                break
            step = min(step * 2, MAX_PASS_SAMPLES) if st["decisions"] <= 1 and st["left"] > 0 else MAX_PASS_SAMPLES
        st = ad.state()
        ad.close()
        if denoise:
            # The guides of the first round: its exact passes and the albedo of its samples.
            film.guides(0, min(warmup, st["lo"]))
        return RenderOutput(scene, film, st["hi"], st)
    if denoise:
        film.fuse_guides(True)
    done, step = 0, 1
    while done < samples:
        n = min(step, samples - done)
        film.render(done, n)
        done += n
        step = min(step * 2, MAX_PASS_SAMPLES)
        if spent():
            break
    return RenderOutput(scene, film, done)


def render(rsb: bytes, samples: int | None = None, budget: float | None = None):
    """(scene, film, samples rendered) after the progressive loop, samples defaulting to the scene's."""
    out = render_until(rsb, samples or render_settings(rsb)["max_samples"] or 16, budget)
    return out.scene, out.film, out.samples


def denoised(out: RenderOutput, strength: float) -> Planes:
    """The film with its radiance replaced by the denoiser's at `strength` (denoise_film_at,
    lib.rs:97-150): the denoised sums are those of `samples` samples in every pixel (a film whose
    pixels have their own counts is rescaled first), so its weight is `samples` everywhere."""
    sums = out.film.denoise(out.samples, strength=strength)
    weight = np.full((out.film.h, out.film.w), np.float32(out.samples), np.float32)
    return Planes(np.ascontiguousarray(sums[..., :3]), weight, out.scene)


def main(argv=None) -> int:
    ap = parser()
    args = ap.parse_args(argv)
    try:
        if args.example == (args.scene is not None):
            raise ValueError("no scene given: pass a .rsb file or --example" if not args.example
                             else "only one scene can be rendered at a time")
        fmt, bits = output_spec(args.format, args.bits, args.output)
        if args.example:
            from . import scenes
            rsb = scenes.to_rsb(scenes.example_scene())
        else:
            rsb = Path(args.scene).read_bytes()
        rsb, samples, budget = apply(rsb, args)
    except ValueError as e:
        ap.error(str(e))
    settings = render_settings(rsb)
    t0 = time.perf_counter()
    out = render_until(rsb, samples, budget)
    dt = time.perf_counter() - t0
    scene = out.scene
    ad = out.adaptive
    note = f", adaptive {ad['lo']}..{ad['hi']} spp in {ad['decisions']} rounds" if ad else ""
    print(f"{scene.width}x{scene.height}, {out.samples} spp{note}, {dt:.3f} s", file=sys.stderr)

    def write(path, film):
        path = Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        path.write_bytes(encode_film(film, args.ev, args.tonemap, fmt, bits))
        print(f"wrote {path}")

    strength = settings["denoise_strength"]
    if settings["denoise"] & DENOISE_IMAGE and strength > 0.0:
        t1 = time.perf_counter()
        clean = denoised(out, strength)
        print(f"denoised in {time.perf_counter() - t1:.3f} s", file=sys.stderr)
        write(args.output, clean)
        if settings["denoise"] & DENOISE_KEEP_NOISY:
            write(noisy_path(args.output), out.film)
    else:
        write(args.output, out.film)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
