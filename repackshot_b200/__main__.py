"""Renders an RSB scene on the GPU and writes a PNG: the progressive loop of the reference's
command line (engine/crates/rt-cli/src/lib.rs:239-368, cli.rs:841-843) on this library.

    python -m repackshot_b200 SCENE.rsb -o OUT.png [--samples N] [--budget SECONDS]
                              [--ev STOPS] [--tonemap 0..4] [--bits 8|16]

Samples go in passes of 1, 2, 4, ... up to 16 sample indices (MAX_PASS_SAMPLES), each pass one
rtg_render_progressive call; with a time budget, rendering stops between passes once it is spent.
The result does not depend on the pass sizes: each pixel's samples are added in index order.
Exposure and tone curve default to the scene's RNDR settings.
"""
from __future__ import annotations

import argparse
import sys
import time

MAX_PASS_SAMPLES = 16


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


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m repackshot_b200", description=__doc__.splitlines()[0])
    ap.add_argument("scene", help="an RSB file")
    ap.add_argument("-o", "--output", required=True, help="PNG file to write")
    ap.add_argument("--samples", type=int, default=None, help="samples per pixel (default: the scene's)")
    ap.add_argument("--budget", type=float, default=None, help="stop between passes after this many seconds")
    ap.add_argument("--ev", type=float, default=None, help="exposure in stops (default: the scene's)")
    ap.add_argument("--tonemap", type=int, default=None, help="0 linear, 1 ACES, 2 filmic, 3 AgX, 4 standard")
    ap.add_argument("--bits", type=int, choices=(8, 16), default=8)
    args = ap.parse_args(argv)
    from .image import write_png
    with open(args.scene, "rb") as f:
        rsb = f.read()
    t0 = time.perf_counter()
    scene, film, done = render(rsb, args.samples, args.budget)
    write_png(args.output, film.srgb(args.ev, args.tonemap, args.bits))
    dt = time.perf_counter() - t0
    print(f"{scene.width}x{scene.height}, {done} spp, {dt:.3f} s, {scene.width * scene.height * done / dt / 1e6:.1f} Mpaths/s -> "
          f"{args.output}", file=sys.stderr)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
