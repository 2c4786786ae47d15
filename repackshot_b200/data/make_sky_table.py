"""Writes repackshot_b200/data/sky_table.f32: the physical sky's coefficient table.

The Repackshot engine's physical daylight sky (ENVR.sky_model 0, its E5c scene) evaluates the
Hosek-Wilkie functional form with coefficients the Repackshot authors fitted to their own
atmosphere simulation (engine/crates/rt-sky, seed 0xe5c5c1e) and published as data in
engine/crates/rt-core/src/sky_table.rs. A film with that sky is reproducible to the bit only with
those exact numbers, so they are carried here as data: 3240 coefficients ([turbidity 1..10]
[ground albedo 0, 1][R, G, B][Bezier control point 0..5][A..I]) then 360 radiances
([turbidity][albedo][R, G, B][control point]), little-endian f32. The script checks the SHA-256
the reference states for exactly these values before writing.

Usage: python repackshot_b200/data/make_sky_table.py /path/to/reference
"""
from __future__ import annotations

import hashlib
import re
import struct
import sys
from pathlib import Path

OUT = Path(__file__).resolve().parent / "sky_table.f32"
N_COEFFICIENTS, N_RADIANCE = 3240, 360


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python repackshot_b200/data/make_sky_table.py /path/to/reference (the Repackshot checkout to read)")
    src = (Path(sys.argv[1]) / "engine" / "crates" / "rt-core" / "src" / "sky_table.rs").read_text()
    want = re.search(r'pub const SHA256: &str = "([0-9a-f]{64})";', src).group(1)

    def block(name, n):
        body = src[src.index(f"pub const {name}: [f32; {n}] = ["):]
        body = body[body.index("[", body.index("=")) + 1:body.index("];")]
        vals = [float(t) for t in re.findall(r"-?\d+(?:\.\d+)?(?:e-?\d+)?", body)]
        assert len(vals) == n, (name, len(vals))
        return vals

    vals = block("COEFFICIENTS", N_COEFFICIENTS) + block("RADIANCE", N_RADIANCE)
    data = struct.pack(f"<{len(vals)}f", *vals)
    got = hashlib.sha256(data).hexdigest()
    if got != want:
        sys.exit(f"SHA-256 {got} does not match the reference's {want}")
    OUT.write_bytes(data)
    print(f"wrote {OUT} ({len(vals)} values, SHA-256 {got})")


if __name__ == "__main__":
    main()
