"""Inputs of the adaptive-sampling tests, restated from engine/crates/rt-core/src/adaptive/tests.rs
in float32 with the reference's order of operations: grey pixels of n samples (tests.rs:33), the
half-noisy image (tests.rs:77), the image with one noisy block (tests.rs:142), the synthetic image
and the six decisions over it that the reference pins (tests.rs:459-534).

A decision function here has the signature of rt_adaptive_decide (rt-wasm/src/lib.rs:660):
``decide(width, height, ev, target, cap, counts, sums_rgba, lum2) -> (active bytes, six words)``;
the oracle's and the CUDA path's both fit it.
"""
import struct

import numpy as np

f32 = np.float32


def grey(n, mean, spread):
    """Sums and squared sums of n samples of luminance mean +- spread, half each way."""
    s, l2 = f32(0.0), f32(0.0)
    for i in range(n):
        v = f32(f32(mean) + f32(spread)) if i % 2 == 0 else f32(f32(mean) - f32(spread))
        s = f32(s + v)
        l2 = f32(l2 + f32(v * v))
    return s, l2


def half_noisy(width, height, split, spread, n):
    noisy, clean = grey(n, 0.5, spread), grey(n, 0.5, 0.0)
    sums = np.zeros((height, width, 4), f32)
    lum2 = np.zeros((height, width), f32)
    for x in range(width):
        s, l2 = noisy if x < split else clean
        sums[:, x, :3] = s
        sums[:, x, 3] = f32(n)
        lum2[:, x] = l2
    return sums, lum2


def one_noisy_block(counts):
    """64 x 64, block 0 +-0.3 around 0.5, the rest +-0.001; RGBA sums (alpha = n, unused)."""
    sums = np.zeros((64, 64, 4), f32)
    lum2 = np.zeros((64, 64), f32)
    cache = {}
    for y in range(64):
        for x in range(64):
            spread = 0.3 if x < 8 and y < 8 else 0.001
            n = int(counts[(y // 8) * 8 + x // 8])
            key = (n, spread)
            if key not in cache:
                cache[key] = grey(n, 0.5, spread)
            s, l2 = cache[key]
            sums[y, x] = (s, s, s, f32(n))
            lum2[y, x] = l2
    return sums, lum2


def _hash(x):
    x = x.astype(np.uint32)
    x ^= x >> np.uint32(16)
    x = (x * np.uint32(0x7FEB352D)).astype(np.uint32)
    x ^= x >> np.uint32(15)
    x = (x * np.uint32(0x846CA68B)).astype(np.uint32)
    x ^= x >> np.uint32(16)
    return x


def synthetic(samples, width, height, rnd):
    """The synthetic image of tests.rs:459 for per-block samples `samples` (rows x cols)."""
    with np.errstate(over="ignore"):
        p = np.arange(width * height, dtype=np.uint32).reshape(height, width)
        v = _hash((p * np.uint32(2654435761)) ^ np.uint32((rnd * 0x9E3779B9) & 0xFFFFFFFF))
    ys, xs = np.mgrid[0:height, 0:width]
    n = samples[ys // 8, xs // 8].astype(f32)
    c = [(v >> np.uint32(s) & np.uint32(0xFF)).astype(f32) / f32(255.0) for s in (0, 8, 16)]
    band = np.where(xs < width // 3, f32(0.5), f32(0.05)).astype(f32)
    corner = np.where(ys < 9, f32(2.0), f32(1.0)).astype(f32)
    spread = ((v >> np.uint32(24) & np.uint32(0xFF)).astype(f32) / f32(255.0) * band).astype(f32) * corner
    lum = (f32(0.2126) * c[0] + f32(0.7152) * c[1]).astype(f32) + f32(0.0722) * c[2]
    sums = np.stack([c[0] * n, c[1] * n, c[2] * n, n], axis=-1).astype(f32)
    lum2 = ((lum * lum + spread * spread).astype(f32) * n).astype(f32)
    return sums, lum2


def fnv1a(data: bytes) -> int:
    h = 0x811C9DC5
    for b in data:
        h = ((h ^ b) * 0x01000193) & 0xFFFFFFFF
    return h


def synthetic_decisions(decide, rounds=6):
    """tests.rs:500: the hash of the decisions over `rounds` synthetic images of a 45 x 37 image
    (a target of 2 %, an exposure of +0.5, a cap of 200), the round state kept as
    Adaptive::{new, advance, decide} keep it (adaptive.rs:349-535)."""
    w, h, cap = 45, 37, 200
    cols, rows = (w + 7) // 8, (h + 7) // 8
    counts = np.zeros(rows * cols, np.int64)
    active = np.ones(rows * cols, bool)
    rnd_samples = min(16, cap)
    out = bytearray()
    for rnd in range(rounds):
        quota = np.where(active, np.minimum(rnd_samples, np.maximum(cap - counts, 0)), 0)
        counts = counts + quota
        sums, lum2 = synthetic(counts.reshape(rows, cols), w, h, rnd)
        act, words = decide(w, h, 0.5, 0.02, cap, counts.astype(np.uint32), sums, lum2)
        out += struct.pack("<6I", *(int(x) for x in words))
        out += bytes(np.asarray(act, np.uint8))
        active = np.asarray(act, bool)
        rnd_samples = int(words[0])
        if rnd_samples == 0:
            break
    return fnv1a(bytes(out))


def words_as_floats(words):
    return [struct.unpack("<f", struct.pack("<I", int(x)))[0] for x in words[3:6]]
