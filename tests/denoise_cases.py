"""Inputs of the denoiser tests (engine/crates/rt-post/src/denoise/tests.rs): the example with its
guide passes at n samples (tests.rs:338 example_with_guides) through the oracle, and the denoised
means a pinned hash is taken over (tests.rs:361)."""
import numpy as np


def rgba_sums(rgb, alpha):
    """denoise.rs:321 rgba_sums: radiance and coverage, 4 per pixel."""
    return np.concatenate([np.asarray(rgb, np.float32).reshape(-1, 3), np.asarray(alpha, np.float32).reshape(-1, 1)], axis=1)


def means(sums, samples):
    """tests.rs:361: the RGB means sum * (1 / n) of RGBA sums, in float32."""
    inv = np.float32(1.0) / np.float32(samples)
    return (np.asarray(sums, np.float32).reshape(-1, 4)[:, :3] * inv).astype(np.float32)


def fnv1a_floats(values) -> int:
    h = 0x811C9DC5
    for b in np.ascontiguousarray(values, np.float32).tobytes():
        h = ((h ^ b) * 0x01000193) & 0xFFFFFFFF
    return h


def example_input(oracle_lib, samples):
    """The example's film and guides at `samples` samples, as the denoiser's input words."""
    from repackshot_b200 import scenes
    o = oracle_lib.OracleScene(scenes.to_rsb(scenes.example_scene()))
    rgb, _, alpha, lum2, _ = o.render_film(0, samples, threads=8)
    albedo, normal, depth, part, material = o.guides(samples)
    words = oracle_lib.denoise_words(rgba_sums(rgb, alpha), lum2, albedo, normal, depth, part, material)
    return o, words, (rgb, alpha, lum2), (albedo, normal, depth, part, material)
