"""The command line on the GPU (python -m repackshot_b200, the reference's `rt` for one scene).

* --denoise at 4 spp on the example: the 32-bit TIFF at 0 stops holds the denoised means the
  reference pins (rt-post/src/denoise/tests.rs:369-378, 587-592), and --keep-noisy's file the
  example's pinned film (render.rs:1036-1065).
* --size renders the resized scene, pixel for pixel the oracle's image of it.
* --noise / --adaptive give the film of one rtg_adaptive_run to convergence, whatever the passes;
  with --denoise, the adaptive film denoised with its first round's guides (lib.rs:97-150).
* a spent time budget stops after the first pass; a denoise strength of 0 writes the plain image.
"""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


def run(tmp_path: Path, name: str, *argv) -> Path:
    from repackshot_b200.__main__ import main
    out = tmp_path / name
    assert main(["-o", str(out), *argv]) == 0
    return out


def tiff_floats(path: Path) -> np.ndarray:
    from test_image_files import read_tiff
    _, px = read_tiff(path.read_bytes())
    return np.frombuffer(px, "<f4").copy()


def test_denoised_example_keeps_the_reference_pins(rtg, tmp_path, pins):
    out = run(tmp_path, "example.tif", "--example", "--samples", "4", "--denoise", "--keep-noisy", "--bits", "32", "--ev", "0")
    assert rtg.fnv1a(tiff_floats(out)) == pins["denoised"]["example_4spp"]
    assert rtg.fnv1a(tiff_floats(tmp_path / "example-noisy.tif")) == pins["film_hashes"]["example_4spp"]


def test_size_renders_the_resized_scene(rtg, tmp_path, oracle_lib):
    from repackshot_b200 import scenes
    from repackshot_b200.__main__ import with_render_settings
    from repackshot_b200.image import read_png
    got = read_png(run(tmp_path, "small.png", "--example", "--size", "48x32", "--samples", "2").read_bytes())
    assert got.shape == (32, 48, 3)
    rsb = with_render_settings(scenes.to_rsb(scenes.example_scene()), width=48, height=32)
    rgb, wt, _, _, _ = oracle_lib.OracleScene(rsb).render_film(0, 2, threads=8)
    ev, tonemap, _ = rtg.Scene(rsb).output()
    want, _ = oracle_lib.film_encode(rgb, wt, ev, tonemap)
    assert np.array_equal(got.reshape(-1, 3), want)


def adaptive_rsb():
    from repackshot_b200 import scenes
    from repackshot_b200.__main__ import with_render_settings
    return with_render_settings(scenes.to_rsb(scenes.example_scene()), width=96, height=64, adaptive=1, noise_threshold=0.05)


def test_adaptive_flags_give_the_adaptive_film(rtg, tmp_path):
    got = tiff_floats(run(tmp_path, "ad.tif", "--example", "--size", "96x64", "--noise", "5", "--samples", "48", "--bits", "32",
                          "--ev", "0"))
    s = rtg.Scene(adaptive_rsb())
    f = s.film()
    ad = rtg.Adaptive(s, f, 48)
    ad.run(0)
    st = ad.state()
    ad.close()
    assert st["converged"] and st["lo"] < st["hi"]
    want = f.linear(0.0).reshape(-1)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_adaptive_film_is_denoised_with_its_first_round_guides(rtg, tmp_path, oracle_lib):
    got = tiff_floats(run(tmp_path, "adn.tif", "--example", "--size", "96x64", "--noise", "5", "--samples", "48", "--denoise",
                          "--denoise-strength", "0.5", "--bits", "32", "--ev", "0"))
    s = rtg.Scene(adaptive_rsb())
    f = s.film()
    ad = rtg.Adaptive(s, f, 48)
    ad.run(0)
    hi = ad.state()["hi"]
    ad.close()
    f.guides(0, 16)
    den = f.denoise(hi, strength=0.5)
    want = oracle_lib.film_linear(den[..., :3], np.full(den.shape[:2], np.float32(hi), np.float32), 0.0).reshape(-1)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_a_spent_budget_stops_after_the_first_pass(rtg, tmp_path, oracle_lib):
    from repackshot_b200 import scenes
    from repackshot_b200.image import read_png
    got = read_png(run(tmp_path, "budget.png", "--example", "--samples", "64", "--max-seconds", "0.000001").read_bytes())
    rsb = scenes.to_rsb(scenes.example_scene())
    rgb, wt, _, _, _ = oracle_lib.OracleScene(rsb).render_film(0, 1, threads=8)
    ev, tonemap, _ = rtg.Scene(rsb).output()
    want, _ = oracle_lib.film_encode(rgb, wt, ev, tonemap)
    assert np.array_equal(got.reshape(-1, 3), want)


def test_zero_strength_writes_the_image_without_denoise(rtg, tmp_path, pins):
    out = run(tmp_path, "zero.tif", "--example", "--samples", "4", "--denoise", "--denoise-strength", "0", "--keep-noisy",
              "--bits", "32", "--ev", "0")
    assert rtg.fnv1a(tiff_floats(out)) == pins["film_hashes"]["example_4spp"]
    assert not (tmp_path / "zero-noisy.tif").exists()


def test_encode_planes_is_the_film_encoding(rtg):
    from repackshot_b200 import scenes
    s = rtg.Scene(scenes.to_rsb(scenes.example_scene()))
    f = s.film()
    f.render(0, 3)
    rgb, wt, _, _ = f.read()
    for bits in (8, 16):
        assert np.array_equal(rtg.encode_planes(rgb, wt, 1.5, 3, bits), f.srgb(1.5, 3, bits))
    assert np.array_equal(rtg.encode_planes(rgb, wt, -1.0, 0, 32).view(np.uint32), f.linear(-1.0).view(np.uint32))
