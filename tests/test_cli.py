"""The command line's host logic on the CPU: the RNDR settings read from and written into an RSB
file, the flags applied as Options::apply applies them (engine/crates/rt-cli/src/cli.rs:350-403),
the refusals worded as the reference's parser words them (cli.rs:744-1013), and <out>-noisy paths
(cli.rs:1375-1386). A file the flags rewrote still loads in the oracle with the new settings."""
from types import SimpleNamespace

import numpy as np
import pytest

from repackshot_b200 import scenes
from repackshot_b200.__main__ import (ADAPTIVE_ON, DENOISE_IMAGE, DENOISE_KEEP_NOISY, RNDR_FIELDS, apply, main, noisy_path,
                                      render_settings, with_render_settings)


def flags(**kw):
    base = dict(size=None, denoise=False, keep_noisy=False, denoise_strength=None, caustics=None, pixel_filter=None,
                edge_samples=None, adaptive=False, noise=None, threads=None, samples=None, max_seconds=None)
    base.update(kw)
    return SimpleNamespace(**base)


def test_render_settings_are_the_scene_description():
    sc = scenes.example_scene()
    got = render_settings(scenes.to_rsb(sc))
    for name in ("width", "height", "max_samples", "seed", "tonemap", "max_depth", "pixel_filter", "edge_supersample"):
        assert got[name] == getattr(sc, name), name
    assert got["exposure_ev"] == np.float32(sc.exposure_ev)
    assert got["denoise"] == 0 and got["denoise_strength"] == 1.0 and got["adaptive"] == 0


def test_rewritten_settings_keep_every_other_section_and_load(oracle_lib):
    rsb = scenes.to_rsb(scenes.example_scene())
    new = with_render_settings(rsb, width=32, height=24, denoise=3, noise_threshold=0.25)
    got = render_settings(new)
    assert (got["width"], got["height"], got["denoise"], got["noise_threshold"]) == (32, 24, 3, 0.25)
    assert new[:rsb.index(b"RNDR")] == rsb[:rsb.index(b"RNDR")]
    assert len(new) - new.index(b"RNDR") == 8 + 4 * len(RNDR_FIELDS)
    assert with_render_settings(new) == new
    rgb, weight, _, _, _ = oracle_lib.OracleScene(new).render_film(0, 1, threads=4)
    assert weight.shape == (24, 32) and (weight == 1).all()
    with pytest.raises(KeyError):
        with_render_settings(rsb, colour=1)


def test_a_file_without_render_settings_gets_them():
    rsb = scenes.to_rsb(scenes.example_scene())
    at = rsb.index(b"RNDR")
    bare = rsb[:at]
    assert render_settings(bare)["width"] == 640
    assert render_settings(with_render_settings(bare, width=7))["width"] == 7


def test_flags_change_the_render_settings():
    rsb = scenes.to_rsb(scenes.example_scene())
    sc = scenes.example_scene()
    out, samples, budget = apply(rsb, flags())
    assert out == rsb and samples == sc.max_samples and budget is None
    out, samples, budget = apply(rsb, flags(size="48X32", denoise=True, keep_noisy=True, denoise_strength="0.5",
                                             pixel_filter="fine", edge_samples="4", noise="2.5", samples="8", max_seconds="1.5",
                                             threads="3"))
    s = render_settings(out)
    assert (s["width"], s["height"]) == (48, 32)
    assert s["denoise"] == DENOISE_IMAGE | DENOISE_KEEP_NOISY and s["denoise_strength"] == 0.5
    assert s["pixel_filter"] == 3 and s["edge_supersample"] == 4
    assert s["adaptive"] & ADAPTIVE_ON and s["noise_threshold"] == np.float32(0.025)
    assert samples == 8 and budget == 1.5
    s = render_settings(apply(rsb, flags(adaptive=True))[0])
    assert s["adaptive"] == ADAPTIVE_ON and s["noise_threshold"] == 0.0
    assert apply(rsb, flags(max_seconds="0"))[2] is None
    assert apply(with_render_settings(rsb, max_seconds=2.0, max_samples=0), flags())[1:] == (16, 2.0)


@pytest.mark.parametrize("kw,message", [
    (dict(size="640"), "--size expects WxH such as 1280x720, got '640'"),
    (dict(size="0x10"), "--size must be between 1x1 and 16384x16384"),
    (dict(denoise_strength="1.5"), "--denoise-strength expects a number from 0 to 1, got '1.5'"),
    (dict(pixel_filter="blur"), "--pixel-filter expects none, standard, soft or fine, got 'blur'"),
    (dict(edge_samples="17"), "--edge-samples expects a number from 1 to 16, got '17'"),
    (dict(noise="-1"), "--noise expects a percentage from 0 to 100, got '-1'"),
    (dict(caustics="5000000"), "--caustics expects a number of photons up to 4194304, got '5000000'"),
    (dict(samples="0"), "--samples expects a positive integer, got '0'"),
    (dict(threads="x"), "--threads expects a positive integer, got 'x'"),
    (dict(max_seconds="-2"), "--max-seconds expects a non-negative number of seconds, got '-2'"),
])
def test_flags_are_refused_as_the_reference_refuses_them(kw, message):
    rsb = scenes.to_rsb(scenes.example_scene())
    with pytest.raises(ValueError) as e:
        apply(rsb, flags(**kw))
    assert str(e.value) == message


def test_noisy_paths():
    assert str(noisy_path("out/a.png")) == "out/a-noisy.png"
    assert str(noisy_path("a.tiff")) == "a-noisy.tiff"
    assert str(noisy_path("render")) == "render-noisy"


@pytest.mark.parametrize("argv", [["-o", "a.png"], ["a.rsb", "--example", "-o", "a.png"], ["--example", "-o", "a.png", "--bits", "16"],
                                  ["--example", "-o", "a.dng", "--bits", "8"], ["--example", "-o", "a.png", "--size", "3"]])
def test_bad_command_lines_exit_with_the_usage(argv, capsys):
    with pytest.raises(SystemExit) as e:
        main(argv)
    assert e.value.code == 2
    assert "error:" in capsys.readouterr().err
