"""Film output on the GPU (rtg_film_srgb8 / rtg_film_srgb16 / rtg_film_linear): the bytes of every
tone curve, exposure and bit depth, and the linear exposed floats, equal the oracle's encoding of the
same film sums; the command line (python -m repackshot_b200) writes a PNG whose pixels are the
oracle's image of the example, and the TIFF and DNG files of the reference's command line."""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def film(example_rsb):
    import repackshot_b200 as rtg
    s = rtg.Scene(example_rsb)
    f = s.film()
    f.render(0, 4)
    return f


@pytest.mark.parametrize("tonemap", [0, 1, 2, 3, 4, 9])
@pytest.mark.parametrize("ev", [0.0, 1.5, -2.0])
def test_encoding_matches_the_oracle(film, oracle_lib, tonemap, ev):
    rgb, wt, _, _ = film.read()
    want8, want16 = oracle_lib.film_encode(rgb, wt, ev, tonemap)
    got8 = film.srgb(ev, tonemap, 8)
    got16 = film.srgb(ev, tonemap, 16)
    assert np.array_equal(got8.reshape(-1, 3), want8)
    assert np.array_equal(got16.reshape(-1, 3), want16)


def test_command_line_png(tmp_path, example_rsb, oracle_lib):
    scene_file = tmp_path / "example.rsb"
    scene_file.write_bytes(example_rsb)
    out = tmp_path / "example.png"
    subprocess.run([sys.executable, "-m", "repackshot_b200", str(scene_file), "-o", str(out), "--samples", "4"], check=True,
                   cwd=ROOT)
    from repackshot_b200.image import read_png
    got = read_png(out.read_bytes())
    o = oracle_lib.OracleScene(example_rsb)
    rgb, wt, _, _, _ = o.render_film(0, 4, threads=8)
    import repackshot_b200 as rtg
    ev, tonemap, _ = rtg.Scene(example_rsb).output()
    want, _ = oracle_lib.film_encode(rgb, wt, ev, tonemap)
    assert np.array_equal(got.reshape(-1, 3), want)


@pytest.mark.parametrize("ev", [0.0, 1.5, -2.0, 3.0])
def test_linear_film_matches_the_oracle(film, oracle_lib, ev):
    """rtg_film_linear: the resolved film times 2^ev, bit for bit the oracle's to_linear_exposed."""
    rgb, wt, _, _ = film.read()
    want = oracle_lib.film_linear(rgb, wt, ev)
    got = film.linear(ev)
    assert got.dtype == np.float32 and np.array_equal(got.reshape(-1, 3).view(np.uint32), want.view(np.uint32))


def test_command_line_tiff_and_dng(tmp_path, example_rsb, oracle_lib):
    """The files of rt-cli/tests/tiff_golden.rs:199-262 from a render of the example: the 8-bit TIFF
    holds the PNG's pixels, the 16-bit TIFF the oracle's 16-bit encoding, and the 32-bit TIFF and the
    DNG the same linear light, the oracle's exposed film, with values above 1 kept."""
    from repackshot_b200.__main__ import main
    from repackshot_b200.image import read_png
    from test_image_files import read_tiff
    scene_file = tmp_path / "example.rsb"
    scene_file.write_bytes(example_rsb)

    def run(name, *extra):
        out = tmp_path / name
        assert main([str(scene_file), "-o", str(out), "--samples", "4", *extra]) == 0
        return out.read_bytes()

    import repackshot_b200 as rtg
    ev, tonemap, _ = rtg.Scene(example_rsb).output()
    o = oracle_lib.OracleScene(example_rsb)
    rgb, wt, _, _, _ = o.render_film(0, 4, threads=8)
    want8, want16 = oracle_lib.film_encode(rgb, wt, ev, tonemap)
    linear = oracle_lib.film_linear(rgb, wt, ev)

    png = read_png(run("example.png"))
    f8, p8 = read_tiff(run("example-8.tif"))
    assert struct_shorts(f8[258]) == [8, 8, 8] and struct_shorts(f8[262]) == [2] and 339 not in f8
    assert np.array_equal(np.frombuffer(p8, np.uint8), png.reshape(-1))
    assert np.array_equal(png.reshape(-1, 3), want8)
    f16, p16 = read_tiff(run("example-16.tif", "--bits", "16"))
    assert struct_shorts(f16[258]) == [16, 16, 16]
    assert np.array_equal(np.frombuffer(p16, "<u2").reshape(-1, 3), want16)
    for name, extra in (("example-32.tif", ("--bits", "32")), ("example.dng", ())):
        fields, px = read_tiff(run(name, *extra))
        assert struct_shorts(fields[258]) == [32, 32, 32] and struct_shorts(fields[339]) == [3, 3, 3]
        got = np.frombuffer(px, "<f4").reshape(-1, 3)
        assert np.array_equal(got.view(np.uint32), linear.view(np.uint32))
        assert np.isfinite(got).all() and (got > 1.0).any()
    assert struct_shorts(read_tiff(run("example-forced.out", "--format", "tiff"))[0][262]) == [2]
    assert run("example-still.tif", "--format", "png")[:8] == b"\x89PNG\r\n\x1a\n"


def struct_shorts(entry):
    kind, count, data = entry
    assert kind == 3
    return list(np.frombuffer(data, "<u2")[:count])
