"""Film output on the GPU (rtg_film_srgb8 / rtg_film_srgb16): the bytes of every tone curve,
exposure and bit depth equal the oracle's encoding of the same film sums, and the command line
(python -m repackshot_b200) writes a PNG whose pixels are the oracle's image of the example."""
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
