"""The oracle's section view (Q1) against the reference (engine/crates/rt-core/src/render/
section_tests.rs, geometry/section.rs, scene/rsb.rs:1070): the Q1 fixture (E5 cut in two by a capped
plane, the floor exempt from it) at 4 spp has the pinned hash; the same file without its SECT
section, or with a plane that cuts nothing, is the E5 scene of before, bit for bit; the reader
refuses a zero normal and a second SECT with the reference's words."""
import struct
from pathlib import Path

import numpy as np
import pytest

from repackshot_b200.__main__ import _sections

GOLDEN = Path(__file__).resolve().parent / "golden"


def q1() -> bytes:
    return (GOLDEN / "q1.rsb").read_bytes()


def with_section(rsb: bytes, payload: bytes | None, copies: int = 1) -> bytes:
    """The file with its SECT section replaced by `payload` (None: removed), `copies` times."""
    for tag, start, at, n in _sections(rsb):
        if tag == b"SECT":
            new = b"" if payload is None else (b"SECT" + struct.pack("<I", len(payload)) + payload) * copies
            return rsb[:start] + new + rsb[at + n:]
    raise AssertionError("no SECT section")


def film_hash(oracle_lib, rsb: bytes, samples: int = 4) -> int:
    o = oracle_lib.OracleScene(rsb)
    rgb, w, _, _, _ = o.render_film(0, samples, threads=16)
    return oracle_lib.fnv1a(oracle_lib.resolve(rgb, w))


def test_q1_has_the_pinned_hash(oracle_lib, pins):
    assert film_hash(oracle_lib, q1()) == pins["film_hashes"]["q1_section_4spp"]


@pytest.mark.parametrize("payload", [None, struct.pack("<I4f", 1, 0.0, 0.0, 1.0, 1.0e5)], ids=["no section", "far plane"])
def test_a_section_that_cuts_nothing_is_the_scene_of_before(oracle_lib, pins, payload):
    # section_tests.rs:28-44: without the section, or with everything on the kept side, the E5 film.
    assert film_hash(oracle_lib, with_section(q1(), payload)) == pins["film_hashes"]["e5_hdri_4spp"]


def test_the_reader_refuses_a_zero_normal_and_a_second_section(oracle_lib):
    with pytest.raises(Exception, match="RSB section SECT is invalid: section normal is zero"):
        oracle_lib.OracleScene(with_section(q1(), struct.pack("<I4f", 1, 0.0, 0.0, 0.0, 5.0)))
    with pytest.raises(Exception, match="RSB section SECT appears more than once"):
        oracle_lib.OracleScene(with_section(q1(), struct.pack("<I4f", 1, 1.0, 0.0, 0.0, 0.0), copies=2))


def test_an_uncapped_cut_differs_from_the_capped_one(oracle_lib, pins):
    # Without the cap flag the cut spheres show their inside: the image changes.
    assert film_hash(oracle_lib, with_section(q1(), struct.pack("<I4f", 0, 1.0, 0.0, 0.0, 0.0))) != \
        pins["film_hashes"]["q1_section_4spp"]


# ---- the rules one by one, on a synthetic scene (repackshot_b200.scenes.section_scene) -------------

CAP = 0xFFFFFFFF


def synthetic(oracle_lib):
    from repackshot_b200 import scenes
    return oracle_lib.OracleScene(scenes.to_rsb(scenes.section_scene()))


def test_closed_solids_are_capped_and_open_or_thin_ones_are_not(oracle_lib):
    from rays import random_rays
    o = synthetic(oracle_lib)
    rays = random_rays(60000, (-250, -400, 5), (250, 400, 150), seed=41)
    hits, _ = o.trace(rays, camera=False)
    caps = hits[hits[:, 1] == CAP, 0]
    counts = {i: int((caps == i).sum()) for i in range(8)}
    # 0: the welded, rotated and scaled cube; 1: the inward cube; 4: the cube hidden to the camera.
    assert counts[0] > 50 and counts[1] > 50 and counts[4] > 50, counts
    # 2: the open box; 3: the thin-walled cube; 5, 6: exempt; 7: the slices (open).
    assert counts[2] == counts[3] == counts[5] == counts[6] == counts[7] == 0, counts
    seen, _ = o.trace(rays, camera=True)
    assert not ((seen[:, 0] == 4) & (seen[:, 1] == CAP)).any(), "camera rays see no cap of a hidden instance"


def ray(origin, direction, t_max=np.inf):
    return np.array([[*origin, *direction, 1.0e-3, t_max]], np.float32)


def test_the_studio_is_found_behind_at_most_48_surfaces(oracle_lib):
    o = synthetic(oracle_lib)
    # Inside the exempt hollow box on the removed side, looking along +x at its wall (x = 320):
    # behind 13 slices the wall is found, behind 56 the search gives up and the ray sees nothing.
    near, _ = o.trace(ray((280.25, 0.0, 75.0), (1.0, 0.0, 0.0)))
    assert near[0, 0] == 6 and near[0, 1] != CAP
    far, _ = o.trace(ray((215.75, 0.0, 75.0), (1.0, 0.0, 0.0)))
    assert far[0, 0] == 0xFFFFFFFF
    assert o.occluded(ray((280.25, 0.0, 75.0), (1.0, 0.0, 0.0)))[0] == 1
    assert o.occluded(ray((215.75, 0.0, 75.0), (1.0, 0.0, 0.0)))[0] == 0

