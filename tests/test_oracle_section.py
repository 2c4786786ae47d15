"""The oracle's section view (Q1) against the reference (engine/crates/rt-core/src/render/
section_tests.rs, geometry/section.rs, scene/rsb.rs:1070): the Q1 fixture (E5 cut in two by a capped
plane, the floor exempt from it) at 4 spp has the pinned hash; the same file without its SECT
section, or with a plane that cuts nothing, is the E5 scene of before, bit for bit; the reader
refuses a zero normal and a second SECT with the reference's words."""
import struct
from pathlib import Path

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
