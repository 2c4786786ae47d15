"""The C-ABI library on the CPU: it loads, exports every function include/repackshot_b200.h
declares (and the Python table binds exactly those), and its host-side logic answers the
reference's way without a GPU: status codes for bad handles and null pointers
(engine/crates/rt-wasm/src/lib.rs:37-53), parse errors and "unsupported:" refusals at load
(rt_scene_load, ffi.rs:56-66), and a loud CUDA error, not a fallback, when no GPU is present.
No test here launches a kernel.
"""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "repackshot_b200.h"


def header_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:uint32_t|void)\s+(rtg_\w+)\s*\(", text, flags=re.M)))


def header_define(name):
    """The value of an integer #define: a literal or a shift such as (1ull << 22)."""
    m = re.search(rf"#define\s+{name}\s+([^/\n]+)", HEADER.read_text())
    expr = re.sub(r"(?<=[0-9a-fA-F])(ull|ul|u)\b", "", m.group(1).strip())
    assert re.fullmatch(r"[0-9a-fxA-FX()<\s]+", expr), expr
    return int(eval(expr))


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    from repackshot_b200 import build
    build.build()  # no-op when the library is up to date
    rtg.lib()
    return rtg


def test_header_declares_the_entry_points():
    names = header_functions()
    assert "rtg_scene_load" in names and "rtg_render_progressive" in names
    assert len(names) >= 20


def test_library_exports_every_declared_function(rtg):
    L = ctypes.CDLL(str(rtg.LIB_PATH))
    missing = [n for n in header_functions() if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_table_binds_exactly_the_header(rtg):
    assert sorted(rtg.ABI) == header_functions()


def test_version_and_constants(rtg):
    assert rtg.lib().rtg_version() == header_define("RTG_ABI_VERSION")
    assert rtg.MAX_TILE_PIXELS == header_define("RTG_MAX_TILE_PIXELS")
    for name in ("OK", "BAD_HANDLE", "BAD_TILE", "NULL_POINTER", "BAD_SCENE", "CUDA_ERROR", "STACK_OVERFLOW", "BAD_FILM"):
        assert getattr(rtg, "STATUS_" + name) == header_define("RTG_STATUS_" + name)


def test_features_are_the_reference_bits_of_what_loads(rtg):
    # rt_features (ffi.rs:22): FEATURE_SECTION = 4 (Q1), FEATURE_IES = 8 (L5) and FEATURE_CAMERAS = 16
    # (K3), rt-core lib.rs:88,93,100; the texture, program, drop, glass, weather and nesting bits stay clear.
    bits = header_define("RTG_FEATURE_SECTION") | header_define("RTG_FEATURE_IES") | header_define("RTG_FEATURE_CAMERAS")
    assert rtg.features() == bits == 28
    assert (rtg.FEATURE_SECTION, rtg.FEATURE_IES, rtg.FEATURE_CAMERAS) == (4, 8, 16)


def test_bad_handles_and_null_pointers(rtg):
    L = rtg.lib()
    out = (ctypes.c_float * 12)()
    assert L.rtg_scene_free(0) == rtg.STATUS_BAD_HANDLE
    assert L.rtg_scene_free(4096) == rtg.STATUS_BAD_HANDLE
    assert L.rtg_render_tile(4096, 0, 0, 2, 2, 0, out) == rtg.STATUS_BAD_HANDLE
    assert L.rtg_render_tile_rgba(4096, 0, 0, 1, 1, 0, out) == rtg.STATUS_BAD_HANDLE
    assert L.rtg_render_tile_alpha(4096, 0, 0, 4, 4, 0, out) == rtg.STATUS_BAD_HANDLE
    assert L.rtg_render_tile_alpha(4096, 0, 0, 4, 4, 0, None) == rtg.STATUS_NULL_POINTER
    assert L.rtg_film_free(4096) == rtg.STATUS_BAD_FILM
    assert L.rtg_film_linear(4096, 0.0, out) == rtg.STATUS_BAD_FILM
    assert L.rtg_encode_planes(None, out, 2, 2, 0.0, 0, 8, out) == rtg.STATUS_NULL_POINTER
    assert L.rtg_encode_planes(out, out, 0, 2, 0.0, 0, 8, out) == rtg.STATUS_BAD_TILE
    assert L.rtg_encode_planes(out, out, 2, 2, 0.0, 0, 12, out) == rtg.STATUS_BAD_ARGUMENT
    assert L.rtg_film_create(4096, 0, 0, 4, 4) == 0
    assert L.rtg_render_progressive(4096, 1, 0, 1, None) == rtg.STATUS_BAD_HANDLE
    assert L.rtg_scene_update(4096, b"RSB1", 4) == rtg.STATUS_BAD_HANDLE
    assert L.rtg_scene_load(None, 0) == 0
    assert rtg.error_message() == "null pointer"
    # adaptive sampling: null pointers and empty images before any device work
    planes = (ctypes.c_uint32 * 16)()
    assert L.rtg_adaptive_decide(8, 8, 0.0, 0.0, 0, planes, None, planes, planes, planes) == rtg.STATUS_NULL_POINTER
    assert L.rtg_adaptive_decide(0, 8, 0.0, 0.0, 0, planes, planes, planes, planes, planes) == rtg.STATUS_BAD_TILE
    assert L.rtg_render_block_rgba(4096, 0, 0, 1, 1, 0, 0, None) == rtg.STATUS_NULL_POINTER
    assert L.rtg_render_block_rgba(4096, 0, 0, 1, 1, 0, 0, out) == rtg.STATUS_BAD_HANDLE
    assert L.rtg_adaptive_create(4096, 1, 0) == 0
    assert L.rtg_adaptive_run(4096, 16, 0, None, None) == rtg.STATUS_BAD_HANDLE
    assert L.rtg_adaptive_state(0, planes) == rtg.STATUS_BAD_HANDLE
    assert L.rtg_adaptive_free(4096) == rtg.STATUS_BAD_HANDLE


def test_malformed_scenes_are_refused_with_a_message(rtg, example_rsb):
    assert rtg.scene_load(b"not a scene") == 0
    assert rtg.error_message()
    assert rtg.scene_load(example_rsb[: len(example_rsb) // 2]) == 0
    assert rtg.error_message()


@pytest.mark.parametrize("change, words", [
    (lambda s: setattr(s.materials[0], "scatter_mm", 5.0) or setattr(s.materials[0], "transmission", 1.0), "scattering media"),
    (lambda s: setattr(s, "floor_mode", 2), "shadow catcher"),
    (lambda s: setattr(s.materials[0], "bevel_mm", 1.0), "bevel"),
    (lambda s: setattr(s.materials[0], "abbe", 30.0) or setattr(s.materials[0], "transmission", 1.0), "dispersive"),
    (lambda s: setattr(s, "caustic_photons", 100000), "caustic photon maps"),
])
def test_features_outside_the_path_are_refused(rtg, change, words):
    from repackshot_b200 import scenes
    s = scenes.cfg0_scene()
    change(s)
    assert rtg.scene_load(scenes.to_rsb(s)) == 0
    msg = rtg.error_message()
    assert msg.startswith("unsupported:") and words in msg


def test_without_a_gpu_a_valid_scene_fails_loudly(rtg, cfg0_rsb):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert rtg.scene_load(cfg0_rsb) == 0
    assert "CUDA" in rtg.error_message()


@pytest.mark.parametrize("section, copies, words", [
    ((1, 0.0, 0.0, 0.0, 5.0), 1, "RSB section SECT is invalid: section normal is zero"),
    ((1, 1.0, 0.0, 0.0, 0.0), 2, "RSB section SECT appears more than once"),
])
def test_bad_sections_are_refused_as_the_reference_refuses_them(rtg, section, copies, words):
    # rsb.rs:1070 parse_section and set_once: the load stops before any device work.
    from repackshot_b200 import scenes
    s = scenes.example_scene()
    s.section = section
    rsb = scenes.to_rsb(s)
    if copies == 2:
        rsb += rsb[rsb.index(b"SECT"):]
    assert rtg.scene_load(rsb) == 0
    assert rtg.error_message() == words
