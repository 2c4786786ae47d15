"""Writes tests/golden/reference_pins.json: the known answers the Repackshot reference pins for
its path tracer, read from the reference's own source tree (run where it is checked out):

* the FNV-1a film hashes of the example scene (engine/crates/rt-core/src/render.rs:1036-1065);
* the PCG32 demo outputs and the mix64 value (engine/crates/rt-core/src/rng.rs:62-108);
* the first Sobol points (engine/crates/rt-core/src/sampler.rs:403-430);
* SHA-256 of the six energy tables (engine/crates/rt-core/src/bsdf/energy_table.rs), as the
  little-endian bytes of their u16 values and f32 bit patterns;
* SHA-256 of the example scene file (tests/fixtures/example.rsb);
* the FNV-1a film hashes of the E5 scene with its HDRI and with the classic sky (render.rs:1106-1109)
  and SHA-256 of the HDRI scene's file (tests/fixtures/e5.rsb); the E5c scene's hash with the
  physical sky (render.rs:1128);
* the E11 film hash (render.rs:1250) and SHA-256 of the Blackman-Harris inverse-CDF table
  (pixel_filter.rs:64, 256 little-endian f32);
* the L5 film hash (render.rs:1531), SHA-256 of its file (tests/fixtures/l5.rsb), and the two
  hand-written test profiles it carries (tests/fixtures/ies/*.ies), written to
  tests/golden/ies_profiles.json;
* the hash of six adaptive-sampling decisions of the synthetic 45 x 37 image
  (engine/crates/rt-core/src/adaptive/tests.rs:497-534);
* the three K3 interior views (tests/fixtures/k3-{plan,panorama,fisheye}.rsb, copied beside this
  script as test inputs) and their pinned 4-spp film hashes (render/k3_tests.rs:17-22);
* the hashes of the denoised example: the full filter at 4 spp and the viewport's at 2 and 4 spp
  (engine/crates/rt-post/src/denoise/tests.rs:392, 527-528).
* the Q1 section view (tests/fixtures/q1.rsb, copied beside this script as a test input) and its
  pinned 4-spp film hash (render/section_tests.rs:11);
* the hashes of the exact passes and the 4-sample albedo and alpha of the example and the E5 example
  (engine/crates/rt-core/src/render/passes_tests.rs:365-398, 865-868);
* the golden TIFF and DNG files the reference's writers must reproduce byte for byte
  (tests/fixtures/tiff/*, made by engine/crates/rt-cli/tests/tiff_golden.rs:48-80 from 4 x 4 and
  50 x 60 images of closed-form samples), copied to tests/golden/tiff/.

Usage: python tests/golden/make_golden.py /path/to/reference
"""
from __future__ import annotations

import hashlib
import json
import re
import struct
import sys
from pathlib import Path

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py /path/to/reference (the Repackshot checkout to read)")
REF = Path(sys.argv[1])
CORE = REF / "engine" / "crates" / "rt-core" / "src"
OUT = Path(__file__).resolve().parent / "reference_pins.json"
TIFF_GOLDEN = ("rgb8.tif", "rgba8.tif", "rgb16.tif", "rgba16-300dpi.tif", "rgb32.tif", "rgba32.tif", "strips.tif",
               "linear.dng")


def pinned(src: str, name: str) -> int:
    m = re.search(r"const " + name + r": u32 = (0x[0-9a-f_]+);", src)
    return int(m.group(1).replace("_", ""), 16)


def main():
    render = (CORE / "render.rs").read_text()
    denoise = (REF / "engine" / "crates" / "rt-post" / "src" / "denoise" / "tests.rs").read_text()
    rng = (CORE / "rng.rs").read_text()
    sampler = (CORE / "sampler.rs").read_text()
    table = (CORE / "bsdf" / "energy_table.rs").read_text()
    pins = {
        "example_4spp": pinned(render, "PINNED_EXAMPLE_4SPP"),
        "tile_centre_240_176_s3": pinned(render, "PINNED_CENTRE"),
        "tile_small_sphere_48_144_s3": pinned(render, "PINNED_SMALL_SPHERE"),
        "e5_hdri_4spp": pinned(render, "PINNED_E5_HDRI_4SPP"),
        "e5_sky_4spp": pinned(render, "PINNED_E5_SKY_4SPP"),
        "e5c_physical_sky_4spp": pinned(render, "PINNED_E5C_SKY_4SPP"),
        "e11_edges_4spp": pinned(render, "PINNED_E11_EDGES_4SPP"),
        "l5_ies_4spp": pinned(render, "PINNED_L5_IES_4SPP"),
    }
    block = rng[rng.index("fn matches_the_reference_implementation"):]
    block = block[:block.index("]")]
    pcg = [int(h.replace("_", ""), 16) for h in re.findall(r"0x[0-9a-f_]+", block)]
    m = re.search(r"mix64\((0x[0-9A-F_]+)\), (0x[0-9A-F_]+)\)", rng)
    sob = sampler[sampler.index("fn the_first_points_match_the_published_sequence"):]
    sob = sob[sob.index("let expected"):sob.index("];")]
    points = [[float(x) for x in row.split(",") if x.strip()] for row in re.findall(r"\[([0-9., ]+)\]", sob)]
    tables = {}
    for name in ["ALBEDO", "SCHLICK", "CLEAR_IN", "CLEAR_OUT", "ALBEDO_AVG", "SCHLICK_AVG"]:
        mm = re.search(r"pub static " + name + r": \[(u16|f32); \d+\] = \[(.*?)\];", table, re.S)
        vals = [v.strip() for v in mm.group(2).split(",") if v.strip()]
        if mm.group(1) == "u16":
            raw = struct.pack("<%dH" % len(vals), *[int(v) for v in vals])
        else:
            raw = struct.pack("<%df" % len(vals), *[float(v) for v in vals])
        tables[name] = {"count": len(vals), "sha256": hashlib.sha256(raw).hexdigest()}
    pf = (CORE / "pixel_filter.rs").read_text()
    body = pf[pf.index("pub const BLACKMAN_HARRIS_INV_CDF"):]
    body = body[body.index("= [") + 3:body.index("];")]
    bh = [float(v) for v in re.findall(r"-?\d+\.\d+(?:e-?\d+)?", body)]
    bh_raw = struct.pack("<%df" % len(bh), *bh)
    example = (REF / "tests" / "fixtures" / "example.rsb").read_bytes()
    e5 = (REF / "tests" / "fixtures" / "e5.rsb").read_bytes()
    l5 = (REF / "tests" / "fixtures" / "l5.rsb").read_bytes()
    ies = {name: (REF / "tests" / "fixtures" / "ies" / (name + ".ies")).read_text() for name in ("downlight-symmetric", "wall-washer")}
    (OUT.parent / "ies_profiles.json").write_text(json.dumps(ies, indent=1) + "\n")
    # The three interior views of K3 as the reference writes them (rt --write-k3-*-example), kept
    # as test inputs: the room's split boxes, cylinder and sphere, the disk uplight, the physical
    # sky through a thin pane, an orthographic plan with its ceiling hidden to the camera and the
    # panoramic cameras; their films at 4 spp are pinned in render/k3_tests.rs.
    k3 = (CORE / "render" / "k3_tests.rs").read_text()
    for view in ("plan", "panorama", "fisheye"):
        data = (REF / "tests" / "fixtures" / f"k3-{view}.rsb").read_bytes()
        (OUT.parent / f"k3-{view}.rsb").write_bytes(data)
        pins[f"k3_{view}_4spp"] = pinned(k3, f"PINNED_K3_{view.upper()}_4SPP")
    # The TIFF and DNG files rt-cli/tests/tiff_golden.rs compares rt_core::tiff and rt_core::dng with.
    (OUT.parent / "tiff").mkdir(exist_ok=True)
    for name in TIFF_GOLDEN:
        (OUT.parent / "tiff" / name).write_bytes((REF / "tests" / "fixtures" / "tiff" / name).read_bytes())
    # The Q1 parity scene: E5 cut in two by a capped section, the floor exempt from it.
    (OUT.parent / "q1.rsb").write_bytes((REF / "tests" / "fixtures" / "q1.rsb").read_bytes())
    pins["q1_section_4spp"] = pinned((CORE / "render" / "section_tests.rs").read_text(), "PINNED_Q1_SECTION_4SPP")
    passes_src = (CORE / "render" / "passes_tests.rs").read_text()
    pass_keys = ("albedo", "normal", "depth", "part_id", "material_id", "coc")
    passes = {
        "example": {k: pinned(passes_src, "PINNED_PASS_" + k.upper()) for k in pass_keys},
        "e5_hdri": {k: pinned(passes_src, "PINNED_E5_PASS_" + k.upper()) for k in pass_keys},
    }
    passes["example"]["alpha"] = pinned(passes_src, "PINNED_PASS_ALPHA")
    passes["e5_hdri"]["alpha"] = pinned(passes_src, "PINNED_E5_PASS_ALPHA")
    out = {
        "source": "Repackshot reference tree (engine crate rt-core), read by tests/golden/make_golden.py",
        "film_hashes": pins,
        "pcg32_seed42_stream54": pcg,
        "mix64": [int(m.group(1).replace("_", ""), 16), int(m.group(2).replace("_", ""), 16)],
        "sobol_first_points_gray_order": points,
        "energy_tables": tables,
        "example_rsb": {"bytes": len(example), "sha256": hashlib.sha256(example).hexdigest()},
        "e5_rsb": {"bytes": len(e5), "sha256": hashlib.sha256(e5).hexdigest()},
        "l5_rsb": {"bytes": len(l5), "sha256": hashlib.sha256(l5).hexdigest()},
        "blackman_harris_inv_cdf": {"count": len(bh), "sha256": hashlib.sha256(bh_raw).hexdigest()},
        "e10_synthetic_decisions": pinned((CORE / "adaptive" / "tests.rs").read_text(), "PINNED_E10_DECISIONS"),
        "passes_4spp": passes,
        "denoised": {k: pinned(denoise, "PINNED_DENOISED_" + k.upper()) for k in
                     ("example_4spp", "viewport_example_2spp", "viewport_example_4spp")},
    }
    OUT.write_text(json.dumps(out, indent=1) + "\n")
    print(OUT)


if __name__ == "__main__":
    main()
