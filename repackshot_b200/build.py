"""Build recipe of the native library: the energy-table generator, the sm_100a kernels and the
C-ABI engine, linked into ``repackshot_b200/librtg.so`` (CUDA runtime linked statically, so the
library carries no dependency on a Python package).

Device code is compiled with ``-fmad=false -prec-div=true -prec-sqrt=true -ftz=false`` and host
code with ``-ffp-contract=off``: every floating-point operation is one IEEE round-to-nearest
step, as the Repackshot engine's arithmetic is.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
GEN = CSRC / "_gen"
OBJ = PKG / "_build"
LIB = PKG / "librtg.so"

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CUDA_HOME = Path(NVCC).resolve().parent.parent
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
DEVICE_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
                "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-Xptxas", "-v"]
# RTG_SHADE_MIN_BLOCKS (environment): blocks per SM the shade kernels are compiled for (default 8);
# RTG_SHORT_STACK (environment): traversal stack entries kept in shared memory (default 16).
# RTG_LEAF_STEP (environment): triangles of a leaf tested per traversal step (default 0: all).
# RTG_TRACE_MIN_BLOCKS (environment): blocks per SM the traversal kernels are compiled for (default 8).
# RTG_REFILL_MIN, RTG_SHADOW_REFILL_MIN (environment): idle lanes a k_extend / k_shadow warp waits
# for before it refills (default 8).
for _name in ("RTG_SHADE_MIN_BLOCKS", "RTG_SHORT_STACK", "RTG_LEAF_STEP", "RTG_TRACE_MIN_BLOCKS", "RTG_REFILL_MIN",
              "RTG_SHADOW_REFILL_MIN"):
    if os.environ.get(_name, "").isdigit():
        DEVICE_FLAGS.append(f"-D{_name}={os.environ[_name]}")
HOST_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-pthread", f"-I{CUDA_HOME}/include"]

HOST_SOURCES = ["rtg_scene.cpp", "rtg_section.cpp", "rtg_bitmap.cpp", "rtg_ies.cpp", "rtg_tables.cpp", "rtg_energy.cpp", "rtg_adaptive.cpp", "rtg_engine.cpp"]
DEVICE_SOURCES = ["rtg_kernels.cu", "rtg_noalloc.cu", "rtg_adaptive.cu", "rtg_denoise.cu"]


SKY_TABLE = PKG / "data" / "sky_table.f32"
# SHA-256 of the physical sky's table (little-endian f32: 3240 coefficients, then 360 radiances),
# as engine/crates/rt-core/src/sky_table.rs states it.
SKY_TABLE_SHA256 = "2329ac7376204749a317d5b31e23e17fa27950515be0f0d50018cd9c16e8a721"


def sky_table_inc() -> str:
    """The sky table as C float literals (hexadecimal: exact), after checking its SHA-256."""
    import hashlib
    import struct
    data = SKY_TABLE.read_bytes()
    if hashlib.sha256(data).hexdigest() != SKY_TABLE_SHA256:
        raise RuntimeError(f"{SKY_TABLE} does not have the physical sky table's SHA-256")
    vals = struct.unpack(f"<{len(data) // 4}f", data)
    return ",\n".join(", ".join(f"{float(v).hex()}f" for v in vals[i:i + 6]) for i in range(0, len(vals), 6)) + "\n"


def _run(cmd, log=None):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        log.write(" ".join(map(str, cmd)) + "\n" + res.stdout + res.stderr + "\n")
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(map(str, cmd))}")
    return res


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Builds ``librtg.so`` if any source is newer; returns its path."""
    GEN.mkdir(exist_ok=True)
    OBJ.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "repackshot_b200.h"]
    log = open(OBJ / "build.log", "w")
    # 1. energy tables (generated, then compiled in)
    gen_exe = OBJ / "rtg_energy_gen"
    inc = GEN / "rtg_energy_tables.inc"
    gen_deps = [CSRC / "rtg_energy_gen.cpp"] + headers
    if force or _stale(gen_exe, gen_deps):
        _run([CXX, *HOST_FLAGS, "-O2", str(CSRC / "rtg_energy_gen.cpp"), "-o", str(gen_exe)], log)
    if force or _stale(inc, [gen_exe]):
        _run([str(gen_exe), str(inc)], log)
    # 2. the physical sky's fitted table (data, checked against its SHA-256, compiled in)
    sky_inc = GEN / "rtg_sky_table.inc"
    if force or _stale(sky_inc, [SKY_TABLE]):
        sky_inc.write_text(sky_table_inc())
    objs = []
    for src in HOST_SOURCES:
        o = OBJ / (src + ".o")
        deps = [CSRC / src, inc, sky_inc] + headers
        if force or _stale(o, deps):
            _run([CXX, *HOST_FLAGS, "-c", str(CSRC / src), "-o", str(o)], log)
        objs.append(o)
    for src in DEVICE_SOURCES:
        o = OBJ / (src + ".o")
        deps = [CSRC / src] + headers
        if force or _stale(o, deps):
            _run([NVCC, *ARCH, *DEVICE_FLAGS, "-c", str(CSRC / src), "-o", str(o)], log)
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs), "-lpthread"], log)
    log.close()
    if verbose:
        sys.stdout.write((OBJ / "build.log").read_text())
    return LIB


def build_oracle() -> Path | None:
    """Builds the oracle library (test infrastructure) with its Makefile; None without make."""
    oracle = PKG.parent / "oracle"
    if not (oracle / "Makefile").exists() or shutil.which("make") is None:
        return None
    _run(["make", "-s", "-C", str(oracle)])
    return oracle / "_build" / "liborc.so"


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
