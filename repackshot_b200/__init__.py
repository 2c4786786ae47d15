"""repackshot_b200: a B200-native (sm_100a) drop-in for the progressive sample-and-accumulate
render of the Repackshot engine's path tracer.

The native library ``librtg.so`` (built by ``repackshot_b200.build``) exports the C ABI declared
in ``include/repackshot_b200.h``; this module binds it with ctypes and mirrors the Rust host API
of the reference's rt-wasm crate (engine/crates/rt-wasm/src/lib.rs: ``scene_load``,
``scene_free``, ``error_message``, ``render_tile``, ``render_tile_rgba``), with the same status
codes, plus device films for progressive rendering.

There is no CPU fallback: every call runs the CUDA kernels, and importing the binding without the
built library (or without a GPU at call time) raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path
from typing import Optional

import numpy as np

STATUS_OK = 0
STATUS_BAD_HANDLE = 1
STATUS_BAD_TILE = 2
STATUS_NULL_POINTER = 3
STATUS_BAD_SCENE = 4
STATUS_CUDA_ERROR = 16
STATUS_STACK_OVERFLOW = 17
STATUS_BAD_FILM = 18
STATUS_BAD_ARGUMENT = 19
MAX_TILE_PIXELS = 1 << 22
QUEUE_GRAPH = 1
ADJOINT_CORRELATED = 1

LIB_PATH = Path(__file__).resolve().parent / "librtg.so"
_lib: Optional[ctypes.CDLL] = None

_u32, _u64, _f = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p
# The ABI of include/repackshot_b200.h: name -> (restype, argtypes).
ABI = {
    "rtg_version": (_u32, []),
    "rtg_features": (_u32, []),
    "rtg_scene_load": (_u32, [ctypes.c_char_p, _u32]),
    "rtg_scene_update": (_u32, [_u32, ctypes.c_char_p, _u32]),
    "rtg_scene_error_len": (_u32, []),
    "rtg_scene_error_copy": (None, [ctypes.c_void_p]),
    "rtg_scene_free": (_u32, [_u32]),
    "rtg_render_tile": (_u32, [_u32, _u32, _u32, _u32, _u32, _u32, _f]),
    "rtg_render_tile_rgba": (_u32, [_u32, _u32, _u32, _u32, _u32, _u32, _f]),
    "rtg_film_create": (_u32, [_u32, _u32, _u32, _u32, _u32]),
    "rtg_film_free": (_u32, [_u32]),
    "rtg_film_clear": (_u32, [_u32]),
    "rtg_render_progressive": (_u32, [_u32, _u32, _u32, _u32, ctypes.POINTER(_u64)]),
    "rtg_render_progressive_noalloc": (_u32, [_u32, _u32, _u32, _u32, ctypes.POINTER(_u64)]),
    "rtg_queue_create": (_u32, [_u32]),
    "rtg_queue_add": (_u32, [_u32, ctypes.c_char_p, _u32, _u32, _u32, ctypes.POINTER(_u32)]),
    "rtg_queue_run": (_u32, [_u32, _u32, ctypes.POINTER(_u64)]),
    "rtg_queue_free": (_u32, [_u32]),
    "rtg_adjoint_params": (_u32, [_u32, ctypes.POINTER(_u32), ctypes.POINTER(_u32)]),
    "rtg_render_adjoint": (_u32, [_u32, _u32, _f, _u32, _u32, _u32, ctypes.POINTER(ctypes.c_float), _f, _u32, _f]),
    "rtg_film_srgb8": (_u32, [_u32, ctypes.c_float, _u32, _f]),
    "rtg_film_srgb16": (_u32, [_u32, ctypes.c_float, _u32, _f]),
    "rtg_film_linear": (_u32, [_u32, ctypes.c_float, _f]),
    "rtg_encode_planes": (_u32, [_f, _f, _u32, _u32, ctypes.c_float, _u32, _u32, _f]),
    "rtg_mesh_solid": (_u32, [_f, _u32, _f, _u32, _f]),
    "rtg_scene_output": (_u32, [_u32, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(_u32), ctypes.POINTER(_u32)]),
    "rtg_film_read": (_u32, [_u32, _f, _f, _f, _f]),
    "rtg_film_device": (_u32, [_u32, _f, _f, _f, _f]),
    "rtg_render_paths": (_u32, [_u32, _f, _u32, _f]),
    "rtg_trace_rays": (_u32, [_u32, _f, _u32, _u32, _f]),
    "rtg_scene_stats": (_u32, [_u32, _f]),
    "rtg_set_path_capacity": (_u32, [_u32, _u32]),
    "rtg_set_tuning": (_u32, [_u32, _f, _u32]),
    "rtg_get_tuning": (_u32, [_u32, _f, _u32]),
    "rtg_autotune": (_u32, [_u32, _u32, _u32, _u32, _u32, _u32, _u32, _f, _u32, ctypes.POINTER(_u32)]),
    "rtg_timing": (_u32, [_u32, _u32, _u32, _f]),
    "rtg_set_stream": (_u32, [_u32, ctypes.c_void_p]),
    "rtg_synchronize": (_u32, [_u32]),
    "rtg_adaptive_decide": (_u32, [_u32, _u32, ctypes.c_float, ctypes.c_float, _u32, _f, _f, _f, _f, _f]),
    "rtg_render_block_rgba": (_u32, [_u32, _u32, _u32, _u32, _u32, _u32, _u32, _f]),
    "rtg_adaptive_create": (_u32, [_u32, _u32, _u32]),
    "rtg_adaptive_run": (_u32, [_u32, _u32, _u32, ctypes.POINTER(_u32), ctypes.POINTER(_u64)]),
    "rtg_adaptive_state": (_u32, [_u32, _f]),
    "rtg_adaptive_counts": (_u32, [_u32, _f, _f]),
    "rtg_adaptive_free": (_u32, [_u32]),
    "rtg_render_tile_passes": (_u32, [_u32, _u32, _u32, _u32, _u32, _u32, _f]),
    "rtg_render_tile_albedo": (_u32, [_u32, _u32, _u32, _u32, _u32, _u32, _f]),
    "rtg_render_tile_alpha": (_u32, [_u32, _u32, _u32, _u32, _u32, _u32, _f]),
    "rtg_denoise": (_u32, [_u32, _u32, _u32, _u32, _u32, _u32, _u32, _f, _f]),
    "rtg_denoise_with": (_u32, [_u32, ctypes.c_float, _u32, _u32, _u32, _u32, _u32, _u32, _u32, _f, _f]),
    "rtg_denoise_halo": (_u32, [_u32]),
    "rtg_film_guides": (_u32, [_u32, _u32, _u32, _u32]),
    "rtg_film_guides_fused": (_u32, [_u32, _u32, _u32]),
    "rtg_film_denoise": (_u32, [_u32, _u32, ctypes.c_float, _u32, _f]),
}


class RtgError(RuntimeError):
    """A non-zero status of the C ABI, with the library's last error message."""

    def __init__(self, status: int, message: str = ""):
        super().__init__(f"status {status}: {message}" if message else f"status {status}")
        self.status = status


def lib() -> ctypes.CDLL:
    """The loaded native library. Raises when it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m repackshot_b200.build`")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in ABI.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def error_message() -> str:
    """The last error (rt_scene_error_len / rt_scene_error_copy)."""
    L = lib()
    n = L.rtg_scene_error_len()
    buf = ctypes.create_string_buffer(max(n, 1))
    L.rtg_scene_error_copy(buf)
    return buf.raw[:n].decode("utf-8", "replace")


def _check(status: int):
    if status != STATUS_OK:
        raise RtgError(status, error_message() if status in (STATUS_CUDA_ERROR, STATUS_STACK_OVERFLOW) else "")


def scene_load(rsb: bytes) -> int:
    """rt_scene_load: a handle > 0, or 0 with ``error_message()`` set."""
    return lib().rtg_scene_load(rsb, len(rsb))


def scene_free(handle: int) -> int:
    return lib().rtg_scene_free(handle)


def render_tile(handle: int, x: int, y: int, w: int, h: int, sample_index: int, rgba: bool = False):
    """rt_render_tile(_rgba): (status, w*h*3 or w*h*4 float32 array)."""
    out = np.zeros(w * h * (4 if rgba else 3), np.float32) if 0 < w * h <= MAX_TILE_PIXELS else np.zeros(0, np.float32)
    fn = lib().rtg_render_tile_rgba if rgba else lib().rtg_render_tile
    status = fn(handle, x, y, w, h, sample_index, _ptr(out) if out.size else None)
    return status, out


class Scene:
    """A loaded scene (owns its handle)."""

    def __init__(self, rsb: bytes):
        self.handle = scene_load(rsb)
        if self.handle == 0:
            raise RtgError(STATUS_BAD_SCENE, error_message())
        self._read_stats()

    def _read_stats(self):
        st = np.zeros(8, np.float64)
        _check(lib().rtg_scene_stats(self.handle, _ptr(st)))
        self.width, self.height, self.max_depth = int(st[0]), int(st[1]), int(st[2])
        self.triangles, self.nodes, self.leaf_triangles, self.build_seconds = int(st[3]), int(st[4]), int(st[5]), float(st[6])

    def update(self, rsb: bytes):
        """rt_scene_update: replaces the scene; a file without MESH sections keeps the meshes (and,
        with unchanged instances, the device trees). On error raises and the scene is unchanged."""
        status = lib().rtg_scene_update(self.handle, rsb, len(rsb))
        if status != STATUS_OK:
            raise RtgError(status, error_message())
        self._read_stats()

    def close(self):
        if self.handle:
            scene_free(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render_tile(self, x, y, w, h, sample_index, rgba=False) -> np.ndarray:
        status, out = render_tile(self.handle, x, y, w, h, sample_index, rgba)
        _check(status)
        return out

    def film(self, x=0, y=0, w=None, h=None) -> "Film":
        return Film(self, x, y, self.width if w is None else w, self.height if h is None else h)

    def render_paths(self, xys: np.ndarray) -> np.ndarray:
        """Radiance of explicit (x, y, sample) paths: (n, 5) = r, g, b, alpha, 0."""
        xys = np.ascontiguousarray(xys, dtype=np.uint32).reshape(-1, 3)
        out = np.zeros((len(xys), 5), np.float32)
        _check(lib().rtg_render_paths(self.handle, _ptr(xys), len(xys), _ptr(out)))
        return out

    def trace(self, rays: np.ndarray, camera=False, any_hit=False) -> np.ndarray:
        """Nearest hits (n, 3) u32 = instance, triangle, t bits; or any-hit flags (n,)."""
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = len(rays)
        out = np.zeros(n if any_hit else 3 * n, np.uint32)
        mode = (1 if camera else 0) | (2 if any_hit else 0)
        _check(lib().rtg_trace_rays(self.handle, _ptr(rays), n, mode, _ptr(out)))
        return out if any_hit else out.reshape(n, 3)

    def adjoint_params(self):
        """(materials, lights): the adjoint's gradient has 4 entries per material, 1 per light."""
        nm, nl = _u32(0), _u32(0)
        _check(lib().rtg_adjoint_params(self.handle, ctypes.byref(nm), ctypes.byref(nl)))
        return int(nm.value), int(nl.value)

    def adjoint(self, film: "Film", target: np.ndarray, first: int, count: int, correlated: bool = False):
        """rtg_render_adjoint: (loss, gradients, residual). gradients: per material d/d base R, G,
        B and d/d alpha, then per light d/d power. By default decorrelated by sample halves, the
        second drawn with the seed adjoint_seed_b(seed) (an unbiased gradient for fitting);
        `correlated` gives the derivative of this very estimate."""
        nm, nl = self.adjoint_params()
        target = np.ascontiguousarray(target, dtype=np.float32).reshape(-1)
        grads = np.zeros(4 * nm + nl, np.float32)
        residual = np.zeros(2, np.float32)
        loss = ctypes.c_float(0.0)
        status = lib().rtg_render_adjoint(self.handle, film.handle, _ptr(target), first, count, ADJOINT_CORRELATED if correlated else 0,
                                          ctypes.byref(loss), _ptr(grads), len(grads), _ptr(residual))
        if status != STATUS_OK:
            raise RtgError(status, error_message())
        return float(loss.value), grads, residual

    def output(self):
        """(exposure in stops, tone curve, samples per pixel) of the scene's RNDR section."""
        ev, tm, spp = ctypes.c_float(0.0), _u32(0), _u32(0)
        _check(lib().rtg_scene_output(self.handle, ctypes.byref(ev), ctypes.byref(tm), ctypes.byref(spp)))
        return float(ev.value), int(tm.value), int(spp.value)

    def set_path_capacity(self, paths: int):
        _check(lib().rtg_set_path_capacity(self.handle, paths))

    def set_tuning(self, ray_bits: int | None = None, shadow_sort: bool | None = None, material_sort: bool | None = None,
                   capacity: int | None = None, l2_persist: bool | None = None, tail_paths: int | None = None):
        """rtg_set_tuning: how the scene's waves order their rays and paths (None keeps a value)."""
        cur = self.tuning()
        new = [cur["ray_bits"] if ray_bits is None else int(ray_bits),
               cur["shadow_sort"] if shadow_sort is None else int(bool(shadow_sort)),
               cur["material_sort"] if material_sort is None else int(bool(material_sort)),
               cur["capacity"] if capacity is None else int(capacity),
               cur["l2_persist"] if l2_persist is None else int(bool(l2_persist)),
               cur["tail_paths"] if tail_paths is None else int(tail_paths)]
        v = np.array(new, np.uint32)
        _check(lib().rtg_set_tuning(self.handle, _ptr(v), 6))

    def autotune(self, first: int, count: int, x: int = 0, y: int = 0, w: int | None = None, h: int | None = None) -> dict:
        """rtg_autotune: times candidate tunings on samples [first, first + count) of the rectangle
        (default: the whole image) and keeps the fastest; returns it and every candidate's time."""
        w = self.width if w is None else w
        h = self.height if h is None else h
        report = np.zeros((24, 7), np.float64)
        n = _u32(0)
        _check(lib().rtg_autotune(self.handle, x, y, w, h, first, count, _ptr(report), 24, ctypes.byref(n)))
        tried = [{"ray_bits": int(r[0]), "shadow_sort": int(r[1]), "material_sort": int(r[2]), "capacity": int(r[3]),
                  "l2_persist": int(r[4]), "tail_paths": int(r[5]), "ms": float(r[6])} for r in report[:int(n.value)]]
        return {"chosen": self.tuning(), "tried": tried}

    def tuning(self) -> dict:
        """rtg_get_tuning: ray-sort bits, shadow sort, material sort, paths per wave (0: automatic),
        the L2 window, the tail limit (0: off)."""
        v = np.zeros(6, np.uint32)
        _check(lib().rtg_get_tuning(self.handle, _ptr(v), 6))
        return {"ray_bits": int(v[0]), "shadow_sort": int(v[1]), "material_sort": int(v[2]), "capacity": int(v[3]),
                "l2_persist": int(v[4]), "tail_paths": int(v[5])}

    def timing(self, enable: bool, reset: bool = False):
        """(extend ms, extend launches, camera+extension rays, shadow rays, kernels launched)
        since the last reset."""
        out = np.zeros(5, np.float64)
        _check(lib().rtg_timing(self.handle, int(enable), int(reset), _ptr(out)))
        return float(out[0]), int(out[1]), int(out[2]), int(out[3]), int(out[4])

    def set_stream(self, stream_ptr: int | None):
        """Runs this scene's work on a caller-owned cudaStream_t (e.g. torch's current stream)."""
        _check(lib().rtg_set_stream(self.handle, stream_ptr))

    def synchronize(self):
        _check(lib().rtg_synchronize(self.handle))


class Film:
    """A device film over an image rectangle (rt-core Film): rgb, weight, alpha, lum2 sums."""

    def __init__(self, scene: Scene, x: int, y: int, w: int, h: int, handle: int = 0):
        self.scene, self.x, self.y, self.w, self.h = scene, x, y, w, h
        self.handle = handle or lib().rtg_film_create(scene.handle, x, y, w, h)
        if self.handle == 0:
            raise RtgError(STATUS_BAD_FILM, error_message())

    def render(self, first: int, count: int) -> int:
        """Accumulates samples [first, first + count); returns the rays cast."""
        rays = _u64(0)
        _check(lib().rtg_render_progressive(self.scene.handle, self.handle, first, count, ctypes.byref(rays)))
        return int(rays.value)

    def render_noalloc(self, first: int, count: int) -> int:
        """As ``render``, with the path state in the library's fixed device array
        (rtg_render_progressive_noalloc): no device memory is allocated."""
        rays = _u64(0)
        _check(lib().rtg_render_progressive_noalloc(self.scene.handle, self.handle, first, count, ctypes.byref(rays)))
        return int(rays.value)

    def read(self, out=None):
        """(rgb (h, w, 3), weight, alpha, lum2 (h, w)) copied to host."""
        n = self.w * self.h
        if out is None:
            out = (np.zeros(3 * n, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32))
        _check(lib().rtg_film_read(self.handle, *[_ptr(a) for a in out]))
        rgb, w, a, l2 = out
        return rgb.reshape(self.h, self.w, 3), w.reshape(self.h, self.w), a.reshape(self.h, self.w), l2.reshape(self.h, self.w)

    def srgb(self, ev: float | None = None, tonemap: int | None = None, bits: int = 8) -> np.ndarray:
        """Film::to_srgb8_tonemapped / to_srgb16_tonemapped: (h, w, 3) uint8 or uint16. Exposure and
        tone curve default to the scene's RNDR settings."""
        sev, stm, _ = self.scene.output()
        ev = sev if ev is None else ev
        tonemap = stm if tonemap is None else tonemap
        out = np.zeros((self.h, self.w, 3), np.uint8 if bits == 8 else np.uint16)
        fn = lib().rtg_film_srgb8 if bits == 8 else lib().rtg_film_srgb16
        _check(fn(self.handle, ev, tonemap, _ptr(out)))
        return out

    def linear(self, ev: float | None = None) -> np.ndarray:
        """Film::to_linear_exposed (image.rs:218): (h, w, 3) float32, the resolved film times 2^ev,
        no tone curve and no clamp. Exposure defaults to the scene's RNDR setting."""
        ev = self.scene.output()[0] if ev is None else ev
        out = np.zeros((self.h, self.w, 3), np.float32)
        _check(lib().rtg_film_linear(self.handle, ev, _ptr(out)))
        return out

    def resolve(self) -> np.ndarray:
        """Film::resolve (image.rs:158): rgb * (1 / weight), black where no sample."""
        rgb, w, _, _ = self.read()
        inv = np.where(w > 0, np.float32(1.0) / np.where(w > 0, w, np.float32(1.0)), np.float32(0.0)).astype(np.float32)
        return (rgb * inv[..., None]).astype(np.float32)

    def clear(self):
        _check(lib().rtg_film_clear(self.handle))

    def guides(self, first: int, count: int):
        """Renders the film's guide passes: the exact passes, and the albedo of samples
        [first, first + count) added to its albedo sums (rtg_film_guides)."""
        _check(lib().rtg_film_guides(self.scene.handle, self.handle, first, count))

    def fuse_guides(self, enable: bool = True):
        """rtg_film_guides_fused: the exact passes now, and the albedo of every later render
        taken from its own camera rays."""
        _check(lib().rtg_film_guides_fused(self.scene.handle, self.handle, int(enable)))

    def denoise(self, samples: int, preset: int = 0, strength: float = 1.0, out=None):
        """The film denoised on the device (rtg_film_denoise): (h, w, 4) RGBA sums; ``out=False``
        leaves the result on the device and returns None."""
        if out is False:
            _check(lib().rtg_film_denoise(self.handle, preset, float(strength), samples, None))
            return None
        out = np.zeros((self.h, self.w, 4), np.float32) if out is None else out
        _check(lib().rtg_film_denoise(self.handle, preset, float(strength), samples, _ptr(out)))
        return out

    def close(self):
        if self.handle:
            lib().rtg_film_free(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def adaptive_decide(width: int, height: int, ev: float, target: float, cap: int, counts, sums, lum2):
    """rt_adaptive_decide (rt-wasm/src/lib.rs:660) through rtg_adaptive_decide: (active bytes per
    block, six u32 words: round, active blocks, blocks, then the bits of the threshold, the largest
    error and the remaining pixel-samples). ``sums`` holds 4 floats a pixel (RGBA)."""
    cols, rows = (width + 7) // 8, (height + 7) // 8
    counts = np.ascontiguousarray(counts, np.uint32).reshape(-1)
    sums = np.ascontiguousarray(sums, np.float32).reshape(-1)
    lum2 = np.ascontiguousarray(lum2, np.float32).reshape(-1)
    if counts.size != cols * rows or sums.size != 4 * width * height or lum2.size != width * height:
        raise ValueError("plane sizes do not match the image")
    active = np.zeros(max(cols * rows, 1), np.uint8)
    words = np.zeros(6, np.uint32)
    _check(lib().rtg_adaptive_decide(width, height, float(ev), float(target), cap, _ptr(counts), _ptr(sums), _ptr(lum2), _ptr(active),
                                     _ptr(words)))
    return active[:cols * rows], words


def render_block_rgba(handle: int, x: int, y: int, w: int, h: int, sample_index: int, iteration: int = 0):
    """rt_render_block_rgba: (status, w*h*4 float32 array)."""
    out = np.zeros(w * h * 4, np.float32) if 0 < w * h <= MAX_TILE_PIXELS else np.zeros(0, np.float32)
    status = lib().rtg_render_block_rgba(handle, x, y, w, h, sample_index, iteration, _ptr(out) if out.size else None)
    return status, out


STATUS_BAD_DENOISE = 5


def denoise(words, width: int, height: int, samples: int, preset: int = 0, strength: float = 1.0, origin_y: int = 0, rows=None,
            y0=None, y1=None):
    """rt_denoise_with through rtg_denoise_with: the denoised RGBA sums of rows y0..y1 of the band.
    ``words`` holds the band's planes as u32 words (14 a pixel)."""
    rows = height if rows is None else rows
    y0 = origin_y if y0 is None else y0
    y1 = origin_y + rows if y1 is None else y1
    words = np.ascontiguousarray(words, np.uint32)
    out = np.zeros(max((y1 - y0) * width * 4, 1), np.float32)
    _check(lib().rtg_denoise_with(preset, float(strength), width, height, origin_y, rows, samples, y0, y1, _ptr(words), _ptr(out)))
    return out[:(y1 - y0) * width * 4]


def tile_passes(handle: int, x: int, y: int, w: int, h: int, mask: int = 0x3E):
    """rt_render_tile_passes: the planes of ``mask`` as u32 words (status, words)."""
    per = sum(c for bit, c in ((2, 3), (4, 1), (8, 1), (16, 1), (32, 1)) if mask & bit)
    out = np.zeros(max(w * h * per, 1), np.uint32)
    st = lib().rtg_render_tile_passes(handle, x, y, w, h, mask, _ptr(out))
    return st, out[:w * h * per]


def tile_albedo(handle: int, x: int, y: int, w: int, h: int, sample_index: int):
    """rt_render_tile_albedo: (status, w*h*3 float32)."""
    out = np.zeros(max(w * h * 3, 1), np.float32)
    st = lib().rtg_render_tile_albedo(handle, x, y, w, h, sample_index, _ptr(out))
    return st, out[:w * h * 3]


def adjoint_seed_b(seed: int) -> int:
    """The render seed the decorrelated adjoint draws its second half of samples with: the seed's
    complement (32 bits)."""
    return (~int(seed)) & 0xFFFFFFFF


def tile_alpha(handle: int, x: int, y: int, w: int, h: int, sample_index: int):
    """rt_render_tile_alpha: (status, w*h float32 coverage)."""
    out = np.zeros(max(w * h, 1), np.float32)
    st = lib().rtg_render_tile_alpha(handle, x, y, w, h, sample_index, _ptr(out))
    return st, out[:w * h]


FEATURE_SECTION, FEATURE_IES, FEATURE_CAMERAS = 4, 8, 16


def encode_planes(rgb: np.ndarray, weight: np.ndarray, ev: float, tonemap: int, bits: int) -> np.ndarray:
    """rtg_encode_planes: film planes in host memory ((h, w, 3) sums and (h, w) weights) encoded on
    the device as Film.srgb (bits 8 or 16) or Film.linear (bits 32) encode a render's film."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    weight = np.ascontiguousarray(weight, np.float32)
    h, w = weight.shape
    if rgb.shape != (h, w, 3):
        raise ValueError("rgb must be (h, w, 3) and weight (h, w)")
    dtype = {8: np.uint8, 16: np.uint16, 32: np.float32}.get(bits)
    if dtype is None:
        raise ValueError("bits must be 8, 16 or 32")
    out = np.zeros((h, w, 3), dtype)
    _check(lib().rtg_encode_planes(_ptr(rgb), _ptr(weight), w, h, ev, tonemap, bits, _ptr(out)))
    return out


def mesh_solid(positions: np.ndarray, indices: np.ndarray) -> int:
    """rtg_mesh_solid: 0 open, 1 closed and wound outward, 2 closed and wound inward (solid.rs)."""
    p = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    i = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    out = _u32(0)
    _check(lib().rtg_mesh_solid(_ptr(p), len(p), _ptr(i), len(i), ctypes.byref(out)))
    return int(out.value)


def features() -> int:
    """rt_features: the reference's FEATURE_* bits this engine reads (section views, IES lights, interior
    cameras)."""
    return int(lib().rtg_features())


class Adaptive:
    """An adaptive render (E10, rt-core/src/adaptive.rs) of a scene into one of its whole-image
    films, to convergence or ``cap`` samples a pixel (0: none)."""

    def __init__(self, scene: Scene, film: Film, cap: int):
        self.scene, self.film = scene, film
        self.handle = lib().rtg_adaptive_create(scene.handle, film.handle, cap)
        if self.handle == 0:
            raise RtgError(STATUS_BAD_ARGUMENT, error_message())

    def run(self, pass_samples: int = 16, max_passes: int = 0):
        """Renders passes until converged (or ``max_passes``): (passes, rays)."""
        passes, rays = _u32(0), _u64(0)
        _check(lib().rtg_adaptive_run(self.handle, pass_samples, max_passes, ctypes.byref(passes), ctypes.byref(rays)))
        return int(passes.value), int(rays.value)

    def state(self) -> dict:
        w = np.zeros(16, np.uint32)
        _check(lib().rtg_adaptive_state(self.handle, _ptr(w)))
        keys = ("round", "done", "left", "iteration", "converged", "decisions", "lo", "hi")
        out = {k: int(v) for k, v in zip(keys, w[:8])}
        out["last"] = w[8:14].copy()
        out["cols"], out["rows"] = int(w[14]), int(w[15])
        return out

    def counts(self):
        """(samples per block now, (rows, cols) u32; active blocks, (rows, cols) u8)."""
        st = self.state()
        samples = np.zeros(st["rows"] * st["cols"], np.uint32)
        active = np.zeros(st["rows"] * st["cols"], np.uint8)
        _check(lib().rtg_adaptive_counts(self.handle, _ptr(samples), _ptr(active)))
        return samples.reshape(st["rows"], st["cols"]), active.reshape(st["rows"], st["cols"])

    def close(self):
        if self.handle:
            lib().rtg_adaptive_free(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Queue:
    """A batched render queue over a loaded scene (rtg_queue_*): jobs are variants of the scene
    (RSB files without MESH sections) with sample ranges, rendered together by ``run``."""

    def __init__(self, scene: Scene):
        self.scene = scene
        self.handle = lib().rtg_queue_create(scene.handle)
        if self.handle == 0:
            raise RtgError(STATUS_BAD_HANDLE, error_message())

    def add(self, rsb: bytes, first: int, count: int, width: int, height: int) -> Film:
        """Queues samples [first, first + count) of the variant ``rsb`` (whose image is width x
        height); returns the film it will render into."""
        film = _u32(0)
        status = lib().rtg_queue_add(self.handle, rsb, len(rsb), first, count, ctypes.byref(film))
        if status != STATUS_OK:
            raise RtgError(status, error_message())
        return Film(self.scene, 0, 0, width, height, handle=int(film.value))

    def run(self, graph: bool = False) -> int:
        """Renders every queued job; returns the rays cast."""
        rays = _u64(0)
        status = lib().rtg_queue_run(self.handle, QUEUE_GRAPH if graph else 0, ctypes.byref(rays))
        if status != STATUS_OK:
            raise RtgError(status, error_message())
        return int(rays.value)

    def close(self):
        if self.handle:
            lib().rtg_queue_free(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fnv1a(values: np.ndarray) -> int:
    """FNV-1a over the little-endian bytes of float32 values (the reference's film hash)."""
    b = np.ascontiguousarray(values, dtype="<f4").view(np.uint8)
    h = 0x811C9DC5
    for byte in b.tobytes():
        h = ((h ^ byte) * 0x01000193) & 0xFFFFFFFF
    return h
