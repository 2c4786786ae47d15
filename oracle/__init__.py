"""ORACLE (test infrastructure only): ctypes binding of the C++ restatement of the Repackshot
engine's path tracer (oracle/*.cpp, built by oracle/Makefile into oracle/_build/liborc.so).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use it, as the CPU results
the device's are compared with and as the timed CPU reference; the product (repackshot_b200) never
imports it.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liborc.so"
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ctypes.CDLL(str(LIB))
        v, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
        sig = {
            "orc_scene_load": (u32, [ctypes.c_char_p, u32]),
            "orc_error": (u32, [v, u32]),
            "orc_scene_free": (u32, [u32]),
            "orc_scene_info": (u32, [u32, v]),
            "orc_render_film": (u64, [u32, u32, u32, u32, u32, u32, u32, u32, u32, v, v, v, v, v]),
            "orc_render_tile": (u64, [u32, u32, u32, u32, u32, u32, v, v]),
            "orc_paths": (None, [u32, v, u32, v, u32]),
            "orc_trace": (None, [u32, v, u32, u32, u32, v, v, u32]),
            "orc_occluded": (None, [u32, v, u32, v]),
            "orc_energy_tables": (None, [v, v]),
            "orc_enable_merged_stats": (u32, [u32]),
            "orc_pcg32": (None, [u64, u64, u32, v]),
            "orc_mix64": (u64, [u64]),
            "orc_sobol": (u32, [u32, u32]),
            "orc_sampler_get1": (ctypes.c_float, [u32, u32, u32, u32, u32]),
            "orc_fmath": (None, [u32, v, u32, v]),
            "orc_film_encode": (None, [v, v, u32, ctypes.c_float, u32, v, v]),
            "orc_film_linear": (None, [v, v, u32, ctypes.c_float, v]),
            "orc_mesh_solid": (u32, [v, u32, v, u32]),
            "orc_color": (None, [u32, v, u32, v]),
            "orc_agx_identity": (None, [v]),
            "orc_light_count": (u32, [u32]),
            "orc_light_flux_pmf": (ctypes.c_float, [u32, u32]),
            "orc_light_sample": (u32, [u32, v, ctypes.c_float, ctypes.c_float, ctypes.c_float, v]),
            "orc_light_sky": (None, [u32, v, v]),
            "orc_light_crossed": (None, [u32, v, ctypes.c_float, v]),
            "orc_bitmap": (u32, [u32, u32, u32, ctypes.c_char_p, u32, v, v, u32, v, v]),
            "orc_dist2d": (u32, [u32, u32, v, u32, v, v]),
            "orc_filter_offset": (None, [u32, v, u32, v]),
            "orc_ies": (u32, [ctypes.c_char_p, u32, v, u32, v, v, u32, v, v]),
            "orc_blackman_harris_table": (None, [v]),
            "orc_set_sky_table": (None, [v, u32]),
            "orc_adjoint_reference": (u32, [u32, u32, u32, u32, u32, u32, u32, u32, v, u32, v, v]),
            "orc_edge_mask": (None, [u32, v]),
            "orc_adaptive_decide": (u32, [u32, u32, ctypes.c_float, ctypes.c_float, u32, v, v, v, v, v]),
            "orc_adaptive_film": (u32, [u32, u32, u32, u32, v, v, v, v, v, v]),
            "orc_pixel_error": (ctypes.c_float, [ctypes.c_float] * 4 + [u32, ctypes.c_float]),
            "orc_render_passes": (u32, [u32, u32, u32, u32, u32, v, v, v, v]),
            "orc_render_albedo": (u32, [u32, u32, u32, u32, u32, u32, v]),
            "orc_render_alpha": (u32, [u32, u32, u32, u32, u32, u32, v]),
            "orc_denoise": (u32, [u32, ctypes.c_float, u32, u32, u32, u32, u32, u32, u32, v, u32, v]),
            "orc_denoise_halo": (u32, [u32]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        # the physical sky's fitted table: the same data file the product compiles in
        table = np.fromfile(HERE.parent / "repackshot_b200" / "data" / "sky_table.f32", dtype="<f4")
        L.orc_set_sky_table(table.ctypes.data_as(ctypes.c_void_p), len(table))
        _lib = L
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib().orc_error(buf, 1024)
    return buf.value.decode()


class OracleScene:
    def __init__(self, rsb: bytes):
        self.handle = lib().orc_scene_load(rsb, len(rsb))
        if not self.handle:
            raise ValueError(error())
        info = np.zeros(8, np.uint32)
        lib().orc_scene_info(self.handle, _p(info))
        (self.width, self.height, self.seed, self.max_depth, self.instances, self.triangles, self.n_materials,
         self.n_lights) = map(int, info)

    def close(self):
        if self.handle:
            lib().orc_scene_free(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render_film(self, first=0, count=1, x=0, y=0, w=None, h=None, tile=32, threads=1):
        """Film sums of samples [first, first+count) over a rectangle: (rgb, weight, alpha, lum2,
        stats=(rays, nearest queries, their node visits, packet tests, any-hit queries, their node
        visits, packet tests, then the nearest and any-hit node visits and packet tests in the
        merged single tree when enable_merged_stats() was called) with the reference's BVH8 layout."""
        w = self.width if w is None else w
        h = self.height if h is None else h
        n = w * h
        rgb, wt, al, l2 = (np.zeros(3 * n, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32))
        st = np.zeros(11, np.uint64)
        lib().orc_render_film(self.handle, x, y, w, h, first, count, tile, threads, _p(rgb), _p(wt), _p(al), _p(l2), _p(st))
        return rgb.reshape(h, w, 3), wt.reshape(h, w), al.reshape(h, w), l2.reshape(h, w), tuple(int(v) for v in st)

    def enable_merged_stats(self):
        """Also count visits in one reference-layout BVH8 over all identity instances."""
        lib().orc_enable_merged_stats(self.handle)

    def render_tile(self, x, y, w, h, sample, rgba=False):
        rgb = np.zeros(3 * w * h, np.float32)
        al = np.zeros(w * h, np.float32)
        lib().orc_render_tile(self.handle, x, y, w, h, sample, _p(rgb), _p(al))
        if not rgba:
            return rgb
        return np.concatenate([rgb.reshape(-1, 3), al.reshape(-1, 1)], axis=1).reshape(-1)

    def paths(self, xys, threads=0):
        """Per-path radiance (r, g, b, alpha, rays) of (x, y, sample) triples; `threads` workers
        (0: the host's cores)."""
        xys = np.ascontiguousarray(xys, dtype=np.uint32).reshape(-1, 3)
        out = np.zeros((len(xys), 5), np.float32)
        lib().orc_paths(self.handle, _p(xys), len(xys), _p(out), int(threads))
        return out

    def adjoint_reference(self, target, first, count, x=0, y=0, w=None, h=None, threads=0, correlated=False):
        """The CPU reference of the device adjoint (orc_adjoint_reference): (loss, gradients as
        float64: 4 per material -- base R, G, B, alpha -- then one per scene light's power);
        decorrelated by sample halves unless `correlated`."""
        w = self.width if w is None else w
        h = self.height if h is None else h
        t = np.ascontiguousarray(target, np.float32).reshape(-1)
        assert t.size == 3 * w * h
        n = 4 * self.n_materials + self.n_lights
        grads = np.zeros(n, np.float64)
        loss = np.zeros(1, np.float64)
        if lib().orc_adjoint_reference(self.handle, x, y, w, h, first, count, int(correlated), _p(t), int(threads), _p(grads),
                                       _p(loss)):
            raise ValueError("orc_adjoint_reference: bad arguments")
        return float(loss[0]), grads

    def trace(self, rays, camera=False, brute=False, threads=0):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        hits = np.zeros((len(rays), 3), np.uint32)
        st = np.zeros(2, np.uint64)
        lib().orc_trace(self.handle, _p(rays), len(rays), int(camera), int(brute), _p(hits), _p(st), int(threads))
        return hits, (int(st[0]), int(st[1]))

    def light_count(self):
        return int(lib().orc_light_count(self.handle))

    def light_flux_pmf(self, entry):
        """Probability of a selection entry under the static selection, by flux."""
        return float(lib().orc_light_flux_pmf(self.handle, entry))

    def light_sample(self, x, u_select, u):
        """Lights::sample at x: (wi, distance, radiance, pdf, delta, shadow) or None."""
        xs = np.asarray(x, np.float32)
        out = np.zeros(10, np.float32)
        if not lib().orc_light_sample(self.handle, _p(xs), float(u_select), float(u[0]), float(u[1]), _p(out)):
            return None
        return out[0:3].copy(), float(out[3]), out[4:7].copy(), float(out[7]), bool(out[8]), bool(out[9])

    def light_sky(self, direction):
        """The sky a camera ray sees along a unit direction (environment and sun discs)."""
        d = np.asarray(direction, np.float32)
        out = np.zeros(3, np.float32)
        lib().orc_light_sky(self.handle, _p(d), _p(out))
        return out

    def light_crossed(self, origin, direction, t_max=float("inf"), bsdf_pdf=None, t_min=1.0e-3):
        """Lights a ray crosses: seen by the camera (bsdf_pdf None) or MIS-weighted for a BSDF
        sample of that density, with the selection at the ray's origin."""
        r = np.array([*origin, *direction, t_min, t_max], np.float32)
        out = np.zeros(3, np.float32)
        lib().orc_light_crossed(self.handle, _p(r), -1.0 if bsdf_pdf is None else float(bsdf_pdf), _p(out))
        return out

    def edge_mask(self):
        """One byte per pixel: 1 on the pixels that take the edge samples."""
        out = np.zeros((self.height, self.width), np.uint8)
        lib().orc_edge_mask(self.handle, _p(out))
        return out

    def adaptive_film(self, cap, pass_samples=16, threads=8):
        """The scene rendered adaptively to convergence or `cap` samples a pixel
        (adaptive/tests.rs:294): (rgb, weight, alpha, lum2, counts per block (rows, cols),
        (fewest, most samples of a pixel, decisions taken, rays mod 2^32))."""
        w, h = self.width, self.height
        n = w * h
        rgb, wt, al, l2 = (np.zeros(3 * n, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32))
        cols, rows = (w + 7) // 8, (h + 7) // 8
        counts = np.zeros(cols * rows, np.uint32)
        st = np.zeros(4, np.uint32)
        if lib().orc_adaptive_film(self.handle, cap, pass_samples, threads, _p(rgb), _p(wt), _p(al), _p(l2), _p(counts), _p(st)):
            raise ValueError("bad scene handle")
        return (rgb.reshape(h, w, 3), wt.reshape(h, w), al.reshape(h, w), l2.reshape(h, w), counts.reshape(rows, cols),
                tuple(int(v) for v in st))

    def passes(self, x=0, y=0, w=None, h=None):
        """The exact passes of the rectangle's centre rays (rt_render_tile_passes): normal (h, w, 3),
        depth, part id, material id (h, w)."""
        w = self.width if w is None else w
        h = self.height if h is None else h
        normal, depth = np.zeros((h, w, 3), np.float32), np.zeros((h, w), np.float32)
        part, material = np.zeros((h, w), np.uint32), np.zeros((h, w), np.uint32)
        lib().orc_render_passes(self.handle, x, y, w, h, _p(normal), _p(depth), _p(part), _p(material))
        return normal, depth, part, material

    def albedo(self, sample, x=0, y=0, w=None, h=None):
        """The albedo of sample `sample` of the rectangle (rt_render_tile_albedo): (h, w, 3)."""
        w = self.width if w is None else w
        h = self.height if h is None else h
        out = np.zeros((h, w, 3), np.float32)
        lib().orc_render_albedo(self.handle, x, y, w, h, sample, _p(out))
        return out

    def alpha(self, sample, x=0, y=0, w=None, h=None):
        """The coverage of sample `sample` of the rectangle (rt_render_tile_alpha): (h, w)."""
        w = self.width if w is None else w
        h = self.height if h is None else h
        out = np.zeros((h, w), np.float32)
        lib().orc_render_alpha(self.handle, x, y, w, h, sample, _p(out))
        return out

    def guides(self, samples):
        """The denoiser's guides of the whole image (rt-post denoise/tests.rs:338): the albedo
        summed over samples 0..samples in order and divided as Film::resolve divides, and the
        exact passes."""
        acc = np.zeros((self.height, self.width, 3), np.float32)
        for s in range(samples):
            acc = (acc + self.albedo(s)).astype(np.float32)
        albedo = (acc * (np.float32(1.0) / np.float32(samples))).astype(np.float32) if samples else acc
        normal, depth, part, material = self.passes()
        return albedo, normal, depth, part, material

    def occluded(self, rays):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        out = np.zeros(len(rays), np.uint8)
        lib().orc_occluded(self.handle, _p(rays), len(rays), _p(out))
        return out


def bitmap(fmt, w, h, data, lookups=()):
    """Bitmap::decode of a BMAP payload: (texels (h, w, 3), bilinear lookups (n, 3)) or raises
    ValueError with the reason."""
    wh = np.zeros(2, np.uint32)
    uvw = np.asarray(lookups, np.float32).reshape(-1, 3)
    out = np.zeros((len(uvw), 3), np.float32)
    st = lib().orc_bitmap(fmt, w, h, bytes(data), len(data), _p(wh), None, len(uvw), _p(uvw), _p(out))
    if st:
        raise ValueError(error())
    tex = np.zeros((int(wh[1]), int(wh[0]), 3), np.float32)
    lib().orc_bitmap(fmt, w, h, bytes(data), len(data), _p(wh), _p(tex), 0, None, None)
    return tex, out


def dist2d(w, h, weights, samples):
    """Distribution2D over w x h weights: (u, v, pdf, pdf at (u, v)) per sample, or None."""
    wts = np.ascontiguousarray(weights, np.float32)
    s = np.ascontiguousarray(samples, np.float32).reshape(-1, 2)
    out = np.zeros((len(s), 4), np.float32)
    if lib().orc_dist2d(w, h, _p(wts), len(s), _p(s), _p(out)):
        return None
    return out


def ies(text, angles=(), dirs=()):
    """IesProfile::parse: (peak, flux, symmetry, intensities at (gamma, phi) pairs, shapes towards
    local directions), or raises ValueError with the reason."""
    data = text.encode() if isinstance(text, str) else bytes(text)
    gp = np.ascontiguousarray(angles, np.float32).reshape(-1, 2)
    dd = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
    out3 = np.zeros(3, np.float32)
    inten = np.zeros(len(gp), np.float32)
    shp = np.zeros(len(dd), np.float32)
    if lib().orc_ies(data, len(data), _p(out3), len(gp), _p(gp), _p(inten), len(dd), _p(dd), _p(shp)):
        raise ValueError(error())
    return float(out3[0]), float(out3[1]), int(out3[2]), inten, shp


def adaptive_decide(width, height, ev, target, cap, counts, sums, lum2):
    """rt_adaptive_decide (rt-wasm/src/lib.rs:660): (active bytes per block, six words: round,
    active, blocks, and the bits of threshold, max_error, remaining)."""
    cols, rows = (width + 7) // 8, (height + 7) // 8
    counts = np.ascontiguousarray(counts, np.uint32).reshape(-1)
    sums = np.ascontiguousarray(sums, np.float32).reshape(-1)
    lum2 = np.ascontiguousarray(lum2, np.float32).reshape(-1)
    if counts.size != cols * rows or sums.size != 4 * width * height or lum2.size != width * height:
        raise ValueError("plane sizes do not match the image")
    active = np.zeros(max(cols * rows, 1), np.uint8)
    words = np.zeros(6, np.uint32)
    st = lib().orc_adaptive_decide(width, height, float(ev), float(target), cap, _p(counts), _p(sums), _p(lum2), _p(active), _p(words))
    if st:
        raise ValueError(f"status {st}")
    return active[:cols * rows], words


def denoise_words(sums_rgba, lum2, albedo, normal, depth, part, material, counts=None):
    """The denoiser's input (rt-wasm/src/lib.rs:420): the planes one after another as u32 words."""
    planes = [np.ascontiguousarray(a, np.float32).reshape(-1).view(np.uint32) for a in (sums_rgba, lum2, albedo, normal, depth)]
    planes += [np.ascontiguousarray(a, np.uint32).reshape(-1) for a in (part, material)]
    if counts is not None:
        planes.append(np.ascontiguousarray(counts, np.float32).reshape(-1).view(np.uint32))
    return np.concatenate(planes)


def denoise(words, width, height, samples, preset=0, strength=1.0, origin_y=0, rows=None, y0=None, y1=None):
    """rt_denoise_with: the denoised RGBA sums of rows y0..y1 of the band (float32, (y1 - y0) * width * 4)."""
    rows = height if rows is None else rows
    y0 = origin_y if y0 is None else y0
    y1 = origin_y + rows if y1 is None else y1
    words = np.ascontiguousarray(words, np.uint32)
    per_pixel = words.size // max(width * rows, 1)
    out = np.zeros(max((y1 - y0) * width * 4, 1), np.float32)
    st = lib().orc_denoise(preset, float(strength), width, height, origin_y, rows, samples, y0, y1, _p(words), per_pixel, _p(out))
    if st:
        raise ValueError(f"status {st}")
    return out[:(y1 - y0) * width * 4]


def denoise_halo(preset):
    return int(lib().orc_denoise_halo(preset))


def pixel_error(r, g, b, lum2, n, floor):
    return float(lib().orc_pixel_error(float(r), float(g), float(b), float(lum2), int(n), float(floor)))


def filter_offset(filter_kind, us):
    u = np.ascontiguousarray(us, np.float32)
    out = np.zeros_like(u)
    lib().orc_filter_offset(filter_kind, _p(u), len(u), _p(out))
    return out


def blackman_harris_table():
    out = np.zeros(256, np.float32)
    lib().orc_blackman_harris_table(_p(out))
    return out


def energy_tables():
    u16 = np.zeros(2048 + 2 * 17408, np.uint16)
    f = np.zeros(64, np.float32)
    lib().orc_energy_tables(_p(u16), _p(f))
    return {"albedo": u16[:1024], "schlick": u16[1024:2048], "clear_in": u16[2048:2048 + 17408],
            "clear_out": u16[2048 + 17408:], "albedo_avg": f[:32], "schlick_avg": f[32:]}


def fnv1a(values) -> int:
    h = 0x811C9DC5
    for byte in np.ascontiguousarray(values, dtype="<f4").tobytes():
        h = ((h ^ byte) * 0x01000193) & 0xFFFFFFFF
    return h


def resolve(rgb, weight):
    """Film::resolve (image.rs:158): rgb * (1 / weight) in f32, black where weight is 0."""
    w = np.asarray(weight, np.float32)
    inv = np.where(w > 0, np.float32(1.0) / np.where(w > 0, w, np.float32(1.0)), np.float32(0.0)).astype(np.float32)
    return (np.asarray(rgb, np.float32) * inv[..., None]).astype(np.float32)


def film_encode(rgb, weight, ev, tonemap):
    """image.rs to_srgb8_tonemapped / to_srgb16_tonemapped of film sums: (u8 (n, 3), u16 (n, 3))."""
    rgb = np.ascontiguousarray(rgb, np.float32).reshape(-1)
    weight = np.ascontiguousarray(weight, np.float32).reshape(-1)
    n = weight.size
    out8 = np.zeros(3 * n, np.uint8)
    out16 = np.zeros(3 * n, np.uint16)
    lib().orc_film_encode(_p(rgb), _p(weight), n, ev, tonemap, _p(out8), _p(out16))
    return out8.reshape(n, 3), out16.reshape(n, 3)


def film_linear(rgb, weight, ev):
    """image.rs to_linear_exposed of film sums: float32 (n, 3), the resolved film times 2^ev."""
    rgb = np.ascontiguousarray(rgb, np.float32).reshape(-1)
    weight = np.ascontiguousarray(weight, np.float32).reshape(-1)
    n = weight.size
    out = np.zeros(3 * n, np.float32)
    lib().orc_film_linear(_p(rgb), _p(weight), n, ev, _p(out))
    return out.reshape(n, 3)


def mesh_solid(positions, indices):
    """solid.rs analyse of a mesh: 0 open, 1 closed and wound outward, 2 inward."""
    p = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    i = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    return int(lib().orc_mesh_solid(_p(p), len(p), _p(i), len(i)))


def color(which, xs):
    """orc_color: 0 exposure, 1 ACES, 2 sRGB encode, 3 + k Tonemap k on a grey (its green)."""
    xs = np.ascontiguousarray(xs, np.float32)
    out = np.zeros_like(xs)
    lib().orc_color(which, _p(xs), xs.size, _p(out))
    return out


def agx_identity():
    out = np.zeros(9, np.float32)
    lib().orc_agx_identity(_p(out))
    return out.reshape(3, 3)
