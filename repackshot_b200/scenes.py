"""Scene construction for the renders this package is measured on: an RSB writer (the format of
engine/crates/rt-core/src/scene/rsb.rs:1-140), the reference's example scene
(engine/crates/rt-core/src/example.rs:20-228) and the synthetic product scenes of the
benchmark workloads.

Geometry that the reference builds in f32 (the icosphere) is built here with the same f32
operations, so the example's bytes are the reference's ``tests/fixtures/example.rsb``.

Units follow the reference: millimetres, Z up. The benchmark workloads are described Y-up in
metres; ``yup_m_to_mm`` maps (x, y, z) to 1000 * (x, -z, y).
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

f32 = np.float32

# ---- RSB writer ----------------------------------------------------------------------------------


@dataclass
class Material:
    kind: int = 0
    base_color: Tuple[float, float, float] = (0.8, 0.8, 0.8)
    metallic: float = 0.0
    roughness: float = 0.5
    ior: float = 1.5
    transmission: float = 0.0
    coat: float = 0.0
    coat_roughness: float = 0.0
    emission: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    emission_power: float = 0.0
    flags: int = 0
    opacity: float = 1.0
    anisotropy: float = 0.0
    absorption_mm: float = 0.0
    bevel_mm: float = 0.0
    scatter_mm: float = 0.0
    scatter_color: Tuple[float, float, float] = (1.0, 1.0, 1.0)
    scatter_g: float = 0.0
    abbe: float = 0.0


@dataclass
class Light:
    kind: int = 0  # 0 rect, 1 disk, 2 sun, 3 point (a sphere of diameter size_x), 4 spot
    position: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    direction: Tuple[float, float, float] = (0.0, 0.0, -1.0)
    up: Tuple[float, float, float] = (0.0, 1.0, 0.0)
    size_x: float = 100.0
    size_y: float = 100.0
    color: Tuple[float, float, float] = (1.0, 1.0, 1.0)
    power: float = 1.0
    spread_deg: float = 180.0
    angle_deg: float = 0.0
    flags: int = 3  # glossy | camera
    profile: int = 0xFFFFFFFF  # kind 5 (IES): its profile among the scene's IESP sections


@dataclass
class Bitmap:
    """A BMAP section: format 0 (sRGB RGB8), 1 (sRGB RGBA8), 2 (linear f32 RGB) or 16 (a
    Radiance file, width and height 0), and its data bytes."""
    format: int
    width: int
    height: int
    data: bytes


@dataclass
class Mesh:
    positions: np.ndarray  # (n, 3) float32
    normals: np.ndarray  # (n, 3) float32 (zeros: none)
    indices: np.ndarray  # (m,) uint32
    material_id: int = 0


@dataclass
class Instance:
    mesh: int
    rows: Sequence[float] = (1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0)
    material_id: int = 0
    flags: int = 0


@dataclass
class Scene:
    camera_position: Tuple[float, float, float] = (0.0, -1000.0, 0.0)
    camera_target: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    camera_up: Tuple[float, float, float] = (0.0, 0.0, 1.0)
    focal_mm: float = 50.0
    sensor_mm: float = 36.0
    fstop: float = 0.0
    focus_dist: float = 1000.0
    ortho: int = 0
    ortho_width: float = 1000.0
    materials: List[Material] = field(default_factory=list)
    meshes: List[Mesh] = field(default_factory=list)
    instances: List[Instance] = field(default_factory=list)
    lights: List[Light] = field(default_factory=list)
    bitmaps: List[Bitmap] = field(default_factory=list)
    profiles: List[bytes] = field(default_factory=list)  # IES LM-63 files (IESP sections)
    env_kind: int = 0  # 0 studio, 1 flat, 2 sky, 3 HDRI
    env_floor: float = 0.1
    env_horizon: float = 0.3
    env_zenith: float = 0.6
    env_strength: float = 1.0
    env_rotation: float = 0.0
    background_color: Tuple[float, float, float] = (0.05, 0.05, 0.05)
    background_mode: int = 0  # 0 environment, 1 colour, 2 transparent, 3 backplate
    hdri_map: int = 0xFFFFFFFF
    backplate_map: int = 0xFFFFFFFF
    backplate_fit: int = 0  # 0 fill, 1 fit, 2 stretch
    sky_turbidity: float = 3.0
    sun_azimuth_deg: float = 0.0
    sun_elevation_deg: float = 45.0
    backplate_rect: Tuple[float, float, float, float] = (0.0, 0.0, 1.0, 1.0)
    sky_model: int = 0
    floor_mode: int = 0
    floor_z: float = 0.0
    floor_color: Tuple[float, float, float] = (0.5, 0.5, 0.5)
    width: int = 640
    height: int = 360
    max_samples: int = 64
    seed: int = 0
    max_seconds: float = 0.0
    exposure_ev: float = 0.0
    tonemap: int = 1
    max_depth: int = 8
    clamp_indirect: float = 0.0
    pixel_filter: int = 0  # 0 standard, 1 none, 2 tent, 3 Blackman-Harris
    edge_supersample: int = 1  # samples per sample index of an edge pixel
    caustic_photons: int = 0  # photons of the caustic maps a sample index (0: none)
    adaptive: int = 0  # bit 0: the host samples adaptively (E10)
    noise_threshold: float = 0.0  # relative error a block stops at (0: none)
    # SECT (Q1): (flags, normal x, y, z, distance); flags bit 0 caps the cut solids. None: no section.
    section: Optional[Tuple[int, float, float, float, float]] = None


def _sec(tag: bytes, payload: bytes) -> bytes:
    return tag + struct.pack("<I", len(payload)) + payload


def _f(*v) -> bytes:
    return struct.pack("<%df" % len(v), *[float(f32(x)) for x in v])


def _u(*v) -> bytes:
    return struct.pack("<%dI" % len(v), *v)


def to_rsb(s: Scene, meshes: bool = True) -> bytes:
    """Serialises a scene as RSB version 1, sections in the reference writer's order (CAMR, MATL,
    MESH, INST, LGHT, ENVR, FLOR, RNDR) and payload sizes (rsb.rs:1645-1990). Without ``meshes``
    the MESH sections are left out: the file of a scene update that keeps the loaded geometry
    (rt_scene_update). BMAP sections follow the lights, as the reference writes them."""
    out = [b"RSB1", _u(0)]
    out.append(_sec(b"CAMR", _f(*s.camera_position, *s.camera_target, *s.camera_up, s.focal_mm, s.sensor_mm, s.fstop,
                                s.focus_dist) + _u(s.ortho) + _f(s.ortho_width)))
    for m in s.materials:
        out.append(_sec(b"MATL", _u(m.kind) + _f(*m.base_color, m.metallic, m.roughness, m.ior, m.transmission, m.coat,
                                                 m.coat_roughness, *m.emission, m.emission_power) + _u(m.flags) +
                        _f(m.opacity, m.anisotropy, m.absorption_mm, m.bevel_mm, m.scatter_mm, *m.scatter_color,
                           m.scatter_g, m.abbe)))
    for mesh in (s.meshes if meshes else []):
        p = np.ascontiguousarray(mesh.positions, dtype="<f4")
        n = np.ascontiguousarray(mesh.normals, dtype="<f4")
        i = np.ascontiguousarray(mesh.indices, dtype="<u4")
        out.append(_sec(b"MESH", _u(len(p), len(i)) + p.tobytes() + n.tobytes() + i.tobytes() + _u(mesh.material_id)))
    for inst in s.instances:
        out.append(_sec(b"INST", _u(inst.mesh) + _f(*inst.rows) + _u(inst.material_id, inst.flags)))
    for l in s.lights:
        out.append(_sec(b"LGHT", _u(l.kind) + _f(*l.position, *l.direction, *l.up, l.size_x, l.size_y, *l.color, l.power,
                                                 l.spread_deg, l.angle_deg) + _u(l.flags) + (_u(l.profile) if l.kind == 5 else b"")))
    for p in s.profiles:
        out.append(_sec(b"IESP", _u(len(p)) + bytes(p) + bytes((4 - len(p) % 4) % 4)))
    for b in s.bitmaps:
        out.append(_sec(b"BMAP", _u(b.format, b.width, b.height, len(b.data)) + bytes(b.data) + bytes((4 - len(b.data) % 4) % 4)))
    out.append(_sec(b"ENVR", _u(s.env_kind) + _f(s.env_floor, s.env_horizon, s.env_zenith, s.env_strength, s.env_rotation,
                                                 *s.background_color) + _u(s.background_mode) +
                    _u(s.hdri_map, s.backplate_map, s.backplate_fit) +
                    _f(s.sky_turbidity, s.sun_azimuth_deg, s.sun_elevation_deg, *s.backplate_rect) + _u(s.sky_model)))
    out.append(_sec(b"FLOR", _u(s.floor_mode) + _f(s.floor_z, *s.floor_color)))
    out.append(_sec(b"RNDR", _u(s.width, s.height, s.max_samples, s.seed) + _f(s.max_seconds, s.exposure_ev) +
                    _u(s.tonemap, s.max_depth) + _f(s.clamp_indirect) + _u(0, 0, s.caustic_photons) + _f(0.0, 1.0) +
                    _u(s.pixel_filter, s.edge_supersample) +
                    (_u(s.adaptive) + _f(s.noise_threshold) if s.adaptive or s.noise_threshold else b"")))
    if s.section is not None:  # rsb.rs:1884, written only when the scene has one
        out.append(_sec(b"SECT", _u(s.section[0]) + _f(*s.section[1:])))
    return b"".join(out)


# ---- f32 geometry helpers ----------------------------------------------------------------------


def _normalize32(v):
    x, y, z = f32(v[0]), f32(v[1]), f32(v[2])
    ln = np.sqrt(f32(f32(f32(x * x) + f32(y * y)) + f32(z * z)))
    if ln > 0 and np.isfinite(ln):
        return (f32(x / ln), f32(y / ln), f32(z / ln))
    return (x, y, z)


def icosphere(center, radius: float, subdivisions: int, material_id: int = 0) -> Mesh:
    """The reference's icosphere (example.rs:20) in f32: icosahedron, midpoint subdivision,
    vertices pushed onto the sphere; normals are the unit radial directions."""
    with np.errstate(all="ignore"):
        t = f32(f32(1.0) + np.sqrt(f32(5.0))) / f32(2.0)
        base = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
                (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
        dirs = [_normalize32(v) for v in base]
        faces = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6],
                 [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
                 [8, 6, 7], [9, 8, 1]]
        for _ in range(subdivisions):
            mids = {}

            def midpoint(a, b):
                key = (min(a, b), max(a, b))
                if key not in mids:
                    da, db = dirs[a], dirs[b]
                    dirs.append(_normalize32((f32(da[0] + db[0]), f32(da[1] + db[1]), f32(da[2] + db[2]))))
                    mids[key] = len(dirs) - 1
                return mids[key]

            nxt = []
            for a, b, c in faces:
                ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
                nxt += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
            faces = nxt
        d = np.array(dirs, dtype=np.float32)
        pos = (np.asarray(center, dtype=np.float32)[None, :] + d * f32(radius)).astype(np.float32)
    return Mesh(pos, d, np.array(faces, dtype=np.uint32).reshape(-1), material_id)


def floor_quad(z: float, half: float, material_id: int) -> Mesh:
    """example.rs:87: a quad at height z spanning [-half, half] on X and Y, facing up."""
    p = np.array([(-half, -half, z), (half, -half, z), (half, half, z), (-half, half, z)], dtype=np.float32)
    n = np.array([(0, 0, 1)] * 4, dtype=np.float32)
    return Mesh(p, n, np.array([0, 1, 2, 0, 2, 3], dtype=np.uint32), material_id)


def example_scene() -> Scene:
    """The reference's example scene (example.rs:113): a 100 mm icosphere on a floor quad, a
    half-size second instance, one 5 W rect light, the studio dome, an 85 mm camera at f/11."""
    cam = (560.0, -900.0, 400.0)
    target = (0.0, 0.0, 90.0)
    light_pos = (250.0, -450.0, 650.0)
    fd = np.float32(0)
    dv = [f32(target[i]) - f32(cam[i]) for i in range(3)]
    fd = np.sqrt(f32(f32(f32(dv[0] * dv[0]) + f32(dv[1] * dv[1])) + f32(dv[2] * dv[2])))
    ld = _normalize32([f32(target[i]) - f32(light_pos[i]) for i in range(3)])
    return Scene(
        camera_position=cam, camera_target=target, camera_up=(0.0, 0.0, 1.0), focal_mm=85.0, sensor_mm=36.0,
        fstop=11.0, focus_dist=float(fd), ortho=0, ortho_width=600.0,
        materials=[Material(base_color=(0.92, 0.38, 0.22), roughness=0.35),
                   Material(base_color=(0.3, 0.3, 0.32), roughness=0.8),
                   Material(base_color=(0.2, 0.42, 0.85), roughness=0.25)],
        meshes=[icosphere((0.0, 0.0, 100.0), 100.0, 2), floor_quad(0.0, 900.0, 1)],
        instances=[Instance(0, material_id=0), Instance(1, material_id=1),
                   Instance(0, rows=(0.5, 0, 0, -330.0, 0, 0.5, 0, 120.0, 0, 0, 0.5, 0), material_id=2)],
        lights=[Light(kind=0, position=light_pos, direction=tuple(float(x) for x in ld), up=(0.0, 0.0, 1.0), size_x=400.0,
                      size_y=400.0, power=5.0, flags=3)],
        env_kind=0, env_floor=0.05, env_horizon=0.12, env_zenith=0.3, env_strength=1.0, background_color=(0.05, 0.05, 0.05),
        width=512, height=384, max_samples=16, seed=1, tonemap=1, max_depth=8)


LIGHT_SUN, LIGHT_POINT, LIGHT_SPOT = 2, 3, 4
MATERIAL_GLASS, MATERIAL_FLAG_THIN = 1, 2
MATERIAL_EMISSIVE, MATERIAL_FLAG_LIGHT = 2, 1  # scene/mod.rs:367-370: an emitter; sampled as a light
INSTANCE_ONE_SIDED = 1  # geometry/mod.rs:54


def _rgb_to_rgbe(c) -> bytes:
    """hdr.rs:60 rgb_to_rgbe in f32: the shared exponent of the largest channel, mantissas truncated."""
    clean = [f32(v) if (np.isfinite(v) and v > 0) else f32(0.0) for v in c]
    m = max(max(clean[0], clean[1]), clean[2])
    if m < f32(1.0e-32):
        return bytes(4)
    e = int((int(np.array(m, np.float32).view(np.uint32)) >> 23) & 0xFF) - 126
    e = min(e, 127)
    scale = f32(2.0) ** f32(8 - e) if -126 <= 8 - e <= 127 else f32(math.ldexp(1.0, 8 - e))
    q = [min(int(f32(v * scale)), 255) for v in clean]
    return bytes([q[0], q[1], q[2], e + 128])


def _rle_channel(data: bytes) -> bytes:
    """hdr.rs:261 encode_channel: runs of four or more as (128 + n, value), literals of up to 128."""
    out = bytearray()
    n, i = len(data), 0
    while i < n:
        run = 1
        while i + run < n and run < 127 and data[i + run] == data[i]:
            run += 1
        if run >= 4:
            out += bytes([128 + run, data[i]])
            i += run
            continue
        start = i
        while i < n and i - start < 128:
            ahead = 1
            while i + ahead < n and ahead < 4 and data[i + ahead] == data[i]:
                ahead += 1
            if ahead >= 4:
                break
            i += 1
        out.append(i - start)
        out += data[start:i]
    return bytes(out)


def hdr_encode(width: int, height: int, rgb) -> bytes:
    """hdr.rs:295 encode: a Radiance file (-Y h +X w, the new run-length encoding where the width
    allows it) of 3 w h linear floats, rows top to bottom."""
    rgb = np.asarray(rgb, np.float32).reshape(height, width, 3)
    out = bytearray(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {height} +X {width}\n".encode())
    rle = 8 <= width <= 0x7FFF
    for y in range(height):
        px = [_rgb_to_rgbe(rgb[y, x]) for x in range(width)]
        if not rle:
            out += b"".join(px)
            continue
        out += bytes([2, 2, width >> 8, width & 0xFF])
        for c in range(4):
            out += _rle_channel(bytes(p[c] for p in px))
    return bytes(out)


def e5_scene(sky: bool = False) -> Scene:
    """example.rs:232 e5_scene: the example at 160 x 120 and depth 12 with clear blue glass
    (absorption 80 mm), a lacquered floor, brushed metal (anisotropy 0.8), a thin glass card and a
    cut-out card (opacity 0.4), lit by its rect light and a 64 x 32 HDRI panorama (a grey gradient
    with two bright panels, rotated 30 degrees) over a 16 x 8 background image. With `sky`, the
    classic sky (sun 35 degrees up at azimuth -60) seen as the background, lit by a sun of
    irradiance 3 and a disc of 0.545 degrees instead of the rect light."""
    s = example_scene()
    s.width, s.height, s.max_depth = 160, 120, 12
    s.materials = [
        Material(kind=MATERIAL_GLASS, base_color=(0.3, 0.5, 0.95), roughness=0.05, ior=1.5, transmission=1.0, absorption_mm=80.0),
        Material(base_color=(0.3, 0.3, 0.32), roughness=0.6, coat=1.0, coat_roughness=0.05),
        Material(base_color=(0.9, 0.85, 0.8), metallic=1.0, roughness=0.35, anisotropy=0.8),
        Material(kind=MATERIAL_GLASS, base_color=(0.9, 0.6, 0.6), roughness=0.0, transmission=1.0, flags=MATERIAL_FLAG_THIN),
        Material(base_color=(0.9, 0.9, 0.2), opacity=0.4),
    ]
    for x, material in ((150.0, 3), (-80.0, 4)):
        p = np.array([(x - 60.0, -260.0, 0.0), (x + 60.0, -260.0, 0.0), (x + 60.0, -260.0, 160.0), (x - 60.0, -260.0, 160.0)], np.float32)
        s.meshes.append(Mesh(p, np.zeros((4, 3), np.float32), np.array([0, 1, 2, 0, 2, 3], np.uint32), 0))
        s.instances.append(Instance(len(s.meshes) - 1, material_id=material))
    w, h = 64, 32
    rgb = np.zeros((h, w, 3), np.float32)
    for y in range(h):
        up = f32(1.0) - f32(y) / f32(h)
        for x in range(w):
            panel = f32(8.0) if (20 <= x < 28 and 8 <= y < 14) else (f32(12.0) if (44 <= x < 47 and 6 <= y < 18) else f32(0.0))
            rgb[y, x] = (f32(f32(0.05) + f32(0.2) * up) + panel, f32(f32(0.06) + f32(0.2) * up) + panel,
                         f32(f32(0.08) + f32(0.25) * up) + panel)
    plate = bytes(v for i in range(16 * 8) for v in ((i * 13) % 256, 120, 255 - (i * 7) % 256))
    s.bitmaps = [Bitmap(16, 0, 0, hdr_encode(w, h, rgb)), Bitmap(0, 16, 8, plate)]
    s.env_kind, s.hdri_map, s.backplate_map, s.background_mode = 3, 0, 1, 3
    s.env_floor, s.env_horizon, s.env_zenith, s.env_strength, s.env_rotation = 0.1, 0.3, 0.6, 1.0, 30.0
    s.background_color = (0.05, 0.05, 0.05)
    if sky:
        s.env_kind, s.sky_model, s.background_mode = 2, 1, 0
        s.sun_azimuth_deg, s.sun_elevation_deg = -60.0, 35.0
        s.lights = [Light(kind=LIGHT_SUN, position=(0.0, 0.0, 1000.0), direction=(-0.41, 0.71, -0.574), up=(0.0, 1.0, 0.0),
                          size_x=500.0, size_y=500.0, color=(1.0, 0.91, 0.83), power=3.0, angle_deg=0.545, flags=3)]
    return s


def e5c_scene() -> Scene:
    """example.rs:361 e5c_scene: the E5 sky scene under the physical sky (turbidity 2.5, the sun 12
    degrees up at azimuth -60). The sun light points along the sky's sun, -(cos e cos a, cos e sin a,
    sin e), from the reference's deterministic sin/cos of those angles (fmath.rs), written here as
    the f32 values they give; its colour is (1, 0.78, 0.6)."""
    s = e5_scene(sky=True)
    s.sky_model, s.sky_turbidity = 0, 2.5
    s.sun_azimuth_deg, s.sun_elevation_deg = -60.0, 12.0
    s.lights[0].direction = (float.fromhex("-0x1.f4cfc2p-2"), float.fromhex("0x1.b1b73p-1"), float.fromhex("-0x1.a9cd9cp-3"))
    s.lights[0].color = (1.0, 0.78, 0.6)
    return s


def e11_scene() -> Scene:
    """example.rs:1440 e11_scene: the example with the Blackman-Harris pixel filter and two samples
    per sample index on its edges."""
    s = example_scene()
    s.pixel_filter, s.edge_supersample = 3, 2
    return s


LIGHT_IES = 5


def l5_scene(downlight: bytes, wall_washer: bytes) -> Scene:
    """example.rs:1453 l5_scene: the example at 160 x 120 lit by its panel at 1 W and two IES
    lights: a downlight profile on a sphere of 24 mm above and in front of the big sphere, and a
    wall-washer profile as a warm point on the left, turned about its axis (`up`) so that its
    horizontal angles do not line up with the world. The two profiles are the files' bytes."""
    s = example_scene()
    s.width, s.height = 160, 120
    s.lights[0].power = 1.0
    above, washer = (0.0, -250.0, 760.0), (-620.0, -180.0, 380.0)
    to = lambda a, b: tuple(float(v) for v in _normalize32([f32(b[i]) - f32(a[i]) for i in range(3)]))
    s.profiles = [bytes(downlight), bytes(wall_washer)]
    s.lights.append(Light(kind=LIGHT_IES, position=above, direction=to(above, (0.0, 0.0, 100.0)), up=(0.0, 1.0, 0.0),
                          size_x=24.0, size_y=24.0, color=(1.0, 1.0, 1.0), power=18.0, spread_deg=180.0, angle_deg=0.0,
                          flags=3, profile=0))
    s.lights.append(Light(kind=LIGHT_IES, position=washer, direction=to(washer, (-330.0, 120.0, 60.0)), up=(0.35, -0.2, 0.9),
                          size_x=0.0, size_y=0.0, color=(1.0, 0.82, 0.62), power=7.0, spread_deg=180.0, angle_deg=0.0,
                          flags=1, profile=1))
    return s


def sun_triangle_scene() -> Scene:
    """render.rs:752-786: one Lambertian triangle (albedo 0.8, ior 1) facing a camera at y = -100
    that looks along +Y, lit by a delta sun of irradiance pi shining along +Y, in a black world
    with a black background colour; 16 x 16 pixels. Its centre pixel is albedo * E / pi = 0.8."""
    tri = Mesh(np.array([(-10.0, 0.0, -10.0), (10.0, 0.0, -10.0), (0.0, 0.0, 10.0)], np.float32),
               np.array([(0.0, -1.0, 0.0)] * 3, np.float32), np.array([0, 1, 2], np.uint32), 0)
    return Scene(camera_position=(0.0, -100.0, 0.0), camera_target=(0.0, 0.0, 0.0), focal_mm=50.0, sensor_mm=36.0,
                 materials=[Material(base_color=(0.8, 0.8, 0.8), ior=1.0)], meshes=[tri], instances=[Instance(0)],
                 lights=[Light(kind=LIGHT_SUN, position=(0.0, 0.0, 1000.0), direction=(0.0, 1.0, 0.0), size_x=500.0,
                               size_y=500.0, power=math.pi, angle_deg=0.0, flags=3)],
                 env_strength=0.0, background_color=(0.0, 0.0, 0.0), background_mode=1, width=16, height=16)


def light_kinds_scene(width: int = 256, height: int = 192) -> Scene:
    """The example scene lit by every light kind of the path at once: its rect softbox, a sun with
    a disc of 3 degrees, a point light, a sphere light of 60 mm and a spot with a soft edge, the
    last two seen by the camera and in reflections, over a dim dome (2 + 5 selection entries)."""
    s = example_scene()
    s.width, s.height = width, height
    s.lights.append(Light(kind=LIGHT_SUN, direction=(-0.3, 0.5, -0.81), power=2.0, angle_deg=3.0, flags=3))
    s.lights.append(Light(kind=LIGHT_POINT, position=(-300.0, -250.0, 320.0), size_x=0.0, size_y=0.0, power=6.0,
                          color=(1.0, 0.8, 0.6), flags=1))
    s.lights.append(Light(kind=LIGHT_POINT, position=(200.0, 150.0, 260.0), size_x=60.0, size_y=60.0, power=4.0,
                          color=(0.6, 0.8, 1.0), flags=3))
    s.lights.append(Light(kind=LIGHT_SPOT, position=(-150.0, -500.0, 700.0), direction=(0.2, 0.6, -0.77),
                          size_x=20.0, size_y=20.0, power=40.0, spread_deg=40.0, angle_deg=8.0, flags=3))
    return s


# ---- benchmark workloads -----------------------------------------------------------------------------------


def yup_m_to_mm(p):
    """Y-up metres -> Z-up millimetres: (x, y, z) -> 1000 * (x, -z, y)."""
    return (1000.0 * p[0], -1000.0 * p[2], 1000.0 * p[1])


def focal_for_vfov(vfov_deg: float, width: int, height: int, sensor_mm: float = 36.0) -> float:
    """Focal length giving a vertical field of view on a W x H image whose longer side spans
    `sensor_mm` (scene/mod.rs:306-313)."""
    sh = sensor_mm * min(1.0, height / width)
    return (sh / 2.0) / math.tan(math.radians(vfov_deg) / 2.0)


def rect_power(radiance: float, size_x_m: float, size_y_m: float) -> float:
    """Flux in watts of a rect light of the given radiance (light.rs:731: L = P / (pi A))."""
    return radiance * math.pi * size_x_m * size_y_m


def cfg0_scene() -> Scene:
    """Plain forward render, small: 256x256, 16 spp, depth 8, seed 1; pinhole 40 deg vertical FOV
    at (0,1,4) looking at the origin; icosphere (subdivision 4, radius 1, centre (0,1,0)) on a
    20x20 floor quad at y=0; GGX conductor F0 (0.95,0.64,0.54) alpha 0.3 on the sphere, Lambert
    0.8 on the floor; one 2x2 rect light at y=4 of radiance 10; constant dome 0.1."""
    w = h = 256
    return Scene(
        camera_position=yup_m_to_mm((0, 1, 4)), camera_target=(0.0, 0.0, 0.0), camera_up=(0.0, 0.0, 1.0),
        focal_mm=focal_for_vfov(40.0, w, h), sensor_mm=36.0, fstop=0.0, focus_dist=1000.0,
        materials=[Material(base_color=(0.95, 0.64, 0.54), metallic=1.0, roughness=math.sqrt(0.3)),
                   Material(base_color=(0.8, 0.8, 0.8), metallic=0.0, roughness=1.0, ior=1.0)],
        meshes=[icosphere(yup_m_to_mm((0, 1, 0)), 1000.0, 4, 0), floor_quad(0.0, 10000.0, 1)],
        instances=[Instance(0, material_id=0), Instance(1, material_id=1)],
        lights=[Light(kind=0, position=yup_m_to_mm((0, 4, 0)), direction=(0.0, 0.0, -1.0), up=(0.0, 1.0, 0.0),
                      size_x=2000.0, size_y=2000.0, power=rect_power(10.0, 2.0, 2.0), flags=3)],
        env_kind=1, env_floor=0.1, env_horizon=0.1, env_zenith=0.1, env_strength=1.0,
        width=w, height=h, max_samples=16, seed=1, max_depth=8)


def emissive_scene(width: int = 96, height: int = 96, spp: int = 8) -> Scene:
    """The small scene with two emissive meshes sampled as lights beside its rect light: a warm
    two-sided icosphere (subdivision 1, radius 0.25 m) above the floor to the left and a one-sided
    0.6 m square facing down-right, both in materials flagged as lights (light.rs:440-495)."""
    s = cfg0_scene()
    s.width, s.height, s.max_samples = width, height, spp
    s.materials += [Material(kind=MATERIAL_EMISSIVE, emission=(1.0, 0.8, 0.6), emission_power=6.0, flags=MATERIAL_FLAG_LIGHT),
                    Material(kind=MATERIAL_EMISSIVE, emission=(0.6, 0.8, 1.0), emission_power=12.0, flags=MATERIAL_FLAG_LIGHT)]
    s.meshes.append(icosphere(yup_m_to_mm((-1.3, 0.5, 0.6)), 250.0, 1, 2))
    q = np.array([(900.0, -300.0, 1500.0), (900.0, 300.0, 1500.0), (1500.0, 300.0, 2100.0), (1500.0, -300.0, 2100.0)], np.float32)
    s.meshes.append(Mesh(q, np.zeros((4, 3), np.float32), np.array([0, 2, 1, 0, 3, 2], np.uint32), 3))
    s.instances += [Instance(2, material_id=2), Instance(3, material_id=3, flags=INSTANCE_ONE_SIDED)]
    return s


def box_mesh(lo, hi, material_id: int = 0, inward: bool = False, skip_faces=()) -> Mesh:
    """An axis-aligned box of 24 vertices (4 per face, each with its face's normal), the faces wound
    counter-clockwise seen from outside, or from inside with `inward`. `skip_faces` leaves out faces
    by (axis, side) with side 0 the low face: an open box."""
    lo, hi = np.asarray(lo, np.float32), np.asarray(hi, np.float32)
    pos, nrm, idx = [], [], []
    for axis in range(3):
        for side in (0, 1):
            if (axis, side) in skip_faces:
                continue
            u, v = (axis + 1) % 3, (axis + 2) % 3
            corners = []
            for cu, cv in ((0, 0), (1, 0), (1, 1), (0, 1)):
                c = np.zeros(3, np.float32)
                c[axis] = hi[axis] if side else lo[axis]
                c[u] = hi[u] if cu else lo[u]
                c[v] = hi[v] if cv else lo[v]
                corners.append(c)
            out = np.zeros(3, np.float32)
            out[axis] = 1.0 if side else -1.0
            if (np.dot(np.cross(corners[1] - corners[0], corners[2] - corners[0]), out) < 0) != inward:
                corners.reverse()
            base = len(pos)
            pos += corners
            nrm += [-out if inward else out] * 4
            idx += [base, base + 1, base + 2, base, base + 2, base + 3]
    return Mesh(np.array(pos, np.float32), np.array(nrm, np.float32), np.array(idx, np.uint32), material_id)


def section_scene(width: int = 96, height: int = 64, spp: int = 4) -> Scene:
    """A section view that takes every rule of geometry/section.rs: a plane of normal (1, 0.2, 0)
    (normalised on load) at 10 mm cutting
    * a closed cube of 24 vertices (closed once welded), rotated 30 degrees and scaled (1.5, 0.8, 1.2):
      capped;
    * a cube wound inward: capped, its inside the front of its triangles;
    * an open box (no top) and a cube of a thin-walled material: cut but never capped;
    * a cube hidden to the camera: capped for every ray but camera rays;
    and, exempt from the section (the studio), the floor and a hollow box on the removed side that
    holds 60 parallel slices of the cut model: a ray looking for the box's wall from behind more
    than 48 of them gives up."""
    ang = math.radians(30.0)
    c, sn = math.cos(ang), math.sin(ang)
    def placed(scale, t):
        sx, sy, sz = scale
        return (c * sx, -sn * sy, 0.0, t[0], sn * sx, c * sy, 0.0, t[1], 0.0, 0.0, sz, t[2])
    slices_p, slices_i = [], []
    for k in range(60):  # quads perpendicular to x at x = 210 + 1.5 k
        x = 210.0 + 1.5 * k
        b = len(slices_p)
        slices_p += [(x, -80.0, 10.0), (x, 80.0, 10.0), (x, 80.0, 140.0), (x, -80.0, 140.0)]
        slices_i += [b, b + 1, b + 2, b, b + 2, b + 3]
    slices = Mesh(np.array(slices_p, np.float32), np.zeros((len(slices_p), 3), np.float32), np.array(slices_i, np.uint32), 0)
    return Scene(
        camera_position=(700.0, -500.0, 420.0), camera_target=(40.0, 0.0, 60.0), focal_mm=35.0, focus_dist=900.0,
        materials=[Material(base_color=(0.9, 0.45, 0.2), roughness=0.4),
                   Material(kind=MATERIAL_GLASS, base_color=(0.9, 0.95, 1.0), transmission=1.0, roughness=0.05, ior=1.5),
                   Material(kind=MATERIAL_GLASS, base_color=(0.9, 0.95, 1.0), transmission=1.0, roughness=0.05, flags=MATERIAL_FLAG_THIN),
                   Material(base_color=(0.5, 0.5, 0.52), roughness=0.8),
                   Material(base_color=(0.3, 0.6, 0.3), roughness=0.6)],
        meshes=[box_mesh((-50, -50, -50), (50, 50, 50)), box_mesh((-50, -50, -50), (50, 50, 50), inward=True),
                box_mesh((-50, -50, -50), (50, 50, 50), skip_faces=((2, 1),)), floor_quad(0.0, 900.0, 3),
                box_mesh((200, -100, 0), (320, 100, 150)), slices],
        instances=[Instance(0, rows=placed((1.5, 0.8, 1.2), (0.0, -140.0, 70.0)), material_id=0),
                   Instance(1, rows=(0.8, 0, 0, 0.0, 0, 0.8, 0, 0.0, 0, 0, 0.8, 60.0), material_id=1),
                   Instance(2, rows=(1, 0, 0, 0.0, 0, 1, 0, 140.0, 0, 0, 1, 60.0), material_id=0),
                   Instance(0, rows=(1, 0, 0, 0.0, 0, 1, 0, 280.0, 0, 0, 1, 60.0), material_id=2),
                   Instance(0, rows=(1, 0, 0, 60.0, 0, 1, 0, -290.0, 0, 0, 1, 60.0), material_id=4, flags=4),
                   Instance(3, material_id=3, flags=2),
                   Instance(4, material_id=4, flags=2),
                   Instance(5, material_id=0)],
        lights=[Light(kind=0, position=(200.0, -300.0, 700.0), direction=(-0.2, 0.3, -0.93), up=(0.0, 1.0, 0.0), size_x=300.0,
                      size_y=300.0, power=6.0)],
        env_kind=0, env_floor=0.05, env_horizon=0.12, env_zenith=0.3,
        width=width, height=height, max_samples=spp, seed=3, max_depth=8,
        section=(1, 1.0, 0.2, 0.0, 10.0))


def _value_noise3(p: np.ndarray, seed: int) -> np.ndarray:
    """Trilinear value noise on the unit lattice, lattice values hashed from (seed, cell) with the
    SplitMix64 finaliser; p (n, 3) float64 -> (n,) float64 in [-1, 1]."""
    c = np.floor(p).astype(np.int64)
    f = p - c
    f = f * f * (3.0 - 2.0 * f)

    def lattice(ix, iy, iz):
        z = (ix.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15) ^ iy.astype(np.uint64) * np.uint64(0xC2B2AE3D27D4EB4F)
             ^ iz.astype(np.uint64) * np.uint64(0x165667B19E3779F9) ^ np.uint64(seed) * np.uint64(0xD6E8FEB86659FD93))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
        return (z >> np.uint64(40)).astype(np.float64) / float(1 << 24) * 2.0 - 1.0

    out = 0.0
    with np.errstate(over="ignore"):
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    wgt = (f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1]) * (f[:, 2] if dz else 1 - f[:, 2])
                    out = out + wgt * lattice(c[:, 0] + dx, c[:, 1] + dy, c[:, 2] + dz)
    return out


def torus_knot(p: int = 2, q: int = 3, seg_u: int = 1024, seg_v: int = 512, radius: float = 1.0, tube: float = 0.12,
               amplitude: float = 0.02, noise_seed: int = 7, noise_scale: float = 6.0):
    """A (p, q) torus-knot tube of seg_u x seg_v quads (2 seg_u seg_v triangles), its surface
    displaced along the tube's radial direction by amplitude * tube * noise (3-D value noise,
    seeded). Returns positions (n, 3), normals (n, 3) float32 (Y-up, metres) and indices."""
    u = np.arange(seg_u, dtype=np.float64) / seg_u * 2 * math.pi
    v = np.arange(seg_v, dtype=np.float64) / seg_v * 2 * math.pi

    def curve(t):
        r = radius * (2 + np.cos(q * t)) / 3.0
        return np.stack([r * np.cos(p * t), radius * -np.sin(q * t) / 3.0, r * np.sin(p * t)], axis=-1)

    c = curve(u)
    tangent = curve(u + 1e-4) - curve(u - 1e-4)
    tangent /= np.linalg.norm(tangent, axis=1, keepdims=True)
    ref = np.array([0.0, 1.0, 0.0])
    n1 = np.cross(tangent, ref)
    n1 /= np.linalg.norm(n1, axis=1, keepdims=True)
    n2 = np.cross(tangent, n1)
    cv, sv = np.cos(v), np.sin(v)
    radial = n1[:, None, :] * cv[None, :, None] + n2[:, None, :] * sv[None, :, None]  # (U, V, 3)
    base = c[:, None, :] + tube * radial
    disp = _value_noise3(base.reshape(-1, 3) * noise_scale, noise_seed).reshape(seg_u, seg_v)
    pos = c[:, None, :] + (tube * (1.0 + amplitude * disp))[:, :, None] * radial
    # Normals: the tube's radial direction corrected by the displacement gradient (finite differences).
    du = np.roll(pos, -1, axis=0) - np.roll(pos, 1, axis=0)
    dv = np.roll(pos, -1, axis=1) - np.roll(pos, 1, axis=1)
    nrm = np.cross(du, dv)
    nrm /= np.linalg.norm(nrm, axis=2, keepdims=True)
    nrm *= np.sign(np.sum(nrm * radial, axis=2, keepdims=True))
    iu, iv = np.meshgrid(np.arange(seg_u), np.arange(seg_v), indexing="ij")
    a = iu * seg_v + iv
    b = ((iu + 1) % seg_u) * seg_v + iv
    cc = ((iu + 1) % seg_u) * seg_v + (iv + 1) % seg_v
    d = iu * seg_v + (iv + 1) % seg_v
    tris = np.stack([np.stack([a, b, cc], -1), np.stack([a, cc, d], -1)], axis=2).reshape(-1, 3)
    return pos.reshape(-1, 3).astype(np.float32), nrm.reshape(-1, 3).astype(np.float32), tris.astype(np.uint32)


def product_materials(seed: int = 7):
    """The 16-material table of the product scene, drawn from PCG32 (seed, stream 1): 6 GGX
    conductors (alpha U(0.05, 0.5)), 4 dielectrics (ior 1.5, alpha U(0, 0.2)), 6 Lambert (albedo
    U(0.1, 0.9))."""
    rng = Pcg32(seed, 1)
    f0s = [(0.95, 0.64, 0.54), (0.91, 0.92, 0.92), (1.0, 0.77, 0.34), (0.56, 0.57, 0.58), (0.97, 0.96, 0.91), (0.66, 0.62, 0.57)]
    mats = []
    for k in range(6):
        alpha = 0.05 + 0.45 * rng.next_f32()
        mats.append(Material(base_color=f0s[k], metallic=1.0, roughness=math.sqrt(alpha)))
    for _ in range(4):
        alpha = 0.2 * rng.next_f32()
        mats.append(Material(kind=1, base_color=(1.0, 1.0, 1.0), transmission=1.0, ior=1.5, roughness=math.sqrt(alpha)))
    for _ in range(6):
        a = 0.1 + 0.8 * rng.next_f32()
        mats.append(Material(base_color=(a, a, a), metallic=0.0, ior=1.0, roughness=1.0))
    return mats


def adjoint_scene(width: int = 512, height: int = 512, spp: int = 32, depth: int = 6, perturb_seed: int = 0,
                  subdivisions: int = 4) -> Scene:
    """The differentiable render's scene: the small scene's geometry (camera, icosphere of radius 1
    on a 20 x 20 floor) with the icosphere split round-robin by triangle into 16 meshes carrying
    the product scene's 16-material table, GGX alphas drawn U(0.05, 0.8), and three rect lights.
    With perturb_seed > 0, every base colour, alpha and light power is scaled by U(0.8, 1.2)
    drawn from PCG32 (perturb_seed, 3): the parameters of a target image. The floor (material 16)
    is not a parameter."""
    base = cfg0_scene()
    sphere = icosphere(yup_m_to_mm((0, 1, 0)), 1000.0, subdivisions, 0)
    tris = np.asarray(sphere.indices, np.uint32).reshape(-1, 3)
    meshes, insts = [], []
    for k in range(16):
        sel = tris[k::16]
        used, inv = np.unique(sel.reshape(-1), return_inverse=True)
        meshes.append(Mesh(np.asarray(sphere.positions, np.float32)[used], np.asarray(sphere.normals, np.float32)[used],
                           inv.astype(np.uint32), k))
        insts.append(Instance(k, material_id=k))
    meshes.append(floor_quad(0.0, 10000.0, 16))
    insts.append(Instance(16, material_id=16))
    rng = Pcg32(3, 5)
    mats = []
    for m in product_materials():
        alpha = 0.05 + 0.75 * rng.next_f32()
        mats.append(Material(kind=m.kind, base_color=m.base_color, metallic=m.metallic, transmission=m.transmission, ior=m.ior,
                             roughness=math.sqrt(alpha)))
    mats.append(Material(base_color=(0.8, 0.8, 0.8), metallic=0.0, ior=1.0, roughness=1.0))
    lights = [base.lights[0],
              Light(0, (3000.0, -2500.0, 2500.0), tuple(_normalize_py((-3000.0, 2500.0, -1500.0))), (0.0, 0.0, 1.0), 1500.0, 1500.0,
                    (1.0, 0.9, 0.8), rect_power(6.0, 1.5, 1.5), flags=3),
              Light(0, (-3000.0, 1000.0, 3000.0), tuple(_normalize_py((3000.0, -1000.0, -2000.0))), (0.0, 0.0, 1.0), 1000.0, 2000.0,
                    (0.8, 0.9, 1.0), rect_power(8.0, 1.0, 2.0), flags=3)]
    if perturb_seed:
        g = Pcg32(perturb_seed, 3)
        u = lambda: 0.8 + 0.4 * g.next_f32()
        for k in range(16):
            m = mats[k]
            m.base_color = tuple(c * u() for c in m.base_color)
            m.roughness = math.sqrt(min(m.roughness ** 2 * u(), 1.0))
        for l in lights:
            l.power *= u()
    base.meshes, base.instances, base.materials, base.lights = meshes, insts, mats, lights
    base.width, base.height, base.max_samples, base.max_depth = width, height, spp, depth
    base.focal_mm = focal_for_vfov(40.0, width, height)
    return base


_GEOMETRY_CACHE: dict = {}


def _product_geometry(seg_u: int, seg_v: int):
    """The product scene's 17 meshes (16 knot parts, one per material, and the floor) and their
    instances; built once per size."""
    key = (seg_u, seg_v)
    if key not in _GEOMETRY_CACHE:
        pos, nrm, tris = torus_knot(seg_u=seg_u, seg_v=seg_v)
        pos_mm = np.stack([pos[:, 0], -pos[:, 2], pos[:, 1]], axis=1) * np.float32(1000.0)
        nrm_mm = np.stack([nrm[:, 0], -nrm[:, 2], nrm[:, 1]], axis=1)
        lift = np.float32(-pos_mm[:, 2].min() + 20.0)
        pos_mm[:, 2] += lift
        meshes, insts = [], []
        for k in range(16):
            sel = tris[k::16]
            used, inv = np.unique(sel.reshape(-1), return_inverse=True)
            meshes.append(Mesh(pos_mm[used].astype(np.float32), nrm_mm[used].astype(np.float32), inv.astype(np.uint32), k))
            insts.append(Instance(k, material_id=k))
        meshes.append(floor_quad(0.0, 20000.0, 16))
        insts.append(Instance(16, material_id=16))
        _GEOMETRY_CACHE[key] = (meshes, tuple(insts))
    return _GEOMETRY_CACHE[key]


JOB_RESOLUTIONS = ((256, 256), (512, 512), (1280, 720), (1920, 1080), (2048, 1152))
JOB_SPP = (4, 16, 64, 256)


def light_rig(rig: int) -> List[Light]:
    """Light rig `rig` of the batched queue's workload: 1-4 rect softboxes (count, placement,
    size and radiance 1-20 drawn from PCG32 seeded with the rig number), aimed at the knot."""
    g = Pcg32(rig, 11)
    n = 1 + (g.next_u32() % 4)
    target = (0.0, 0.0, 500.0)
    out = []
    for _ in range(n):
        az = 2.0 * math.pi * g.next_f32()
        el = math.radians(20.0 + 45.0 * g.next_f32())
        dist = 3000.0 + 2500.0 * g.next_f32()
        pos = (dist * math.cos(el) * math.sin(az), -dist * math.cos(el) * math.cos(az), target[2] + dist * math.sin(el))
        d = _normalize_py(tuple(t - p for t, p in zip(target, pos)))
        sx, sy = 800.0 + 1700.0 * g.next_f32(), 800.0 + 1700.0 * g.next_f32()
        radiance = 1.0 + 19.0 * g.next_f32()
        out.append(Light(0, pos, tuple(d), (0.0, 0.0, 1.0), sx, sy, (1.0, 1.0, 1.0), rect_power(radiance, sx / 1000.0, sy / 1000.0),
                         flags=3))
    return out


def product_jobs(n_jobs: int = 64, seg_u: int = 1024, seg_v: int = 512, spp_scale: float = 1.0) -> List[Scene]:
    """The batched render queue's workload on the product geometry: job j uses camera j % 8 (orbit
    angle 45 * (j % 8) degrees, focal length 35-135 mm) and light rig j // 8 (light_rig); its
    resolution (from JOB_RESOLUTIONS), samples per pixel (from JOB_SPP, times spp_scale) and seed are
    drawn from PCG32 seeded with the job id. Each job is a Scene whose max_samples is its spp."""
    jobs = []
    rigs = [light_rig(r) for r in range((n_jobs + 7) // 8)]
    for j in range(n_jobs):
        g = Pcg32(j, 7)
        w, h = JOB_RESOLUTIONS[g.next_u32() % len(JOB_RESOLUTIONS)]
        spp = max(1, int(round(JOB_SPP[g.next_u32() % len(JOB_SPP)] * spp_scale)))
        cam = j % 8
        jobs.append(product_scene(width=w, height=h, spp=spp, seg_u=seg_u, seg_v=seg_v, seed=1 + (g.next_u32() & 0xFFFF),
                                  camera_angle_deg=45.0 * cam, focal_mm=35.0 + 100.0 * cam / 7.0, rig=rigs[j // 8]))
    return jobs


def product_scene(width: int = 1920, height: int = 1080, spp: int = 64, depth: int = 12, seg_u: int = 1024,
                  seg_v: int = 512, seed: int = 1, camera_angle_deg: float = 0.0, focal_mm: float = 50.0,
                  rig: Sequence[Light] | None = None) -> Scene:
    """The 1080p product scene: a displaced (2,3) torus knot of seg_u x seg_v quads (about 1 M
    triangles at 1024 x 512) split round-robin by triangle id into 16 meshes, one per material
    (materials are per instance in the reference), on a floor quad, lit by three rect softboxes
    of radiance 5-20 and a gradient dome (floor 0.05, horizon 0.3, zenith 0.6)."""
    meshes, insts = _product_geometry(seg_u, seg_v)
    insts = list(insts)
    mats = product_materials() + [Material(base_color=(0.6, 0.6, 0.6), ior=1.0, roughness=1.0)]
    if rig is None:
        rig = [
            Light(0, (2500.0, -2500.0, 3000.0), tuple(_normalize_py((-2500.0, 2500.0, -2600.0))), (0.0, 0.0, 1.0), 1500.0,
                  1500.0, (1.0, 1.0, 1.0), rect_power(20.0, 1.5, 1.5), flags=3),
            Light(0, (-3000.0, -1500.0, 2000.0), tuple(_normalize_py((3000.0, 1500.0, -1600.0))), (0.0, 0.0, 1.0), 1200.0,
                  2000.0, (1.0, 0.95, 0.9), rect_power(10.0, 1.2, 2.0), flags=3),
            Light(0, (0.0, 3500.0, 2500.0), tuple(_normalize_py((0.0, -3500.0, -2100.0))), (0.0, 0.0, 1.0), 2500.0, 1000.0,
                  (0.9, 0.95, 1.0), rect_power(5.0, 2.5, 1.0), flags=3),
        ]
    ang = math.radians(camera_angle_deg)
    dist = 5200.0
    cam = (dist * math.sin(ang), -dist * math.cos(ang), 1600.0)
    target = (0.0, 0.0, 500.0)
    return Scene(camera_position=cam, camera_target=target, camera_up=(0.0, 0.0, 1.0), focal_mm=focal_mm, sensor_mm=36.0,
                 materials=mats, meshes=meshes, instances=insts, lights=list(rig), env_kind=0, env_floor=0.05,
                 env_horizon=0.3, env_zenith=0.6, env_strength=1.0, width=width, height=height, max_samples=spp,
                 seed=seed, max_depth=depth)


def displaced_sphere(triangles: int = 10000, material_id: int = 0) -> Mesh:
    """rt-cli/src/bench.rs:113 displaced_sphere: a latitude/longitude grid of about `triangles`
    triangles (lat = sqrt(triangles / 4), lon = 2 lat: 10,000 exactly at 10,000) whose radius of
    about 100 mm is modulated by a few waves; no vertex normals."""
    lat = max(int(math.sqrt(triangles / 4.0)), 2)
    lon = lat * 2
    i, j = np.meshgrid(np.arange(lat + 1, dtype=np.float32), np.arange(lon, dtype=np.float32), indexing="ij")
    theta = np.float32(math.pi) * i / np.float32(lat)
    phi = np.float32(2.0 * math.pi) * j / np.float32(lon)
    r = np.float32(100.0) * (np.float32(1.0) + np.float32(0.12) * np.sin(np.float32(7.0) * theta) * np.cos(np.float32(5.0) * phi)
                             + np.float32(0.04) * np.sin(np.float32(23.0) * theta + np.float32(3.0) * phi))
    pos = np.stack([r * np.sin(theta) * np.cos(phi), r * np.sin(theta) * np.sin(phi), r * np.cos(theta)], axis=-1).reshape(-1, 3)
    ii, jj = np.meshgrid(np.arange(lat, dtype=np.uint32), np.arange(lon, dtype=np.uint32), indexing="ij")
    a = ii * lon + jj
    b = ii * lon + (jj + 1) % lon
    c, d = a + lon, b + lon
    idx = np.stack([a, c, b, b, c, d], axis=-1).reshape(-1).astype(np.uint32)
    return Mesh(pos.astype(np.float32), np.zeros_like(pos, dtype=np.float32), idx, material_id)


def _random_rotation(g: "Pcg32"):
    """A uniform random rotation (Shoemake's quaternion from three uniforms) as 3 x 3 rows."""
    u1, u2, u3 = g.next_f32(), g.next_f32(), g.next_f32()
    a, b = math.sqrt(1.0 - u1), math.sqrt(u1)
    qx, qy, qz, qw = a * math.sin(2 * math.pi * u2), a * math.cos(2 * math.pi * u2), b * math.sin(2 * math.pi * u3), b * math.cos(2 * math.pi * u3)
    return ((1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qz * qw), 2 * (qx * qz + qy * qw)),
            (2 * (qx * qy + qz * qw), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qx * qw)),
            (2 * (qx * qz - qy * qw), 2 * (qy * qz + qx * qw), 1 - 2 * (qx * qx + qy * qy)))


def cfg4_scene(width: int = 3840, height: int = 2160, spp: int = 256, depth: int = 16, n_instances: int = 1000,
               rig: Sequence[Light] | None = None, seed: int = 1) -> Scene:
    """The large stress scene: `n_instances` (1000: 10 M triangles) instances of one 10,000-triangle
    displaced sphere under random rigid transforms (PCG32 seed 11: a uniform rotation and a
    position in a 6 x 6 x 1.6 m box over the floor), instance i with material i % 16 of the product
    table, on the product floor, lit by light rig `rig` (default: rig 0) and the gradient dome.
    Instances share the sphere's tree (two levels), as the reference's instanced geometry does."""
    g = Pcg32(11, 0)
    mats = product_materials() + [Material(base_color=(0.6, 0.6, 0.6), ior=1.0, roughness=1.0)]
    meshes = [displaced_sphere(10000), floor_quad(0.0, 20000.0, 16)]
    insts = []
    for k in range(n_instances):
        rot = _random_rotation(g)
        t = (6000.0 * (g.next_f32() - 0.5), 6000.0 * (g.next_f32() - 0.5), 150.0 + 1600.0 * g.next_f32())
        rows = tuple(v for r in range(3) for v in (*rot[r], t[r]))
        insts.append(Instance(0, rows=rows, material_id=k % 16))
    insts.append(Instance(1, material_id=16))
    cam = (0.0, -7800.0, 3200.0)
    return Scene(camera_position=cam, camera_target=(0.0, 0.0, 700.0), camera_up=(0.0, 0.0, 1.0), focal_mm=35.0, sensor_mm=36.0,
                 materials=mats, meshes=meshes, instances=insts, lights=list(rig if rig is not None else light_rig(0)), env_kind=0,
                 env_floor=0.05, env_horizon=0.3, env_zenith=0.6, env_strength=1.0, width=width, height=height,
                 max_samples=spp, seed=seed, max_depth=depth)


def _normalize_py(v):
    n = math.sqrt(sum(x * x for x in v))
    return [x / n for x in v]


class Pcg32:
    """PCG-XSH-RR 64/32 (rng.rs:21), for seeded scene parameters."""

    M = 6364136223846793005

    def __init__(self, seed: int, stream: int):
        self.state = 0
        self.inc = ((stream << 1) | 1) & 0xFFFFFFFFFFFFFFFF
        self.next_u32()
        self.state = (self.state + seed) & 0xFFFFFFFFFFFFFFFF
        self.next_u32()

    def next_u32(self) -> int:
        old = self.state
        self.state = (old * self.M + self.inc) & 0xFFFFFFFFFFFFFFFF
        xs = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xs >> rot) | (xs << ((32 - rot) & 31))) & 0xFFFFFFFF

    def next_f32(self) -> float:
        return float(np.float32(self.next_u32() >> 8) * np.float32(1.0 / 16777216.0))
