// Host-side scene assembly: RSB subset reader, binned-SAH BVH build, quantised flattening and
// light preparation. See rtg_scene.h.
#include "rtg_scene.h"

#include "rtg_lights.cuh"

#include "rtg_tables.h"

#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>

namespace rtg {

// ---- RSB reader (engine/crates/rt-core/src/scene/rsb.rs:556-1640, the sections of this path) --
namespace {
struct Reader {
    const uint8_t* d;
    size_t n, pos = 0;
    std::string tag;
    std::string* err;
    bool fail = false;
    size_t remaining() const { return n - pos; }
    bool too_short() { if (!fail) *err = "RSB section " + tag + " is shorter than its layout requires"; fail = true; return false; }
    bool invalid(const char* why) { if (!fail) *err = "RSB section " + tag + " is invalid: " + why; fail = true; return false; }
    bool u32(uint32_t& v) { if (fail) return false; if (remaining() < 4) return too_short(); std::memcpy(&v, d + pos, 4); pos += 4; return true; }
    bool f32(float& v) { uint32_t u; if (!u32(u)) return false; v = bitsf(u); if (!finitef(v)) return invalid("non-finite number"); return true; }
    bool vec3(V3& v) { return f32(v.x) && f32(v.y) && f32(v.z); }
    bool f3(float* c) { return f32(c[0]) && f32(c[1]) && f32(c[2]); }
    bool ou32(uint32_t& v, uint32_t def) { if (remaining() >= 4) return u32(v); v = def; return !fail; }
    bool of32(float& v, float def) { if (remaining() >= 4) return f32(v); v = def; return !fail; }
};
std::string tag_text(const uint8_t* t) {
    std::string s;
    for (int i = 0; i < 4; ++i) s += (t[i] >= 33 && t[i] <= 126) ? (char)t[i] : '?';
    return s;
}

// Mesh::with_width validation and inside_out (geometry/mesh.rs:136-200).
const char* make_mesh(HMesh& m, std::vector<V3>&& p, std::vector<V3>&& nn, std::vector<uint32_t>&& idx, uint32_t mat) {
    if (idx.size() % 3 != 0) return "index_count is not a multiple of 3";
    if (idx.size() / 3 > (size_t)((1u << 28) - 2) || p.size() >= 0xffffffffull) return "too many triangles or vertices";
    for (uint32_t i : idx) if (i >= p.size()) return "vertex index out of range";
    if (!nn.empty() && nn.size() != p.size()) return "normals are not one per vertex";
    for (const V3& v : p) if (!vfinite(v)) return "non-finite vertex position";
    for (const V3& v : nn) if (!vfinite(v)) return "non-finite vertex normal";
    bool any = false;
    for (const V3& v : nn) if (!veq(v, v3(0, 0, 0))) { any = true; break; }
    m.positions = std::move(p);
    m.normals = any ? std::move(nn) : std::vector<V3>();
    m.indices = std::move(idx);
    m.material_id = mat;
    V3 lo = v3(f_inf(), f_inf(), f_inf()), hi = v3(-f_inf(), -f_inf(), -f_inf());
    for (const V3& v : m.positions) {
        lo = v3(rmin(lo.x, v.x), rmin(lo.y, v.y), rmin(lo.z, v.z));
        hi = v3(rmax(hi.x, v.x), rmax(hi.y, v.y), rmax(hi.z, v.z));
    }
    m.bmin = lo; m.bmax = hi;
    m.empty_bounds = m.positions.empty();
    m.inside_out = false;
    if (!m.normals.empty()) {
        float agreement = 0.0f;
        for (size_t t = 0; t < m.triangles(); ++t) {
            V3 a = m.positions[m.indices[3 * t]], b = m.positions[m.indices[3 * t + 1]], c = m.positions[m.indices[3 * t + 2]];
            V3 w = cross(b - a, c - a);
            V3 n = v3(0, 0, 0);
            for (int k = 0; k < 3; ++k) n = n + m.normals[m.indices[3 * t + k]];
            agreement += dot(normalize(w), n);
        }
        m.inside_out = agreement < 0.0f;
    }
    return "";
}
}  // namespace

bool parse_rsb(const uint8_t* bytes, size_t len, HScene& s, std::string& error, const std::vector<HMesh>* kept, bool* used_kept,
               const std::vector<HImage>* kept_bitmaps) {
    s = HScene();
    if (used_kept) *used_kept = false;
    bool seen_mesh = false;
    if (len < 4 || std::memcmp(bytes, "RSB1", 4) != 0) { error = "not an RSB file (missing RSB1 magic)"; return false; }
    if (len < 8) { error = "RSB file is truncated in header"; return false; }
    uint32_t header_len;
    std::memcpy(&header_len, bytes + 4, 4);
    size_t pos = 8 + (size_t)header_len;
    if (pos > len) { error = "RSB file is truncated in header"; return false; }
    bool seen_cam = false, seen_env = false, seen_floor = false, seen_render = false, seen_section = false;
    while (pos < len) {
        if (len - pos < 8) { error = "RSB file is truncated in section header"; return false; }
        const uint8_t* tag = bytes + pos;
        uint32_t n;
        std::memcpy(&n, bytes + pos + 4, 4);
        if ((size_t)n > len - pos - 8) { error = "RSB file is truncated in section payload"; return false; }
        Reader r{bytes + pos + 8, n, 0, tag_text(tag), &error};
        pos += 8 + (size_t)n;
        auto is = [&](const char* t) { return std::memcmp(tag, t, 4) == 0; };
        auto once = [&](bool& seen) {
            if (seen) { error = "RSB section " + r.tag + " appears more than once"; return false; }
            seen = true;
            return true;
        };
        if (is("CAMR")) {
            if (!once(seen_cam)) return false;
            if (!(r.vec3(s.cam_position) && r.vec3(s.cam_target) && r.vec3(s.cam_up) && r.f32(s.focal_mm) && r.f32(s.sensor_mm) &&
                  r.f32(s.fstop) && r.f32(s.focus_dist) && r.u32(s.ortho) && r.f32(s.ortho_width) && r.ou32(s.projection, 0) &&
                  r.of32(s.fov_x, 360) && r.of32(s.fov_y, 180) && r.of32(s.exterior, 1)))
                return false;
            s.ortho = s.ortho != 0;
            if (s.focal_mm <= 0.0f || s.sensor_mm <= 0.0f) return r.invalid("focal_mm and sensor_mm must be positive");
            if (s.fstop < 0.0f || s.focus_dist < 0.0f || s.ortho_width < 0.0f)
                return r.invalid("fstop, focus_dist and ortho_width must not be negative");
            if (!(s.fov_x > 0.0f && s.fov_x <= 3600.0f) || !(s.fov_y > 0.0f && s.fov_y <= 3600.0f))
                return r.invalid("fov_x_deg and fov_y_deg must be positive and at most 3600");
            if (s.exterior < 0.0f) return r.invalid("exterior must not be negative");
        } else if (is("MESH")) {
            seen_mesh = true;
            uint32_t vc, ic;
            if (!(r.u32(vc) && r.u32(ic))) return false;
            if (((uint64_t)vc * 6 + ic + 1) * 4 > r.remaining()) return r.too_short();
            if (ic % 3 != 0) return r.invalid("index_count is not a multiple of 3");
            std::vector<V3> p(vc), nn(vc);
            for (auto& v : p) if (!r.vec3(v)) return false;
            for (auto& v : nn) if (!r.vec3(v)) return false;
            std::vector<uint32_t> idx(ic);
            for (auto& i : idx) {
                if (!r.u32(i)) return false;
                if (i >= vc) return r.invalid("vertex index out of range");
            }
            uint32_t mat;
            if (!r.u32(mat)) return false;
            HMesh m;
            const char* e = make_mesh(m, std::move(p), std::move(nn), std::move(idx), mat);
            if (*e) return r.invalid(e);
            if (r.remaining() >= 4) {  // UV sets of textured files: read and ignored
                uint32_t sets = 0;
                if (!r.u32(sets)) return false;
                if (sets > 2) return r.invalid("at most 2 UV sets");
                if ((uint64_t)sets * vc * 8 > r.remaining()) return r.too_short();
                for (uint64_t k = 0; k < (uint64_t)sets * vc * 2; ++k) { float f; if (!r.f32(f)) return false; }
            }
            s.meshes.push_back(std::move(m));
        } else if (is("INST")) {
            HInstance in;
            if (!r.u32(in.mesh)) return false;
            for (int k = 0; k < 12; ++k) if (!r.f32(in.rows[k])) return false;
            if (!(r.u32(in.material_id) && r.u32(in.flags))) return false;
            s.instances.push_back(in);
        } else if (is("MATL")) {
            HMaterial m;
            if (!(r.u32(m.kind) && r.f3(m.base) && r.f32(m.metallic) && r.f32(m.roughness) && r.f32(m.ior) && r.f32(m.transmission) &&
                  r.f32(m.coat) && r.f32(m.coat_roughness) && r.f3(m.emission) && r.f32(m.emission_power) && r.ou32(m.flags, 0) &&
                  r.of32(m.opacity, 1) && r.of32(m.anisotropy, 0) && r.of32(m.absorption_mm, 0) && r.of32(m.bevel_mm, 0) &&
                  r.of32(m.scatter_mm, 0) && r.of32(m.scatter_color[0], 1) && r.of32(m.scatter_color[1], 1) &&
                  r.of32(m.scatter_color[2], 1) && r.of32(m.scatter_g, 0) && r.of32(m.abbe, 0)))
                return false;
            if (r.remaining() >= 4 && r.pos == 100) {
                uint32_t version = 0;
                r.u32(version);
                if (version == 1) { error = "unsupported: material texture block"; return false; }
            }
            s.materials.push_back(m);
        } else if (is("LGHT")) {
            HLight l;
            if (!r.u32(l.kind)) return false;
            if (l.kind > 5) return r.invalid("unknown light kind");
            if (!(r.vec3(l.position) && r.vec3(l.direction) && r.vec3(l.up) && r.f32(l.size_x) && r.f32(l.size_y) && r.f3(l.color) &&
                  r.f32(l.power) && r.f32(l.spread_deg) && r.f32(l.angle_deg) && r.u32(l.flags)))
                return false;
            if (l.kind == 5 && !r.ou32(l.profile, 0xffffffffu)) return false;  // rsb.rs:1006
            s.lights.push_back(l);
        } else if (is("ENVR")) {
            if (!once(seen_env)) return false;
            if (!r.u32(s.env_kind)) return false;
            if (s.env_kind > 3) return r.invalid("unknown environment kind");
            if (!(r.f32(s.env_floor) && r.f32(s.env_horizon) && r.f32(s.env_zenith) && r.f32(s.env_strength) && r.f32(s.env_rotation) &&
                  r.f3(s.background_color) && r.u32(s.background_mode)))
                return false;
            if (!(r.ou32(s.hdri_map, 0xffffffffu) && r.ou32(s.backplate_map, 0xffffffffu) && r.ou32(s.backplate_fit, 0) &&
                  r.of32(s.sky_turbidity, 3.0f) && r.of32(s.sun_azimuth_deg, 0.0f) && r.of32(s.sun_elevation_deg, 45.0f) &&
                  r.of32(s.backplate_rect[0], 0.0f) && r.of32(s.backplate_rect[1], 0.0f) && r.of32(s.backplate_rect[2], 1.0f) &&
                  r.of32(s.backplate_rect[3], 1.0f) && r.ou32(s.sky_model, 0)))
                return false;
        } else if (is("IESP")) {  // rsb.rs:1018: an IES file
            uint32_t n;
            if (!r.u32(n)) return false;
            if ((size_t)n > r.remaining()) return r.too_short();
            HIes prof;
            std::string reason;
            if (!parse_ies(r.d + r.pos, n, prof, reason)) return r.invalid(reason.c_str());
            r.pos += n;
            s.profiles.push_back(std::move(prof));
        } else if (is("BMAP")) {  // rsb.rs:1057
            uint32_t format, w, h, n;
            if (!(r.u32(format) && r.u32(w) && r.u32(h) && r.u32(n))) return false;
            if ((size_t)n > r.remaining()) return r.too_short();
            HImage img;
            std::string reason;
            bool unsupported = false;
            if (!decode_bitmap(format, w, h, r.d + r.pos, n, img, reason, unsupported)) {
                if (unsupported) { error = reason; return false; }
                return r.invalid(reason.c_str());
            }
            r.pos += n;
            s.bitmaps.push_back(std::move(img));
        } else if (is("SECT")) {  // rsb.rs:1070 parse_section, geometry/section.rs:69 SectionPlane::new
            if (!once(seen_section)) return false;
            uint32_t flags;
            V3 n;
            float d;
            if (!(r.u32(flags) && r.vec3(n) && r.f32(d))) return false;
            const float length = std::sqrt(len2(n));
            if (!(std::isfinite(length) && length > 0.0f)) return r.invalid("section normal is zero");
            s.section_on = 1;
            s.section_cap = (flags & 1u) != 0;
            s.section_n = absf(length - 1.0f) <= 1.0e-6f ? n : n * (1.0f / length);
            s.section_d = d;
        } else if (is("FLOR")) {
            if (!once(seen_floor)) return false;
            if (!(r.u32(s.floor_mode) && r.f32(s.floor_z) && r.f3(s.floor_color))) return false;
            if (s.floor_mode > 2) return r.invalid("unknown floor mode");
            if (s.floor_mode == 2) { error = "unsupported: shadow catcher floor"; return false; }
        } else if (is("RNDR")) {
            if (!once(seen_render)) return false;
            uint32_t passes, denoise, photons;
            float radius, strength;
            if (!(r.u32(s.width) && r.u32(s.height) && r.u32(s.max_samples) && r.u32(s.seed) && r.f32(s.max_seconds) &&
                  r.f32(s.exposure_ev) && r.u32(s.tonemap) && r.ou32(s.max_depth, 8) && r.of32(s.clamp_indirect, 0) &&
                  r.ou32(passes, 0) && r.ou32(denoise, 0) && r.ou32(photons, 0) && r.of32(radius, 0) && r.of32(strength, 1) &&
                  r.ou32(s.pixel_filter, 0) && r.ou32(s.edge_supersample, 1) && r.ou32(s.adaptive, 0) && r.of32(s.noise_threshold, 0)))
                return false;
            if (!(s.noise_threshold >= 0.0f && s.noise_threshold <= 1.0f)) return r.invalid("noise_threshold must be between 0 and 1");
            if (s.edge_supersample > 16) return r.invalid("edge_supersample must be at most 16");
            if (!(strength >= 0.0f && strength <= 1.0f)) return r.invalid("denoise_strength must be between 0 and 1");
            if (photons > (1u << 22)) return r.invalid("caustic_photons must be at most 4194304");
            if (radius < 0.0f) return r.invalid("caustic_radius must not be negative");
            // The photon maps of caustics (caustics.rs) are not built: a scene that asks for them is
            // refused rather than rendered without them.
            if (photons > 0) { error = "unsupported: caustic photon maps (caustic_photons above 0)"; return false; }
            if (s.width < 1 || s.width > 16384 || s.height < 1 || s.height > 16384)
                return r.invalid("width and height must be between 1 and 16384");
            if (s.max_seconds < 0.0f || s.clamp_indirect < 0.0f) return r.invalid("max_seconds and clamp_indirect must not be negative");

        } else {
            static const char* feature_tags[] = {"LENS", "PATN", "IMGS", "PROG", "FXAM",
                                                 "GLAS", "WETP", "WETF", "WTP2", "WETG", "NEST"};
            for (const char* t : feature_tags)
                if (is(t)) { error = std::string("unsupported: RSB section ") + t; return false; }
        }
    }
    if (!seen_mesh && kept) {
        s.meshes = *kept;
        if (used_kept) *used_kept = true;
    }
    if (s.bitmaps.empty() && kept_bitmaps) s.bitmaps = *kept_bitmaps;
    for (const HLight& l : s.lights)  // rsb.rs:1354
        if (l.kind == 5 && l.profile >= s.profiles.size()) {
            error = "RSB section LGHT is invalid: an IES light needs a profile that is an IESP section";
            return false;
        }
    for (uint32_t map : {s.hdri_map, s.backplate_map})
        if (map != 0xffffffffu && map >= s.bitmaps.size()) {
            error = "RSB section ENVR is invalid: bitmap index does not refer to a BMAP section";
            return false;
        }
    size_t nm = s.materials.size();
    for (const HMesh& m : s.meshes)
        if (m.material_id >= nm) { error = "RSB section MESH is invalid: material_id does not refer to a MATL section"; return false; }
    if (s.instances.empty())
        for (size_t i = 0; i < s.meshes.size(); ++i) {
            HInstance in;
            in.mesh = (uint32_t)i;
            in.material_id = s.meshes[i].material_id;
            s.instances.push_back(in);
        }
    for (const HInstance& in : s.instances) {
        if (in.mesh >= s.meshes.size()) { error = "RSB section INST is invalid: mesh_id does not refer to a MESH section"; return false; }
        if (in.material_id >= nm) { error = "RSB section INST is invalid: material_id does not refer to a MATL section"; return false; }
    }
    for (const HMaterial& m : s.materials) {
        bool emissive = m.kind == MATERIAL_EMISSIVE;
        if (m.scatter_mm > 0.0f && m.transmission > 0.0f) { error = "unsupported: scattering media"; return false; }
        if (m.abbe > 0.0f && m.transmission > 0.0f) { error = "unsupported: dispersive glass"; return false; }
        if (m.bevel_mm > 0.0f) { error = "unsupported: edge bevel"; return false; }
    }
    return true;
}

// ---- transforms (geometry/transform.rs) ------------------------------------------------------
namespace {
struct Xf { float r[3][4]; };
Xf xf_of(const float* rows) { Xf x; for (int i = 0; i < 3; ++i) for (int j = 0; j < 4; ++j) x.r[i][j] = rows[4 * i + j]; return x; }
bool xf_identity(const Xf& x) {
    static const float I[3][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}};
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 4; ++j) if (!(x.r[i][j] == I[i][j])) return false;
    return true;
}
V3 xf_point(const Xf& x, V3 p) {
    const float(*r)[4] = x.r;
    return v3(r[0][0] * p.x + r[0][1] * p.y + r[0][2] * p.z + r[0][3], r[1][0] * p.x + r[1][1] * p.y + r[1][2] * p.z + r[1][3],
              r[2][0] * p.x + r[2][1] * p.y + r[2][2] * p.z + r[2][3]);
}
V3 xf_vector(const Xf& x, V3 v) {
    const float(*r)[4] = x.r;
    return v3(r[0][0] * v.x + r[0][1] * v.y + r[0][2] * v.z, r[1][0] * v.x + r[1][1] * v.y + r[1][2] * v.z,
              r[2][0] * v.x + r[2][1] * v.y + r[2][2] * v.z);
}
bool xf_inverse(const Xf& x, Xf& out) {
    const float(*r)[4] = x.r;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 4; ++j) if (!finitef(r[i][j])) return false;
    float det = r[0][0] * (r[1][1] * r[2][2] - r[1][2] * r[2][1]) - r[0][1] * (r[1][0] * r[2][2] - r[1][2] * r[2][0]) +
                r[0][2] * (r[1][0] * r[2][1] - r[1][1] * r[2][0]);
    if (det == 0.0f || !finitef(det)) return false;
    float inv_det = 1.0f / det;
    float c[3][3] = {
        {r[1][1] * r[2][2] - r[1][2] * r[2][1], r[0][2] * r[2][1] - r[0][1] * r[2][2], r[0][1] * r[1][2] - r[0][2] * r[1][1]},
        {r[1][2] * r[2][0] - r[1][0] * r[2][2], r[0][0] * r[2][2] - r[0][2] * r[2][0], r[0][2] * r[1][0] - r[0][0] * r[1][2]},
        {r[1][0] * r[2][1] - r[1][1] * r[2][0], r[0][1] * r[2][0] - r[0][0] * r[2][1], r[0][0] * r[1][1] - r[0][1] * r[1][0]}};
    Xf t;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) t.r[i][j] = c[i][j] * inv_det;
    float tr[3] = {r[0][3], r[1][3], r[2][3]};
    for (int i = 0; i < 3; ++i) t.r[i][3] = -(t.r[i][0] * tr[0] + t.r[i][1] * tr[1] + t.r[i][2] * tr[2]);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 4; ++j) if (!finitef(t.r[i][j])) return false;
    out = t;
    return true;
}

struct Box {
    V3 lo = v3(f_inf(), f_inf(), f_inf()), hi = v3(-f_inf(), -f_inf(), -f_inf());
    bool empty() const { return lo.x > hi.x || lo.y > hi.y || lo.z > hi.z; }
    Box uni(const Box& o) const {
        Box b;
        b.lo = v3(rmin(lo.x, o.lo.x), rmin(lo.y, o.lo.y), rmin(lo.z, o.lo.z));
        b.hi = v3(rmax(hi.x, o.hi.x), rmax(hi.y, o.hi.y), rmax(hi.z, o.hi.z));
        return b;
    }
    Box ext(V3 p) const {
        Box b;
        b.lo = v3(rmin(lo.x, p.x), rmin(lo.y, p.y), rmin(lo.z, p.z));
        b.hi = v3(rmax(hi.x, p.x), rmax(hi.y, p.y), rmax(hi.z, p.z));
        return b;
    }
    V3 centroid() const { return (lo + hi) * 0.5f; }
    float area() const {
        if (empty()) return 0.0f;
        V3 d = hi - lo;
        return 2.0f * (d.x * d.y + d.y * d.z + d.z * d.x);
    }
};
Box xf_box(const Xf& x, const Box& b) {
    if (b.empty()) return Box();
    Box out;
    for (int corner = 0; corner < 8; ++corner) {
        V3 p = v3((corner & 1) == 0 ? b.lo.x : b.hi.x, (corner & 2) == 0 ? b.lo.y : b.hi.y, (corner & 4) == 0 ? b.lo.z : b.hi.z);
        out = out.ext(xf_point(x, p));
    }
    return out;
}
// geometry/mod.rs:269: a transformed instance's world box, padded against rounding.
Box instance_box(const HMesh& m, const Xf& x) {
    Box b;
    b.lo = m.bmin; b.hi = m.bmax;
    if (m.empty_bounds) b = Box();
    if (xf_identity(x)) return b;
    Box w = xf_box(x, b);
    float scale = rmax(rmax(rmax(absf(w.lo.x), absf(w.hi.x)), rmax(absf(w.lo.y), absf(w.hi.y))), rmax(absf(w.lo.z), absf(w.hi.z)));
    V3 pad = v3(scale * 1.0e-5f, scale * 1.0e-5f, scale * 1.0e-5f);
    w.lo = w.lo - pad;
    w.hi = w.hi + pad;
    return w;
}

// ---- binned SAH build (geometry/bvh.rs:246-420) ------------------------------------------------
constexpr int BINS = 16;
struct BNode { Box box; uint32_t left = 0, right = 0, first = 0, count = 0; };
struct SahBuilder {
    const std::vector<Box>& boxes;
    const std::vector<V3>& cents;
    int leaf_target, leaf_max;
    std::vector<uint32_t> order;
    std::vector<BNode> nodes;

    static size_t bin_of(float c, float lo, float scale) {
        float v = (c - lo) * scale;
        uint32_t b = f2u32_floor_nonneg(v);
        return b < (uint32_t)(BINS - 1) ? b : (size_t)(BINS - 1);
    }
    uint32_t build(size_t b, size_t e, uint32_t depth) {
        Box bb, cb;
        for (size_t i = b; i < e; ++i) { bb = bb.uni(boxes[order[i]]); cb = cb.ext(cents[order[i]]); }
        uint32_t index = (uint32_t)nodes.size();
        BNode n;
        n.box = bb; n.first = (uint32_t)b; n.count = (uint32_t)(e - b);
        nodes.push_back(n);
        if (e - b <= (size_t)leaf_target) return index;
        size_t mid;
        if (!split(b, e, bb, cb, depth, mid)) return index;
        uint32_t l = build(b, mid, depth + 1);
        uint32_t r = build(mid, e, depth + 1);
        nodes[index].left = l; nodes[index].right = r; nodes[index].count = 0;
        return index;
    }
    bool split(size_t b, size_t e, const Box& bb, const Box& cb, uint32_t depth, size_t& mid) {
        size_t count = e - b, median = b + count / 2;
        if (depth >= 32) { mid = median; return true; }
        uint32_t counts[3][BINS] = {};
        Box bins[3][BINS];
        float scales[3] = {0, 0, 0};
        bool usable[3] = {false, false, false};
        for (int a = 0; a < 3; ++a) {
            float ext = comp(cb.hi, a) - comp(cb.lo, a);
            if (ext > 0.0f && finitef(ext)) { usable[a] = true; scales[a] = (float)BINS / ext; }
        }
        bool have = false;
        int best_axis = 0, best_plane = 0;
        float best_cost = 0;
        if (usable[0] || usable[1] || usable[2]) {
            for (size_t i = b; i < e; ++i) {
                uint32_t p = order[i];
                for (int a = 0; a < 3; ++a)
                    if (usable[a]) {
                        size_t k = bin_of(comp(cents[p], a), comp(cb.lo, a), scales[a]);
                        counts[a][k] += 1;
                        bins[a][k] = bins[a][k].uni(boxes[p]);
                    }
            }
            for (int a = 0; a < 3; ++a) {
                if (!usable[a]) continue;
                float right_area[BINS] = {};
                uint32_t right_count[BINS] = {};
                Box acc;
                uint32_t nn = 0;
                for (int pl = BINS - 2; pl >= 0; --pl) {
                    acc = acc.uni(bins[a][pl + 1]);
                    nn += counts[a][pl + 1];
                    right_area[pl] = acc.area();
                    right_count[pl] = nn;
                }
                acc = Box();
                nn = 0;
                for (int pl = 0; pl < BINS - 1; ++pl) {
                    acc = acc.uni(bins[a][pl]);
                    nn += counts[a][pl];
                    if (nn == 0 || right_count[pl] == 0) continue;
                    float cost = acc.area() * (float)nn + right_area[pl] * (float)right_count[pl];
                    if (!have || cost < best_cost) { have = true; best_axis = a; best_plane = pl; best_cost = cost; }
                }
            }
        }
        if (!have) {
            if (count > (size_t)leaf_max) { mid = median; return true; }
            return false;
        }
        float area = bb.area();
        float split_cost = (area > 0.0f && finitef(area)) ? 1.0f + 1.0f * best_cost / area : 1.0f;
        if (count <= (size_t)leaf_max && 1.0f * (float)count <= split_cost) return false;
        float lo = comp(cb.lo, best_axis);
        float scale = (float)BINS / (comp(cb.hi, best_axis) - lo);
        size_t i = b, j = e;
        while (i < j) {
            if (bin_of(comp(cents[order[i]], best_axis), lo, scale) <= (size_t)best_plane) ++i;
            else { --j; std::swap(order[i], order[j]); }
        }
        mid = (i == b || i == e) ? median : i;
        return true;
    }
};

// ---- 8-wide collapse (bvh.rs:439) and quantisation -------------------------------------------------
// The decoded lower/upper plane of a child, with the kernels' operations.
inline float decode(float p, uint32_t q, float scale) { return p + (float)q * scale; }

struct Flattener {
    Flat& F;
    const std::vector<BNode>* bn = nullptr;
    const std::vector<uint32_t>* order = nullptr;
    // emit(prims) -> leaf reference
    std::function<uint32_t(const uint32_t*, uint32_t)> emit;
    uint32_t max_depth = 0;
    // The top level: a child box that is flat on an axis but not at its node's lower corner
    // there (a floor under instances whose rotated boxes reach below it) is wrapped into a node
    // of its own, whose origin is the box itself, so that it decodes to the exact plane and the
    // slab test drops the hits just before t_min as the reference's tree does.
    bool exact_flat = false;
    bool wrapped = false;

    void quantise(QNode& q, const Box* kids, int nk) {
        Box nb;
        for (int k = 0; k < nk; ++k) nb = nb.uni(kids[k]);
        float p[3] = {nb.lo.x, nb.lo.y, nb.lo.z};
        q.px = p[0]; q.py = p[1]; q.pz = p[2];
        uint8_t* es[3] = {&q.ex, &q.ey, &q.ez};
        for (int a = 0; a < 3; ++a) {
            float extent = comp(nb.hi, a) - p[a];
            int e = 1;  // biased exponent, 2^(e-127); at least the smallest normal
            if (extent > 0.0f) {
                int ex;
                std::frexp((double)extent / 255.0, &ex);  // extent/255 < 2^ex
                e = ex + 127;
                if (e < 1) e = 1;
            }
            for (;; ++e) {
                if (e > 254) e = 254;
                float scale = bitsf((uint32_t)e << 23);
                bool ok = true;
                uint8_t lo[8], hi[8];
                for (int k = 0; k < nk && ok; ++k) {
                    float clo = comp(kids[k].lo, a), chi = comp(kids[k].hi, a);
                    double ql = std::floor(((double)clo - (double)p[a]) / (double)scale);
                    double qh = std::ceil(((double)chi - (double)p[a]) / (double)scale);
                    long a0 = (long)std::max(0.0, ql), a1 = (long)std::min(255.0, std::max(0.0, qh));
                    while (a0 > 0 && decode(p[a], (uint32_t)a0, scale) > clo) --a0;
                    while (a1 < 255 && decode(p[a], (uint32_t)a1, scale) < chi) ++a1;
                    if (decode(p[a], (uint32_t)a0, scale) > clo || decode(p[a], (uint32_t)a1, scale) < chi) ok = false;
                    lo[k] = (uint8_t)a0;
                    hi[k] = (uint8_t)a1;
                }
                if (ok || e == 254) {
                    *es[a] = (uint8_t)e;
                    for (int k = 0; k < 8; ++k) {
                        q.qlo[a][k] = k < nk ? lo[k] : 255;
                        q.qhi[a][k] = k < nk ? hi[k] : 0;
                    }
                    break;
                }
            }
        }
        q.nchild = (uint8_t)nk;
    }
    // Reference of the subtree replacing binary node b (Collapser::reference).
    uint32_t reference(uint32_t b, uint32_t depth) {
        const BNode& node = (*bn)[b];
        if (node.count > 0) return emit(order->data() + node.first, node.count);
        if (depth + 1 > max_depth) max_depth = depth + 1;
        uint32_t index = (uint32_t)F.nodes.size();
        F.nodes.push_back(QNode());
        uint32_t kids[8] = {};
        kids[0] = node.left;
        kids[1] = node.right;
        int n = 2;
        while (n < 8) {
            int widest = -1;
            float warea = 0;
            for (int s = 0; s < n; ++s) {
                const BNode& k = (*bn)[kids[s]];
                if (k.count == 0) {
                    float a = k.box.area();
                    if (widest < 0 || a > warea) { widest = s; warea = a; }
                }
            }
            if (widest < 0) break;
            BNode opened = (*bn)[kids[widest]];
            for (int s = n - 1; s >= widest + 1; --s) kids[s + 1] = kids[s];
            kids[widest] = opened.left;
            kids[widest + 1] = opened.right;
            ++n;
        }
        Box boxes[8];
        for (int s = 0; s < n; ++s) boxes[s] = (*bn)[kids[s]].box;
        uint32_t refs[8];
        for (int s = 0; s < n; ++s) refs[s] = reference(kids[s], depth + 1);
        if (exact_flat) {
            Box nb;
            for (int s = 0; s < n; ++s) nb = nb.uni(boxes[s]);
            for (int s = 0; s < n; ++s)
                for (int a = 0; a < 3; ++a) {
                    const float lo = comp(boxes[s].lo, a);
                    if (lo != comp(boxes[s].hi, a) || lo == comp(nb.lo, a)) continue;
                    QNode qw;
                    std::memset(&qw, 0, sizeof(qw));
                    quantise(qw, &boxes[s], 1);
                    qw.child[0] = refs[s];
                    for (int k = 1; k < 8; ++k) qw.child[k] = NODE_EMPTY;
                    refs[s] = (uint32_t)F.nodes.size();
                    F.nodes.push_back(qw);
                    wrapped = true;
                    break;
                }
        }
        QNode q;
        std::memset(&q, 0, sizeof(q));
        quantise(q, boxes, n);
        for (int s = 0; s < 8; ++s) q.child[s] = s < n ? refs[s] : NODE_EMPTY;
        F.nodes[index] = q;
        return index;
    }
};
}  // namespace

// ---- light preparation (light.rs:245-995) ----------------------------------------------------------
static bool prepare_lights(const HScene& s, const Box& scene_box, LightsDev& L, Flat& F, std::string& error) {
    std::memset(&L, 0, sizeof(L));
    V3 centre;
    float radius;
    if (scene_box.empty()) { centre = v3(0, 0, 0); radius = 1000.0f; }
    else { centre = scene_box.centroid(); radius = rmax(0.5f * len(scene_box.hi - scene_box.lo), 1.0f); }
    float radius_m = radius * 1.0e-3f;
    auto reach = [&](V3 p, const V3* normal) {
        V3 to_centre = centre - p;
        float d = len(to_centre) * 1.0e-3f;
        float facing = normal ? 0.05f + 0.95f * rmax(dot(*normal, normalize(to_centre)), 0.0f) : 1.0f;
        d = rmax(d, radius_m);
        return facing / (d * d);
    };
    // Each kind is collected in scene order; the selection entries keep the scene's order and
    // point into lights[] once the kinds are laid out as areas, then suns, then spheres.
    std::vector<float> weights;
    std::vector<LightDev> kinds[3];
    // The IES lights' tables, laid out once so that the lights can point into them.
    std::vector<size_t> ies_at(s.lights.size(), 0);
    F.ies_data.clear();
    for (size_t li = 0; li < s.lights.size(); ++li)
        if (s.lights[li].kind == 5) {
            const HIes& p = s.profiles[s.lights[li].profile];
            ies_at[li] = F.ies_data.size();
            F.ies_data.insert(F.ies_data.end(), p.vertical.begin(), p.vertical.end());
            F.ies_data.insert(F.ies_data.end(), p.horizontal.begin(), p.horizontal.end());
            F.ies_data.insert(F.ies_data.end(), p.candela.begin(), p.candela.end());
        }
    std::vector<std::pair<uint32_t, uint32_t>> refs;  // (kind, index in its kind) per entry
    auto put3 = [](float* d, V3 v) { d[0] = v.x; d[1] = v.y; d[2] = v.z; };
    for (size_t li = 0; li < s.lights.size(); ++li) {
        const HLight& l = s.lights[li];
        float power = rmax(l.power, 0.0f);
        uint32_t entry = (uint32_t)refs.size();
        float color[3] = {rmax(l.color[0], 0.0f), rmax(l.color[1], 0.0f), rmax(l.color[2], 0.0f)};
        float lum = 0.2126f * color[0] + 0.7152f * color[1] + 0.0722f * color[2];
        LightDev a;
        std::memset(&a, 0, sizeof(a));
        a.glossy = (l.flags & 1u) != 0;
        a.camera = (l.flags & 2u) != 0;
        a.shadow = (l.flags & 4u) == 0;
        a.entry = entry;
        a.source = (uint32_t)li;
        if (l.kind == 2) {  // sun (light.rs:755)
            V3 to_sun = -normalize(l.direction);
            if (len2(to_sun) < 0.5f) continue;
            float half = rmin(0.5f * rmax(l.angle_deg, 0.0f) * (PI / 180.0f), FRAC_PI_2);
            Rgb irr = rgb(color[0] * power, color[1] * power, color[2] * power);
            if (!(luminance(irr) > 0.0f)) continue;
            a.kind = LIGHT_SUN;
            a.delta = half < 1.0e-5f;
            float sh, ch;
            sin_cos(0.5f * half, sh, ch);
            a.one_minus_cos_max = 2.0f * sh * sh;
            float sin_max, cos_half;
            sin_cos(half, sin_max, cos_half);
            Rgb rad = a.delta ? irr : irr * (1.0f / (PI * sin_max * sin_max));
            a.radiance[0] = rad.r; a.radiance[1] = rad.g; a.radiance[2] = rad.b;
            weights.push_back(PI * luminance(irr));
            Frame f = frame_from_normal(to_sun);
            put3(a.fx, f.x); put3(a.fy, f.y); put3(a.fz, f.z);
            a.cos_max = 1.0f - a.one_minus_cos_max;
            a.solid_angle = TAU * a.one_minus_cos_max;
            a.base = luminance(irr);
        } else if (l.kind == 3 || l.kind == 4 || l.kind == 5) {  // point light, spot or IES light (light.rs:780)
            a.kind = LIGHT_SPHERE;
            float k = power / (4.0f * PI);
            a.intensity[0] = color[0] * k; a.intensity[1] = color[1] * k; a.intensity[2] = color[2] * k;
            const float r_light = 0.5f * absf(l.size_x);
            a.radius = finitef(r_light) ? r_light : 0.0f;
            V3 axis = v3(0.0f, 0.0f, -1.0f);
            const HIes* ies = nullptr;
            if (l.kind == 5) {  // L5: masked by its profile in the frame of its axis and its up
                ies = &s.profiles[l.profile];
                V3 z = normalize(l.direction);
                V3 y = normalize(l.up - z * dot(z, l.up));
                Frame f;
                if (len2(y) < 0.5f) f = frame_from_normal(z);
                else { f.x = cross(y, z); f.y = y; f.z = z; }
                if (len2(f.z) < 0.5f) continue;
                put3(a.fx, f.x); put3(a.fy, f.y);
                axis = f.z;
                a.ies = F.ies_data.data() + ies_at[li];
                a.ies_nv = (uint32_t)ies->vertical.size();
                a.ies_nh = (uint32_t)ies->horizontal.size();
                a.ies_sym = ies->symmetry;
                a.ies_peak = ies->peak;
            }
            if (l.kind == 4) {
                axis = normalize(l.direction);
                if (len2(axis) < 0.5f) continue;
                float half = 0.5f * rclamp(l.spread_deg, 1.0f, 180.0f) * (PI / 180.0f);
                float soft = rmax(l.angle_deg, 0.0f) * (PI / 180.0f);
                float inner = rmax(half - soft, 0.0f);
                a.cos_outer = fcos(half);
                a.cos_inner = fcos(inner);
            } else {
                a.cos_outer = -2.0f;
                a.cos_inner = -2.0f;
            }
            put3(a.fz, axis);
            float flux = lum * power;
            if (!(flux > 0.0f)) continue;
            float r_m = a.radius * 1.0e-3f;
            if (a.radius > 0.0f) {
                float kr = 1.0f / (PI * r_m * r_m);
                a.radiance[0] = a.intensity[0] * kr; a.radiance[1] = a.intensity[1] * kr; a.radiance[2] = a.intensity[2] * kr;
            }
            put3(a.centre, l.position);
            a.base = luminance(rgb(a.intensity[0], a.intensity[1], a.intensity[2]));
            a.near2 = rmax(r_m * r_m, 1.0e-6f);
            // An IES light inside the sphere that bounds the scene sends it its whole flux:
            // flux / (4 pi peak) of its peak's worth.
            const float toward = (ies && len(l.position - centre) <= radius) ? ies->flux / (4.0f * PI * ies->peak)
                                                                               : 0.05f + 0.95f * sphere_mask(a, centre);
            weights.push_back(flux * toward * reach(l.position, nullptr));
        } else {  // rect or disk
            a.kind = LIGHT_AREA;
            a.rect = l.kind == 0;
            if (a.rect) {
                a.half_x = 0.5f * absf(l.size_x);
                a.half_y = 0.5f * absf(l.size_y);
                a.area = 4.0f * a.half_x * a.half_y;
                a.bound = sqrt_(a.half_x * a.half_x + a.half_y * a.half_y);
            } else {
                a.radius = 0.5f * absf(l.size_x);
                a.area = PI * a.radius * a.radius;
                a.bound = a.radius;
            }
            // light_frame (light.rs:245)
            V3 z = normalize(l.direction);
            V3 y = normalize(l.up - z * dot(z, l.up));
            Frame f;
            if (len2(y) < 0.5f) f = frame_from_normal(z);
            else { f.x = cross(y, z); f.y = y; f.z = z; }
            if (!(a.area > 0.0f) || len2(f.z) < 0.5f) continue;
            float k = power / (PI * a.area * 1.0e-6f);
            a.radiance[0] = color[0] * k; a.radiance[1] = color[1] * k; a.radiance[2] = color[2] * k;
            if (l.spread_deg >= 180.0f) a.exponent = 0.0f;
            else {
                float half = 0.5f * rmax(l.spread_deg, 1.0f) * (PI / 180.0f);
                a.exponent = -1.0f / flog2(fcos(half));
            }
            float flux = lum * power * 2.0f / (a.exponent + 2.0f);
            if (!(flux > 0.0f)) continue;
            weights.push_back(flux * reach(l.position, &f.z));
            put3(a.centre, l.position);
            put3(a.fx, f.x); put3(a.fy, f.y); put3(a.fz, f.z);
            a.base = luminance(rgb(a.radiance[0], a.radiance[1], a.radiance[2])) * a.area * 1.0e-6f;
        }
        if (refs.size() >= (size_t)MAX_LIGHTS) { error = "unsupported: more than 63 lights"; return false; }
        refs.push_back({a.kind, (uint32_t)kinds[a.kind].size()});
        kinds[a.kind].push_back(a);
    }
    // Emissive meshes (light.rs:867-958): every instance whose material is an emitter flagged as a
    // light, sampled by area over its world-space triangles; entries after the scene's lights.
    std::vector<LightDev> meshes;
    F.mesh_light_data.clear();
    for (size_t i = 0; i < s.instances.size(); ++i) {
        const HInstance& in = s.instances[i];
        if (in.material_id >= s.materials.size()) continue;
        const HMaterial& m = s.materials[in.material_id];
        if (m.kind != MATERIAL_EMISSIVE || !(m.flags & 1u)) continue;
        const Rgb radiance = rgb(rmax(m.emission[0] * m.emission_power, 0.0f), rmax(m.emission[1] * m.emission_power, 0.0f),
                                 rmax(m.emission[2] * m.emission_power, 0.0f));
        if (!(luminance(radiance) > 0.0f)) continue;
        if (in.mesh >= s.meshes.size()) continue;
        const HMesh& M = s.meshes[in.mesh];
        const Xf xf = xf_of(in.rows);
        Xf inv;
        if (!xf_inverse(xf, inv)) continue;  // never hit, so never lit either
        std::vector<std::array<V3, 3>> corners;
        std::vector<V3> normals;
        std::vector<float> tri_areas;
        V3 centroid = v3(0, 0, 0);
        for (size_t t = 0; t < M.triangles(); ++t) {
            const uint32_t ia = M.indices[3 * t], ib = M.indices[3 * t + 1], ic = M.indices[3 * t + 2];
            if (ia >= M.positions.size() || ib >= M.positions.size() || ic >= M.positions.size()) continue;
            const std::array<V3, 3> w = {xf_point(xf, M.positions[ia]), xf_point(xf, M.positions[ib]), xf_point(xf, M.positions[ic])};
            const V3 c = cross(w[1] - w[0], w[2] - w[0]);
            const float a = 0.5f * len(c);
            if (!(a > 0.0f && finitef(a))) continue;
            centroid = centroid + (w[0] + w[1] + w[2]) * (a / 3.0f);
            corners.push_back(w);
            normals.push_back(normalize(c));
            tri_areas.push_back(a);
        }
        float area = 0.0f, total = 0.0f;
        for (float a : tri_areas) area += a;
        total = area;
        if (!(total > 0.0f && finitef(total))) continue;  // build_cdf (light.rs:652): no CDF, no light
        LightDev e;
        std::memset(&e, 0, sizeof(e));
        e.kind = LIGHT_MESH;
        e.glossy = 1;
        e.shadow = 1;
        e.source = 0xffffffffu;
        e.entry = (uint32_t)(refs.size() + meshes.size());
        e.two_sided = (in.flags & 1u) == 0;
        const float sides = e.two_sided ? 2.0f : 1.0f;
        const float flux = luminance(radiance) * PI * area * 1.0e-6f * sides;
        centroid = centroid / area;
        float bound = 0.0f;
        for (const auto& w : corners)
            for (const V3& q : w) bound = rmax(bound, len(q - centroid));
        V3 mean = v3(0, 0, 0);
        for (size_t k = 0; k < normals.size(); ++k) mean = mean + normals[k] * tri_areas[k];
        const float length = len(mean);
        V3 axis = v3(0, 0, 1);
        if (e.two_sided || length <= 1.0e-3f * area) {
            e.cos_o = -1.0f;
            e.sin_o = 0.0f;
        } else {
            axis = mean / length;
            float c = 1.0f;
            for (const V3& n : normals) c = rmin(c, dot(n, axis));
            e.cos_o = rclamp(c, -1.0f, 1.0f);
            e.sin_o = sqrt_(rmax(1.0f - e.cos_o * e.cos_o, 0.0f));
        }
        weights.push_back(flux * reach(centroid, nullptr));
        put3(e.centre, centroid);
        put3(e.fz, axis);
        e.bound = bound;
        e.area = area;
        e.radiance[0] = radiance.r; e.radiance[1] = radiance.g; e.radiance[2] = radiance.b;
        e.base = luminance(radiance) * area * 1.0e-6f;
        // The triangles: corners, the cumulative area fraction (light.rs:652 build_cdf) in a's w,
        // the unit normal; their offset in the scene's mesh-light data until upload.
        e.n_tris = (uint32_t)corners.size();
        e.tris = reinterpret_cast<const float4*>(F.mesh_light_data.size());
        float acc = 0.0f;
        for (size_t k = 0; k < corners.size(); ++k) {
            acc += tri_areas[k];
            const float cdf = k + 1 == corners.size() ? 1.0f : acc / total;
            const V3& a = corners[k][0];
            const V3& b = corners[k][1];
            const V3& c = corners[k][2];
            const V3& n = normals[k];
            const float rec[16] = {a.x, a.y, a.z, cdf, b.x, b.y, b.z, 0.0f, c.x, c.y, c.z, 0.0f, n.x, n.y, n.z, 0.0f};
            F.mesh_light_data.insert(F.mesh_light_data.end(), rec, rec + 16);
        }
        F.instances[i].emitter = (uint32_t)meshes.size() + 1;  // made absolute below
        meshes.push_back(e);
        if (refs.size() + meshes.size() > (size_t)MAX_LIGHTS) { error = "unsupported: more than 63 lights"; return false; }
    }
    uint32_t first[3] = {0, (uint32_t)kinds[0].size(), (uint32_t)(kinds[0].size() + kinds[1].size())};
    for (int k = 0; k < 3; ++k)
        for (size_t i = 0; i < kinds[k].size(); ++i) L.lights[first[k] + i] = kinds[k][i];
    L.n_areas = (int)kinds[0].size();
    L.n_suns = (uint32_t)kinds[1].size();
    L.n_spheres = (uint32_t)kinds[2].size();
    const uint32_t first_mesh = (uint32_t)refs.size();
    for (size_t i = 0; i < meshes.size(); ++i) L.lights[first_mesh + i] = meshes[i];
    for (DevInstance& d : F.instances)
        if (d.emitter) d.emitter += first_mesh;
    L.n_lights = (uint32_t)(refs.size() + meshes.size());
    for (const auto& r : refs) L.entries[L.n_entries++] = (int)(first[r.first] + r.second);
    for (size_t i = 0; i < meshes.size(); ++i) L.entries[L.n_entries++] = (int)(first_mesh + i);
    // EnvLight::new (environment.rs:335): an HDRI with its bitmap is a map (black when it has no
    // light), any other kind the ramp (flat: three equal stops; an HDRI without a bitmap: the dome).
    float strength = rmax(s.env_strength, 0.0f);
    float f0 = s.env_kind == 1 ? s.env_horizon : s.env_floor, h0 = s.env_horizon, z0 = s.env_kind == 1 ? s.env_horizon : s.env_zenith;
    F.env_image = nullptr;
    if (s.env_kind == 2) {  // the sky, tabulated; scale 1 and no rotation
        F.sky = sky_image(s);
        if (build_env_map(F.sky, 1.0f, 0.0f, F.env_map)) {
            L.env_is_map = 1;
            F.env_image = &F.sky;
        } else {
            f0 = h0 = z0 = 0.0f;
        }
    } else if (s.env_kind == 3 && s.hdri_map < s.bitmaps.size()) {
        if (build_env_map(s.bitmaps[s.hdri_map], strength, s.env_rotation, F.env_map)) {
            L.env_is_map = 1;
            F.env_image = &s.bitmaps[s.hdri_map];
        } else {
            f0 = h0 = z0 = 0.0f;
        }
    }
    L.env_floor = rmax(f0 * strength, 0.0f);
    L.env_horizon = rmax(h0 * strength, 0.0f);
    L.env_zenith = rmax(z0 * strength, 0.0f);
    L.env_lower = 0.5f * (L.env_floor + L.env_horizon);
    float upper = 0.5f * (L.env_horizon + L.env_zenith);
    L.env_total = L.env_lower + upper;
    const float mean = L.env_is_map ? F.env_map.mean_luminance : 0.5f * L.env_total;
    const bool black = L.env_is_map ? (mean != mean || mean <= 0.0f) : L.env_total <= 0.0f;
    if (L.env_is_map) {
        const HEnvMap& m = F.env_map;
        L.env_map.width = F.env_image->width;
        L.env_map.height = F.env_image->height;
        L.env_map.scale = m.scale;
        L.env_map.rot_s = m.rot_s;
        L.env_map.rot_c = m.rot_c;
        L.env_map.gw = m.gw;
        L.env_map.gh = m.gh;
        L.env_map.mean = m.mean;
    }
    L.env_base = PI * mean;
    if (!black) {
        if (L.n_entries >= MAX_ENTRIES) { error = "unsupported: more than 64 lights"; return false; }
        weights.push_back(4.0f * PI * PI * mean);
        L.env_is_entry = 1;
        L.env_entry = (uint32_t)L.n_entries;
        L.entries[L.n_entries++] = -1;
    }
    // build_cdf (light.rs:649)
    float total = 0.0f;
    for (float w : weights) total += w;
    if (!(total > 0.0f && finitef(total))) {
        L.n_entries = 0;
        L.env_is_entry = 0;
    } else {
        float acc = 0.0f;
        for (size_t e = 0; e < weights.size(); ++e) { acc += weights[e]; L.cdf[e] = acc / total; }
        L.cdf[weights.size() - 1] = 1.0f;
        for (size_t e = 0; e < weights.size(); ++e) L.flux_pmf[e] = L.cdf[e] - (e == 0 ? 0.0f : L.cdf[e - 1]);
    }
    L.per_point = L.n_entries >= 2 && L.n_entries <= MAX_ENTRIES;
    return true;
}

std::string geometry_key(const HScene& s) {
    std::string k;
    auto put = [&](const void* p, size_t n) { k.append(static_cast<const char*>(p), n); };
    uint64_t nm = s.meshes.size(), ni = s.instances.size();
    put(&nm, 8);
    put(&ni, 8);
    for (const HInstance& in : s.instances) {
        uint32_t vis = in.flags & 5u;  // one-sided, hidden to the camera: stored in the leaves
        put(&in.mesh, 4);
        put(in.rows, sizeof(in.rows));
        put(&vis, 4);
    }
    return k;
}

bool flatten_scene(const HScene& s, Flat& F, std::string& error, bool geometry) {
    auto t0 = std::chrono::steady_clock::now();
    F = Flat();
    const size_t ni = s.instances.size();
    // Vertices, normals and triangle indices, global.
    std::vector<uint32_t> vtx_base(s.meshes.size()), tri_base(s.meshes.size());
    uint32_t nv = 0, nt = 0;
    for (size_t m = 0; m < s.meshes.size(); ++m) {
        vtx_base[m] = nv;
        tri_base[m] = nt;
        nv += (uint32_t)s.meshes[m].positions.size();
        nt += (uint32_t)s.meshes[m].triangles();
    }
    if (geometry) {
        F.positions.resize((size_t)nv * 4);
        F.normals.assign((size_t)nv * 4, 0.0f);
        F.tri_index.resize((size_t)nt * 4);
        for (size_t m = 0; m < s.meshes.size(); ++m) {
            const HMesh& M = s.meshes[m];
            for (size_t v = 0; v < M.positions.size(); ++v) {
                float* p = &F.positions[((size_t)vtx_base[m] + v) * 4];
                p[0] = M.positions[v].x; p[1] = M.positions[v].y; p[2] = M.positions[v].z; p[3] = 0;
                if (!M.normals.empty()) {
                    float* n = &F.normals[((size_t)vtx_base[m] + v) * 4];
                    n[0] = M.normals[v].x; n[1] = M.normals[v].y; n[2] = M.normals[v].z;
                }
            }
            for (size_t t = 0; t < M.triangles(); ++t) {
                uint32_t* ti = &F.tri_index[((size_t)tri_base[m] + t) * 4];
                ti[0] = vtx_base[m] + M.indices[3 * t];
                ti[1] = vtx_base[m] + M.indices[3 * t + 1];
                ti[2] = vtx_base[m] + M.indices[3 * t + 2];
                ti[3] = (uint32_t)m;
            }
        }
    }
    // Instances.
    Box scene_box;
    std::vector<Xf> xf(ni), inv(ni);
    std::vector<bool> live(ni), ident(ni);
    for (size_t i = 0; i < ni; ++i) {
        const HInstance& in = s.instances[i];
        const HMesh& M = s.meshes[in.mesh];
        xf[i] = xf_of(in.rows);
        bool has_inv = xf_inverse(xf[i], inv[i]);
        if (!has_inv) inv[i] = xf_of(HInstance().rows);
        live[i] = M.triangles() > 0 && has_inv;
        ident[i] = xf_identity(xf[i]);
        DevInstance d;
        std::memset(&d, 0, sizeof(d));
        std::memcpy(d.to_local, &inv[i].r[0][0], 48);
        std::memcpy(d.to_world, &xf[i].r[0][0], 48);
        d.identity = ident[i];
        d.active = live[i];
        d.material = in.material_id;
        d.mesh = in.mesh;
        d.flags = in.flags;
        d.inside_out = M.inside_out;
        d.has_normals = !M.normals.empty();
        d.tri_base = tri_base[in.mesh];
        const HMaterial& mat = s.materials[in.material_id];
        // Shadow rays cross cut-outs and thin walls (integrator/mod.rs:371).
        const bool thin = (mat.flags & MATERIAL_FLAG_THIN) != 0;
        d.passable = mat.kind != MATERIAL_EMISSIVE &&
                     (mat.opacity < 1.0f || (thin && mat.transmission > 0.0f && (mat.metallic < 1.0f || mat.kind == MATERIAL_GLASS)));
        // Tangent axes of anisotropic materials (integrator/mod.rs:396).
        if (!(mat.anisotropy != mat.anisotropy || mat.anisotropy <= 0.0f || mat.kind == MATERIAL_EMISSIVE)) {
            d.tangent_on = 1;
            V3 c = xf_point(xf[i], (v3(M.bmin.x, M.bmin.y, M.bmin.z) + M.bmax) * 0.5f);
            if (M.empty_bounds) c = xf_point(xf[i], (v3(f_inf(), f_inf(), f_inf()) + v3(-f_inf(), -f_inf(), -f_inf())) * 0.5f);
            V3 ax = normalize(xf_vector(xf[i], v3(0, 0, 1)));
            V3 xa = normalize(xf_vector(xf[i], v3(1, 0, 0)));
            d.tan_centre[0] = c.x; d.tan_centre[1] = c.y; d.tan_centre[2] = c.z;
            d.tan_axis[0] = ax.x; d.tan_axis[1] = ax.y; d.tan_axis[2] = ax.z;
            d.tan_x[0] = xa.x; d.tan_x[1] = xa.y; d.tan_x[2] = xa.z;
        }
        F.instances.push_back(d);
        if (live[i]) scene_box = scene_box.uni(instance_box(M, xf[i]));
        if (live[i]) F.instanced_triangles += M.triangles();
    }
    // The box the ray sort grids: the instances that hold at least 1% of the triangles (where
    // most rays start; a large floor quad of two triangles would otherwise spread the grid thin),
    // or the whole scene's.
    {
        uint64_t total = 0;
        for (size_t i = 0; i < ni; ++i)
            if (live[i]) total += s.meshes[s.instances[i].mesh].triangles();
        Box bulk;
        for (size_t i = 0; i < ni; ++i) {
            const HMesh& M = s.meshes[s.instances[i].mesh];
            if (live[i] && (uint64_t)M.triangles() * 100 >= total) bulk = bulk.uni(instance_box(M, xf[i]));
        }
        if (bulk.empty()) bulk = scene_box;
        F.box_lo[0] = bulk.lo.x; F.box_lo[1] = bulk.lo.y; F.box_lo[2] = bulk.lo.z;
        F.box_hi[0] = bulk.hi.x; F.box_hi[1] = bulk.hi.y; F.box_hi[2] = bulk.hi.z;
    }
    // Materials.
    for (const HMaterial& m : s.materials) {
        DevMaterial d;
        std::memset(&d, 0, sizeof(d));
        d.kind = m.kind; d.flags = m.flags;
        for (int c = 0; c < 3; ++c) d.base[c] = m.base[c];
        d.metallic = m.metallic; d.roughness = m.roughness; d.ior = m.ior; d.transmission = m.transmission;
        d.coat = m.coat; d.coat_roughness = m.coat_roughness; d.anisotropy = m.anisotropy; d.absorption_mm = m.absorption_mm;
        d.opacity = m.opacity;
        if (m.kind == MATERIAL_EMISSIVE)
            for (int c = 0; c < 3; ++c) d.emission[c] = rmax(m.emission[c] * m.emission_power, 0.0f);
        // medium_of (integrator/mod.rs:298)
        bool clear = m.transmission > 0.0f && m.metallic < 1.0f && (m.flags & MATERIAL_FLAG_THIN) == 0;
        if (clear && m.absorption_mm > 0.0f && m.kind != MATERIAL_EMISSIVE) {
            for (int c = 0; c < 3; ++c) d.sigma[c] = -fln(rclamp(m.base[c], 1.0e-4f, 1.0f)) / m.absorption_mm;
            d.has_medium = d.sigma[0] > 0.0f || d.sigma[1] > 0.0f || d.sigma[2] > 0.0f;
        }
        F.materials.push_back(d);
    }
    // Bsdf::surface_at (bsdf.rs:382) of every material, entering and leaving, and the floor's
    // Bsdf::lambert: a BSDF depends on the material and the side only, so the kernels read it.
    {
        const EnergyData& ed = energy_data();
        EnergyTables E{ed.albedo.data(), ed.schlick.data(), ed.clear_in.data(), ed.clear_out.data(), ed.albedo_avg.data(),
                       ed.schlick_avg.data()};
        for (const DevMaterial& d : F.materials) {
            F.bsdfs.push_back(bsdf_surface(E, d, true));
            F.bsdfs.push_back(bsdf_surface(E, d, false));
        }
        F.bsdfs.push_back(bsdf_lambert(rgb(s.floor_color[0], s.floor_color[1], s.floor_color[2])));
    }
    if (geometry) {
        // Bottom level: one world-space tree over the triangles of every identity instance (the
        // nearest hit does not depend on the tree, so they can share one), one object-space tree per
        // mesh used by a transformed instance.
        Flattener fl{F};
        uint32_t blas_depth = 0;
        std::vector<BlasInst> tlas_leaves;
        std::vector<Box> tlas_boxes;
        {
            std::vector<std::pair<uint32_t, uint32_t>> prims;  // (instance, triangle)
            for (size_t i = 0; i < ni; ++i)
                if (live[i] && ident[i])
                    for (uint32_t t = 0; t < s.meshes[s.instances[i].mesh].triangles(); ++t) prims.push_back({(uint32_t)i, t});
            if (!prims.empty()) {
                std::vector<Box> boxes(prims.size());
                std::vector<V3> cents(prims.size());
                Box all;
                for (size_t k = 0; k < prims.size(); ++k) {
                    const HMesh& M = s.meshes[s.instances[prims[k].first].mesh];
                    uint32_t t = prims[k].second;
                    Box b = Box().ext(M.positions[M.indices[3 * t]]).ext(M.positions[M.indices[3 * t + 1]]).ext(M.positions[M.indices[3 * t + 2]]);
                    boxes[k] = b;
                    cents[k] = b.centroid();
                    all = all.uni(b);
                }
                SahBuilder sb{boxes, cents, 4, 8, {}, {}};
                sb.order.resize(prims.size());
                for (size_t k = 0; k < prims.size(); ++k) sb.order[k] = (uint32_t)k;
                sb.build(0, prims.size(), 0);
                fl.bn = &sb.nodes;
                fl.order = &sb.order;
                fl.max_depth = 0;
                fl.emit = [&](const uint32_t* p, uint32_t n) {
                    uint32_t first = (uint32_t)F.tris.size();
                    for (uint32_t k = 0; k < n; ++k) {
                        uint32_t inst = prims[p[k]].first, t = prims[p[k]].second;
                        const HMesh& M = s.meshes[s.instances[inst].mesh];
                        TriRec r;
                        const V3& a = M.positions[M.indices[3 * t]];
                        const V3& b = M.positions[M.indices[3 * t + 1]];
                        const V3& c = M.positions[M.indices[3 * t + 2]];
                        r.v0[0] = a.x; r.v0[1] = a.y; r.v0[2] = a.z; r.tri = t;
                        r.v1[0] = b.x; r.v1[1] = b.y; r.v1[2] = b.z; r.inst = inst;
                        r.v2[0] = c.x; r.v2[1] = c.y; r.v2[2] = c.z;
                        r.flags = (s.instances[inst].flags & 1u) | ((s.instances[inst].flags & 4u) ? 2u : 0u);
                        F.tris.push_back(r);
                    }
                    return make_leaf(first, n);
                };
                uint32_t root = fl.reference(0, 0);
                blas_depth = std::max(blas_depth, fl.max_depth);
                BlasInst bi;
                std::memset(&bi, 0, sizeof(bi));
                bi.root = root;
                bi.identity = 1;
                bi.instance = 0xffffffffu;
                tlas_leaves.push_back(bi);
                tlas_boxes.push_back(all);
            }
        }
        std::map<uint32_t, uint32_t> mesh_root;
        for (size_t i = 0; i < ni; ++i) {
            if (!live[i] || ident[i]) continue;
            uint32_t m = s.instances[i].mesh;
            if (!mesh_root.count(m)) {
                const HMesh& M = s.meshes[m];
                size_t n = M.triangles();
                std::vector<Box> boxes(n);
                std::vector<V3> cents(n);
                for (size_t t = 0; t < n; ++t) {
                    boxes[t] = Box().ext(M.positions[M.indices[3 * t]]).ext(M.positions[M.indices[3 * t + 1]]).ext(M.positions[M.indices[3 * t + 2]]);
                    cents[t] = boxes[t].centroid();
                }
                SahBuilder sb{boxes, cents, 4, 8, {}, {}};
                sb.order.resize(n);
                for (size_t k = 0; k < n; ++k) sb.order[k] = (uint32_t)k;
                sb.build(0, n, 0);
                fl.bn = &sb.nodes;
                fl.order = &sb.order;
                fl.max_depth = 0;
                fl.emit = [&](const uint32_t* p, uint32_t cnt) {
                    uint32_t first = (uint32_t)F.tris.size();
                    for (uint32_t k = 0; k < cnt; ++k) {
                        uint32_t t = p[k];
                        TriRec r;
                        const V3& a = M.positions[M.indices[3 * t]];
                        const V3& b = M.positions[M.indices[3 * t + 1]];
                        const V3& c = M.positions[M.indices[3 * t + 2]];
                        r.v0[0] = a.x; r.v0[1] = a.y; r.v0[2] = a.z; r.tri = t;
                        r.v1[0] = b.x; r.v1[1] = b.y; r.v1[2] = b.z; r.inst = 0xffffffffu;
                        r.v2[0] = c.x; r.v2[1] = c.y; r.v2[2] = c.z; r.flags = 0;
                        F.tris.push_back(r);
                    }
                    return make_leaf(first, cnt);
                };
                mesh_root[m] = fl.reference(0, 0);
                blas_depth = std::max(blas_depth, fl.max_depth);
            }
            BlasInst bi;
            std::memset(&bi, 0, sizeof(bi));
            std::memcpy(bi.to_local, &inv[i].r[0][0], 48);
            bi.root = mesh_root[m];
            bi.identity = 0;
            bi.instance = (uint32_t)i;
            bi.flags = (s.instances[i].flags & 1u) | ((s.instances[i].flags & 4u) ? 2u : 0u);
            tlas_leaves.push_back(bi);
            tlas_boxes.push_back(instance_box(s.meshes[m], xf[i]));
        }
        // Top level over the placed trees (one per leaf).
        F.blas = tlas_leaves;
        uint32_t tlas_depth = 0;
        if (!tlas_leaves.empty()) {
            std::vector<V3> cents(tlas_boxes.size());
            for (size_t k = 0; k < cents.size(); ++k) cents[k] = tlas_boxes[k].centroid();
            SahBuilder sb{tlas_boxes, cents, 1, 1, {}, {}};
            sb.order.resize(tlas_boxes.size());
            for (size_t k = 0; k < tlas_boxes.size(); ++k) sb.order[k] = (uint32_t)k;
            sb.build(0, tlas_boxes.size(), 0);
            fl.bn = &sb.nodes;
            fl.order = &sb.order;
            fl.max_depth = 0;
            fl.emit = [&](const uint32_t* p, uint32_t) { return make_leaf(p[0], 1); };
            fl.exact_flat = true;
            fl.wrapped = false;
            F.tlas_root = fl.reference(0, 0);
            fl.exact_flat = false;
            tlas_depth = fl.max_depth + (fl.wrapped ? 1 : 0);  // a wrapper adds one level
        }
        F.stack_need = 7 * (tlas_depth + blas_depth) + 2;
        if (F.stack_need > 96) { error = "unsupported: BVH too deep for the traversal stack"; return false; }
        if (F.tris.size() >= (1u << 27) - 16) { error = "unsupported: more than 2^27 triangles"; return false; }
    }
    if (!prepare_lights(s, scene_box, F.lights, F, error)) return false;

    // Scene constants: camera basis (scene/mod.rs:158) and render settings.
    SceneDev& S = F.scene;
    std::memset(&S, 0, sizeof(S));
    V3 forward = normalize(s.cam_target - s.cam_position);
    if (len2(forward) == 0.0f) forward = v3(0, 1, 0);
    V3 right = normalize(cross(forward, s.cam_up));
    if (len2(right) < 0.5f) {
        V3 axis = absf(forward.z) < 0.9f ? v3(0, 0, 1) : v3(1, 0, 0);
        right = normalize(cross(forward, axis));
    }
    V3 up = cross(right, forward);
    S.cam_pos[0] = s.cam_position.x; S.cam_pos[1] = s.cam_position.y; S.cam_pos[2] = s.cam_position.z;
    S.cam_fwd[0] = forward.x; S.cam_fwd[1] = forward.y; S.cam_fwd[2] = forward.z;
    S.cam_right[0] = right.x; S.cam_right[1] = right.y; S.cam_right[2] = right.z;
    S.cam_up[0] = up.x; S.cam_up[1] = up.y; S.cam_up[2] = up.z;
    S.focal_mm = s.focal_mm; S.sensor_mm = s.sensor_mm; S.focus_dist = s.focus_dist;
    const bool panoramic = s.projection == 1 || s.projection == 2;  // K3: a pinhole, no lens sample
    S.lens_radius = (s.fstop > 0.0f && s.focus_dist > 0.0f && !s.ortho && !panoramic) ? s.focal_mm / s.fstop * 0.5f : 0.0f;
    S.ortho_width = s.ortho_width; S.ortho = s.ortho; S.exterior = s.exterior;
    S.projection = panoramic ? s.projection : 0;
    S.fov_x_deg = s.fov_x; S.fov_y_deg = s.fov_y;
    S.width = s.width; S.height = s.height; S.seed = s.seed; S.seed_b = s.seed; S.split_b = 0xffffffffu;
    S.max_depth = s.max_depth == 0 ? 8 : (s.max_depth < 1024 ? s.max_depth : 1024);
    S.pixel_filter = s.pixel_filter;
    S.edge_k = s.edge_supersample < 1 ? 1 : (s.edge_supersample > 16 ? 16 : s.edge_supersample);  // RenderSettings::edge_factor
    S.clamp_indirect = s.clamp_indirect;
    // The background image fitted to the frame (integrator/mod.rs:317); without one a background
    // image shows the colour.
    F.plate = s.backplate_map < s.bitmaps.size() ? &s.bitmaps[s.backplate_map] : nullptr;
    if (F.plate) {
        const float* r = s.backplate_rect;
        const bool ok = r[2] > r[0] && r[3] > r[1];
        for (int k = 0; k < 4; ++k) S.plate_rect[k] = ok ? r[k] : (k < 2 ? 0.0f : 1.0f);
        const uint32_t w = s.width ? s.width : 1, h = s.height ? s.height : 1;
        S.plate_w = F.plate->width;
        S.plate_h = F.plate->height;
        S.plate_fit = s.backplate_fit;
        S.frame_aspect = ((S.plate_rect[2] - S.plate_rect[0]) * (float)w) / ((S.plate_rect[3] - S.plate_rect[1]) * (float)h);
        S.image_aspect = (float)F.plate->width / (float)F.plate->height;
    }
    S.background = s.background_mode == 1 ? 1 : s.background_mode == 2 ? 2 : s.background_mode == 3 ? (F.plate ? 3 : 1) : 0;
    for (int c = 0; c < 3; ++c) S.background_color[c] = rmax(s.background_color[c], 0.0f);
    for (const DevInstance& d : F.instances) S.any_passable |= d.passable;
    // The section view (geometry/section.rs:180-222, scene/mod.rs:1092-1111): per instance whether
    // the plane caps it (a closed solid that is live, not exempt and not a thin wall) or leaves it
    // alone (the studio), the grown box where caps can be, and the exempt instances' grown boxes.
    F.exempt_boxes.clear();
    if (s.section_on) {
        S.section_on = 1;
        S.section_cap = s.section_cap;
        S.section_n[0] = s.section_n.x; S.section_n[1] = s.section_n.y; S.section_n[2] = s.section_n.z;
        S.section_d = s.section_d;
        auto grown = [](Box b) {
            const V3 d = b.hi - b.lo;
            const float pad = rmax(rmax(d.x, d.y), d.z) * 1.0e-5f + 1.0e-4f;
            b.lo = b.lo - v3(pad, pad, pad);
            b.hi = b.hi + v3(pad, pad, pad);
            return b;
        };
        std::vector<int> solid(s.meshes.size(), -1);  // per mesh, analysed on first use
        Box caps;
        for (size_t i = 0; i < ni; ++i) {
            const HInstance& in = s.instances[i];
            const HMesh& M = s.meshes[in.mesh];
            DevInstance& d = F.instances[i];
            const bool exempt = (in.flags & 2u) != 0;
            if (exempt && d.active) {
                d.exempt = 1;
                const Box b = grown(instance_box(M, xf_of(in.rows)));
                F.exempt_boxes.insert(F.exempt_boxes.end(), {b.lo.x, b.lo.y, b.lo.z, b.hi.x, b.hi.y, b.hi.z});
            }
            const bool thin = (s.materials[in.material_id].flags & MATERIAL_FLAG_THIN) != 0;
            if (!(s.section_cap && !exempt && !thin && d.active)) continue;
            if (solid[in.mesh] < 0) solid[in.mesh] = (int)solid_of(M);
            d.solid = (uint32_t)solid[in.mesh];
            if (d.solid) caps = caps.uni(grown(instance_box(M, xf_of(in.rows))));
        }
        S.cap_any = !caps.empty();
        S.cap_lo[0] = caps.lo.x; S.cap_lo[1] = caps.lo.y; S.cap_lo[2] = caps.lo.z;
        S.cap_hi[0] = caps.hi.x; S.cap_hi[1] = caps.hi.y; S.cap_hi[2] = caps.hi.z;
        S.n_exempt = (uint32_t)(F.exempt_boxes.size() / 6);
    }
    for (const HInstance& in : s.instances) {
        const HMaterial& m = s.materials[in.material_id];
        if (m.kind != MATERIAL_EMISSIVE && m.opacity < 1.0f) S.any_cutout = 1;
    }
    S.floor_mode = s.floor_mode;
    S.floor_z = s.floor_z;
    for (int c = 0; c < 3; ++c) S.floor_color[c] = s.floor_color[c];
    S.tlas_root = F.tlas_root;
    S.n_instances = (uint32_t)ni;
    S.n_materials = (uint32_t)s.materials.size();
    S.stack_need = F.stack_need;
    F.build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return true;
}

}  // namespace rtg
