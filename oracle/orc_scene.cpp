// ORACLE (test infrastructure only). See orc_scene.h.
#include "orc_scene.h"

#include <cstring>

namespace orc {

// ---- scene/mod.rs:158-359 camera -------------------------------------------------------------
void Camera::basis(Vec3& forward, Vec3& right, Vec3& upv) const {
    forward = normalize(target - position);
    if (length_squared(forward) == 0.0f) forward = Vec3(0, 1, 0);
    right = normalize(cross(forward, up));
    if (length_squared(right) < 0.5f) {
        Vec3 axis = std::fabs(forward.z) < 0.9f ? Vec3(0, 0, 1) : Vec3(1, 0, 0);
        right = normalize(cross(forward, axis));
    }
    upv = cross(right, forward);
}
bool Camera::panorama_dir(float aspect, float u, float v, Vec3& dir) const {
    Vec3 forward, right, upv;
    basis(forward, right, upv);
    if (projection == 1) {  // equirectangular: longitude across the width, latitude across the height
        float lon = (u - 0.5f) * (fov_x_deg * DEG_TO_RAD);
        float lat = (0.5f - v) * (fov_y_deg * DEG_TO_RAD);
        float s_lat, c_lat, s_lon, c_lon;
        sin_cos(lat, s_lat, c_lat);
        sin_cos(lon, s_lon, c_lon);
        dir = forward * (c_lat * c_lon) + right * (c_lat * s_lon) + upv * s_lat;
        return true;
    }
    if (projection == 2) {  // equidistant fisheye: the angle from the axis grows with the distance from the centre
        float k = fov_x_deg * DEG_TO_RAD;
        float x = (u - 0.5f) * k;
        float y = (0.5f - v) * k / rmax(aspect, 1.0e-6f);
        float theta = std::sqrt(x * x + y * y);
        if (theta != theta || theta > PI) return false;
        if (theta == 0.0f) { dir = forward; return true; }
        float s, c;
        sin_cos(theta, s, c);
        dir = forward * c + (right * x + upv * y) * (s / theta);
        return true;
    }
    return false;
}
Ray Camera::generate_ray(float aspect, float u, float v, float lx, float ly) const {
    Vec3 forward, right, upv;
    basis(forward, right, upv);
    if (panoramic()) {  // scene/mod.rs:227 panorama_ray
        Vec3 dir;
        if (panorama_dir(aspect, u, v, dir)) return Ray(position, dir);
        Ray r(position, forward);
        r.t_max = 0.0f;
        return r;
    }
    if (ortho) {
        float w = ortho_width;
        Vec3 origin = position + right * ((u - 0.5f) * w) + upv * ((0.5f - v) * w / aspect);
        return Ray(origin, forward);
    }
    float sw, sh;
    if (aspect >= 1.0f) { sw = sensor_mm; sh = sensor_mm / aspect; }
    else { sw = sensor_mm * aspect; sh = sensor_mm; }
    float x = (u - 0.5f) * sw;
    float y = (0.5f - v) * sh;
    Vec3 dir = normalize(forward * focal_mm + right * x + upv * y);
    float radius = lens_radius();
    if (radius == 0.0f) return Ray(position, dir);
    Vec3 focus_point = position + dir * (focus_dist / dot(dir, forward));
    Vec3 origin = position + (right * lx + upv * ly) * radius;
    return Ray(origin, normalize(focus_point - origin));
}

// ---- scene/rsb.rs subset reader -------------------------------------------------------------------
namespace {
struct Reader {
    const uint8_t* data;
    size_t len, pos = 0;
    char tag[5];
    std::string* err;
    bool fail = false;
    Reader(const uint8_t* d, size_t n, const uint8_t* t, std::string* e) : data(d), len(n), err(e) {
        for (int i = 0; i < 4; ++i) tag[i] = (t[i] >= 33 && t[i] <= 126) ? (char)t[i] : '?';
        tag[4] = 0;
    }
    size_t remaining() const { return len - pos; }
    bool too_short() {
        if (!fail) *err = std::string("RSB section ") + tag + " is shorter than its layout requires";
        fail = true;
        return false;
    }
    bool invalid(const char* why) {
        if (!fail) *err = std::string("RSB section ") + tag + " is invalid: " + why;
        fail = true;
        return false;
    }
    bool u32(uint32_t& v) {
        if (fail) return false;
        if (remaining() < 4) return too_short();
        std::memcpy(&v, data + pos, 4);
        pos += 4;
        return true;
    }
    bool f32(float& v) {
        uint32_t u;
        if (!u32(u)) return false;
        v = bitsf(u);
        if (!finite(v)) return invalid("non-finite number");
        return true;
    }
    bool vec3(Vec3& v) { return f32(v.x) && f32(v.y) && f32(v.z); }
    bool rgb(Rgb& c) { return f32(c.r) && f32(c.g) && f32(c.b); }
    bool opt_u32(uint32_t& v, uint32_t d) { if (remaining() >= 4) return u32(v); v = d; return !fail; }
    bool opt_f32(float& v, float d) { if (remaining() >= 4) return f32(v); v = d; return !fail; }
};
}  // namespace

bool read_rsb(const uint8_t* bytes, size_t len, Scene& scene, std::string& error) {
    if (len < 4 || std::memcmp(bytes, "RSB1", 4) != 0) { error = "not an RSB file (missing RSB1 magic)"; return false; }
    if (len < 8) { error = "RSB file is truncated in header"; return false; }
    uint32_t header_len;
    std::memcpy(&header_len, bytes + 4, 4);
    size_t pos = 8 + (size_t)header_len;
    if (pos > len) { error = "RSB file is truncated in header"; return false; }
    bool have_cam = false, have_env = false, have_floor = false, have_render = false, have_section = false;
    SectionPlane section;
    std::vector<Mesh> meshes;
    std::vector<Instance> instances;
    scene = Scene();
    while (pos < len) {
        if (len - pos < 8) { error = "RSB file is truncated in section header"; return false; }
        const uint8_t* tag = bytes + pos;
        uint32_t n;
        std::memcpy(&n, bytes + pos + 4, 4);
        if ((size_t)n > len - pos - 8) { error = "RSB file is truncated in section payload"; return false; }
        const uint8_t* payload = bytes + pos + 8;
        pos += 8 + (size_t)n;
        Reader r(payload, n, tag, &error);
        auto is = [&](const char* t) { return std::memcmp(tag, t, 4) == 0; };
        auto dup = [&](bool& seen) {
            if (seen) { error = std::string("RSB section ") + r.tag + " appears more than once"; return true; }
            seen = true;
            return false;
        };
        if (is("CAMR")) {
            if (dup(have_cam)) return false;
            Camera& c = scene.camera;
            uint32_t ortho;
            if (!(r.vec3(c.position) && r.vec3(c.target) && r.vec3(c.up) && r.f32(c.focal_mm) && r.f32(c.sensor_mm) &&
                  r.f32(c.fstop) && r.f32(c.focus_dist) && r.u32(ortho) && r.f32(c.ortho_width) &&
                  r.opt_u32(c.projection, 0) && r.opt_f32(c.fov_x_deg, 360) && r.opt_f32(c.fov_y_deg, 180) &&
                  r.opt_f32(c.exterior, 1)))
                return false;
            c.ortho = ortho != 0;
            if (c.focal_mm <= 0.0f || c.sensor_mm <= 0.0f) return r.invalid("focal_mm and sensor_mm must be positive");
            if (c.fstop < 0.0f || c.focus_dist < 0.0f || c.ortho_width < 0.0f)
                return r.invalid("fstop, focus_dist and ortho_width must not be negative");
            auto field = [](float v) { return v > 0.0f && v <= 3600.0f; };
            if (!field(c.fov_x_deg) || !field(c.fov_y_deg)) return r.invalid("fov_x_deg and fov_y_deg must be positive and at most 3600");
            if (c.exterior < 0.0f) return r.invalid("exterior must not be negative");
        } else if (is("MESH")) {
            uint32_t vc, ic;
            if (!(r.u32(vc) && r.u32(ic))) return false;
            uint64_t words = (uint64_t)vc * 6 + ic + 1;
            if (words * 4 > r.remaining()) return r.too_short();
            if (ic % 3 != 0) return r.invalid("index_count is not a multiple of 3");
            std::vector<Vec3> p(vc), nn(vc);
            for (auto& v : p) if (!r.vec3(v)) return false;
            for (auto& v : nn) if (!r.vec3(v)) return false;
            std::vector<uint32_t> idx(ic);
            for (auto& i : idx) {
                if (!r.u32(i)) return false;
                if (i >= vc) return r.invalid("vertex index out of range");
            }
            uint32_t mat;
            if (!r.u32(mat)) return false;
            Mesh m;
            const char* e = Mesh::make(m, p, nn, idx, mat);
            if (*e) return r.invalid(e);
            if (r.remaining() >= 4) {  // M2b UV sets: read and ignored (no textures in this subset)
                uint32_t sets;
                r.u32(sets);
                if (sets > 2) return r.invalid("at most 2 UV sets");
                if ((uint64_t)sets * vc * 8 > r.remaining()) return r.too_short();
                for (uint64_t k = 0; k < (uint64_t)sets * vc * 2; ++k) { float f; if (!r.f32(f)) return false; }
            }
            meshes.push_back(std::move(m));
        } else if (is("INST")) {
            Instance in;
            if (!r.u32(in.mesh)) return false;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 4; ++j)
                    if (!r.f32(in.transform.r[i][j])) return false;
            if (!(r.u32(in.material_id) && r.u32(in.flags))) return false;
            instances.push_back(in);
        } else if (is("MATL")) {
            Material m;
            if (!(r.u32(m.kind) && r.rgb(m.base_color) && r.f32(m.metallic) && r.f32(m.roughness) && r.f32(m.ior) &&
                  r.f32(m.transmission) && r.f32(m.coat) && r.f32(m.coat_roughness) && r.rgb(m.emission) &&
                  r.f32(m.emission_power) && r.opt_u32(m.flags, 0) && r.opt_f32(m.opacity, 1) &&
                  r.opt_f32(m.anisotropy, 0) && r.opt_f32(m.absorption_mm, 0) && r.opt_f32(m.bevel_mm, 0) &&
                  r.opt_f32(m.scatter_mm, 0) && r.opt_f32(m.scatter_color.r, 1) && r.opt_f32(m.scatter_color.g, 1) &&
                  r.opt_f32(m.scatter_color.b, 1) && r.opt_f32(m.scatter_g, 0) && r.opt_f32(m.abbe, 0)))
                return false;
            if (r.remaining() >= 4 && r.pos == 100) {
                uint32_t version;
                r.u32(version);
                if (version == 1) { error = "unsupported: material texture block"; return false; }
            }
            scene.materials.push_back(m);
        } else if (is("LGHT")) {
            Light l;
            if (!r.u32(l.kind)) return false;
            if (l.kind > 5) return r.invalid("unknown light kind");
            if (!(r.vec3(l.position) && r.vec3(l.direction) && r.vec3(l.up) && r.f32(l.size_x) && r.f32(l.size_y) &&
                  r.rgb(l.color) && r.f32(l.power) && r.f32(l.spread_deg) && r.f32(l.angle_deg) && r.u32(l.flags)))
                return false;
            if (l.kind == 5) {  // rsb.rs:1006: the profile, an IESP section's position
                uint32_t profile;
                if (!r.opt_u32(profile, 0xffffffffu)) return false;
                l.profile = profile == 0xffffffffu ? -1 : (int)profile;
                if (profile > 0x7fffffffu) l.profile = -2;  // refers to no section
            }
            scene.lights.push_back(l);
        } else if (is("ENVR")) {
            if (dup(have_env)) return false;
            Environment& e = scene.environment;
            if (!r.u32(e.kind)) return false;
            if (e.kind > 3) return r.invalid("unknown environment kind");
            if (!(r.f32(e.floor) && r.f32(e.horizon) && r.f32(e.zenith) && r.f32(e.strength) && r.f32(e.rotation_deg) &&
                  r.rgb(e.background_color) && r.u32(e.background_mode)))
                return false;
            if (!(r.opt_u32(e.hdri_map, NO_BITMAP) && r.opt_u32(e.backplate_map, NO_BITMAP) && r.opt_u32(e.backplate_fit, 0) &&
                  r.opt_f32(e.sky_turbidity, 3.0f) && r.opt_f32(e.sun_azimuth_deg, 0.0f) && r.opt_f32(e.sun_elevation_deg, 45.0f) &&
                  r.opt_f32(e.backplate_rect[0], 0.0f) && r.opt_f32(e.backplate_rect[1], 0.0f) && r.opt_f32(e.backplate_rect[2], 1.0f) &&
                  r.opt_f32(e.backplate_rect[3], 1.0f) && r.opt_u32(e.sky_model, 0)))
                return false;
        } else if (is("IESP")) {  // rsb.rs:1018
            uint32_t n;
            if (!r.u32(n)) return false;
            if ((size_t)n > r.remaining()) return r.too_short();
            IesProfile prof;
            std::string reason;
            if (!IesProfile::parse(r.data + r.pos, n, prof, reason)) return r.invalid(reason.c_str());
            r.pos += n;
            scene.profiles.push_back(std::move(prof));
        } else if (is("BMAP")) {  // rsb.rs:1057
            uint32_t format, w, h, n;
            if (!(r.u32(format) && r.u32(w) && r.u32(h) && r.u32(n))) return false;
            if ((size_t)n > r.remaining()) return r.too_short();
            Image img;
            std::string reason;
            bool unsupported = false;
            if (!decode_bitmap(format, w, h, r.data + r.pos, n, img, reason, unsupported)) {
                if (unsupported) { error = reason; return false; }
                return r.invalid(reason.c_str());
            }
            r.pos += n;
            scene.bitmaps.push_back(std::move(img));
        } else if (is("SECT")) {  // rsb.rs:1070 parse_section
            if (dup(have_section)) return false;
            uint32_t flags;
            Vec3 normal;
            float distance;
            if (!(r.u32(flags) && r.vec3(normal) && r.f32(distance))) return false;
            if (!SectionPlane::make(normal, distance, (flags & 1u) != 0, section)) return r.invalid("section normal is zero");
        } else if (is("FLOR")) {
            if (dup(have_floor)) return false;
            Floor& f = scene.floor;
            if (!(r.u32(f.mode) && r.f32(f.z) && r.rgb(f.color))) return false;
            if (f.mode > 2) return r.invalid("unknown floor mode");
            if (f.mode == 2) { error = "unsupported: shadow catcher floor"; return false; }
        } else if (is("RNDR")) {
            if (dup(have_render)) return false;
            RenderSettings& s = scene.render;
            if (!(r.u32(s.width) && r.u32(s.height) && r.u32(s.max_samples) && r.u32(s.seed) && r.f32(s.max_seconds) &&
                  r.f32(s.exposure_ev) && r.u32(s.tonemap) && r.opt_u32(s.max_depth, 8) && r.opt_f32(s.clamp_indirect, 0) &&
                  r.opt_u32(s.passes, 0) && r.opt_u32(s.denoise, 0) && r.opt_u32(s.caustic_photons, 0) &&
                  r.opt_f32(s.caustic_radius, 0) && r.opt_f32(s.denoise_strength, 1) && r.opt_u32(s.pixel_filter, 0) &&
                  r.opt_u32(s.edge_supersample, 1) && r.opt_u32(s.adaptive, 0) && r.opt_f32(s.noise_threshold, 0)))
                return false;
            if (!(s.noise_threshold >= 0.0f && s.noise_threshold <= 1.0f)) return r.invalid("noise_threshold must be between 0 and 1");
            if (s.edge_supersample > 16) return r.invalid("edge_supersample must be at most 16");
            if (!(s.denoise_strength >= 0.0f && s.denoise_strength <= 1.0f)) return r.invalid("denoise_strength must be between 0 and 1");
            if (s.caustic_photons > (1u << 22)) return r.invalid("caustic_photons must be at most 4194304");
            if (s.caustic_radius < 0.0f) return r.invalid("caustic_radius must not be negative");
            if (s.caustic_photons > 0) { error = "unsupported: caustic photon maps (caustic_photons above 0)"; return false; }
            if (s.width < 1 || s.width > 16384 || s.height < 1 || s.height > 16384)
                return r.invalid("width and height must be between 1 and 16384");
            if (s.max_seconds < 0.0f || s.clamp_indirect < 0.0f) return r.invalid("max_seconds and clamp_indirect must not be negative");

        } else {
            static const char* feature_tags[] = {"LENS", "PATN", "IMGS", "PROG", "FXAM", "GLAS",
                                                 "WETP", "WETF", "WTP2", "WETG", "NEST"};
            for (const char* t : feature_tags)
                if (is(t)) { error = std::string("unsupported: RSB section ") + t; return false; }
        }
    }
    for (const Light& l : scene.lights)  // rsb.rs:1354
        if (l.kind == 5 && !(l.profile >= 0 && (size_t)l.profile < scene.profiles.size())) {
            error = "RSB section LGHT is invalid: an IES light needs a profile that is an IESP section";
            return false;
        }
    for (uint32_t map : {scene.environment.hdri_map, scene.environment.backplate_map})
        if (map != NO_BITMAP && map >= scene.bitmaps.size()) {
            error = "RSB section ENVR is invalid: bitmap index does not refer to a BMAP section";
            return false;
        }
    size_t nm = scene.materials.size();
    for (const Mesh& m : meshes)
        if (m.material_id >= nm) { error = "RSB section MESH is invalid: material_id does not refer to a MATL section"; return false; }
    if (instances.empty())
        for (size_t i = 0; i < meshes.size(); ++i) {
            Instance in;
            in.mesh = (uint32_t)i;
            in.material_id = meshes[i].material_id;
            instances.push_back(in);
        }
    for (const Instance& in : instances) {
        if (in.mesh >= meshes.size()) { error = "RSB section INST is invalid: mesh_id does not refer to a MESH section"; return false; }
        if (in.material_id >= nm) { error = "RSB section INST is invalid: material_id does not refer to a MATL section"; return false; }
    }
    // Material features outside this path (their branches of the reference integrator).
    for (const Material& m : scene.materials) {
        if (m.scatter_mm > 0.0f && m.transmission > 0.0f) { error = "unsupported: scattering media"; return false; }
        if (m.abbe > 0.0f && m.transmission > 0.0f) { error = "unsupported: dispersive glass"; return false; }
        if (m.bevel_mm > 0.0f) { error = "unsupported: edge bevel"; return false; }
    }
    const char* e = Geometry::make(scene.geometry, std::move(meshes), std::move(instances));
    if (*e) { error = e; return false; }
    if (have_section) {  // Scene::apply_section (scene/mod.rs:1092-1111): a thin wall has no inside to cap
        std::vector<bool> capped;
        for (const Instance& in : scene.geometry.instances)
            capped.push_back((scene.materials[in.material_id].flags & MATERIAL_FLAG_THIN) == 0);
        scene.geometry.set_section(&section, capped);
    }
    return true;
}

// ---- environment.rs:275-441 --------------------------------------------------------------------
Ramp Ramp::make(float f, float h, float z, float strength) {
    Ramp r;
    r.floor = rmax(f * strength, 0.0f);
    r.horizon = rmax(h * strength, 0.0f);
    r.zenith = rmax(z * strength, 0.0f);
    r.lower_mass = 0.5f * (r.floor + r.horizon);
    float upper = 0.5f * (r.horizon + r.zenith);
    r.total_mass = r.lower_mass + upper;
    return r;
}
float Ramp::value(float z) const {
    z = rclamp(z, -1.0f, 1.0f);
    if (z < 0.0f) return floor * -z + horizon * (1.0f + z);
    return horizon * (1.0f - z) + zenith * z;
}
float Ramp::pdf(Vec3 dir) const {
    if (total_mass <= 0.0f) return 0.0f;
    return value(dir.z) / (TAU * total_mass);
}
static float invert_linear(float a, float b, float u) {
    float c = u * 0.5f * (a + b);
    float denom = a + std::sqrt(rmax(a * a + 2.0f * (b - a) * c, 0.0f));
    return denom > 0.0f ? rclamp(2.0f * c / denom, 0.0f, 1.0f) : 0.0f;
}
bool Ramp::sample(float u0, float u1, Vec3& dir, float& p) const {
    if (total_mass <= 0.0f) return false;
    float target = u0 * total_mass;
    float z;
    if (target < lower_mass) {
        z = -1.0f + invert_linear(floor, horizon, target / lower_mass);
    } else {
        float upper = total_mass - lower_mass;
        float fraction = rclamp((target - lower_mass) / upper, 0.0f, 1.0f);
        z = invert_linear(horizon, zenith, fraction);
    }
    z = rclamp(z, -1.0f, 1.0f);
    float rr = std::sqrt(rmax((1.0f - z) * (1.0f + z), 0.0f));
    float s, c;
    sin_cos(TAU * u1, s, c);
    dir = Vec3(rr * c, rr * s, z);
    p = pdf(dir);
    return p > 0.0f;
}

// ---- light.rs ----------------------------------------------------------------------------------
static float orientation_bound(Vec3 v, float d2, Vec3 axis, float cos_o, float sin_o, float bound) {  // light.rs:260
    if (d2 <= bound * bound) return 1.0f;
    float inv_d = 1.0f / std::sqrt(d2);
    float sin_u = bound * inv_d;
    float cos_u = std::sqrt(rmax(1.0f - sin_u * sin_u, 0.0f));
    float cos_s = cos_o * cos_u - sin_o * sin_u;
    float sin_s = sin_o * cos_u + cos_o * sin_u;
    if (sin_s < 0.0f) return 1.0f;
    float cos_t = dot(v, axis) * inv_d;
    if (cos_t >= cos_s) return 1.0f;
    float sin_t = std::sqrt(rmax(1.0f - cos_t * cos_t, 0.0f));
    return rmax(cos_t * cos_s + sin_t * sin_s, 0.0f);
}
Vec3 AreaLight::sample_point(float u0, float u1) const {
    float x, y;
    if (rect) { x = (2.0f * u0 - 1.0f) * half_x; y = (2.0f * u1 - 1.0f) * half_y; }
    else { concentric_disk(u0, u1, x, y); x = x * radius; y = y * radius; }
    return centre + frame.x * x + frame.y * y;
}
bool AreaLight::intersect(const Ray& ray, float t_max, float& t, float& cos) const {
    Vec3 n = frame.z;
    float denom = dot(ray.dir, n);
    if (denom >= 0.0f) return false;
    t = dot(centre - ray.origin, n) / denom;
    if (!(t > ray.t_min && t < t_max)) return false;
    Vec3 q = ray.at(t) - centre;
    float x = dot(q, frame.x), y = dot(q, frame.y);
    bool inside = rect ? (std::fabs(x) <= half_x && std::fabs(y) <= half_y) : (x * x + y * y <= radius * radius);
    if (!inside) return false;
    cos = -denom;
    return true;
}
float MeshEmitter::weight(Vec3 x) const {  // light.rs:468: lum(L) A cos' / max(d^2, A) from its centroid
    Vec3 v = x - centroid;
    float d2 = length_squared(v);
    float o = cos_o <= -1.0f ? 1.0f : orientation_bound(v, d2, axis, cos_o, sin_o, bound);
    if (o <= 0.0f) return 0.0f;
    return base * o / (rmax(d2, area) * 1.0e-6f);
}
float AreaLight::weight(Vec3 x) const {
    Vec3 v = x - centre;
    float d2 = length_squared(v);
    float o = orientation_bound(v, d2, frame.z, 1.0f, 0.0f, bound);
    if (o <= 0.0f) return 0.0f;
    return base * o / (rmax(d2, area) * 1.0e-6f);
}
static Frame light_frame(Vec3 normal, Vec3 up) {  // light.rs:245
    Vec3 z = normalize(normal);
    Vec3 y = normalize(up - z * dot(z, up));
    if (length_squared(y) < 0.5f) return Frame::from_normal(z);
    Frame f;
    f.x = cross(y, z);
    f.y = y;
    f.z = z;
    return f;
}
static float spread_exponent(float spread_deg) {
    if (spread_deg >= 180.0f) return 0.0f;
    float half = 0.5f * rmax(spread_deg, 1.0f) * DEG_TO_RAD;
    return -1.0f / log2(fcos(half));
}
static std::vector<float> build_cdf(const std::vector<float>& w) {  // light.rs:649
    float total = 0.0f;
    for (float x : w) total += x;
    if (!(total > 0.0f && finite(total))) return {};
    std::vector<float> cdf;
    float acc = 0.0f;
    for (float x : w) { acc += x; cdf.push_back(acc / total); }
    cdf.back() = 1.0f;
    return cdf;
}
static void pick(const std::vector<float>& cdf, float u, size_t& i, float& rest) {  // light.rs:634
    size_t k = 0;
    while (k < cdf.size() && cdf[k] <= u) ++k;
    i = k < cdf.size() - 1 ? k : cdf.size() - 1;
    float lo = i == 0 ? 0.0f : cdf[i - 1];
    float width = cdf[i] - lo;
    rest = width > 0.0f ? rclamp((u - lo) / width, 0.0f, 0.99999994f) : 0.0f;
}

static Vec3 uniform_cone(float u0, float u1, float one_minus_cos_max) {  // warp.rs:38
    float one_minus_cos = u0 * one_minus_cos_max;
    float cos = 1.0f - one_minus_cos;
    float sin = std::sqrt(rmax(one_minus_cos * (2.0f - one_minus_cos), 0.0f));
    float sp, cp;
    sin_cos(TAU * u1, sp, cp);
    return Vec3(sin * cp, sin * sp, cos);
}
float SphereLight::mask(Vec3 x) const {  // light.rs:368
    if (ies) {
        Vec3 d = x - centre;
        float len2 = length_squared(d);
        if (!(len2 > 0.0f)) return 0.0f;
        return ies->shape(ies_frame.to_local(d / std::sqrt(len2)));
    }
    if (cos_outer < -1.0f) return 1.0f;
    Vec3 d = x - centre;
    float len2 = length_squared(d);
    if (!(len2 > 0.0f)) return 0.0f;
    float c = dot(d, axis) / std::sqrt(len2);
    if (c <= cos_outer) return 0.0f;
    if (c >= cos_inner) return 1.0f;
    float t = (c - cos_outer) / (cos_inner - cos_outer);
    return t * t * (3.0f - 2.0f * t);
}
bool SphereLight::cone(float dist2, float& omc) const {  // light.rs:398
    float r2 = radius * radius;
    if (!(dist2 - r2 > 0.0f)) return false;
    float sin2 = r2 / dist2;
    omc = sin2 / (1.0f + std::sqrt(rmax(1.0f - sin2, 0.0f)));
    if (omc < 1.0e-7f) omc = 0.0f;  // POINT_CONE
    return true;
}
bool SphereLight::intersect(const Ray& ray, float t_max, float& t) const {  // light.rs:409
    if (!(radius > 0.0f)) return false;
    Vec3 oc = ray.origin - centre;
    float r2 = radius * radius;
    if (length_squared(oc) <= r2) return false;
    float b = dot(oc, ray.dir);
    float disc = r2 - length_squared(oc - ray.dir * b);
    if (disc < 0.0f) return false;
    t = -b - std::sqrt(disc);
    return t > ray.t_min && t < t_max;
}
float SphereLight::weight(Vec3 x) const {  // light.rs:430
    float m = mask(x);
    if (m <= 0.0f) return 0.0f;
    float d2 = length_squared(x - centre) * 1.0e-6f;
    return base * m / rmax(d2, near2);
}

Lights Lights::make(const Scene& scene) {  // light.rs:673
    Lights L;
    Aabb bounds = scene.geometry.bounds;
    Vec3 centre;
    float radius;
    if (bounds.is_empty()) { centre = Vec3(0, 0, 0); radius = 1000.0f; }
    else { centre = bounds.centroid(); radius = rmax(0.5f * length(bounds.max - bounds.min), 1.0f); }
    float radius_m = radius * 1.0e-3f;
    auto reach = [&](Vec3 p, const Vec3* normal) {
        Vec3 to_centre = centre - p;
        float d = length(to_centre) * 1.0e-3f;
        float facing = normal ? 0.05f + 0.95f * rmax(dot(*normal, normalize(to_centre)), 0.0f) : 1.0f;
        d = rmax(d, radius_m);
        return facing / (d * d);
    };
    std::vector<float> weights;
    for (size_t li = 0; li < scene.lights.size(); ++li) {
        const Light& light = scene.lights[li];
        bool glossy = (light.flags & LIGHT_FLAG_GLOSSY) != 0;
        bool camera = (light.flags & LIGHT_FLAG_CAMERA) != 0;
        bool shadow = (light.flags & LIGHT_FLAG_NO_SHADOW) == 0;
        float power = rmax(light.power, 0.0f);
        uint32_t entry = (uint32_t)L.entries.size();
        Rgb color(rmax(light.color.r, 0.0f), rmax(light.color.g, 0.0f), rmax(light.color.b, 0.0f));
        if (light.kind == (uint32_t)LightKind::Sun) {  // light.rs:755
            Vec3 to_sun = -normalize(light.direction);
            if (length_squared(to_sun) < 0.5f) continue;
            float half = rmin(0.5f * rmax(light.angle_deg, 0.0f) * DEG_TO_RAD, FRAC_PI_2);
            Rgb irradiance = color * power;
            if (!(irradiance.luminance() > 0.0f)) continue;
            SunLight sun{};
            sun.delta = half < 1.0e-5f;
            float s = fsin(0.5f * half);
            sun.one_minus_cos_max = 2.0f * s * s;
            float sin_max = fsin(half);
            sun.radiance = sun.delta ? irradiance : irradiance * (1.0f / (PI * sin_max * sin_max));
            weights.push_back(PI * irradiance.luminance());
            L.entries.push_back({LightRef::Sun, (uint32_t)L.suns.size()});
            sun.frame = Frame::from_normal(to_sun);
            sun.cos_max = 1.0f - sun.one_minus_cos_max;
            sun.solid_angle = TAU * sun.one_minus_cos_max;
            sun.glossy = glossy;
            sun.camera = camera;
            sun.shadow = shadow;
            sun.entry = entry;
            sun.base = irradiance.luminance();
            sun.source = (uint32_t)li;
            L.suns.push_back(sun);
            continue;
        }
        if (light.kind == (uint32_t)LightKind::Point || light.kind == (uint32_t)LightKind::Spot ||
            light.kind == (uint32_t)LightKind::Ies) {  // light.rs:780
            SphereLight sp{};
            sp.intensity = color * (power / (4.0f * PI));
            float r_light = 0.5f * std::fabs(light.size_x);
            sp.radius = finite(r_light) ? r_light : 0.0f;
            if (light.kind == (uint32_t)LightKind::Ies) {  // L5: masked by its profile in its own frame
                sp.ies = &scene.profiles[light.profile];
                sp.ies_frame = light_frame(light.direction, light.up);
                if (length_squared(sp.ies_frame.z) < 0.5f) continue;
            }
            if (light.kind == (uint32_t)LightKind::Spot) {
                Vec3 axis = normalize(light.direction);
                if (length_squared(axis) < 0.5f) continue;
                float half = 0.5f * rclamp(light.spread_deg, 1.0f, 180.0f) * DEG_TO_RAD;
                float soft = rmax(light.angle_deg, 0.0f) * DEG_TO_RAD;
                float inner = rmax(half - soft, 0.0f);
                sp.axis = axis;
                sp.cos_outer = fcos(half);
                sp.cos_inner = fcos(inner);
            } else {
                sp.axis = Vec3(0, 0, -1);
                sp.cos_outer = -2.0f;
                sp.cos_inner = -2.0f;
            }
            float flux = color.luminance() * power;
            if (!(flux > 0.0f)) continue;
            float r_m = sp.radius * 1.0e-3f;
            sp.radiance = sp.radius > 0.0f ? sp.intensity * (1.0f / (PI * r_m * r_m)) : BLACK;
            sp.centre = light.position;
            sp.glossy = glossy;
            sp.camera = camera;
            sp.shadow = shadow;
            sp.entry = entry;
            sp.base = sp.intensity.luminance();
            sp.near2 = rmax(r_m * r_m, 1.0e-6f);  // MIN_DISTANCE2_M2
            sp.source = (uint32_t)li;
            // An IES light inside the sphere that bounds the scene sends it its whole flux.
            float toward = (sp.ies && length(light.position - centre) <= radius) ? sp.ies->efficiency() : 0.05f + 0.95f * sp.mask(centre);
            weights.push_back(flux * toward * reach(light.position, nullptr));
            L.entries.push_back({LightRef::Sphere, (uint32_t)L.spheres.size()});
            L.spheres.push_back(sp);
            continue;
        }
        AreaLight a{};
        a.rect = light.kind == 0;
        if (a.rect) {
            a.half_x = 0.5f * std::fabs(light.size_x);
            a.half_y = 0.5f * std::fabs(light.size_y);
            a.area = 4.0f * a.half_x * a.half_y;
            a.bound = std::sqrt(a.half_x * a.half_x + a.half_y * a.half_y);
        } else {
            a.radius = 0.5f * std::fabs(light.size_x);
            a.area = PI * a.radius * a.radius;
            a.bound = a.radius;
        }
        a.frame = light_frame(light.direction, light.up);
        if (!(a.area > 0.0f) || length_squared(a.frame.z) < 0.5f) continue;
        a.radiance = color * (power / (PI * a.area * 1.0e-6f));
        a.exponent = spread_exponent(light.spread_deg);
        float flux = color.luminance() * power * 2.0f / (a.exponent + 2.0f);
        if (!(flux > 0.0f)) continue;
        weights.push_back(flux * reach(light.position, &a.frame.z));
        L.entries.push_back({LightRef::Area, (uint32_t)L.areas.size()});
        a.centre = light.position;
        a.glossy = glossy;
        a.camera = camera;
        a.shadow = shadow;
        a.entry = entry;
        a.base = a.radiance.luminance() * a.area * 1.0e-6f;
        a.source = (uint32_t)li;
        L.areas.push_back(a);
    }
    // light.rs:867-958: every emissive instance whose material is flagged as a light, sampled by
    // area over its world-space triangles.
    const Geometry& geo = scene.geometry;
    L.instance_emitter.assign(geo.instances.size(), -1);
    for (size_t i = 0; i < geo.instances.size(); ++i) {
        const Instance& inst = geo.instances[i];
        if (inst.material_id >= scene.materials.size()) continue;
        const Material& mat = scene.materials[inst.material_id];
        Rgb radiance = mat.radiance();
        if (!(mat.flags & MATERIAL_FLAG_LIGHT) || !(radiance.luminance() > 0.0f)) continue;
        if (inst.mesh >= geo.meshes.size()) continue;
        const Mesh& mesh = geo.meshes[inst.mesh];
        Transform inv;
        if (!inst.transform.inverse(inv)) continue;  // never hit, so never lit either
        MeshEmitter em{};
        std::vector<float> tri_areas;
        Vec3 centroid(0, 0, 0);
        for (size_t t = 0; t < mesh.triangle_count(); ++t) {
            uint32_t ia = mesh.indices[3 * t], ib = mesh.indices[3 * t + 1], ic = mesh.indices[3 * t + 2];
            if (ia >= mesh.positions.size() || ib >= mesh.positions.size() || ic >= mesh.positions.size()) continue;
            std::array<Vec3, 3> w = {inst.transform.point(mesh.positions[ia]), inst.transform.point(mesh.positions[ib]),
                                     inst.transform.point(mesh.positions[ic])};
            Vec3 c = cross(w[1] - w[0], w[2] - w[0]);
            float a = 0.5f * length(c);
            if (!(a > 0.0f && finite(a))) continue;
            centroid = centroid + (w[0] + w[1] + w[2]) * (a / 3.0f);
            em.corners.push_back(w);
            em.normals.push_back(normalize(c));
            tri_areas.push_back(a);
        }
        float area = 0.0f;
        for (float a : tri_areas) area += a;
        em.cdf = build_cdf(tri_areas);
        if (em.cdf.empty()) continue;
        em.two_sided = (inst.flags & INSTANCE_ONE_SIDED) == 0;
        float sides = em.two_sided ? 2.0f : 1.0f;
        float flux = radiance.luminance() * PI * area * 1.0e-6f * sides;
        centroid = centroid / area;
        float bound = 0.0f;
        for (const auto& w : em.corners)
            for (const Vec3& q : w) bound = rmax(bound, length(q - centroid));
        Vec3 mean(0, 0, 0);
        for (size_t k = 0; k < em.normals.size(); ++k) mean = mean + em.normals[k] * tri_areas[k];
        float len = length(mean);
        if (em.two_sided || len <= 1.0e-3f * area) {
            em.axis = Vec3(0, 0, 1);
            em.cos_o = -1.0f;
            em.sin_o = 0.0f;
        } else {
            em.axis = mean / len;
            float c = 1.0f;
            for (const Vec3& n : em.normals) c = rmin(c, dot(n, em.axis));
            em.cos_o = rclamp(c, -1.0f, 1.0f);
            em.sin_o = std::sqrt(rmax(1.0f - em.cos_o * em.cos_o, 0.0f));
        }
        weights.push_back(flux * reach(centroid, nullptr));
        em.entry = (uint32_t)L.entries.size();
        L.entries.push_back({LightRef::Mesh, (uint32_t)L.meshes.size()});
        L.instance_emitter[i] = (int)L.meshes.size();
        em.area = area;
        em.radiance = radiance;
        em.centroid = centroid;
        em.bound = bound;
        em.base = radiance.luminance() * area * 1.0e-6f;
        L.meshes.push_back(std::move(em));
    }
    L.env = EnvLight::make(scene.environment, scene.bitmaps);
    L.env_base = PI * L.env.mean_radiance();
    if (!L.env.is_black()) {
        weights.push_back(4.0f * PI * PI * L.env.mean_radiance());
        L.env_is_entry = true;
        L.env_entry = (uint32_t)L.entries.size();
        L.entries.push_back({LightRef::Environment, 0});
    }
    L.cdf = build_cdf(weights);
    if (L.cdf.empty()) { L.entries.clear(); L.env_is_entry = false; }
    for (size_t e = 0; e < L.cdf.size(); ++e) L.flux_pmf.push_back(L.cdf[e] - (e == 0 ? 0.0f : L.cdf[e - 1]));
    L.per_point = L.entries.size() >= 2 && L.entries.size() <= 64;
    return L;
}

float Lights::weight(size_t entry, Vec3 x) const {  // light.rs:1014
    const LightRef& e = entries[entry];
    switch (e.kind) {
        case LightRef::Area: return areas[e.index].weight(x);
        case LightRef::Sun: return suns[e.index].base;
        case LightRef::Sphere: return spheres[e.index].weight(x);
        case LightRef::Mesh: return meshes[e.index].weight(x);
        default: return env_base;
    }
}
Selection Lights::select(Vec3 x) const {  // light.rs:1026
    size_t n = entries.size();
    if (!per_point || n == 0) return select_by_flux(x);
    Selection s;
    s.point = x;
    s.total = 0.0f;
    s.by_flux = false;
    for (size_t e = 0; e < n; ++e) {
        float w = weight(e, x);
        if (e < 8) s.weights[e] = w;
        s.total += w;
    }
    return s;
}
float Lights::pmf(uint32_t entry, const Selection& from) const {  // light.rs:1076
    if (entry >= entries.size()) return 0.0f;
    if (from.by_flux) return flux_pmf[entry];
    if (!(from.total > 0.0f && finite(from.total))) return 0.0f;
    return weight_at(entry, from) / from.total;
}
void Lights::pick_at(const Selection& s, float u, size_t& idx, float& rest, float& pmf_out) const {  // light.rs:1118
    float total = s.total;
    size_t last = entries.size() - 1;
    float acc = 0.0f, lo = 0.0f;
    for (size_t e = 0; e <= last; ++e) {
        float w = weight_at(e, s);
        acc += w;
        float hi = e == last ? 1.0f : acc / total;
        if (hi > u || e == last) {
            float width = hi - lo;
            rest = width > 0.0f ? rclamp((u - lo) / width, 0.0f, 0.99999994f) : 0.0f;
            idx = e;
            pmf_out = w / total;
            return;
        }
        lo = hi;
    }
    idx = last; rest = 0.0f; pmf_out = 0.0f;
}
bool Lights::sample_selected(const Selection& from, float u_select, float u0, float u1, LightSample& out) const {  // light.rs:1150
    size_t n = entries.size();
    if (n == 0) return false;
    Vec3 x = from.point;
    size_t index;
    float rest, pmf_v;
    if (from.by_flux) {
        pick(cdf, u_select, index, rest);
        pmf_v = pmf((uint32_t)index, from);
    } else {
        if (!(from.total > 0.0f && finite(from.total))) return false;
        pick_at(from, u_select, index, rest, pmf_v);
    }
    if (!(pmf_v > 0.0f)) return false;
    const LightRef& e = entries[index];
    if (e.kind == LightRef::Sun) {  // light.rs:1197
        const SunLight& sun = suns[e.index];
        if (sun.delta) {
            out = {sun.frame.z, F_INF, sun.radiance, pmf_v, true, sun.glossy, sun.glossy, sun.shadow, (int)sun.source};
        } else {
            Vec3 local = uniform_cone(u0, u1, sun.one_minus_cos_max);
            out = {normalize(sun.frame.to_world(local)), F_INF, sun.radiance, pmf_v / sun.solid_angle, false, sun.glossy,
                   sun.glossy, sun.shadow, (int)sun.source};
        }
    } else if (e.kind == LightRef::Sphere) {  // light.rs:1224
        const SphereLight& light = spheres[e.index];
        float m = light.mask(x);
        Vec3 d = light.centre - x;
        float dist2 = length_squared(d);
        if (!(m > 0.0f && dist2 > 0.0f)) return false;
        float dist = std::sqrt(dist2);
        Vec3 towards = d / dist;
        float omc = 0.0f;
        if (light.radius > 0.0f && !light.cone(dist2, omc)) return false;
        if (omc == 0.0f) {
            out = {towards, dist, light.intensity * (m / (dist2 * 1.0e-6f)), pmf_v, true, light.glossy, false, light.shadow,
                   (int)light.source};
        } else {
            Vec3 local = uniform_cone(u0, u1, omc);
            Vec3 wi = normalize(Frame::from_normal(towards).to_world(local));
            float b = dot(wi, d);
            float r2 = light.radius * light.radius;
            float near = b - std::sqrt(rmax(r2 - length_squared(d - wi * b), 0.0f));
            out = {wi, rmax(near, 0.0f), light.radiance * m, pmf_v / (TAU * omc), false, light.glossy, false, light.shadow,
                   (int)light.source};
        }
    } else if (e.kind == LightRef::Area) {
        const AreaLight& light = areas[e.index];
        Vec3 p = light.sample_point(u0, u1);
        Vec3 d = p - x;
        float dist2 = length_squared(d);
        float distance = std::sqrt(dist2);
        Vec3 wi = d / distance;
        float cos = -dot(wi, light.frame.z);
        if (!(cos > 0.0f && distance > 0.0f)) return false;
        out = {wi, distance, light.radiance_at(cos), pmf_v * dist2 / (light.area * cos), false, light.glossy, light.glossy,
               light.shadow, (int)light.source};
    } else if (e.kind == LightRef::Mesh) {  // light.rs:1270: a triangle by area, a point on it uniformly
        const MeshEmitter& em = meshes[e.index];
        size_t t;
        float unused;
        pick(em.cdf, rest, t, unused);
        const std::array<Vec3, 3>& c = em.corners[t];
        float su = std::sqrt(u0);  // warp.rs:57 uniform_triangle
        float b0 = 1.0f - su, b1 = u1 * su, b2 = 1.0f - b0 - b1;
        Vec3 p = c[0] * b0 + c[1] * b1 + c[2] * b2;
        Vec3 d = p - x;
        float dist2 = length_squared(d);
        float distance = std::sqrt(dist2);
        Vec3 wi = d / distance;
        float facing = -dot(wi, em.normals[t]);
        if (!(distance > 0.0f) || (!em.two_sided && facing <= 0.0f)) return false;
        float cos = std::fabs(facing);
        if (!(cos > 0.0f)) return false;
        out = {wi, distance, em.radiance, pmf_v * dist2 / (em.area * cos), false, true, true, true};
    } else {
        Vec3 wi;
        float p;
        if (!env.sample(u0, u1, wi, p)) return false;
        out = {wi, F_INF, env.radiance(wi), pmf_v * p, false, true, false, true};
    }
    return out.pdf > 0.0f && finite(out.pdf) && out.radiance.luminance() > 0.0f;
}
Rgb Lights::crossed_from(const Ray& ray, float t_max, const float* bsdf_pdf, const Selection* from, float offset, int only,
                         Rgb* part) const {
    Rgb sum = BLACK;  // light.rs:1354 crossed_areas, then light.rs:1387 crossed_spheres
    if (part) *part = BLACK;
    for (const AreaLight& light : areas) {
        bool visible = bsdf_pdf ? light.glossy : light.camera;
        if (!visible) continue;
        float t, cos;
        if (!light.intersect(ray, t_max, t, cos)) continue;
        float w = 1.0f;
        if (bsdf_pdf) {
            float d = offset + t;
            float light_pdf = pmf(light.entry, *from) * d * d / (light.area * cos);
            w = power_heuristic(*bsdf_pdf, light_pdf);
        }
        sum = sum + light.radiance_at(cos) * w;
        if (part && (int)light.source == only) *part = *part + light.radiance_at(cos) * w;
    }
    for (const SphereLight& light : spheres) {
        bool visible = bsdf_pdf ? light.glossy : light.camera;
        if (!visible) continue;
        float t;
        if (!light.intersect(ray, t_max, t)) continue;
        Vec3 vertex = ray.origin - ray.dir * offset;
        float m = light.mask(vertex);
        if (!(m > 0.0f)) continue;
        float w = 1.0f;
        if (bsdf_pdf) {
            float omc;
            if (light.cone(length_squared(light.centre - vertex), omc) && omc > 0.0f)
                w = power_heuristic(*bsdf_pdf, pmf(light.entry, *from) / (TAU * omc));
            else
                w = 0.0f;
        }
        sum = sum + light.radiance * (m * w);
        if (part && (int)light.source == only) *part = *part + light.radiance * (m * w);
    }
    return sum;
}
float Lights::emitter_weight(uint32_t instance, float bsdf_pdf, const Selection& from, float t, float cos) const {
    if (instance >= instance_emitter.size() || instance_emitter[instance] < 0) return 1.0f;
    const MeshEmitter& em = meshes[(size_t)instance_emitter[instance]];
    float light_pdf = pmf(em.entry, from) * t * t / (em.area * rmax(std::fabs(cos), 1.0e-7f));
    return power_heuristic(bsdf_pdf, light_pdf);  // light.rs:1090 found_weight
}
bool Lights::camera_sees_panel(const Ray& ray, float t_max) const {
    for (const AreaLight& a : areas) {
        float t, cos;
        if (a.camera && a.intersect(ray, t_max, t, cos)) return true;
    }
    for (const SphereLight& l : spheres) {
        float t;
        if (l.camera && l.intersect(ray, t_max, t) && l.mask(ray.origin) > 0.0f) return true;
    }
    return false;
}
Rgb Lights::escaped(Vec3 dir, const float* bsdf_pdf, const Selection* from, int only, Rgb* part) const {  // light.rs:1502
    Rgb sum = env.radiance(dir);
    if (part) *part = BLACK;
    if (bsdf_pdf && env_is_entry) sum = sum * power_heuristic(*bsdf_pdf, pmf(env_entry, *from) * env.pdf(dir));
    for (const SunLight& sun : suns) {
        bool visible = bsdf_pdf ? sun.glossy : sun.camera;
        if (!(visible && sun.contains(dir))) continue;
        float w = bsdf_pdf ? power_heuristic(*bsdf_pdf, pmf(sun.entry, *from) / sun.solid_angle) : 1.0f;
        sum = sum + sun.radiance * w;
        if (part && (int)sun.source == only) *part = *part + sun.radiance * w;
    }
    return sum;
}

}  // namespace orc
