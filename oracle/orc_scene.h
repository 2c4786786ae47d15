// ORACLE (test infrastructure only). Scene model, RSB subset reader, lights, environment ramp and
// camera, restated from engine/crates/rt-core/src/{scene/mod.rs, scene/rsb.rs, light.rs,
// environment.rs}.
#pragma once
#include <array>
#include <memory>
#include <string>
#include <vector>

#include "orc_bsdf.h"
#include "orc_geometry.h"

namespace orc {

struct Camera {  // scene/mod.rs:91
    Vec3 position{0, -1000, 0}, target{0, 0, 0}, up{0, 0, 1};
    float focal_mm = 50, sensor_mm = 36, fstop = 0, focus_dist = 1000;
    bool ortho = false;
    float ortho_width = 1000;
    uint32_t projection = 0;
    float fov_x_deg = 360, fov_y_deg = 180, exterior = 1;
    void basis(Vec3& forward, Vec3& right, Vec3& upv) const;
    bool panoramic() const { return projection == 1 || projection == 2; }  // K3 (scene/mod.rs:178)
    // A panoramic camera takes no lens sample (scene/mod.rs:338 sample_ray is a pinhole for it).
    float lens_radius() const { return (fstop > 0.0f && focus_dist > 0.0f && !ortho && !panoramic()) ? focal_mm / fstop * 0.5f : 0.0f; }
    // scene/mod.rs:196 panorama_dir: false where a fisheye sees nothing (more than 180 degrees from its axis)
    bool panorama_dir(float aspect, float u, float v, Vec3& dir) const;
    // scene/mod.rs:294 generate_ray; a panoramic camera's ray where it sees nothing has t_max 0
    Ray generate_ray(float aspect, float u, float v, float lx, float ly) const;
};
enum class LightKind : uint32_t { Rect = 0, Disk = 1, Sun = 2, Point = 3, Spot = 4, Ies = 5 };
constexpr uint32_t LIGHT_FLAG_GLOSSY = 1, LIGHT_FLAG_CAMERA = 2, LIGHT_FLAG_NO_SHADOW = 4;
// ies.rs: an IES LM-63 type C photometric profile (candela by vertical and horizontal angle)
struct IesProfile {
    enum Symmetry : uint32_t { Rotational, Quadrant, Bilateral0, Bilateral90, Full } symmetry = Rotational;
    std::vector<float> vertical, horizontal, candela;  // degrees; horizontal.size() rows of vertical.size()
    float peak = 0, flux = 0;
    // IesProfile::parse (ies.rs:227): false with the reference's reason
    static bool parse(const uint8_t* bytes, size_t len, IesProfile& out, std::string& reason);
    float intensity(float gamma, float phi) const;  // candela, degrees
    float shape(Vec3 local) const;                  // intensity towards a local unit direction over the peak
    float efficiency() const { return flux / (4.0f * PI * peak); }
    float fold(float phi) const;
    float row_integral(size_t row) const;
    float integrate() const;
};
struct Light {
    uint32_t kind = 0;
    int profile = -1;  // an IES light's profile among the scene's
    Vec3 position, direction{0, 0, -1}, up{0, 1, 0};
    float size_x = 0, size_y = 0;
    Rgb color = WHITE;
    float power = 0, spread_deg = 180, angle_deg = 0;
    uint32_t flags = 0;
};
constexpr uint32_t NO_BITMAP = 0xffffffffu;
struct Environment {  // scene/mod.rs:739
    uint32_t kind = 0;  // 0 studio, 1 flat, 2 sky, 3 HDRI
    float floor = 0.1f, horizon = 0.3f, zenith = 0.6f, strength = 1.0f, rotation_deg = 0.0f;
    Rgb background_color = Rgb::splat(0.05f);
    uint32_t background_mode = 0;  // 0 environment, 1 colour, 2 transparent, 3 backplate
    uint32_t hdri_map = NO_BITMAP, backplate_map = NO_BITMAP, backplate_fit = 0;  // fit: 0 fill, 1 fit, 2 stretch
    float sky_turbidity = 3.0f, sun_azimuth_deg = 0.0f, sun_elevation_deg = 45.0f;
    float backplate_rect[4] = {0.0f, 0.0f, 1.0f, 1.0f};
    uint32_t sky_model = 0;
};

// ---- bitmap.rs, hdr.rs: decoded images ------------------------------------------------------------
struct Image {  // bitmap.rs:90
    uint32_t width = 0, height = 0;
    bool srgb8 = false;           // sRGB bytes (3 per pixel), else linear floats (3 per pixel)
    std::vector<uint8_t> bytes;
    std::vector<float> linear;
    Rgb texel(uint32_t x, uint32_t y) const;
    Rgb bilinear(float u, float v, bool wrap_u) const;
};
// Bitmap::decode (bitmap.rs:236): formats 0 (sRGB RGB8), 1 (sRGB RGBA8), 2 (linear f32 RGB) and
// 16 (a Radiance file). False with the reason on a bad size or file; OpenEXR (17) is refused.
bool decode_bitmap(uint32_t format, uint32_t width, uint32_t height, const uint8_t* data, size_t len, Image& out,
                   std::string& reason, bool& unsupported);
const float* srgb_table();

struct Distribution2D {  // bitmap.rs:330
    size_t width = 0, height = 0;
    std::vector<float> weights, conditional, marginal;
    float mean = 0;
    static bool make(size_t w, size_t h, std::vector<float> weights, Distribution2D& out);
    void sample(float s0, float s1, float& u, float& v, float& pdf) const;
    float pdf(float u, float v) const;
};
struct Floor { uint32_t mode = 0; float z = 0; Rgb color = Rgb::splat(0.5f); };
struct RenderSettings {  // scene/mod.rs:911
    uint32_t width = 640, height = 360, max_samples = 64, seed = 0;
    float max_seconds = 0, exposure_ev = 0;
    uint32_t tonemap = 1, max_depth = 8;
    float clamp_indirect = 0;
    uint32_t passes = 0, denoise = 0, caustic_photons = 0;
    float caustic_radius = 0, denoise_strength = 1;
    uint32_t pixel_filter = 0, edge_supersample = 1, adaptive = 0;
    float noise_threshold = 0;
    uint32_t depth() const { return max_depth == 0 ? 8 : (max_depth < 1024 ? max_depth : 1024); }
};
struct Scene {
    Camera camera;
    std::vector<Image> bitmaps;
    std::vector<IesProfile> profiles;
    std::vector<Material> materials;
    Geometry geometry;
    std::vector<Light> lights;
    Environment environment;
    Floor floor;
    RenderSettings render;
};
// Parses the RSB subset (CAMR, MESH, MATL, LGHT, ENVR, FLOR, RNDR, INST; unknown tags skipped).
// Sections of features outside the path tracer's core (LENS, BMAP, PATN, IMGS, PROG, FXAM,
// GLAS, WET*, NEST) and scene values that need them are refused with a message; SECT (the section
// view) and IESP (IES profiles) are read.
bool read_rsb(const uint8_t* bytes, size_t len, Scene& out, std::string& error);

// ---- environment.rs: the dome / flat ramp ------------------------------------------------------
struct Ramp {
    float floor = 0, horizon = 0, zenith = 0, lower_mass = 0, total_mass = 0;
    static Ramp make(float f, float h, float z, float strength);
    float value(float z) const;
    float pdf(Vec3 dir) const;
    bool sample(float u0, float u1, Vec3& dir, float& pdf_out) const;
    float mean_radiance() const { return 0.5f * total_mass; }
    bool is_black() const { return total_mass <= 0.0f; }
};

// environment.rs:49-130: an equirectangular map (an HDRI), importance-sampled by its luminance
struct EnvMap {
    const Image* image = nullptr;
    float scale = 0, rot_s = 0, rot_c = 1;
    Distribution2D dist;
    float mean_luminance = 0;
    static bool make(const Image* image, float scale, float rotation_deg, EnvMap& out);
    Vec3 to_image(Vec3 d) const { return Vec3(rot_c * d.x + rot_s * d.y, -rot_s * d.x + rot_c * d.y, d.z); }
    Vec3 to_world(Vec3 d) const { return Vec3(rot_c * d.x - rot_s * d.y, rot_s * d.x + rot_c * d.y, d.z); }
    Rgb radiance(Vec3 dir) const;
    float pdf(Vec3 dir) const;
    bool sample(float u0, float u1, Vec3& dir, float& pdf_out) const;
};
// sky.rs:245 the classic sky (Preetham, Shirley and Smits 1999) before scaling
struct Preetham {
    Vec3 sun;
    float coefficients[3][5];
    float zenith_over_perez[3];
    static Preetham make(float azimuth_deg, float elevation_deg, float turbidity);
    Rgb radiance(Vec3 dir) const;
};
// sky.rs:96 the physical sky (the Hosek-Wilkie form with the fitted table) before scaling: up to
// four knots (two turbidities times two ground albedos), blended by radiance.
struct PhysicalSky {
    struct Knot {
        float weight;
        float coefficients[3][9];
        float radiance[3];
    };
    Vec3 sun;
    Knot knots[4];
    int n = 0;
    static PhysicalSky make(float azimuth_deg, float elevation_deg, float turbidity, float albedo);
    Rgb radiance(Vec3 dir) const;
};
// environment.rs:178 sky_image: the sky (physical, or classic with sky_model 1) tabulated into a
// 256 x 128 map
Image sky_image(const Environment& env);

// environment.rs:333 EnvLight: the ramp or a map
struct EnvLight {
    std::shared_ptr<Image> owned;  // the tabulated sky
    bool is_map = false;
    Ramp ramp;
    EnvMap map;
    static EnvLight make(const Environment& env, const std::vector<Image>& bitmaps);
    Rgb radiance(Vec3 dir) const { return is_map ? map.radiance(dir) : Rgb::splat(ramp.value(dir.z)); }
    float pdf(Vec3 dir) const { return is_map ? map.pdf(dir) : ramp.pdf(dir); }
    bool sample(float u0, float u1, Vec3& dir, float& p) const { return is_map ? map.sample(u0, u1, dir, p) : ramp.sample(u0, u1, dir, p); }
    float mean_radiance() const { return is_map ? map.mean_luminance : ramp.mean_radiance(); }
    bool is_black() const { return is_map ? (map.mean_luminance != map.mean_luminance || map.mean_luminance <= 0.0f) : ramp.is_black(); }
};

// ---- light.rs ----------------------------------------------------------------------------------
struct AreaLight {
    bool rect;
    float half_x, half_y, radius;
    Vec3 centre;
    Frame frame;
    float area;
    Rgb radiance;
    float exponent;
    bool glossy, camera, shadow;
    uint32_t entry;
    float base, bound;
    uint32_t source;  // the scene light it was built from
    Rgb radiance_at(float cos) const { return exponent == 0.0f ? radiance : radiance * powf_(cos, exponent); }
    Vec3 sample_point(float u0, float u1) const;
    bool intersect(const Ray& ray, float t_max, float& t, float& cos) const;
    float weight(Vec3 x) const;
};
struct SunLight {  // light.rs:300
    Frame frame;  // z points at the sun
    float cos_max, one_minus_cos_max, solid_angle;
    Rgb radiance;  // of the disc; for a delta sun, the irradiance
    bool delta, glossy, camera, shadow;
    uint32_t entry;
    float base;
    uint32_t source;  // the scene light it was built from
    bool contains(Vec3 dir) const { return !delta && dot(dir, frame.z) >= cos_max; }
};
struct SphereLight {  // light.rs:330 (point lights, spots and IES lights)
    const IesProfile* ies = nullptr;
    Frame ies_frame;  // an IES light's axis (z) and horizontal angle 0 (y)
    Vec3 centre;
    float radius;
    Rgb intensity, radiance;
    Vec3 axis;
    float cos_outer, cos_inner;  // cos_outer below -1: no mask
    bool glossy, camera, shadow;
    uint32_t entry;
    float base, near2;
    uint32_t source;  // the scene light it was built from
    float mask(Vec3 x) const;
    bool cone(float dist2, float& omc) const;
    bool intersect(const Ray& ray, float t_max, float& t) const;
    float weight(Vec3 x) const;
};
struct MeshEmitter {  // light.rs:440: an emissive instance sampled as an area light
    std::vector<std::array<Vec3, 3>> corners;  // world-space corners of each triangle
    std::vector<Vec3> normals;                 // unit normal of each (winding order: the front)
    std::vector<float> cdf;                    // cumulative area fractions
    float area;                                // mm^2
    Rgb radiance;
    bool two_sided;
    uint32_t entry;
    Vec3 centroid;       // area-weighted centre of its triangles
    float bound;         // radius of the sphere around the centroid that holds it
    Vec3 axis;           // the cone of its front faces' normals: axis, cos, sin (cos -1: any)
    float cos_o, sin_o;
    float base;          // lum(L) A, A in m^2
    float weight(Vec3 x) const;
};
struct Selection { Vec3 point; float total = 0; bool by_flux = true; float weights[8] = {}; };
// source: the scene light the sample came from (-1: the environment or an emissive mesh)
struct LightSample { Vec3 wi; float distance; Rgb radiance; float pdf; bool delta, glossy, photon, shadow; int source = -1; };
struct LightRef {  // light.rs:488
    enum Kind : uint32_t { Area, Sun, Sphere, Mesh, Environment } kind;
    uint32_t index;
};
struct Lights {
    std::vector<AreaLight> areas;
    std::vector<SunLight> suns;
    std::vector<SphereLight> spheres;
    std::vector<MeshEmitter> meshes;
    std::vector<int> instance_emitter;  // per instance: its mesh emitter, or -1
    EnvLight env;
    bool env_is_entry = false;
    uint32_t env_entry = 0;
    float env_base = 0;
    std::vector<LightRef> entries;
    std::vector<float> cdf, flux_pmf;
    bool per_point = false;

    static Lights make(const Scene& scene);
    float weight(size_t entry, Vec3 x) const;
    Selection select(Vec3 x) const;
    Selection select_by_flux(Vec3 x) const { Selection s; s.point = x; s.by_flux = true; return s; }
    float weight_at(size_t entry, const Selection& s) const { return entry < 8 ? s.weights[entry] : weight(entry, s.point); }
    float pmf(uint32_t entry, const Selection& from) const;
    void pick_at(const Selection& s, float u, size_t& idx, float& rest, float& pmf_out) const;
    bool sample_selected(const Selection& s, float u_select, float u0, float u1, LightSample& out) const;
    // `only` >= 0: *part receives the share of scene light `only` in the result.
    Rgb crossed_from(const Ray& ray, float t_max, const float* bsdf_pdf, const Selection* from, float offset, int only = -1,
                     Rgb* part = nullptr) const;
    // light.rs:1536-1550: for a BSDF-sampled ray that hit emissive instance `instance` at
    // distance t with `cos` between the ray and the geometric normal, the MIS weight of the emission
    // found (1 when the instance is not a mesh light).
    float emitter_weight(uint32_t instance, float bsdf_pdf, const Selection& from, float t, float cos) const;
    // light.rs:1490: a camera ray meets a light it sees (an area light flagged camera, or a sphere
    // flagged camera lit towards the ray's origin) before t_max.
    bool camera_sees_panel(const Ray& ray, float t_max) const;
    Rgb escaped(Vec3 dir, const float* bsdf_pdf, const Selection* from, int only = -1, Rgb* part = nullptr) const;
};
inline float power_heuristic(float pa, float pb) {  // light.rs:129
    if (!(pa > 0.0f)) return 0.0f;
    float r = pb / pa;
    return 1.0f / (1.0f + r * r);
}

}  // namespace orc
