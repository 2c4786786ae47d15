// Host-side scene assembly of the drop-in: the RSB subset reader, the reference's binned-SAH
// BVH builder (engine/crates/rt-core/src/geometry/bvh.rs:195-505) and its flattening into the
// quantised 8-wide layout of rtg_dev.h, and the light preparation of Lights::new
// (engine/crates/rt-core/src/light.rs:673-995).
#pragma once
#include <string>
#include <vector>

#include "rtg_dev.h"

namespace rtg {

struct HMaterial {
    uint32_t kind = 0;
    float base[3] = {0.8f, 0.8f, 0.8f};
    float metallic = 0, roughness = 0.5f, ior = 1.5f, transmission = 0, coat = 0, coat_roughness = 0;
    float emission[3] = {0, 0, 0};
    float emission_power = 0;
    uint32_t flags = 0;
    float opacity = 1, anisotropy = 0, absorption_mm = 0, bevel_mm = 0, scatter_mm = 0;
    float scatter_color[3] = {1, 1, 1};
    float scatter_g = 0, abbe = 0;
};
struct HLight {
    uint32_t kind = 0;
    V3 position{0, 0, 0}, direction{0, 0, -1}, up{0, 1, 0};
    float size_x = 0, size_y = 0;
    float color[3] = {1, 1, 1};
    float power = 0, spread_deg = 180, angle_deg = 0;
    uint32_t flags = 0;
    uint32_t profile = 0xffffffffu;  // an IES light's profile among the scene's IESP sections
};
struct HMesh {
    std::vector<V3> positions, normals;  // normals empty: none
    std::vector<uint32_t> indices;
    uint32_t material_id = 0;
    V3 bmin{0, 0, 0}, bmax{0, 0, 0};
    bool empty_bounds = true, inside_out = false;
    size_t triangles() const { return indices.size() / 3; }
};
// geometry/solid.rs: what a mesh is as a solid, 0 open, 1 closed and wound outward, 2 inward.
uint32_t solid_of(const HMesh& m);

struct HInstance {
    uint32_t mesh = 0;
    float rows[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
    uint32_t material_id = 0, flags = 0;
};
// An IES LM-63 type C profile (ies.rs:207): vertical and horizontal angles in degrees, the candela
// table (a row of vertical values per horizontal angle, the file's multiplier applied), its
// symmetry, peak and flux (candela steradians of the bilinear interpolant).
enum : uint32_t { IES_ROTATIONAL = 0, IES_QUADRANT = 1, IES_BILATERAL0 = 2, IES_BILATERAL90 = 3, IES_FULL = 4 };
struct HIes {
    uint32_t symmetry = IES_ROTATIONAL;
    std::vector<float> vertical, horizontal, candela;
    float peak = 0, flux = 0;
};
// IesProfile::parse (ies.rs:227): false with the reference's reason.
bool parse_ies(const uint8_t* bytes, size_t len, HIes& out, std::string& reason);

// A decoded bitmap: linear RGB texels (3 per pixel), rows top to bottom.
struct HImage {
    uint32_t width = 0, height = 0;
    std::vector<float> texels;
};
// An environment map's sampling grid (rtg_bitmap.cpp): cell weights, per-row conditional CDFs,
// the marginal CDF over rows, the mean weight, and the map's scale, rotation and mean luminance.
struct HEnvMap {
    uint32_t gw = 0, gh = 0;
    std::vector<float> weights, conditional, marginal;
    float mean = 0, scale = 0, rot_s = 0, rot_c = 1, mean_luminance = 0;
};
// Bitmap::decode (bitmap.rs:236): formats 0 and 1 (8-bit sRGB RGB, RGBA), 2 (linear f32 RGB) and
// 16 (a Radiance file). False with the reason otherwise; `unsupported` for OpenEXR (17).
bool decode_bitmap(uint32_t format, uint32_t width, uint32_t height, const uint8_t* data, size_t len, HImage& out, std::string& reason,
                   bool& unsupported);
// Map::new (environment.rs:60): false when the map has no light to sample.
bool build_env_map(const HImage& img, float scale, float rotation_deg, HEnvMap& out);
// sky_image (environment.rs:178): the scene's sky -- the physical model (sky.rs:96, the Hosek-Wilkie
// form with the Repackshot fit) or the classic one (sky.rs:245, Preetham et al. 1999) --
// tabulated into a 256 x 128 map, scaled to the dome's irradiance, the ground below.
struct HScene;
HImage sky_image(const HScene& s);
struct HScene {
    V3 cam_position{0, -1000, 0}, cam_target{0, 0, 0}, cam_up{0, 0, 1};
    // SECT (Q1): the section plane section_n . p = section_d, normalised as SectionPlane::new does.
    uint32_t section_on = 0, section_cap = 0;
    V3 section_n{0, 0, 1};
    float section_d = 0;
    float focal_mm = 50, sensor_mm = 36, fstop = 0, focus_dist = 1000, ortho_width = 1000;
    uint32_t ortho = 0, projection = 0;
    float fov_x = 360, fov_y = 180, exterior = 1;
    std::vector<HMaterial> materials;
    std::vector<HMesh> meshes;
    std::vector<HInstance> instances;
    std::vector<HLight> lights;
    std::vector<HImage> bitmaps;
    std::vector<HIes> profiles;
    uint32_t env_kind = 0;  // 0 studio, 1 flat, 2 sky, 3 HDRI
    float env_floor = 0.1f, env_horizon = 0.3f, env_zenith = 0.6f, env_strength = 1, env_rotation = 0;
    float background_color[3] = {0.05f, 0.05f, 0.05f};
    uint32_t background_mode = 0;  // 0 environment, 1 colour, 2 transparent, 3 background image
    uint32_t hdri_map = 0xffffffffu, backplate_map = 0xffffffffu, backplate_fit = 0;
    float backplate_rect[4] = {0, 0, 1, 1};
    float sky_turbidity = 3, sun_azimuth_deg = 0, sun_elevation_deg = 45;
    uint32_t sky_model = 0;  // 0 physical, 1 classic
    uint32_t floor_mode = 0;
    float floor_z = 0;
    float floor_color[3] = {0.5f, 0.5f, 0.5f};
    uint32_t width = 640, height = 360, max_samples = 64, seed = 0, tonemap = 1, max_depth = 8;
    float max_seconds = 0, exposure_ev = 0, clamp_indirect = 0;
    uint32_t pixel_filter = 0, edge_supersample = 1;
    uint32_t adaptive = 0;        // RNDR.adaptive (E10): bit 0 asks the host for adaptive sampling
    float noise_threshold = 0;    // RNDR.noise_threshold: the relative error a block stops at (0: none)
};

// Parses the RSB subset the path tracer reads. Returns false with `error` set (the reference's
// wording for format errors, "unsupported: ..." for features outside this path). With `kept`, a
// file without MESH sections takes those meshes instead (Scene::update_from_rsb,
// engine/crates/rt-core/src/scene/rsb.rs:1630): its INST sections, or the implicit instances of
// the kept meshes, refer to them. `used_kept` (may be null) tells whether it did. A file without
// BMAP sections takes `kept_bitmaps` (when given) as its bitmaps, as the reference's update does.
bool parse_rsb(const uint8_t* bytes, size_t len, HScene& out, std::string& error, const std::vector<HMesh>* kept = nullptr,
               bool* used_kept = nullptr, const std::vector<HImage>* kept_bitmaps = nullptr);

// What the device geometry (trees, leaf triangles, hit-detail arrays) of a scene depends on,
// besides the meshes themselves: the instances' meshes, transforms and visibility flags. Two
// scenes over the same meshes with equal keys have identical device geometry.
std::string geometry_key(const HScene& s);

// Flattened, device-ready arrays of a scene.
struct Flat {
    // the environment map's texels and sampling grid, the background image's texels (uploaded
    // with the shading; the pointers in `lights` and `scene` are set on upload)
    HEnvMap env_map;
    HImage sky;  // the tabulated sky of a sky environment
    std::vector<float> ies_data;  // per IES light: vertical angles, horizontal angles, candela
    std::vector<float> mesh_light_data;  // per mesh light's triangle: 16 floats (LightDev::tris)
    std::vector<float> exempt_boxes;     // the section's exempt instances: grown world box lo, hi
    const HImage* env_image = nullptr;
    const HImage* plate = nullptr;
    std::vector<QNode> nodes;
    std::vector<TriRec> tris;
    std::vector<BlasInst> blas;
    std::vector<DevInstance> instances;
    std::vector<float> positions, normals;  // 4 floats per vertex
    std::vector<uint32_t> tri_index;        // 4 per triangle
    std::vector<DevMaterial> materials;
    std::vector<Bsdf> bsdfs;  // 2 per material (entering, leaving), then the floor's
    LightsDev lights;
    SceneDev scene;  // pointers left null
    uint32_t tlas_root = NODE_EMPTY;
    uint32_t stack_need = 0;
    float box_lo[3] = {0, 0, 0}, box_hi[3] = {0, 0, 0};  // the ray sort's box (empty: lo > hi)
    uint64_t instanced_triangles = 0;
    double build_seconds = 0;
};
// Builds the BVHs and the device layout. Returns false with `error` when a limit is exceeded.
// Without `geometry`, only the shading part is built (instances, materials, BSDFs, lights, the
// scene constants); nodes, triangles and vertex arrays stay empty and the tree fields of `scene`
// (tlas_root, stack_need) are left for the caller to take from the geometry it keeps.
bool flatten_scene(const HScene& s, Flat& out, std::string& error, bool geometry = true);

}  // namespace rtg
