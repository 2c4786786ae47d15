// Data layout in device memory shared by the host upload (rtg_scene.cpp) and the kernels
// (rtg_kernels.cu). Everything here is plain data: no torch types, no host pointers.
#pragma once
#include <vector_types.h>

#include <cstdint>

#include "rtg_bsdf.cuh"

namespace rtg {

constexpr uint32_t NODE_EMPTY = 0xffffffffu;
constexpr uint32_t NODE_LEAF = 1u << 31;
// Leaf reference: NODE_LEAF | first << 4 | (count - 1), count in 1..16.
RTG_HD uint32_t make_leaf(uint32_t first, uint32_t count) { return NODE_LEAF | (first << 4) | (count - 1); }

// An 8-wide BVH node with child boxes quantised to 8 bits per plane (96 bytes, six 16-byte
// loads). A child box decodes as p + q * 2^e per axis; the builder checks that every decoded box
// (computed with the same IEEE operations as the kernels) contains the child's exact box, so the
// slab test never drops a hit that the exact box keeps. A flat child at the node's lower corner
// (a floor under the rest of the scene) decodes to its exact plane, so a ray starting within
// t_min of it is culled exactly where the reference's box culls it.
struct alignas(16) QNode {
    float px, py, pz;
    uint8_t ex, ey, ez;   // biased exponents of the per-axis scales 2^(e-127)
    uint8_t nchild;
    uint8_t qlo[3][8];
    uint8_t qhi[3][8];
    uint32_t child[8];    // inner node index, leaf reference or NODE_EMPTY
};
static_assert(sizeof(QNode) == 96, "QNode must be 96 bytes");

// A leaf triangle (48 bytes): corners in its BLAS's space; w lanes carry the triangle's index in
// its mesh, its instance (0xffffffff: the BLAS instance's) and flags (bit 0 one-sided, bit 1
// hidden to camera rays).
struct alignas(16) TriRec {
    float v0[3]; uint32_t tri;
    float v1[3]; uint32_t inst;
    float v2[3]; uint32_t flags;
};

// A TLAS leaf: one bottom-level tree placed in the world.
struct alignas(16) BlasInst {
    float to_local[12];   // world -> object rows (unused when identity)
    uint32_t root;        // node index or leaf reference of the BLAS
    uint32_t identity;    // the BLAS is in world space
    uint32_t instance;    // instance id for BLAS records that carry 0xffffffff
    uint32_t flags;       // bit 0 one-sided, bit 1 hidden to camera rays
};

// Per instance, what hit details and shading read.
struct alignas(16) DevInstance {
    float to_local[12];
    float to_world[12];
    uint32_t identity, active, material, mesh;
    uint32_t flags, inside_out, has_normals, tri_base;  // tri_base: first global triangle of its mesh
    uint32_t tangent_on, passable, emitter, solid;  // passable: shadow rays cross it (cut-out or thin wall);
                                                    // emitter: its mesh light's index in lights[] + 1, or 0;
                                                    // solid: the section caps it, 1 wound outward, 2 inward (0 not)
    float tan_centre[3], tan_axis[3], tan_x[3];
    uint32_t exempt;  // the section neither cuts nor caps it (INST flag 2, the studio)
    float pad3[2];
};

// One light of the selection (light.rs:300-495): an area light (rect or disk), a sun, a sphere
// light (a point light or a spot; radius 0 is a point) or an emissive mesh sampled by area. Each
// kind reads its own fields.
enum : uint32_t { LIGHT_AREA = 0, LIGHT_SUN = 1, LIGHT_SPHERE = 2, LIGHT_MESH = 3 };
struct LightDev {
    float centre[3];
    // area: its frame; sun: a frame whose z points at the sun; sphere: fz is a spot's axis
    float fx[3], fy[3], fz[3];
    float half_x, half_y, radius, area;
    float radiance[3];  // area, sun disc (a delta sun: its irradiance), sphere surface
    float exponent, base, bound;
    float cos_max, one_minus_cos_max, solid_angle;  // sun
    float intensity[3];                             // sphere: W/sr
    float cos_outer, cos_inner, near2;              // sphere: cos_outer below -1 means no mask
    // an IES light (a sphere masked by its profile in the frame fx, fy, fz: axis z, angle 0 along
    // y): vertical angles, horizontal angles, candela rows
    const float* ies;
    uint32_t ies_nv, ies_nh, ies_sym;
    float ies_peak;
    uint32_t kind, rect, delta;
    uint32_t glossy, camera, shadow, entry;
    uint32_t source;  // index of the scene light it was built from (0xffffffff: an emissive mesh)
    // an emissive mesh (light.rs:440): per world-space triangle four float4s -- corner a with the
    // cumulative area fraction in w, corners b and c, the unit normal (winding order: the front);
    // the cone of the front faces' normals about fz (cos_o -1: any direction); centre, bound, area
    // (mm^2), radiance and base as an area light's
    const float4* tris;
    uint32_t n_tris, two_sided;
    float cos_o, sin_o;
};
constexpr int MAX_ENTRIES = 64;
constexpr int MAX_LIGHTS = 63;

// An equirectangular environment map (environment.rs:49): linear RGB texels, rows top to bottom,
// importance-sampled by a piecewise-constant 2-D distribution over a grid of its cells
// (bitmap.rs:330): per-row conditional CDFs, the marginal CDF over rows, the cell weights.
struct EnvMapDev {
    const float* texels;  // 3 per pixel
    uint32_t width, height;
    float scale, rot_s, rot_c;
    const float* weights;      // gw * gh
    const float* conditional;  // gw * gh
    const float* marginal;     // gh
    uint32_t gw, gh;
    float mean;
};

struct LightsDev {
    // lights[] holds the area lights, then the suns, then the sphere lights, each in scene order
    int n_areas, n_entries, per_point, env_is_entry;
    uint32_t env_entry, n_suns, n_spheres, n_lights;  // n_lights counts the mesh lights after the spheres
    float env_floor, env_horizon, env_zenith, env_lower, env_total, env_base;
    uint32_t env_is_map;  // the environment is `env_map`, else the ramp above
    EnvMapDev env_map;
    int entries[MAX_ENTRIES];  // >= 0 index into lights[], -1 environment
    float cdf[MAX_ENTRIES];
    float flux_pmf[MAX_ENTRIES];
    LightDev lights[MAX_LIGHTS];
};

// Everything a launch needs besides the per-path buffers (constant memory).
struct SceneDev {
    // camera (basis precomputed on the host with the reference's operations)
    float cam_pos[3], cam_fwd[3], cam_right[3], cam_up[3];
    float focal_mm, sensor_mm, focus_dist, lens_radius, ortho_width, exterior;
    uint32_t ortho;
    uint32_t projection;        // K3 (scene/mod.rs:55): 0 the standard camera, 1 equirectangular, 2 fisheye
    float fov_x_deg, fov_y_deg;  // a panoramic camera's fields across the width and the height
    // render settings
    uint32_t width, height, seed, max_depth, pixel_filter;
    // Sample indices from split_b on are scrambled with seed_b instead of seed (sample_key). A
    // render keeps split_b = 0xffffffff; the decorrelated adjoint draws its second half with it.
    uint32_t seed_b, split_b;
    float clamp_indirect;
    const float* filter_table;  // the Blackman-Harris inverse CDF, 256 points (pixel filter 3)
    uint32_t edge_k;            // samples per sample index of an edge pixel (1: no edge samples)
    uint32_t background;  // 0 environment, 1 colour, 2 transparent, 3 background image
    float background_color[3];
    // The background image fitted to the frame (integrator/mod.rs:187): linear RGB texels.
    const float* plate;
    uint32_t plate_w, plate_h, plate_fit;  // fit: 0 fill, 1 fit, 2 stretch
    float plate_rect[4], frame_aspect, image_aspect;
    // Some instance lets shadow rays through (a cut-out or a thin wall); some material is a cut-out
    // (paths then pass surfaces without a vertex, and waves run extra rounds).
    uint32_t any_passable, any_cutout;
    uint32_t floor_mode;
    float floor_z;
    float floor_color[3];
    // geometry
    const QNode* nodes;
    const TriRec* tris;
    const BlasInst* blas;
    const DevInstance* instances;
    const float4* positions;  // xyz per vertex (global)
    const float4* normals;    // xyz per vertex (global)
    const uint4* tri_index;   // global vertex indices per global triangle
    const DevMaterial* materials;
    // Bsdf::surface of every material seen from outside (2 m) and from inside (2 m + 1), and the
    // floor's Lambert lobe (2 n_materials): built once on the host, the same bits.
    const Bsdf* bsdfs;
    uint32_t tlas_root, n_instances, n_materials, stack_need;
    EnergyTables energy;
    // The section view (geometry/section.rs): the plane n . p = d removes the side n points to from
    // every query; with section_cap the closed solids it cuts are capped (their instances' `solid`),
    // and a point can only be on a cap inside cap_lo..cap_hi (cap_any: some instance is capped). The
    // exempt instances' world boxes, grown, are 6 floats each (lo, hi).
    uint32_t section_on, section_cap, cap_any, n_exempt;
    float section_n[3], section_d;
    float cap_lo[3], cap_hi[3];
    const float* exempt_boxes;
};

}  // namespace rtg
