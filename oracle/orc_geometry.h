// ORACLE (test infrastructure only). Restatement of the reference's geometry: meshes, the binned
// SAH BVH collapsed to 8-wide nodes, the Woop–Benthin–Wald watertight triangle test, two-level
// traversal and hit details (engine/crates/rt-core/src/geometry/{bvh,mesh,triangle,traverse,
// transform,mod}.rs, bevel.rs:232-252).
#pragma once
#include <cstdint>
#include <vector>

#include "orc_core.h"

namespace orc {

// ---- transform.rs ---------------------------------------------------------------------------
struct Transform {
    float r[3][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}};
    bool is_identity() const {
        static const float I[3][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 4; ++j)
                if (!(r[i][j] == I[i][j])) return false;
        return true;
    }
    Vec3 point(Vec3 p) const {
        return {r[0][0] * p.x + r[0][1] * p.y + r[0][2] * p.z + r[0][3],
                r[1][0] * p.x + r[1][1] * p.y + r[1][2] * p.z + r[1][3],
                r[2][0] * p.x + r[2][1] * p.y + r[2][2] * p.z + r[2][3]};
    }
    Vec3 vector(Vec3 v) const {
        return {r[0][0] * v.x + r[0][1] * v.y + r[0][2] * v.z,
                r[1][0] * v.x + r[1][1] * v.y + r[1][2] * v.z,
                r[2][0] * v.x + r[2][1] * v.y + r[2][2] * v.z};
    }
    Vec3 transpose_vector(Vec3 v) const {
        return {r[0][0] * v.x + r[1][0] * v.y + r[2][0] * v.z,
                r[0][1] * v.x + r[1][1] * v.y + r[2][1] * v.z,
                r[0][2] * v.x + r[1][2] * v.y + r[2][2] * v.z};
    }
    Ray ray(const Ray& ry) const {
        Ray o;
        o.origin = point(ry.origin);
        o.dir = vector(ry.dir);
        o.t_min = ry.t_min;
        o.t_max = ry.t_max;
        return o;
    }
    bool is_finite() const {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 4; ++j)
                if (!finite(r[i][j])) return false;
        return true;
    }
    float determinant() const;
    bool inverse(Transform& out) const;
    Aabb aabb(const Aabb& b) const;
};

// ---- bvh.rs ---------------------------------------------------------------------------------
constexpr uint32_t BVH_EMPTY = 0xffffffffu;
constexpr uint32_t BVH_LEAF = 1u << 31;
inline uint32_t leaf_ref(uint32_t first, uint32_t count) { return BVH_LEAF | (first << 3) | (count - 1); }
inline void leaf_range(uint32_t ref, uint32_t& first, uint32_t& count) {
    first = (ref & ~BVH_LEAF) >> 3;
    count = (ref & 7u) + 1;
}
struct WideNode8 {
    float bounds[3][2][8];  // [axis][min/max][child]
    uint32_t child[8];
};
struct Bvh {
    std::vector<WideNode8> nodes;
    uint32_t root = BVH_EMPTY;
};
struct BinaryNode { Aabb bounds; uint32_t left = 0, right = 0, first = 0, count = 0; };
// Builds the binned-SAH binary tree and its 8-wide collapse; `leaves` receives each leaf's
// primitive list in tree order and returns the reference to store.
template <class EmitLeaf>
Bvh build_bvh(const std::vector<Aabb>& boxes, const std::vector<Vec3>& centroids, int leaf_target, int leaf_max,
              EmitLeaf emit);

// ---- triangle.rs ----------------------------------------------------------------------------
struct PreparedRay {
    float org[3], inv[3];
    bool negative[3];
    int k[3];
    float shear[3];
    float t_min, t_max;
    static PreparedRay make(const Ray& ray);
    bool has_interval() const { return t_min <= t_max; }
};
struct EdgeHit { float t, u, v, w, det; };
enum class Cull { None, Back };
bool watertight(const PreparedRay& r, Vec3 v0, Vec3 v1, Vec3 v2, float t_max, Cull cull, EdgeHit& out);

struct TriPacket { float v[3][3][4]; uint32_t id[4]; };

// ---- mesh.rs --------------------------------------------------------------------------------
struct Mesh {
    std::vector<Vec3> positions;
    std::vector<Vec3> normals;  // empty: no normals
    std::vector<uint32_t> indices;
    uint32_t material_id = 0;
    Aabb bounds;
    Bvh bvh;
    std::vector<TriPacket> packets;
    bool inside_out = false;
    // Returns an error string (empty on success).
    static const char* make(Mesh& out, const std::vector<Vec3>& positions, const std::vector<Vec3>& normals,
                            const std::vector<uint32_t>& indices, uint32_t material_id);
    size_t triangle_count() const { return indices.size() / 3; }
    bool has_normals() const { return !normals.empty(); }
    void corners(uint32_t t, Vec3& a, Vec3& b, Vec3& c) const {
        a = positions[indices[3 * t]];
        b = positions[indices[3 * t + 1]];
        c = positions[indices[3 * t + 2]];
    }
};

// ---- geometry/mod.rs ------------------------------------------------------------------------
constexpr uint32_t INSTANCE_ONE_SIDED = 1, INSTANCE_NO_SECTION = 2, INSTANCE_NO_CAMERA = 4;
struct Instance { uint32_t mesh = 0; Transform transform; uint32_t material_id = 0; uint32_t flags = 0; };
struct PreparedInstance { Transform to_local; bool identity = true; Cull cull = Cull::None; bool active = false; bool camera_hidden = false; };
struct RayHit { uint32_t instance, triangle; float t; };
struct Hit {
    uint32_t instance, triangle;
    float t;
    Vec3 point, normal, geometric_normal;
    float bary[3];
    bool front_face, outside;
};
// Per-query traversal statistics (reference BVH8 layout): inner-node visits and packet tests.
struct TraceStats { uint64_t nodes = 0, packets = 0; };

// ---- geometry/solid.rs, geometry/section.rs ---------------------------------------------------
// What a mesh is as a solid: open (no inside), or closed and wound outward (the back of a triangle
// is the inside) or inward.
enum class Solid : uint8_t { Open, Outward, Inward };
// geometry/mod.rs:284: a mesh's box in the world, padded for a transformed one.
Aabb instance_bounds(const Mesh& mesh, const Transform& t);
Solid analyse_solid(const Mesh& mesh);
inline bool inside_before(Solid s, bool front) { return s == Solid::Outward ? !front : s == Solid::Inward ? front : false; }

// The `triangle` of a hit on the cap of a cut solid.
constexpr uint32_t CAP_TRIANGLE = 0xffffffffu;

// The plane normal . p = distance; the kept side is normal . p <= distance.
struct SectionPlane {
    Vec3 normal;
    float distance = 0.0f;
    bool cap = false;
    // SectionPlane::new: false for a zero or non-finite normal or distance; the normal normalised
    // unless it is unit already to 1e-6.
    static bool make(Vec3 normal, float distance, bool cap, SectionPlane& out);
    float side(Vec3 p) const { return dot(normal, p) - distance; }
};

struct Section {
    SectionPlane plane;
    std::vector<Solid> caps;           // per instance
    Aabb cap_bounds;                   // the capped instances' world boxes, grown
    std::vector<uint8_t> exempt;       // per instance (empty: none is exempt)
    std::vector<Aabb> exempt_boxes;    // the exempt instances' world boxes, grown
};

struct Geometry {
    std::vector<Mesh> meshes;
    std::vector<Instance> instances;
    std::vector<PreparedInstance> prepared;
    Bvh tlas;
    std::vector<uint32_t> tlas_instances;
    Aabb bounds;
    static const char* make(Geometry& g, std::vector<Mesh> meshes, std::vector<Instance> instances);

    bool has_section = false;
    Section section;
    // Geometry::set_section: `capped[i]` false for an instance the plane may not cap (a thin wall).
    void set_section(const SectionPlane* plane, const std::vector<bool>& capped);

    // The queries, through the section when there is one (geometry/section.rs:224-324).
    bool trace(const Ray& ray, bool camera, RayHit& out, TraceStats* st = nullptr) const;
    bool occluded(const Ray& ray, bool camera, TraceStats* st = nullptr) const;
    // The queries against the whole model.
    bool trace_raw(const Ray& ray, bool camera, RayHit& out, TraceStats* st = nullptr) const;
    bool occluded_raw(const Ray& ray, bool camera, TraceStats* st = nullptr) const;
    bool trace_brute(const Ray& ray, bool camera, RayHit& out) const;
    bool hit_details(const Ray& ray, const RayHit& hit, Hit& out) const;
    // Section::cap_details (section.rs:424-448): on the plane, facing the side the ray came from.
    bool cap_details(const Ray& ray, const RayHit& hit, Hit& out) const;
    Vec3 terminator_point(const Hit& hit) const;
};

}  // namespace orc
