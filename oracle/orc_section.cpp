// Test infrastructure: the oracle's section view (Q1), a CPU restatement of the reference's
// engine/crates/rt-core/src/geometry/section.rs (the plane, the clipped queries, the caps and the
// exempt studio) and geometry/solid.rs (which meshes are closed solids, with the vertex weld of
// geometry/edges.rs:221-330). The CUDA path is checked against it; nothing in the product links it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <tuple>

#include "orc_geometry.h"

namespace orc {

namespace {
constexpr float WELD_TOLERANCE = 1.0e-5f;   // edges.rs:52, of the mesh's extent
constexpr size_t VOLUME_BLOCK = 256;        // solid.rs: terms summed at a time
constexpr float MIN_VOLUME = 1.0e-9f;       // solid.rs: of the cube of the mesh's extent
constexpr int MAX_SKIPS = 48;               // section.rs: surfaces stepped over looking for the studio

uint32_t key_bits(float v) {  // edges.rs:200: +0 and -0 are one position
    if (v == 0.0f) return 0;
    uint32_t b;
    std::memcpy(&b, &v, 4);
    return b;
}

// The weld group of every vertex: vertices at the same position, then unique positions within
// the tolerance on every axis of one another, joined transitively (edges.rs:221-330). Only which
// vertices share a group matters to the solid test, not how the groups are numbered.
std::vector<uint32_t> weld_groups(const Mesh& m) {
    const size_t n = m.positions.size();
    std::vector<uint32_t> order(n);
    for (size_t i = 0; i < n; ++i) order[i] = (uint32_t)i;
    auto key = [&](uint32_t i) {
        const Vec3& p = m.positions[i];
        return std::make_tuple(key_bits(p.x), key_bits(p.y), key_bits(p.z));
    };
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return key(a) != key(b) ? key(a) < key(b) : a < b; });
    std::vector<uint32_t> unique_of(n);
    std::vector<Vec3> unique;
    for (size_t k = 0; k < n; ++k) {
        if (k == 0 || key(order[k]) != key(order[k - 1])) unique.push_back(m.positions[order[k]]);
        unique_of[order[k]] = (uint32_t)unique.size() - 1;
    }
    const Aabb bounds = m.bounds;
    const float extent = bounds.is_empty() ? 0.0f : max_component(bounds.max - bounds.min);
    const float tolerance = extent * WELD_TOLERANCE;
    std::vector<uint32_t> parent(unique.size());
    for (size_t i = 0; i < parent.size(); ++i) parent[i] = (uint32_t)i;
    auto root = [&](uint32_t i) {
        while (parent[i] != i) {
            uint32_t up = parent[parent[i]];
            parent[i] = up;
            i = up;
        }
        return i;
    };
    if (tolerance > 0.0f && std::isfinite(tolerance)) {
        const float cell_size = 2.0f * tolerance;
        using Cell = std::tuple<int64_t, int64_t, int64_t>;
        auto axis = [&](float v, float lo) {
            float c = std::floor((v - lo) / cell_size);
            if (!(c == c)) return (int64_t)0;
            if (c >= 9.2e18f) return INT64_MAX;
            if (c <= -9.2e18f) return INT64_MIN;
            return (int64_t)c;
        };
        auto cell = [&](Vec3 p) { return Cell(axis(p.x, bounds.min.x), axis(p.y, bounds.min.y), axis(p.z, bounds.min.z)); };
        std::vector<std::pair<Cell, uint32_t>> by_cell;
        for (size_t i = 0; i < unique.size(); ++i) by_cell.push_back({cell(unique[i]), (uint32_t)i});
        std::sort(by_cell.begin(), by_cell.end());
        for (size_t i = 0; i < unique.size(); ++i) {
            const Cell c = cell(unique[i]);
            for (int dx = -1; dx <= 1; ++dx)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dz = -1; dz <= 1; ++dz) {
                        const Cell k(std::get<0>(c) + dx, std::get<1>(c) + dy, std::get<2>(c) + dz);
                        auto it = std::lower_bound(by_cell.begin(), by_cell.end(), k,
                                                   [](const std::pair<Cell, uint32_t>& e, const Cell& v) { return e.first < v; });
                        for (; it != by_cell.end() && it->first == k; ++it) {
                            const uint32_t j = it->second;
                            if (j <= i) continue;
                            Vec3 d = vabs(unique[i] - unique[j]);
                            if (d.x <= tolerance && d.y <= tolerance && d.z <= tolerance) {
                                uint32_t a = root((uint32_t)i), b = root(j);
                                parent[std::max(a, b)] = std::min(a, b);
                            }
                        }
                    }
        }
    }
    std::vector<uint32_t> ids(n);
    for (size_t v = 0; v < n; ++v) ids[v] = root(unique_of[v]);
    return ids;
}

Aabb grown(const Aabb& b) {  // section.rs: a crossing point rounded onto a box's face is in it
    const float size = max_component(b.max - b.min);
    const float pad = size * 1.0e-5f + 1.0e-4f;
    return Aabb(b.min - Vec3(pad, pad, pad), b.max + Vec3(pad, pad, pad));
}
}  // namespace

bool SectionPlane::make(Vec3 normal, float distance, bool cap, SectionPlane& out) {
    const float length = std::sqrt(length_squared(normal));
    if (!(vfinite(normal) && std::isfinite(length) && length > 0.0f && std::isfinite(distance))) return false;
    out.normal = std::fabs(length - 1.0f) <= 1.0e-6f ? normal : normal * (1.0f / length);
    out.distance = distance;
    out.cap = cap;
    return true;
}

// solid.rs analyse: closed when, after the weld, every edge of every triangle with an area is shared
// by exactly two triangles running along it in opposite directions; the sign of the enclosed volume
// (summed about the box's centre in blocks of 256 terms) tells outward from inward winding.
Solid analyse_solid(const Mesh& mesh) {
    const size_t triangles = mesh.triangle_count();
    const Aabb bounds = mesh.bounds;
    if (triangles == 0 || bounds.is_empty()) return Solid::Open;
    const std::vector<uint32_t> weld = weld_groups(mesh);
    const Vec3 centre = bounds.centroid();
    std::vector<std::tuple<uint32_t, uint32_t, bool>> halves;
    halves.reserve(triangles * 3);
    float blocks = 0.0f, block = 0.0f;
    size_t in_block = 0;
    for (size_t t = 0; t < triangles; ++t) {
        const uint32_t w[3] = {weld[mesh.indices[3 * t]], weld[mesh.indices[3 * t + 1]], weld[mesh.indices[3 * t + 2]]};
        if (w[0] == w[1] || w[1] == w[2] || w[2] == w[0]) continue;
        Vec3 p0, p1, p2;
        mesh.corners((uint32_t)t, p0, p1, p2);
        if (length_squared(cross(p1 - p0, p2 - p0)) <= 0.0f) continue;
        for (int k = 0; k < 3; ++k) {
            const uint32_t from = w[k], to = w[(k + 1) % 3];
            halves.emplace_back(std::min(from, to), std::max(from, to), from < to);
        }
        block += dot(p0 - centre, cross(p1 - centre, p2 - centre));
        if (++in_block == VOLUME_BLOCK) {
            blocks += block;
            block = 0.0f;
            in_block = 0;
        }
    }
    if (halves.empty()) return Solid::Open;
    std::sort(halves.begin(), halves.end());
    if (halves.size() % 2) return Solid::Open;
    for (size_t i = 0; i < halves.size(); i += 2) {
        const auto& a = halves[i];
        const auto& b = halves[i + 1];
        if (!(std::get<0>(a) == std::get<0>(b) && std::get<1>(a) == std::get<1>(b) && !std::get<2>(a) && std::get<2>(b)))
            return Solid::Open;
    }
    const float extent = max_component(bounds.max - bounds.min);
    const float volume = (blocks + block) / 6.0f;
    if (!std::isfinite(volume) || std::fabs(volume) <= extent * extent * extent * MIN_VOLUME) return Solid::Open;
    return volume > 0.0f ? Solid::Outward : Solid::Inward;
}

// Geometry::set_section (section.rs:180-222): per instance whether it is capped (a closed solid, the
// plane asks for caps, the instance is live, not exempt and `capped`), the grown union of the capped
// instances' boxes, and the exempt (studio) instances with their grown boxes.
void Geometry::set_section(const SectionPlane* plane, const std::vector<bool>& capped) {
    has_section = plane != nullptr;
    section = Section();
    if (!plane) return;
    section.plane = *plane;
    for (size_t i = 0; i < instances.size(); ++i) {
        const Instance& inst = instances[i];
        const Mesh* mesh = inst.mesh < meshes.size() ? &meshes[inst.mesh] : nullptr;
        const bool live = i < prepared.size() && prepared[i].active;
        const bool is_exempt = (inst.flags & INSTANCE_NO_SECTION) != 0;
        if (is_exempt && live && mesh) {
            if (section.exempt.empty()) section.exempt.assign(instances.size(), 0);
            section.exempt[i] = 1;
            section.exempt_boxes.push_back(grown(instance_bounds(*mesh, inst.transform)));
        }
        const bool wanted = plane->cap && !is_exempt && (i < capped.size() ? capped[i] : true);
        const Solid solid = (mesh && wanted && live) ? analyse_solid(*mesh) : Solid::Open;
        if (mesh && solid != Solid::Open) section.cap_bounds = section.cap_bounds.uni(grown(instance_bounds(*mesh, inst.transform)));
        section.caps.push_back(solid);
    }
}

namespace {
enum class SpanKind { Removed, Whole, Enters, Leaves };

// Where the ray is on the kept side (section.rs:127-154).
SpanKind span(const SectionPlane& plane, const Ray& ray, float& t) {
    const float from_plane = dot(plane.normal, ray.origin) - plane.distance;
    const float towards = dot(plane.normal, ray.dir);
    if (towards == 0.0f) return from_plane <= 0.0f ? SpanKind::Whole : SpanKind::Removed;
    t = -from_plane / towards;
    if (towards > 0.0f) {
        if (t < ray.t_min) return SpanKind::Removed;
        if (t >= ray.t_max) return SpanKind::Whole;
        return SpanKind::Leaves;
    }
    if (t <= ray.t_min) return SpanKind::Whole;
    if (t > ray.t_max) return SpanKind::Removed;
    return SpanKind::Enters;
}

bool may_cap(const Section& s, Vec3 p) {
    const Aabb& b = s.cap_bounds;
    return !b.is_empty() && p.x >= b.min.x && p.x <= b.max.x && p.y >= b.min.y && p.y <= b.max.y && p.z >= b.min.z &&
           p.z <= b.max.z;
}

Ray limited(const Ray& ray, float t_min, float t_max) {
    Ray r = ray;
    r.t_min = t_min;
    r.t_max = t_max;
    return r;
}

// Aabb::intersect (math.rs:388-408): the interval where the ray is in the box, clipped to its range.
bool box_interval(const Aabb& b, const Ray& ray, Vec3 inv_dir, float& near, float& far) {
    near = ray.t_min;
    far = ray.t_max;
    const float lo[3] = {b.min.x, b.min.y, b.min.z}, hi[3] = {b.max.x, b.max.y, b.max.z};
    const float o[3] = {ray.origin.x, ray.origin.y, ray.origin.z}, inv[3] = {inv_dir.x, inv_dir.y, inv_dir.z};
    for (int a = 0; a < 3; ++a) {
        const float x = (lo[a] - o[a]) * inv[a], y = (hi[a] - o[a]) * inv[a];
        if (x != x || y != y) continue;  // parallel to the slab, on its boundary
        near = rmax(near, rmin(x, y));
        far = rmin(far, rmax(x, y));
    }
    return near <= far && near < F_INF;
}

float next_up(float t) {
    uint32_t b;
    std::memcpy(&b, &t, 4);
    ++b;
    std::memcpy(&t, &b, 4);
    return t;
}
}  // namespace

bool Geometry::cap_details(const Ray& ray, const RayHit& hit, Hit& out) const {
    if (!has_section || hit.instance >= instances.size()) return false;
    const SectionPlane& plane = section.plane;
    const Vec3 at = ray.at(hit.t);
    const Vec3 point = at - plane.normal * plane.side(at);
    const bool front = dot(plane.normal, ray.dir) < 0.0f;
    const Vec3 normal = front ? plane.normal : -plane.normal;
    out.instance = hit.instance;
    out.triangle = CAP_TRIANGLE;
    out.t = hit.t;
    out.point = point;
    out.normal = normal;
    out.geometric_normal = normal;
    out.bary[0] = 1.0f;
    out.bary[1] = out.bary[2] = 0.0f;
    out.front_face = front;
    out.outside = front;
    return true;
}

namespace {
struct SectionQueries {
    const Geometry& g;
    const Section& s;
    bool camera;
    TraceStats* st;

    bool hidden(uint32_t instance) const { return camera && g.prepared[instance].camera_hidden; }

    // True when `hit` is on a capped instance and the ray meets its triangle from inside the solid.
    bool met_from_inside(const Ray& ray, const RayHit& hit) const {
        if (hit.instance >= s.caps.size() || s.caps[hit.instance] == Solid::Open) return false;
        const PreparedInstance& p = g.prepared[hit.instance];
        if (!p.active) return false;
        const Mesh& mesh = g.meshes[g.instances[hit.instance].mesh];
        if (hit.triangle >= mesh.triangle_count()) return false;
        Vec3 p0, p1, p2;
        mesh.corners(hit.triangle, p0, p1, p2);
        Vec3 winding = cross(p1 - p0, p2 - p0);
        if (!p.identity) winding = p.to_local.transpose_vector(winding);
        return inside_before(s.caps[hit.instance], dot(winding, ray.dir) < 0.0f);
    }

    // The first exempt instance within [near, far], stepping over the others' surfaces.
    bool first_exempt(const Ray& ray, float near, float far, RayHit& out) const {
        float t = near;
        for (int k = 0; k < MAX_SKIPS; ++k) {
            RayHit hit;
            if (!g.trace_raw(limited(ray, t, far), camera, hit, st)) return false;
            if (hit.instance < s.exempt.size() && s.exempt[hit.instance]) { out = hit; return true; }
            t = next_up(rmax(hit.t, 0.0f));
            if (t > far) return false;
        }
        return false;
    }

    // The nearest exempt hit within [from, to] (the removed part of the ray's range).
    bool exempt_in(const Ray& ray, float from, float to, RayHit& out) const {
        if (s.exempt_boxes.empty() || from != from || to != to || from > to) return false;
        const Vec3 inv_dir(1.0f / ray.dir.x, 1.0f / ray.dir.y, 1.0f / ray.dir.z);
        bool found = false;
        for (const Aabb& box : s.exempt_boxes) {
            const float end = found ? rmin(out.t, to) : to;
            float near, far;
            if (!box_interval(box, limited(ray, from, end), inv_dir, near, far)) continue;
            RayHit hit;
            if (first_exempt(ray, near, rmin(far, end), hit) && (!found || hit.t < out.t)) {
                out = hit;
                found = true;
            }
        }
        return found;
    }

    // The cap at t where the ray leaves the kept side having hit nothing: there when the next
    // surface of the whole model along the ray is met from inside its solid.
    bool cap_beyond(const Ray& ray, float t, RayHit& out) const {
        if (!s.plane.cap || !may_cap(s, ray.at(t))) return false;
        RayHit hit;
        if (!g.trace_raw(limited(ray, t, F_INF), false, hit, st)) return false;
        if (!met_from_inside(ray, hit)) return false;
        out = {hit.instance, CAP_TRIANGLE, t};
        return true;
    }

    bool trace(const Ray& ray, RayHit& out) const {
        float t = 0.0f;
        switch (span(s.plane, ray, t)) {
            case SpanKind::Removed: return exempt_in(ray, ray.t_min, ray.t_max, out);
            case SpanKind::Whole: return g.trace_raw(ray, camera, out, st);
            case SpanKind::Leaves: {
                if (g.trace_raw(limited(ray, ray.t_min, t), camera, out, st)) return true;
                RayHit cap;
                if (cap_beyond(ray, t, cap) && !hidden(cap.instance)) { out = cap; return true; }
                return exempt_in(ray, t, ray.t_max, out);
            }
            case SpanKind::Enters: {
                if (exempt_in(ray, ray.t_min, t, out)) return true;
                RayHit nearest;
                const bool got = g.trace_raw(limited(ray, t, ray.t_max), camera, nearest, st);
                if (s.plane.cap && may_cap(s, ray.at(t)) && got && met_from_inside(ray, nearest) && !hidden(nearest.instance)) {
                    out = {nearest.instance, CAP_TRIANGLE, t};
                    return true;
                }
                if (got) out = nearest;
                return got;
            }
        }
        return false;
    }

    bool occluded(const Ray& ray) const {
        float t = 0.0f;
        RayHit unused;
        switch (span(s.plane, ray, t)) {
            case SpanKind::Removed: return exempt_in(ray, ray.t_min, ray.t_max, unused);
            case SpanKind::Whole: return g.occluded_raw(ray, camera, st);
            case SpanKind::Leaves:
                return g.occluded_raw(limited(ray, ray.t_min, t), camera, st) || cap_beyond(ray, t, unused) ||
                       exempt_in(ray, t, ray.t_max, unused);
            case SpanKind::Enters:
                return g.occluded_raw(limited(ray, t, ray.t_max), camera, st) || exempt_in(ray, ray.t_min, t, unused);
        }
        return false;
    }
};
}  // namespace

bool Geometry::trace(const Ray& ray, bool camera, RayHit& out, TraceStats* st) const {
    if (!has_section) return trace_raw(ray, camera, out, st);
    return SectionQueries{*this, section, camera, st}.trace(ray, out);
}

bool Geometry::occluded(const Ray& ray, bool camera, TraceStats* st) const {
    if (!has_section) return occluded_raw(ray, camera, st);
    return SectionQueries{*this, section, camera, st}.occluded(ray);
}

}  // namespace orc

// analyse_solid of a mesh given as arrays: 0 open, 1 outward, 2 inward; 0xffffffff when the mesh is
// invalid (an index out of range, a non-finite position).
extern "C" uint32_t orc_mesh_solid(const float* positions, uint32_t n_vertices, const uint32_t* indices, uint32_t n_indices) {
    using namespace orc;
    std::vector<Vec3> p(n_vertices), n(n_vertices, Vec3(0, 0, 0));
    for (uint32_t v = 0; v < n_vertices; ++v) p[v] = Vec3(positions[3 * v], positions[3 * v + 1], positions[3 * v + 2]);
    std::vector<uint32_t> idx(indices, indices + n_indices);
    Mesh m;
    if (*Mesh::make(m, p, n, idx, 0)) return 0xffffffffu;
    const Solid s = analyse_solid(m);
    return s == Solid::Open ? 0u : s == Solid::Outward ? 1u : 2u;
}
