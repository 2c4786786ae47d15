// Which meshes are closed solids, for the caps of a section view (engine/crates/rt-core/src/
// geometry/solid.rs analyse, with the vertex weld of geometry/edges.rs:221-330).
//
// A mesh is closed when, once the vertices that share a position (or lie within 1e-5 of the mesh's
// extent of one another on every axis, joined transitively) are welded, every edge of every
// triangle with an area is used by exactly two triangles that run along it in opposite
// directions. The sign of the volume it encloses, summed about the box's centre in blocks of 256
// terms, says whether the winding faces out (the back of a triangle is the inside) or in. A mesh
// whose volume is under 1e-9 of its extent cubed is open.
//
// The weld here finds the groups with a hash of cells twice the tolerance wide (a pair within the
// tolerance lies in neighbouring cells) and a union-find over the unique positions: only which
// vertices share a group matters to the test, not how the groups are numbered.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "rtg_scene.h"

namespace rtg {

namespace {
constexpr float WELD_TOLERANCE = 1.0e-5f;
constexpr size_t VOLUME_BLOCK = 256;
constexpr float MIN_VOLUME = 1.0e-9f;

uint32_t position_bits(float v) {  // +0 and -0 are one position
    if (v == 0.0f) return 0;
    uint32_t b;
    std::memcpy(&b, &v, 4);
    return b;
}

struct Key3 {
    int64_t x, y, z;
    bool operator==(const Key3& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct Key3Hash {
    size_t operator()(const Key3& k) const {
        uint64_t h = (uint64_t)k.x * 0x9E3779B97F4A7C15ull;
        h ^= (uint64_t)k.y * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
        h ^= (uint64_t)k.z * 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};

int64_t cell_of(float v, float lo, float size) {
    const float c = std::floor((v - lo) / size);
    if (!(c == c)) return 0;
    if (c >= 9.2e18f) return INT64_MAX;
    if (c <= -9.2e18f) return INT64_MIN;
    return (int64_t)c;
}

// The weld group of every vertex of `m`.
std::vector<uint32_t> weld(const HMesh& m) {
    const size_t n = m.positions.size();
    // Unique positions by their bits.
    std::unordered_map<Key3, uint32_t, Key3Hash> exact;
    std::vector<uint32_t> unique_of(n);
    std::vector<V3> unique;
    for (size_t v = 0; v < n; ++v) {
        const V3 p = m.positions[v];
        const Key3 k{position_bits(p.x), position_bits(p.y), position_bits(p.z)};
        auto it = exact.find(k);
        if (it == exact.end()) {
            it = exact.emplace(k, (uint32_t)unique.size()).first;
            unique.push_back(p);
        }
        unique_of[v] = it->second;
    }
    std::vector<uint32_t> parent(unique.size());
    for (size_t i = 0; i < parent.size(); ++i) parent[i] = (uint32_t)i;
    auto root = [&](uint32_t i) {
        while (parent[i] != i) {
            parent[i] = parent[parent[i]];
            i = parent[i];
        }
        return i;
    };
    const V3 lo = m.bmin, hi = m.bmax;
    const float extent = m.empty_bounds ? 0.0f : rmax(rmax(hi.x - lo.x, hi.y - lo.y), hi.z - lo.z);
    const float tolerance = extent * WELD_TOLERANCE;
    if (tolerance > 0.0f && std::isfinite(tolerance)) {
        const float size = 2.0f * tolerance;
        std::unordered_map<Key3, std::vector<uint32_t>, Key3Hash> cells;
        std::vector<Key3> cell(unique.size());
        for (size_t i = 0; i < unique.size(); ++i) {
            cell[i] = Key3{cell_of(unique[i].x, lo.x, size), cell_of(unique[i].y, lo.y, size), cell_of(unique[i].z, lo.z, size)};
            cells[cell[i]].push_back((uint32_t)i);
        }
        for (size_t i = 0; i < unique.size(); ++i)
            for (int dx = -1; dx <= 1; ++dx)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dz = -1; dz <= 1; ++dz) {
                        auto it = cells.find(Key3{cell[i].x + dx, cell[i].y + dy, cell[i].z + dz});
                        if (it == cells.end()) continue;
                        for (uint32_t j : it->second) {
                            if (j <= i) continue;
                            const V3 a = unique[i], b = unique[j];
                            if (absf(a.x - b.x) <= tolerance && absf(a.y - b.y) <= tolerance && absf(a.z - b.z) <= tolerance) {
                                const uint32_t ra = root((uint32_t)i), rb = root(j);
                                parent[std::max(ra, rb)] = std::min(ra, rb);
                            }
                        }
                    }
    }
    std::vector<uint32_t> ids(n);
    for (size_t v = 0; v < n; ++v) ids[v] = root(unique_of[v]);
    return ids;
}
}  // namespace

uint32_t solid_of(const HMesh& m) {
    const size_t triangles = m.triangles();
    if (triangles == 0 || m.empty_bounds) return 0;
    const std::vector<uint32_t> w = weld(m);
    const V3 centre = (m.bmin + m.bmax) * 0.5f;
    // Each half-edge as (smaller group, larger group) with its direction in bit 0 of a sort key.
    std::vector<uint64_t> halves;
    halves.reserve(triangles * 3);
    float blocks = 0.0f, block = 0.0f;
    size_t in_block = 0;
    for (size_t t = 0; t < triangles; ++t) {
        const uint32_t* ix = &m.indices[3 * t];
        const uint32_t g[3] = {w[ix[0]], w[ix[1]], w[ix[2]]};
        if (g[0] == g[1] || g[1] == g[2] || g[2] == g[0]) continue;
        const V3 p0 = m.positions[ix[0]], p1 = m.positions[ix[1]], p2 = m.positions[ix[2]];
        if (len2(cross(p1 - p0, p2 - p0)) <= 0.0f) continue;
        for (int k = 0; k < 3; ++k) {
            const uint32_t from = g[k], to = g[(k + 1) % 3];
            const uint64_t a = std::min(from, to), b = std::max(from, to);
            halves.push_back((a << 33) | (b << 1) | (uint64_t)(from < to));
        }
        block += dot(p0 - centre, cross(p1 - centre, p2 - centre));
        if (++in_block == VOLUME_BLOCK) {
            blocks += block;
            block = 0.0f;
            in_block = 0;
        }
    }
    if (halves.empty() || halves.size() % 2) return 0;
    std::sort(halves.begin(), halves.end());
    // Sorted, an edge used once each way is the pair (its key with bit 0 clear, then set).
    for (size_t i = 0; i < halves.size(); i += 2)
        if ((halves[i] & 1u) || halves[i + 1] != (halves[i] | 1u)) return 0;
    const V3 d = m.bmax - m.bmin;
    const float extent = rmax(rmax(d.x, d.y), d.z);
    const float volume = (blocks + block) / 6.0f;
    if (!std::isfinite(volume) || absf(volume) <= extent * extent * extent * MIN_VOLUME) return 0;
    return volume > 0.0f ? 1u : 2u;
}

}  // namespace rtg
