// ORACLE (test infrastructure only). See orc_geometry.h.
#include "orc_geometry.h"

#include <algorithm>

namespace orc {

// ---- transform.rs:120-185 ---------------------------------------------------------------------
float Transform::determinant() const {
    return r[0][0] * (r[1][1] * r[2][2] - r[1][2] * r[2][1]) - r[0][1] * (r[1][0] * r[2][2] - r[1][2] * r[2][0]) +
           r[0][2] * (r[1][0] * r[2][1] - r[1][1] * r[2][0]);
}
bool Transform::inverse(Transform& out) const {
    if (!is_finite()) return false;
    float det = determinant();
    if (det == 0.0f || !finite(det)) return false;
    float inv_det = 1.0f / det;
    float c[3][3] = {
        {r[1][1] * r[2][2] - r[1][2] * r[2][1], r[0][2] * r[2][1] - r[0][1] * r[2][2], r[0][1] * r[1][2] - r[0][2] * r[1][1]},
        {r[1][2] * r[2][0] - r[1][0] * r[2][2], r[0][0] * r[2][2] - r[0][2] * r[2][0], r[0][2] * r[1][0] - r[0][0] * r[1][2]},
        {r[1][0] * r[2][1] - r[1][1] * r[2][0], r[0][1] * r[2][0] - r[0][0] * r[2][1], r[0][0] * r[1][1] - r[0][1] * r[1][0]},
    };
    Transform t;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t.r[i][j] = c[i][j] * inv_det;
    float tr[3] = {r[0][3], r[1][3], r[2][3]};
    for (int i = 0; i < 3; ++i) t.r[i][3] = -(t.r[i][0] * tr[0] + t.r[i][1] * tr[1] + t.r[i][2] * tr[2]);
    if (!t.is_finite()) return false;
    out = t;
    return true;
}
Aabb Transform::aabb(const Aabb& b) const {
    if (b.is_empty()) return Aabb();
    Aabb out;
    for (int corner = 0; corner < 8; ++corner) {
        Vec3 p((corner & 1) == 0 ? b.min.x : b.max.x, (corner & 2) == 0 ? b.min.y : b.max.y,
               (corner & 4) == 0 ? b.min.z : b.max.z);
        out = out.extend(point(p));
    }
    return out;
}

// ---- bvh.rs:246-505 --------------------------------------------------------------------------
namespace {
constexpr int BINS = 16;
constexpr uint32_t SAH_DEPTH_LIMIT = 32;

inline size_t bin_of(float c, float lo, float scale) {
    uint64_t b = f2usize((c - lo) * scale);
    return b < (uint64_t)(BINS - 1) ? (size_t)b : (size_t)(BINS - 1);
}

struct Builder {
    const std::vector<Aabb>& bounds;
    const std::vector<Vec3>& centroids;
    int leaf_target, leaf_max;
    std::vector<uint32_t> order;
    std::vector<BinaryNode> nodes;

    void range_bounds(size_t b, size_t e, Aabb& bb, Aabb& cb) const {
        bb = Aabb();
        cb = Aabb();
        for (size_t i = b; i < e; ++i) {
            uint32_t p = order[i];
            bb = bb.uni(bounds[p]);
            cb = cb.extend(centroids[p]);
        }
    }
    uint32_t build(size_t begin, size_t end, uint32_t depth) {
        Aabb bb, cb;
        range_bounds(begin, end, bb, cb);
        uint32_t index = (uint32_t)nodes.size();
        BinaryNode n;
        n.bounds = bb;
        n.first = (uint32_t)begin;
        n.count = (uint32_t)(end - begin);
        nodes.push_back(n);
        if (end - begin <= (size_t)leaf_target) return index;
        size_t mid;
        if (!split(begin, end, bb, cb, depth, mid)) return index;
        uint32_t left = build(begin, mid, depth + 1);
        uint32_t right = build(mid, end, depth + 1);
        nodes[index].left = left;
        nodes[index].right = right;
        nodes[index].count = 0;
        return index;
    }
    bool best_plane(size_t begin, size_t end, const Aabb& cb, int& axis_out, int& plane_out, float& cost_out) const {
        uint32_t counts[3][BINS] = {};
        Aabb boxes[3][BINS];
        float scales[3] = {0, 0, 0};
        bool usable[3] = {false, false, false};
        for (int axis = 0; axis < 3; ++axis) {
            float extent = cb.max[axis] - cb.min[axis];
            if (extent > 0.0f && finite(extent)) {
                usable[axis] = true;
                scales[axis] = (float)BINS / extent;
            }
        }
        if (!usable[0] && !usable[1] && !usable[2]) return false;
        for (size_t i = begin; i < end; ++i) {
            uint32_t p = order[i];
            Vec3 c = centroids[p];
            const Aabb& b = bounds[p];
            for (int axis = 0; axis < 3; ++axis) {
                if (usable[axis]) {
                    size_t bin = bin_of(c[axis], cb.min[axis], scales[axis]);
                    counts[axis][bin] += 1;
                    boxes[axis][bin] = boxes[axis][bin].uni(b);
                }
            }
        }
        bool have = false;
        for (int axis = 0; axis < 3; ++axis) {
            if (!usable[axis]) continue;
            float right_area[BINS] = {};
            uint32_t right_count[BINS] = {};
            Aabb acc;
            uint32_t n = 0;
            for (int plane = BINS - 2; plane >= 0; --plane) {
                acc = acc.uni(boxes[axis][plane + 1]);
                n += counts[axis][plane + 1];
                right_area[plane] = acc.surface_area();
                right_count[plane] = n;
            }
            acc = Aabb();
            n = 0;
            for (int plane = 0; plane < BINS - 1; ++plane) {
                acc = acc.uni(boxes[axis][plane]);
                n += counts[axis][plane];
                if (n == 0 || right_count[plane] == 0) continue;
                float cost = acc.surface_area() * (float)n + right_area[plane] * (float)right_count[plane];
                if (!have || cost < cost_out) {
                    have = true;
                    axis_out = axis;
                    plane_out = plane;
                    cost_out = cost;
                }
            }
        }
        return have;
    }
    bool split(size_t begin, size_t end, const Aabb& bb, const Aabb& cb, uint32_t depth, size_t& mid) {
        size_t count = end - begin;
        size_t median = begin + count / 2;
        if (depth >= SAH_DEPTH_LIMIT) { mid = median; return true; }
        int axis = 0, plane = 0;
        float cost = 0;
        if (!best_plane(begin, end, cb, axis, plane, cost)) {
            if (count > (size_t)leaf_max) { mid = median; return true; }
            return false;
        }
        float area = bb.surface_area();
        float split_cost = (area > 0.0f && finite(area)) ? 1.0f + 1.0f * cost / area : 1.0f;
        if (count <= (size_t)leaf_max && 1.0f * (float)count <= split_cost) return false;
        float lo = cb.min[axis];
        float scale = (float)BINS / (cb.max[axis] - lo);
        size_t i = begin, j = end;
        while (i < j) {
            float c = centroids[order[i]][axis];
            if (bin_of(c, lo, scale) <= (size_t)plane) {
                ++i;
            } else {
                --j;
                std::swap(order[i], order[j]);
            }
        }
        mid = (i == begin || i == end) ? median : i;
        return true;
    }
};

template <class EmitLeaf>
struct Collapser {
    const std::vector<BinaryNode>& bn;
    const std::vector<uint32_t>& order;
    std::vector<WideNode8> nodes;
    EmitLeaf& emit;

    static WideNode8 empty() {
        WideNode8 w;
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 8; ++c) { w.bounds[a][0][c] = F_INF; w.bounds[a][1][c] = -F_INF; }
        for (int c = 0; c < 8; ++c) w.child[c] = BVH_EMPTY;
        return w;
    }
    uint32_t reference(uint32_t b, uint32_t depth) {
        BinaryNode node = bn[b];
        if (node.count > 0) {
            std::vector<uint32_t> prims(order.begin() + node.first, order.begin() + node.first + node.count);
            return emit(prims);
        }
        uint32_t index = (uint32_t)nodes.size();
        nodes.push_back(empty());
        uint32_t kids[8] = {};
        kids[0] = node.left;
        kids[1] = node.right;
        int len = 2;
        while (len < 8) {
            int widest = -1;
            float warea = 0;
            for (int slot = 0; slot < len; ++slot) {
                const BinaryNode& kid = bn[kids[slot]];
                if (kid.count == 0) {
                    float area = kid.bounds.surface_area();
                    if (widest < 0 || area > warea) { widest = slot; warea = area; }
                }
            }
            if (widest < 0) break;
            BinaryNode opened = bn[kids[widest]];
            for (int s = len - 1; s >= widest + 1; --s) kids[s + 1] = kids[s];
            kids[widest] = opened.left;
            kids[widest + 1] = opened.right;
            len += 1;
        }
        WideNode8 wide = empty();
        for (int slot = 0; slot < len; ++slot) {
            const Aabb& bb = bn[kids[slot]].bounds;
            for (int axis = 0; axis < 3; ++axis) {
                wide.bounds[axis][0][slot] = bb.min[axis];
                wide.bounds[axis][1][slot] = bb.max[axis];
            }
            wide.child[slot] = reference(kids[slot], depth + 1);
        }
        nodes[index] = wide;
        return index;
    }
};
}  // namespace

template <class EmitLeaf>
Bvh build_bvh(const std::vector<Aabb>& boxes, const std::vector<Vec3>& centroids, int leaf_target, int leaf_max,
              EmitLeaf emit) {
    Bvh out;
    if (boxes.empty()) return out;
    Builder b{boxes, centroids, leaf_target, leaf_max, {}, {}};
    b.order.resize(boxes.size());
    for (size_t i = 0; i < boxes.size(); ++i) b.order[i] = (uint32_t)i;
    b.build(0, boxes.size(), 0);
    Collapser<EmitLeaf> c{b.nodes, b.order, {}, emit};
    out.root = c.reference(0, 0);
    out.nodes = std::move(c.nodes);
    return out;
}

// ---- triangle.rs:60-160 ----------------------------------------------------------------------
PreparedRay PreparedRay::make(const Ray& ray) {
    PreparedRay r;
    float d[3] = {ray.dir.x, ray.dir.y, ray.dir.z};
    r.inv[0] = 1.0f / d[0];
    r.inv[1] = 1.0f / d[1];
    r.inv[2] = 1.0f / d[2];
    float a[3] = {std::fabs(d[0]), std::fabs(d[1]), std::fabs(d[2])};
    int kz = (a[0] >= a[1] && a[0] >= a[2]) ? 0 : (a[1] >= a[2] ? 1 : 2);
    int kx = (kz + 1) % 3, ky = (kz + 2) % 3;
    if (d[kz] < 0.0f) std::swap(kx, ky);
    float sz = r.inv[kz];
    r.org[0] = ray.origin.x;
    r.org[1] = ray.origin.y;
    r.org[2] = ray.origin.z;
    for (int i = 0; i < 3; ++i) r.negative[i] = std::signbit(r.inv[i]);
    r.k[0] = kx; r.k[1] = ky; r.k[2] = kz;
    r.shear[0] = d[kx] * sz;
    r.shear[1] = d[ky] * sz;
    r.shear[2] = sz;
    r.t_min = ray.t_min;
    r.t_max = rmin(ray.t_max, F_MAX);
    return r;
}

bool watertight(const PreparedRay& r, Vec3 v0, Vec3 v1, Vec3 v2, float t_max, Cull cull, EdgeHit& out) {
    int kx = r.k[0], ky = r.k[1], kz = r.k[2];
    float sx = r.shear[0], sy = r.shear[1], sz = r.shear[2];
    float ox = r.org[kx], oy = r.org[ky], oz = r.org[kz];
    float a_x = v0[kx] - ox, a_y = v0[ky] - oy, a_z = v0[kz] - oz;
    float b_x = v1[kx] - ox, b_y = v1[ky] - oy, b_z = v1[kz] - oz;
    float c_x = v2[kx] - ox, c_y = v2[ky] - oy, c_z = v2[kz] - oz;
    float ax = a_x - sx * a_z, ay = a_y - sy * a_z;
    float bx = b_x - sx * b_z, by = b_y - sy * b_z;
    float cx = c_x - sx * c_z, cy = c_y - sy * c_z;
    float u = cx * by - cy * bx;
    float v = ax * cy - ay * cx;
    float w = bx * ay - by * ax;
    bool negative = u < 0.0f || v < 0.0f || w < 0.0f;
    bool positive = u > 0.0f || v > 0.0f || w > 0.0f;
    bool rejected = cull == Cull::None ? (negative && positive) : negative;
    float det = u + v + w;
    if (rejected || det == 0.0f) return false;
    float az = sz * a_z, bz = sz * b_z, cz = sz * c_z;
    float t = (u * az + v * bz + w * cz) / det;
    if (t >= r.t_min && t <= t_max) {
        out = {t, u, v, w, det};
        return true;
    }
    return false;
}

// ---- mesh.rs:121-248 -------------------------------------------------------------------------
const char* Mesh::make(Mesh& m, const std::vector<Vec3>& positions, const std::vector<Vec3>& normals,
                       const std::vector<uint32_t>& indices, uint32_t material_id) {
    if (indices.size() % 3 != 0) return "index_count is not a multiple of 3";
    if (indices.size() / 3 > (size_t)((1u << 28) - 2) || positions.size() >= 0xffffffffull)
        return "too many triangles or vertices";
    for (uint32_t i : indices)
        if (i >= positions.size()) return "vertex index out of range";
    if (!normals.empty() && normals.size() != positions.size()) return "normals are not one per vertex";
    for (const Vec3& p : positions)
        if (!vfinite(p)) return "non-finite vertex position";
    for (const Vec3& n : normals)
        if (!vfinite(n)) return "non-finite vertex normal";
    m.positions = positions;
    bool any = false;
    for (const Vec3& n : normals)
        if (!(n == Vec3(0, 0, 0))) any = true;
    m.normals = any ? normals : std::vector<Vec3>();
    m.indices = indices;
    m.material_id = material_id;
    Aabb b;
    for (const Vec3& p : positions) b = b.extend(p);
    m.bounds = b;
    // normals_oppose_winding (mesh.rs:181)
    m.inside_out = false;
    if (!m.normals.empty()) {
        float agreement = 0.0f;
        for (size_t t = 0; t < m.triangle_count(); ++t) {
            Vec3 a, bb, c;
            m.corners((uint32_t)t, a, bb, c);
            Vec3 winding = cross(bb - a, c - a);
            Vec3 n(0, 0, 0);
            for (int k = 0; k < 3; ++k) n = n + m.normals[m.indices[3 * t + k]];
            agreement += dot(normalize(winding), n);
        }
        m.inside_out = agreement < 0.0f;
    }
    // build_bvh (mesh.rs:209)
    size_t count = m.triangle_count();
    std::vector<Aabb> boxes(count);
    std::vector<Vec3> centroids(count);
    for (size_t i = 0; i < count; ++i) {
        Vec3 a, bb, c;
        m.corners((uint32_t)i, a, bb, c);
        boxes[i] = Aabb().extend(a).extend(bb).extend(c);
        centroids[i] = boxes[i].centroid();
    }
    m.packets.clear();
    auto emit = [&m](const std::vector<uint32_t>& prims) -> uint32_t {
        uint32_t first = (uint32_t)m.packets.size();
        for (size_t c0 = 0; c0 < prims.size(); c0 += 4) {
            size_t n = std::min<size_t>(4, prims.size() - c0);
            TriPacket p{};
            for (int lane = 0; lane < 4; ++lane) {
                uint32_t id = prims[c0 + (lane < (int)n ? lane : n - 1)];
                p.id[lane] = id;
                Vec3 cs[3];
                m.corners(id, cs[0], cs[1], cs[2]);
                for (int corner = 0; corner < 3; ++corner) {
                    p.v[corner][0][lane] = cs[corner].x;
                    p.v[corner][1][lane] = cs[corner].y;
                    p.v[corner][2][lane] = cs[corner].z;
                }
            }
            m.packets.push_back(p);
        }
        return leaf_ref(first, (uint32_t)m.packets.size() - first);
    };
    m.bvh = build_bvh(boxes, centroids, 4, 8, emit);
    return "";
}

// ---- geometry/mod.rs:294-384 -----------------------------------------------------------------
Aabb instance_bounds(const Mesh& mesh, const Transform& t) {
    if (t.is_identity()) return mesh.bounds;
    Aabb b = t.aabb(mesh.bounds);
    float scale = max_component(vmax(vabs(b.min), vabs(b.max)));
    Vec3 pad(scale * 1.0e-5f, scale * 1.0e-5f, scale * 1.0e-5f);
    return Aabb(b.min - pad, b.max + pad);
}

const char* Geometry::make(Geometry& g, std::vector<Mesh> meshes, std::vector<Instance> instances) {
    g.meshes = std::move(meshes);
    g.instances = std::move(instances);
    g.prepared.clear();
    std::vector<Aabb> boxes;
    std::vector<Vec3> centroids;
    std::vector<uint32_t> active;
    g.bounds = Aabb();
    for (size_t i = 0; i < g.instances.size(); ++i) {
        const Instance& inst = g.instances[i];
        if (inst.mesh >= g.meshes.size()) return "instance refers to a mesh that does not exist";
        const Mesh& mesh = g.meshes[inst.mesh];
        Transform inv;
        bool has_inv = inst.transform.inverse(inv);
        bool live = mesh.triangle_count() > 0 && has_inv;
        PreparedInstance p;
        p.to_local = has_inv ? inv : Transform();
        p.identity = inst.transform.is_identity();
        p.cull = (inst.flags & INSTANCE_ONE_SIDED) ? Cull::Back : Cull::None;
        p.active = live;
        p.camera_hidden = (inst.flags & INSTANCE_NO_CAMERA) != 0;
        g.prepared.push_back(p);
        if (live) {
            Aabb b = instance_bounds(mesh, inst.transform);
            g.bounds = g.bounds.uni(b);
            boxes.push_back(b);
            centroids.push_back(b.centroid());
            active.push_back((uint32_t)i);
        }
    }
    g.tlas_instances.clear();
    auto emit = [&g, &active](const std::vector<uint32_t>& prims) -> uint32_t {
        uint32_t first = (uint32_t)g.tlas_instances.size();
        for (uint32_t p : prims) g.tlas_instances.push_back(active[p]);
        return leaf_ref(first, (uint32_t)prims.size());
    };
    g.tlas = build_bvh(boxes, centroids, 1, 1, emit);
    return "";
}

// ---- traverse.rs -----------------------------------------------------------------------------
namespace {
const float ROBUST_SCALE = 1.0f + 4.0f * F_EPS;
inline float smin(float a, float b) { return a < b ? a : b; }  // simd Vector::min
inline float smax(float a, float b) { return a > b ? a : b; }  // simd Vector::max
inline uint64_t entry(float t, uint32_t ref) { return ((uint64_t)fbits(t) << 32) | (uint64_t)ref; }

struct Stack {
    std::vector<uint64_t> v;
    Stack() { v.reserve(128); }
};

struct Best {
    float t;
    uint32_t instance = 0xffffffffu, triangle = 0xffffffffu;
    void offer(float tt, uint32_t inst, uint32_t tri) {
        if (tt < t || (tt == t && (inst < instance || (inst == instance && tri < triangle)))) {
            t = tt; instance = inst; triangle = tri;
        }
    }
};

// node_test (traverse.rs:184): bit mask of children hit and their entry distances.
inline uint32_t node_test(const WideNode8& node, const PreparedRay& r, float t_max, float near_out[8]) {
    int nx = r.negative[0] ? 1 : 0, ny = r.negative[1] ? 1 : 0, nz = r.negative[2] ? 1 : 0;
    uint32_t bits = 0;
    for (int c = 0; c < 8; ++c) {
        float lx0 = node.bounds[0][nx][c], ly0 = node.bounds[1][ny][c], lz0 = node.bounds[2][nz][c];
        float lx1 = node.bounds[0][1 - nx][c], ly1 = node.bounds[1][1 - ny][c], lz1 = node.bounds[2][1 - nz][c];
        float tx0 = (lx0 - r.org[0]) * r.inv[0];
        float ty0 = (ly0 - r.org[1]) * r.inv[1];
        float tz0 = (lz0 - r.org[2]) * r.inv[2];
        float tx1 = (lx1 - r.org[0]) * r.inv[0];
        float ty1 = (ly1 - r.org[1]) * r.inv[1];
        float tz1 = (lz1 - r.org[2]) * r.inv[2];
        float nr = smax(tz0, smax(ty0, smax(tx0, r.t_min)));
        float fr = smin(tz1, smin(ty1, smin(tx1, t_max))) * ROBUST_SCALE;
        near_out[c] = nr;
        if (nr <= fr) bits |= 1u << c;
    }
    return bits;
}

template <class Leaves>
bool walk(const Bvh& bvh, const PreparedRay& r, bool ordered, Leaves& leaves, Stack& stack, TraceStats* st) {
    size_t base = stack.v.size();
    uint32_t current = bvh.root;
    for (;;) {
        if ((current & BVH_LEAF) == 0) {
            if (current < bvh.nodes.size()) {
                const WideNode8& node = bvh.nodes[current];
                if (st) st->nodes += 1;
                float nr[8];
                uint32_t bits = node_test(node, r, leaves.t_max(), nr);
                if (bits != 0) {
                    if (ordered) {
                        if ((bits & (bits - 1)) == 0) {
                            current = node.child[__builtin_ctz(bits)];
                        } else {
                            uint64_t keys[8];
                            int count = 0;
                            while (bits) {
                                int slot = __builtin_ctz(bits);
                                bits &= bits - 1;
                                uint64_t key = entry(nr[slot], node.child[slot]);
                                int j = count;
                                while (j > 0 && keys[j - 1] < key) { keys[j] = keys[j - 1]; --j; }
                                keys[j] = key;
                                ++count;
                            }
                            for (int k = 0; k < count - 1; ++k) stack.v.push_back(keys[k]);
                            current = (uint32_t)keys[count - 1];
                        }
                    } else {
                        int first = __builtin_ctz(bits);
                        bits &= bits - 1;
                        while (bits) {
                            int slot = __builtin_ctz(bits);
                            bits &= bits - 1;
                            stack.v.push_back(entry(nr[slot], node.child[slot]));
                        }
                        current = node.child[first];
                    }
                    continue;
                }
            }
        } else if (current != BVH_EMPTY && leaves.leaf(current, stack)) {
            stack.v.resize(base);
            return true;
        }
        for (;;) {
            if (stack.v.size() <= base) return false;
            uint64_t e = stack.v.back();
            stack.v.pop_back();
            float t = bitsf((uint32_t)(e >> 32));
            if (t <= leaves.t_max() * ROBUST_SCALE) {
                current = (uint32_t)e;
                break;
            }
        }
    }
}

// packet_hits (triangle.rs:203): the scalar test on every lane, the same operations.
inline uint32_t packet_hits(const PreparedRay& r, const TriPacket& p, float t_max, Cull cull, float t[4]) {
    uint32_t bits = 0;
    for (int lane = 0; lane < 4; ++lane) {
        Vec3 a(p.v[0][0][lane], p.v[0][1][lane], p.v[0][2][lane]);
        Vec3 b(p.v[1][0][lane], p.v[1][1][lane], p.v[1][2][lane]);
        Vec3 c(p.v[2][0][lane], p.v[2][1][lane], p.v[2][2][lane]);
        EdgeHit h;
        if (watertight(r, a, b, c, t_max, cull, h)) {
            bits |= 1u << lane;
            t[lane] = h.t;
        }
    }
    return bits;
}

struct NearestTriangles {
    const Mesh* mesh;
    PreparedRay r;
    Cull cull;
    uint32_t instance;
    Best* best;
    TraceStats* st;
    float t_max() const { return best->t; }
    bool leaf(uint32_t ref, Stack&) {
        uint32_t first, count;
        leaf_range(ref, first, count);
        if ((size_t)first + count > mesh->packets.size()) return false;
        for (uint32_t i = first; i < first + count; ++i) {
            const TriPacket& p = mesh->packets[i];
            if (st) st->packets += 1;
            float t[4];
            uint32_t bits = packet_hits(r, p, best->t, cull, t);
            while (bits) {
                int lane = __builtin_ctz(bits);
                bits &= bits - 1;
                best->offer(t[lane], instance, p.id[lane]);
            }
        }
        return false;
    }
};
struct AnyTriangle {
    const Mesh* mesh;
    PreparedRay r;
    Cull cull;
    float tmax;
    TraceStats* st;
    float t_max() const { return tmax; }
    bool leaf(uint32_t ref, Stack&) {
        uint32_t first, count;
        leaf_range(ref, first, count);
        if ((size_t)first + count > mesh->packets.size()) return false;
        for (uint32_t i = first; i < first + count; ++i) {
            if (st) st->packets += 1;
            float t[4];
            if (packet_hits(r, mesh->packets[i], tmax, cull, t) != 0) return true;
        }
        return false;
    }
};
struct NearestInstances {
    const Geometry* g;
    const Ray* ray;
    PreparedRay world;
    Best best;
    bool camera;
    TraceStats* st;
    float t_max() const { return best.t; }
    bool leaf(uint32_t ref, Stack& stack) {
        uint32_t first, count;
        leaf_range(ref, first, count);
        for (uint32_t slot = first; slot < first + count; ++slot) {
            if (slot >= g->tlas_instances.size()) continue;
            uint32_t inst = g->tlas_instances[slot];
            const PreparedInstance& p = g->prepared[inst];
            if (!p.active) continue;
            if (camera && p.camera_hidden) continue;
            const Mesh& mesh = g->meshes[g->instances[inst].mesh];
            PreparedRay local = p.identity ? world : PreparedRay::make(p.to_local.ray(*ray));
            NearestTriangles leaves{&mesh, local, p.cull, inst, &best, st};
            walk(mesh.bvh, local, true, leaves, stack, st);
        }
        return false;
    }
};
struct AnyInstance {
    const Geometry* g;
    const Ray* ray;
    PreparedRay world;
    float tmax;
    bool camera;
    TraceStats* st;
    float t_max() const { return tmax; }
    bool leaf(uint32_t ref, Stack& stack) {
        uint32_t first, count;
        leaf_range(ref, first, count);
        for (uint32_t slot = first; slot < first + count; ++slot) {
            if (slot >= g->tlas_instances.size()) continue;
            uint32_t inst = g->tlas_instances[slot];
            const PreparedInstance& p = g->prepared[inst];
            if (!p.active) continue;
            if (camera && p.camera_hidden) continue;
            const Mesh& mesh = g->meshes[g->instances[inst].mesh];
            PreparedRay local = p.identity ? world : PreparedRay::make(p.to_local.ray(*ray));
            AnyTriangle leaves{&mesh, local, p.cull, local.t_max, st};
            if (walk(mesh.bvh, local, false, leaves, stack, st)) return true;
        }
        return false;
    }
};

inline bool usable(const Ray& r) { return vfinite(r.origin) && vfinite(r.dir) && !(r.dir == Vec3(0, 0, 0)); }
}  // namespace

bool Geometry::trace_raw(const Ray& ray, bool camera, RayHit& out, TraceStats* st) const {
    if (!usable(ray)) return false;
    PreparedRay r = PreparedRay::make(ray);
    if (!r.has_interval()) return false;
    NearestInstances leaves{this, &ray, r, Best{r.t_max}, camera, st};
    Stack stack;
    walk(tlas, r, true, leaves, stack, st);
    if (leaves.best.instance == 0xffffffffu) return false;
    out = {leaves.best.instance, leaves.best.triangle, leaves.best.t};
    return true;
}

bool Geometry::occluded_raw(const Ray& ray, bool camera, TraceStats* st) const {
    if (!usable(ray)) return false;
    PreparedRay r = PreparedRay::make(ray);
    if (!r.has_interval()) return false;
    AnyInstance leaves{this, &ray, r, r.t_max, camera, st};
    Stack stack;
    return walk(tlas, r, false, leaves, stack, st);
}

// Every triangle of every instance (traverse.rs:883): the brute-force reference.
bool Geometry::trace_brute(const Ray& ray, bool camera, RayHit& out) const {
    if (!usable(ray)) return false;
    PreparedRay world = PreparedRay::make(ray);
    if (!world.has_interval()) return false;
    Best best{world.t_max};
    for (size_t i = 0; i < instances.size(); ++i) {
        const PreparedInstance& p = prepared[i];
        if (!p.active || (camera && p.camera_hidden)) continue;
        const Mesh& mesh = meshes[instances[i].mesh];
        PreparedRay local = p.identity ? world : PreparedRay::make(p.to_local.ray(ray));
        for (uint32_t t = 0; t < mesh.triangle_count(); ++t) {
            Vec3 a, b, c;
            mesh.corners(t, a, b, c);
            EdgeHit h;
            if (watertight(local, a, b, c, best.t, p.cull, h)) best.offer(h.t, (uint32_t)i, t);
        }
    }
    if (best.instance == 0xffffffffu) return false;
    out = {best.instance, best.triangle, best.t};
    return true;
}

// hit_details (geometry/mod.rs:731)
bool Geometry::hit_details(const Ray& ray, const RayHit& hit, Hit& out) const {
    if (hit.instance >= instances.size()) return false;
    if (hit.triangle == CAP_TRIANGLE) return cap_details(ray, hit, out);
    const PreparedInstance& p = prepared[hit.instance];
    if (!p.active) return false;
    const Instance& inst = instances[hit.instance];
    const Mesh& mesh = meshes[inst.mesh];
    if (hit.triangle >= mesh.triangle_count()) return false;
    Vec3 p0, p1, p2;
    mesh.corners(hit.triangle, p0, p1, p2);
    Ray local = p.identity ? ray : p.to_local.ray(ray);
    PreparedRay r = PreparedRay::make(local);
    float bary[3];
    EdgeHit h;
    if (watertight(r, p0, p1, p2, F_MAX, Cull::None, h)) {
        bary[0] = h.u / h.det;
        bary[1] = h.v / h.det;
        bary[2] = h.w / h.det;
    } else {
        bary[0] = bary[1] = bary[2] = 1.0f / 3.0f;
    }
    Vec3 point_local = p0 * bary[0] + p1 * bary[1] + p2 * bary[2];
    auto to_normal = [&](Vec3 n) { return p.identity ? n : p.to_local.transpose_vector(n); };
    Vec3 winding = normalize(to_normal(cross(p1 - p0, p2 - p0)));
    Vec3 incoming = normalize(ray.dir);
    Vec3 geometric = length_squared(winding) > 0.0f ? winding : -incoming;
    bool front_face = dot(winding, ray.dir) < 0.0f;
    Vec3 smooth(0, 0, 0);
    if (mesh.has_normals()) {
        Vec3 n0 = mesh.normals[mesh.indices[3 * hit.triangle]];
        Vec3 n1 = mesh.normals[mesh.indices[3 * hit.triangle + 1]];
        Vec3 n2 = mesh.normals[mesh.indices[3 * hit.triangle + 2]];
        smooth = to_normal(n0 * bary[0] + n1 * bary[1] + n2 * bary[2]);
    }
    Vec3 normal = length_squared(smooth) > 1.0e-12f ? normalize(smooth) : geometric;
    auto face = [&](Vec3 n) { return dot(n, ray.dir) > 0.0f ? -n : n; };
    out.instance = hit.instance;
    out.triangle = hit.triangle;
    out.t = hit.t;
    out.point = p.identity ? point_local : inst.transform.point(point_local);
    out.normal = face(normal);
    out.geometric_normal = face(geometric);
    out.bary[0] = bary[0]; out.bary[1] = bary[1]; out.bary[2] = bary[2];
    out.front_face = front_face;
    out.outside = front_face != mesh.inside_out;
    return true;
}

// terminator_point (geometry/mod.rs:682, Hanika 2021)
Vec3 Geometry::terminator_point(const Hit& hit) const {
    if (hit.instance >= instances.size()) return hit.point;
    const PreparedInstance& p = prepared[hit.instance];
    if (!p.active) return hit.point;
    const Mesh& mesh = meshes[instances[hit.instance].mesh];
    if (hit.triangle >= mesh.triangle_count() || !mesh.has_normals()) return hit.point;
    Vec3 c[3], n[3];
    for (int k = 0; k < 3; ++k) {
        c[k] = mesh.positions[mesh.indices[3 * hit.triangle + k]];
        n[k] = mesh.normals[mesh.indices[3 * hit.triangle + k]];
    }
    float b0 = hit.bary[0], b1 = hit.bary[1], b2 = hit.bary[2];
    Vec3 pt = c[0] * b0 + c[1] * b1 + c[2] * b2;
    Vec3 interpolated = n[0] * b0 + n[1] * b1 + n[2] * b2;
    Vec3 world_normal = p.identity ? interpolated : p.to_local.transpose_vector(interpolated);
    float side = dot(world_normal, hit.geometric_normal) < 0.0f ? -1.0f : 1.0f;
    Vec3 lifted = pt;
    float w[3] = {b0, b1, b2};
    for (int k = 0; k < 3; ++k) {
        Vec3 nn = normalize(n[k]) * side;
        float below = dot(pt - c[k], nn);
        if (below < 0.0f) lifted = lifted - nn * (below * w[k]);
    }
    if (!vfinite(lifted)) return hit.point;
    return p.identity ? lifted : instances[hit.instance].transform.point(lifted);
}

}  // namespace orc
