// Ray queries on the device: the watertight triangle test, the quantised 8-wide slab test and
// the two-level closest-hit / any-hit traversal (engine/crates/rt-core/src/geometry/
// triangle.rs:60-160, traverse.rs:47-802), and the hit details of geometry/mod.rs:682-808.
//
// The answer of a nearest-hit query is the smallest (t, instance, triangle) in lexicographic
// order over the triangles the ray meets in [t_min, t_max] whose enclosing boxes pass the slab
// test. The boxes are conservative except at t_min: a ray that starts within about 1e-3 of a
// large axis-aligned quad can see its flat box end just before t_min while the triangle test
// alone would accept the hit, and the reference drops that hit. The slab test below uses the
// reference's operations in its order on boxes that decode to the same flat planes, so it drops
// the same hits; a padded or FMA-contracted test would not.
#pragma once
#include "rtg_dev.h"

namespace rtg {

constexpr int STACK_CAP = 96;
constexpr uint32_t STACK_RETURN = 0xfffffffeu;
#define RTG_ROBUST 1.00000047683715820312f  // 1 + 4 f32::EPSILON (Ize 2013)

struct PRay {
    float org[3], inv[3];
    bool neg[3];
    int kx, ky, kz;
    float sx, sy, sz;
    float tmin, tmax;
};

RTG_D PRay prepare_ray(V3 o, V3 d, float tmin, float tmax) {  // triangle.rs:60
    PRay r;
    float dd[3] = {d.x, d.y, d.z};
    r.inv[0] = __frcp_rn(d.x);  // 1 / d, correctly rounded (the division's IEEE result)
    r.inv[1] = __frcp_rn(d.y);
    r.inv[2] = __frcp_rn(d.z);
    float a0 = absf(d.x), a1 = absf(d.y), a2 = absf(d.z);
    int kz = (a0 >= a1 && a0 >= a2) ? 0 : (a1 >= a2 ? 1 : 2);
    int kx = (kz + 1) % 3, ky = (kz + 2) % 3;
    if (dd[kz] < 0.0f) { int t = kx; kx = ky; ky = t; }
    float sz = r.inv[kz];
    r.org[0] = o.x; r.org[1] = o.y; r.org[2] = o.z;
    r.neg[0] = signbitf(r.inv[0]);
    r.neg[1] = signbitf(r.inv[1]);
    r.neg[2] = signbitf(r.inv[2]);
    r.kx = kx; r.ky = ky; r.kz = kz;
    r.sx = dd[kx] * sz;
    r.sy = dd[ky] * sz;
    r.sz = sz;
    r.tmin = tmin;
    r.tmax = rmin(tmax, F_MAX);
    return r;
}
RTG_D float pick3(const float* v, int k) { return k == 0 ? v[0] : (k == 1 ? v[1] : v[2]); }

// The scalar watertight test (triangle.rs:123), the reference's operations in its order.
RTG_D bool watertight(const PRay& r, const float* v0, const float* v1, const float* v2, float tmax, bool cull_back,
                      float& t, float& u, float& v, float& w, float& det) {
    float ox = r.org[r.kx], oy = r.org[r.ky], oz = r.org[r.kz];
    float a_x = pick3(v0, r.kx) - ox, a_y = pick3(v0, r.ky) - oy, a_z = pick3(v0, r.kz) - oz;
    float b_x = pick3(v1, r.kx) - ox, b_y = pick3(v1, r.ky) - oy, b_z = pick3(v1, r.kz) - oz;
    float c_x = pick3(v2, r.kx) - ox, c_y = pick3(v2, r.ky) - oy, c_z = pick3(v2, r.kz) - oz;
    float ax = a_x - r.sx * a_z, ay = a_y - r.sy * a_z;
    float bx = b_x - r.sx * b_z, by = b_y - r.sy * b_z;
    float cx = c_x - r.sx * c_z, cy = c_y - r.sy * c_z;
    u = cx * by - cy * bx;
    v = ax * cy - ay * cx;
    w = bx * ay - by * ax;
    bool negative = u < 0.0f || v < 0.0f || w < 0.0f;
    bool positive = u > 0.0f || v > 0.0f || w > 0.0f;
    bool rejected = cull_back ? negative : (negative && positive);
    det = u + v + w;
    if (rejected || det == 0.0f) return false;
    float az = r.sz * a_z, bz = r.sz * b_z, cz = r.sz * c_z;
    t = (u * az + v * bz + w * cz) / det;
    return t >= r.tmin && t <= tmax;
}

RTG_D float smax_(float a, float b) { return a > b ? a : b; }
RTG_D float smin_(float a, float b) { return a < b ? a : b; }

// A plane of a quantised box: p + q s for the byte q (byte k of `word`) and the power of two s.
// q s is exact, so the one rounding of the fused form is the sum's: the bits of p + q * s. The
// byte becomes a float as 2^23 + q (a byte permute into 0x4b0000qq) minus 2^23, both exact.
RTG_D float qplane(uint32_t word, int k, float s, float p) {
    const float q = __uint_as_float(__byte_perm(word, 0x4b000000u, 0x7540u | (uint32_t)k)) - 8388608.0f;
    return __fmaf_rn(q, s, p);
}

// Slab test of the eight children of a quantised node; returns the hit mask and entry distances.
RTG_D uint32_t node_test(const QNode* __restrict__ node, const PRay& r, float tmax, float nr[8], uint32_t child[8]) {
    const float4* q = reinterpret_cast<const float4*>(node);
    float4 w0 = __ldg(q + 0), w1 = __ldg(q + 1), w2 = __ldg(q + 2), w3 = __ldg(q + 3), w4 = __ldg(q + 4), w5 = __ldg(q + 5);
    float px = w0.x, py = w0.y, pz = w0.z;
    uint32_t meta = __float_as_uint(w0.w);
    float sx = __uint_as_float((meta & 0xffu) << 23);
    float sy = __uint_as_float(((meta >> 8) & 0xffu) << 23);
    float sz = __uint_as_float(((meta >> 16) & 0xffu) << 23);
    // qlo x,y,z then qhi x,y,z: 8 bytes each = two words each. The near and far planes of each
    // axis are the low and high ones, swapped where the ray runs towards -axis: chosen here once
    // per node, word by word.
    const uint32_t lo[6] = {__float_as_uint(w1.x), __float_as_uint(w1.y), __float_as_uint(w1.z), __float_as_uint(w1.w),
                            __float_as_uint(w2.x), __float_as_uint(w2.y)};
    const uint32_t hi[6] = {__float_as_uint(w2.z), __float_as_uint(w2.w), __float_as_uint(w3.x), __float_as_uint(w3.y),
                            __float_as_uint(w3.z), __float_as_uint(w3.w)};
    uint32_t nw[6], fw[6];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const bool neg = r.neg[a];
        nw[2 * a] = neg ? hi[2 * a] : lo[2 * a];
        nw[2 * a + 1] = neg ? hi[2 * a + 1] : lo[2 * a + 1];
        fw[2 * a] = neg ? lo[2 * a] : hi[2 * a];
        fw[2 * a + 1] = neg ? lo[2 * a + 1] : hi[2 * a + 1];
    }
    child[0] = __float_as_uint(w4.x); child[1] = __float_as_uint(w4.y); child[2] = __float_as_uint(w4.z); child[3] = __float_as_uint(w4.w);
    child[4] = __float_as_uint(w5.x); child[5] = __float_as_uint(w5.y); child[6] = __float_as_uint(w5.z); child[7] = __float_as_uint(w5.w);
    uint32_t bits = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int word = c >> 2, k = c & 3;
        float tx0 = (qplane(nw[0 + word], k, sx, px) - r.org[0]) * r.inv[0];
        float ty0 = (qplane(nw[2 + word], k, sy, py) - r.org[1]) * r.inv[1];
        float tz0 = (qplane(nw[4 + word], k, sz, pz) - r.org[2]) * r.inv[2];
        float tx1 = (qplane(fw[0 + word], k, sx, px) - r.org[0]) * r.inv[0];
        float ty1 = (qplane(fw[2 + word], k, sy, py) - r.org[1]) * r.inv[1];
        float tz1 = (qplane(fw[4 + word], k, sz, pz) - r.org[2]) * r.inv[2];
        float n = smax_(tz0, smax_(ty0, smax_(tx0, r.tmin)));
        float f = smin_(tz1, smin_(ty1, smin_(tx1, tmax))) * RTG_ROBUST;
        nr[c] = n;
        if (n <= f && child[c] != NODE_EMPTY) bits |= 1u << c;
    }
    return bits;
}

RTG_D uint64_t stack_key(float t, uint32_t ref) { return ((uint64_t)__float_as_uint(t) << 32) | (uint64_t)ref; }

RTG_D V3 xf_point(const float* m, V3 p) {
    return v3(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
              m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]);
}
RTG_D V3 xf_vector(const float* m, V3 v) {
    return v3(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[4] * v.x + m[5] * v.y + m[6] * v.z, m[8] * v.x + m[9] * v.y + m[10] * v.z);
}
RTG_D V3 xf_transpose(const float* m, V3 v) {
    return v3(m[0] * v.x + m[4] * v.y + m[8] * v.z, m[1] * v.x + m[5] * v.y + m[9] * v.z, m[2] * v.x + m[6] * v.y + m[10] * v.z);
}

struct TraceResult { uint32_t inst, tri; float t; };

// A traversal stack in one per-thread array.
struct FlatStack {
    uint64_t* p;
    RTG_D void put(int k, uint64_t v) { p[k] = v; }
    RTG_D uint64_t get(int k) const { return p[k]; }
};

// A traversal stack whose first SHORT_STACK entries sit in shared memory, interleaved by thread
// (entry k of thread i at sm[k * stride + i]), and the deeper ones in a per-thread array. Almost
// every ray stays within the shared part.
// A build may set RTG_SHORT_STACK to trade shared memory (8 bytes x 128 threads per entry and
// block) against spills to the deeper part. 16 entries (16 KB a block) leave 128 KB of the SM's
// shared memory to L1 at 8 blocks per SM, where the node fetches hit; on the 1080p product frame
// 12, 16 and 20 entries measured within 1% of each other, 24 entries 3% slower.
#ifndef RTG_SHORT_STACK
#define RTG_SHORT_STACK 16
#endif
constexpr int SHORT_STACK = RTG_SHORT_STACK;
struct SplitStack {
    uint64_t* sm;   // this thread's column of the shared block
    uint64_t* deep; // STACK_CAP - SHORT_STACK entries
    int stride;
    RTG_D void put(int k, uint64_t v) {
        if (k < SHORT_STACK) sm[k * stride] = v;
        else deep[k - SHORT_STACK] = v;
    }
    RTG_D uint64_t get(int k) const { return k < SHORT_STACK ? sm[k * stride] : deep[k - SHORT_STACK]; }
};

// The traversal state of one ray, advanced one node or leaf per trav_step. A kernel can then give
// a lane whose ray has finished a new ray while the rest of its warp keeps traversing.
struct Trav {
    PRay R;          // the ray in the space of the tree being walked (the world ray at level 0)
    V3 o, d;         // the world ray, rebuilt into R on the way back from an instanced tree
    float tmin, tmax;
    float best_t;
    uint32_t best_i, best_tri, cur, b_inst, b_flags;
    uint32_t leaf_k, leaf_end;  // a leaf being tested a few triangles a step: the next one, the end (0: none)
    int sp, level;
    bool camera;
    bool moved;  // R is in a transformed instance's object space (else it is the world ray)
};

// Triangles of a leaf tested per traversal step (0: the whole leaf in one step). With a bound,
// a lane in a long leaf takes as many steps as its triangles need while the rest of its warp
// walks inner nodes, instead of holding them at one step until its leaf is done. A build may set
// RTG_LEAF_STEP; the answer does not depend on it.
#ifndef RTG_LEAF_STEP
#define RTG_LEAF_STEP 0
#endif

// Sets up a query. False when the ray can meet nothing (non-finite or zero direction, empty
// interval): a miss.
RTG_D bool trav_init(const SceneDev& S, Trav& T, V3 o, V3 d, float tmin, float tmax, bool camera) {
    if (!(vfinite(o) && vfinite(d) && !veq(d, v3(0, 0, 0)))) return false;
    T.R = prepare_ray(o, d, tmin, tmax);
    if (!(T.R.tmin <= T.R.tmax)) return false;
    T.o = o;
    T.d = d;
    T.tmin = T.R.tmin;
    T.tmax = T.R.tmax;
    T.best_t = T.R.tmax;
    T.best_i = 0xffffffffu;
    T.best_tri = 0xffffffffu;
    T.cur = S.tlas_root;
    T.b_inst = 0xffffffffu;
    T.b_flags = 0;
    T.sp = 0;
    T.level = 0;
    T.camera = camera;
    T.leaf_k = 0;
    T.leaf_end = 0;
    T.moved = false;
    return true;
}

// One step of the two-level traversal: the slab test of one node, or the triangles of one leaf,
// then the next node (a child, or the nearest entry of the stack that is still in range).
// `ANY`: stop at the first hit in [t_min, t_max] (shadow rays; children in slot order). Otherwise
// the nearest hit with the reference's tie-break, children nearest first. Returns true when the
// query is over; `hit` then says whether it found one (nearest: in T.best_*). A stack that would
// overflow sets *err bit 0 and ends the query as a miss.
template <bool ANY, class Stack>
RTG_D bool trav_step(const SceneDev& S, Trav& T, Stack& stack, uint32_t* err, bool& hit) {
    const uint32_t cur = T.cur;
    if ((cur & NODE_LEAF) == 0) {
        float nr[8];
        uint32_t child[8];
        const uint32_t bits = node_test(S.nodes + cur, T.R, T.best_t, nr, child);
        // Every array index below is a constant after unrolling, so nr, child and key stay in
        // registers.
        if (bits) {
            uint32_t next = 0;
            if ((bits & (bits - 1)) == 0) {
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    if (bits == (1u << c)) next = child[c];
                T.cur = next;
                return false;
            }
            if (T.sp + 8 > STACK_CAP) { *err |= 1u; hit = false; return true; }
            if (ANY) {
                // Slot order: the lowest slot next, the others pushed lowest first.
                const uint32_t first = bits & (0u - bits);
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    if ((bits >> c) & 1u) {
                        if ((1u << c) == first) next = child[c];
                        else stack.put(T.sp++, stack_key(nr[c], child[c]));
                    }
                }
            } else {
                // Nearest first: push the others farthest first (descending (t, ref) keys), so
                // the nearest remaining child is popped next.
                uint64_t key[8];
#pragma unroll
                for (int c = 0; c < 8; ++c) key[c] = stack_key(nr[c], child[c]);
                uint32_t live = bits;
                for (int left = __popc(bits); left > 1; --left) {
                    uint64_t top = 0;
                    uint32_t pick = 0;
#pragma unroll
                    for (int c = 0; c < 8; ++c)
                        if (((live >> c) & 1u) && (pick == 0 || key[c] > top)) { top = key[c]; pick = 1u << c; }
                    stack.put(T.sp++, top);
                    live &= ~pick;
                }
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    if (live == (1u << c)) next = child[c];
            }
            T.cur = next;
            return false;
        }
    } else if (cur != NODE_EMPTY) {
        uint32_t first = (cur & ~NODE_LEAF) >> 4, count = (cur & 15u) + 1;
        if (T.level == 0) {
            const BlasInst* bi = S.blas + first;
            uint32_t flags = __ldg(&bi->flags);
            if (!(T.camera && (flags & 2u))) {
                if (T.sp + 1 > STACK_CAP) { *err |= 1u; hit = false; return true; }
                stack.put(T.sp++, stack_key(0.0f, STACK_RETURN));
                if (!__ldg(&bi->identity)) {
                    float m[12];
#pragma unroll
                    for (int k = 0; k < 12; ++k) m[k] = __ldg(&bi->to_local[k]);
                    T.R = prepare_ray(xf_point(m, T.o), xf_vector(m, T.d), T.tmin, T.tmax);
                    T.moved = true;
                }
                T.b_inst = __ldg(&bi->instance);
                T.b_flags = flags;
                T.level = 1;
                T.cur = __ldg(&bi->root);
                return false;
            }
        } else {
            uint32_t k = T.leaf_end ? T.leaf_k : first;
            const uint32_t end = T.leaf_end ? T.leaf_end : first + count;
            const uint32_t stop = (RTG_LEAF_STEP > 0 && end - k > (uint32_t)RTG_LEAF_STEP) ? k + (uint32_t)RTG_LEAF_STEP : end;
            for (; k < stop; ++k) {
                const float4* tr = reinterpret_cast<const float4*>(S.tris + k);
                float4 a = __ldg(tr), b = __ldg(tr + 1), c = __ldg(tr + 2);
                uint32_t flags = __float_as_uint(c.w) | T.b_flags;
                if (T.camera && (flags & 2u)) continue;
                float v0[3] = {a.x, a.y, a.z}, v1[3] = {b.x, b.y, b.z}, v2[3] = {c.x, c.y, c.z};
                float t, uu, vv, ww, det;
                if (watertight(T.R, v0, v1, v2, ANY ? T.R.tmax : T.best_t, (flags & 1u) != 0, t, uu, vv, ww, det)) {
                    if (ANY) { T.leaf_end = 0; hit = true; return true; }
                    uint32_t inst = __float_as_uint(b.w);
                    if (inst == 0xffffffffu) inst = T.b_inst;
                    uint32_t tri = __float_as_uint(a.w);
                    if (t < T.best_t || (t == T.best_t && (inst < T.best_i || (inst == T.best_i && tri < T.best_tri)))) {
                        T.best_t = t; T.best_i = inst; T.best_tri = tri;
                    }
                }
            }
            if (k < end) {  // more of this leaf next step
                T.leaf_k = k;
                T.leaf_end = end;
                return false;
            }
            T.leaf_end = 0;
        }
    }
    for (;;) {
        if (T.sp == 0) {
            hit = !ANY && T.best_i != 0xffffffffu;
            return true;
        }
        uint64_t e = stack.get(--T.sp);
        uint32_t ref = (uint32_t)e;
        if (ref == STACK_RETURN) {
            T.level = 0;
            if (T.moved) {  // an identity instance's tree was walked with the world ray itself
                T.R = prepare_ray(T.o, T.d, T.tmin, T.tmax);
                T.moved = false;
            }
            continue;
        }
        float t = __uint_as_float((uint32_t)(e >> 32));
        if (t <= (ANY ? T.tmax : T.best_t) * RTG_ROBUST) { T.cur = ref; return false; }
    }
}

// A whole query: false on a miss. Nearest-hit queries fill `res`.
template <bool ANY, class Stack>
RTG_D bool traverse(const SceneDev& S, V3 o, V3 d, float tmin, float tmax, bool camera, TraceResult& res, uint32_t* err,
                    Stack& stack) {
    Trav T;
    if (!trav_init(S, T, o, d, tmin, tmax, camera)) return false;
    bool hit = false;
    while (!trav_step<ANY>(S, T, stack, err, hit)) {
    }
    if (hit && !ANY) { res.inst = T.best_i; res.tri = T.best_tri; res.t = T.best_t; }
    return hit;
}

// ---- the section view (geometry/section.rs:127-448) --------------------------------------------------
// A query of a scene with a section sees the model as if the side of the plane its normal points to
// were empty: the ray is clipped to the interval where it is on the kept side; where it crosses the
// plane inside a closed solid (the next surface along it is met from behind) it hits the solid's cap
// on the plane; and the studio instances (exempt from the section) are found on the removed side by
// stepping over the cut model's surfaces, at most 48 deep.
constexpr uint32_t CAP_TRIANGLE = 0xffffffffu;  // the `tri` of a hit on a cap
constexpr int SECTION_MAX_SKIPS = 48;
enum : int { SPAN_REMOVED = 0, SPAN_WHOLE = 1, SPAN_ENTERS = 2, SPAN_LEAVES = 3 };

RTG_D int section_span(const SceneDev& S, V3 o, V3 d, float tmin, float tmax, float& t) {
    const V3 n = v3(S.section_n[0], S.section_n[1], S.section_n[2]);
    const float from_plane = dot(n, o) - S.section_d;
    const float towards = dot(n, d);
    if (towards == 0.0f) return from_plane <= 0.0f ? SPAN_WHOLE : SPAN_REMOVED;
    t = -from_plane / towards;
    if (towards > 0.0f) return t < tmin ? SPAN_REMOVED : (t >= tmax ? SPAN_WHOLE : SPAN_LEAVES);
    return t <= tmin ? SPAN_WHOLE : (t > tmax ? SPAN_REMOVED : SPAN_ENTERS);
}

RTG_D bool section_may_cap(const SceneDev& S, V3 p) {
    return S.cap_any && p.x >= S.cap_lo[0] && p.x <= S.cap_hi[0] && p.y >= S.cap_lo[1] && p.y <= S.cap_hi[1] &&
           p.z >= S.cap_lo[2] && p.z <= S.cap_hi[2];
}

RTG_D bool section_hidden(const SceneDev& S, bool camera, uint32_t inst) {
    return camera && inst < S.n_instances && (S.instances[inst].flags & 4u) != 0;  // INSTANCE_NO_CAMERA
}

// True when triangle `tri` of capped instance `inst` is met by direction d from inside its solid.
RTG_D bool section_met_from_inside(const SceneDev& S, V3 d, uint32_t inst, uint32_t tri) {
    if (inst >= S.n_instances) return false;
    const DevInstance* I = S.instances + inst;
    if (!I->active || I->solid == 0u) return false;
    const uint4 idx = __ldg(S.tri_index + I->tri_base + tri);
    const float4 q0 = __ldg(S.positions + idx.x), q1 = __ldg(S.positions + idx.y), q2 = __ldg(S.positions + idx.z);
    const V3 p0 = v3(q0.x, q0.y, q0.z), p1 = v3(q1.x, q1.y, q1.z), p2 = v3(q2.x, q2.y, q2.z);
    V3 w = cross(p1 - p0, p2 - p0);
    if (!I->identity) w = xf_transpose(I->to_local, w);
    const bool front = dot(w, d) < 0.0f;
    return I->solid == 1u ? !front : front;
}

// The first exempt instance within [near, far], stepping over the others' surfaces.
template <class Stack>
RTG_D bool section_first_exempt(const SceneDev& S, V3 o, V3 d, float near, float far, bool camera, TraceResult& res,
                                uint32_t* err, Stack& stack) {
    float t = near;
    for (int k = 0; k < SECTION_MAX_SKIPS; ++k) {
        TraceResult h;
        if (!traverse<false>(S, o, d, t, far, camera, h, err, stack)) return false;
        if (h.inst < S.n_instances && S.instances[h.inst].exempt) { res = h; return true; }
        t = __uint_as_float(__float_as_uint(fmaxf(h.t, 0.0f)) + 1u);  // strictly past the surface
        if (t > far) return false;
    }
    return false;
}

// The nearest exempt hit within [from, to] (a removed part of the ray's range), looked for inside
// each exempt instance's box only (Aabb::intersect, math.rs:388).
template <class Stack>
RTG_D bool section_exempt_in(const SceneDev& S, V3 o, V3 d, float from, float to, bool camera, TraceResult& res, uint32_t* err,
                             Stack& stack) {
    if (S.n_exempt == 0u || from != from || to != to || from > to) return false;
    const float inv[3] = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z}, org[3] = {o.x, o.y, o.z};
    bool found = false;
    for (uint32_t b = 0; b < S.n_exempt; ++b) {
        const float* box = S.exempt_boxes + 6 * b;
        const float end = found ? fminf(res.t, to) : to;
        float near = from, far = end;
        for (int a = 0; a < 3; ++a) {
            const float x = (__ldg(box + a) - org[a]) * inv[a], y = (__ldg(box + 3 + a) - org[a]) * inv[a];
            if (x != x || y != y) continue;  // parallel to the slab, on its boundary
            near = fmaxf(near, fminf(x, y));
            far = fminf(far, fmaxf(x, y));
        }
        if (!(near <= far && near < f_inf())) continue;
        TraceResult h;
        if (section_first_exempt(S, o, d, near, fminf(far, end), camera, h, err, stack) && (!found || h.t < res.t)) {
            res = h;
            found = true;
        }
    }
    return found;
}

// The cap at t where the ray leaves the kept side having hit nothing: there when the next surface of
// the whole model beyond the plane is met from inside its solid.
template <class Stack>
RTG_D bool section_cap_beyond(const SceneDev& S, V3 o, V3 d, float t, TraceResult& res, uint32_t* err, Stack& stack) {
    if (!S.section_cap || !section_may_cap(S, o + d * t)) return false;
    TraceResult h;
    if (!traverse<false>(S, o, d, t, f_inf(), false, h, err, stack)) return false;
    if (!section_met_from_inside(S, d, h.inst, h.tri)) return false;
    res.inst = h.inst;
    res.tri = CAP_TRIANGLE;
    res.t = t;
    return true;
}

// Geometry::trace_sectioned / occluded_sectioned (section.rs:224-324). Out of line: scenes without
// a section never call it, and the kernels that can keep their registers for the plain traversal.
template <bool ANY, class Stack>
RTG_D_NI bool section_query(const SceneDev& S, V3 o, V3 d, float tmin, float tmax, bool camera, TraceResult& res,
                            uint32_t* err, Stack& stack) {
    float t = 0.0f;
    const int span = section_span(S, o, d, tmin, tmax, t);
    TraceResult other;
    if (ANY) {
        switch (span) {
            case SPAN_REMOVED: return section_exempt_in(S, o, d, tmin, tmax, camera, other, err, stack);
            case SPAN_WHOLE: return traverse<true>(S, o, d, tmin, tmax, camera, res, err, stack);
            case SPAN_LEAVES:
                return traverse<true>(S, o, d, tmin, t, camera, res, err, stack) || section_cap_beyond(S, o, d, t, other, err, stack) ||
                       section_exempt_in(S, o, d, t, tmax, camera, other, err, stack);
            default:  // the cap of a ray that enters is at the start of what it can hit anyway
                return traverse<true>(S, o, d, t, tmax, camera, res, err, stack) ||
                       section_exempt_in(S, o, d, tmin, t, camera, other, err, stack);
        }
    }
    switch (span) {
        case SPAN_REMOVED: return section_exempt_in(S, o, d, tmin, tmax, camera, res, err, stack);
        case SPAN_WHOLE: return traverse<false>(S, o, d, tmin, tmax, camera, res, err, stack);
        case SPAN_LEAVES:
            // The kept part; else a cap looked for beyond the plane; else the studio beyond it.
            if (traverse<false>(S, o, d, tmin, t, camera, res, err, stack)) return true;
            if (section_cap_beyond(S, o, d, t, other, err, stack) && !section_hidden(S, camera, other.inst)) {
                res = other;
                return true;
            }
            return section_exempt_in(S, o, d, t, tmax, camera, res, err, stack);
        default: {
            // The studio on the removed side is nearer than anything on the kept one; then the
            // nearest surface beyond the plane, whose side tells whether the crossing is a cap.
            if (section_exempt_in(S, o, d, tmin, t, camera, res, err, stack)) return true;
            const bool got = traverse<false>(S, o, d, t, tmax, camera, other, err, stack);
            if (got && S.section_cap && section_may_cap(S, o + d * t) && section_met_from_inside(S, d, other.inst, other.tri) &&
                !section_hidden(S, camera, other.inst)) {
                res.inst = other.inst;
                res.tri = CAP_TRIANGLE;
                res.t = t;
                return true;
            }
            if (got) res = other;
            return got;
        }
    }
}

// A whole query through the scene's section when it has one.
template <bool ANY, class Stack>
RTG_D bool trace_q(const SceneDev& S, V3 o, V3 d, float tmin, float tmax, bool camera, TraceResult& res, uint32_t* err,
                   Stack& stack) {
    if (!S.section_on) return traverse<ANY>(S, o, d, tmin, tmax, camera, res, err, stack);
    return section_query<ANY>(S, o, d, tmin, tmax, camera, res, err, stack);
}

struct HitInfo {
    V3 point, normal, geometric;
    float bary[3];
    bool front, outside;
    bool cap;  // on a section's cap: no triangle, the plane's normal
};

// geometry/mod.rs:731 hit_details for an instance hit.
RTG_D_NI bool hit_details(const SceneDev& S, V3 o, V3 d, float tmin, float tmax, uint32_t inst, uint32_t tri, float t_hit,
                       HitInfo& h, const DevInstance*& I_out, uint4& idx_out) {
    if (inst >= S.n_instances) return false;
    const DevInstance* I = S.instances + inst;
    I_out = I;
    if (!I->active) return false;
    h.cap = tri == CAP_TRIANGLE;
    if (h.cap) {  // Section::cap_details (section.rs:424-448): on the plane, facing where the ray came from
        if (!S.section_on) return false;
        const V3 n = v3(S.section_n[0], S.section_n[1], S.section_n[2]);
        const V3 at = o + d * t_hit;
        h.point = at - n * (dot(n, at) - S.section_d);
        h.front = dot(n, d) < 0.0f;
        h.normal = h.front ? n : -n;
        h.geometric = h.normal;
        h.bary[0] = 1.0f;
        h.bary[1] = h.bary[2] = 0.0f;
        h.outside = h.front;
        idx_out = make_uint4(0u, 0u, 0u, 0u);
        return true;
    }
    uint4 idx = __ldg(S.tri_index + I->tri_base + tri);
    idx_out = idx;
    float4 q0 = __ldg(S.positions + idx.x), q1 = __ldg(S.positions + idx.y), q2 = __ldg(S.positions + idx.z);
    V3 p0 = v3(q0.x, q0.y, q0.z), p1 = v3(q1.x, q1.y, q1.z), p2 = v3(q2.x, q2.y, q2.z);
    bool identity = I->identity != 0;
    PRay r = identity ? prepare_ray(o, d, tmin, tmax) : prepare_ray(xf_point(I->to_local, o), xf_vector(I->to_local, d), tmin, tmax);
    float v0[3] = {p0.x, p0.y, p0.z}, v1[3] = {p1.x, p1.y, p1.z}, v2[3] = {p2.x, p2.y, p2.z};
    float t, u, v, w, det;
    if (watertight(r, v0, v1, v2, F_MAX, false, t, u, v, w, det)) {
        h.bary[0] = u / det; h.bary[1] = v / det; h.bary[2] = w / det;
    } else {
        h.bary[0] = h.bary[1] = h.bary[2] = 1.0f / 3.0f;
    }
    V3 pl = p0 * h.bary[0] + p1 * h.bary[1] + p2 * h.bary[2];
    V3 cr = cross(p1 - p0, p2 - p0);
    V3 winding = normalize(identity ? cr : xf_transpose(I->to_local, cr));
    V3 incoming = normalize(d);
    V3 geometric = len2(winding) > 0.0f ? winding : -incoming;
    h.front = dot(winding, d) < 0.0f;
    V3 smooth = v3(0, 0, 0);
    if (I->has_normals) {
        float4 m0 = __ldg(S.normals + idx.x), m1 = __ldg(S.normals + idx.y), m2 = __ldg(S.normals + idx.z);
        V3 s = v3(m0.x, m0.y, m0.z) * h.bary[0] + v3(m1.x, m1.y, m1.z) * h.bary[1] + v3(m2.x, m2.y, m2.z) * h.bary[2];
        smooth = identity ? s : xf_transpose(I->to_local, s);
    }
    V3 normal = len2(smooth) > 1.0e-12f ? normalize(smooth) : geometric;
    h.normal = dot(normal, d) > 0.0f ? -normal : normal;
    h.geometric = dot(geometric, d) > 0.0f ? -geometric : geometric;
    h.point = identity ? pl : xf_point(I->to_world, pl);
    h.outside = h.front != (I->inside_out != 0);
    return true;
}

// geometry/mod.rs:682 terminator_point (Hanika 2021).
RTG_D_NI V3 terminator_point(const SceneDev& S, const DevInstance* I, uint4 idx, const HitInfo& h) {
    if (h.cap || !I->has_normals) return h.point;
    float4 q[3] = {__ldg(S.positions + idx.x), __ldg(S.positions + idx.y), __ldg(S.positions + idx.z)};
    float4 m[3] = {__ldg(S.normals + idx.x), __ldg(S.normals + idx.y), __ldg(S.normals + idx.z)};
    V3 c[3], n[3];
    for (int k = 0; k < 3; ++k) { c[k] = v3(q[k].x, q[k].y, q[k].z); n[k] = v3(m[k].x, m[k].y, m[k].z); }
    float b0 = h.bary[0], b1 = h.bary[1], b2 = h.bary[2];
    V3 p = c[0] * b0 + c[1] * b1 + c[2] * b2;
    V3 interp = n[0] * b0 + n[1] * b1 + n[2] * b2;
    bool identity = I->identity != 0;
    V3 wn = identity ? interp : xf_transpose(I->to_local, interp);
    float side = dot(wn, h.geometric) < 0.0f ? -1.0f : 1.0f;
    V3 lifted = p;
    for (int k = 0; k < 3; ++k) {
        V3 nn = normalize(n[k]) * side;
        float below = dot(p - c[k], nn);
        if (below < 0.0f) lifted = lifted - nn * (below * h.bary[k]);
    }
    if (!vfinite(lifted)) return h.point;
    return identity ? lifted : xf_point(I->to_world, lifted);
}

}  // namespace rtg
