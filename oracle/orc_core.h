// ORACLE (test infrastructure only). A plain C++17 restatement of the Repackshot engine's
// deterministic maths, random numbers and sampler, used to check the CUDA path. Nothing in the
// product links this file; only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use
// the oracle library built from it.
//
// Compiled with -ffp-contract=off -fno-fast-math: every float expression below is evaluated in
// the written order with IEEE round-to-nearest and never fused, as the reference promises.
//
// Reference files restated here (paths inside engine/crates/rt-core/src/):
//   fmath.rs:35-270   sin_cos, exp2, log2, powf, atan, atan2, acos
//   math.rs:1-400     Vec3, Ray, Frame::from_normal, offset_origin, Aabb
//   color.rs:45-47    Rgb::luminance
//   rng.rs:1-55       Pcg32, mix64
//   sampler.rs:83-368 LAYOUT, Joe–Kuo direction numbers, sobol, owen_scramble, PixelSampler
//   warp.rs:12-62     concentric_disk, cosine_hemisphere
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

namespace orc {

constexpr float F_INF = std::numeric_limits<float>::infinity();
constexpr float F_MAX = std::numeric_limits<float>::max();
constexpr float F_EPS = std::numeric_limits<float>::epsilon();

inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float bitsf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline bool finite(float x) { return std::isfinite(x); }
inline bool isnan_(float x) { return x != x; }

// Rust f32::min / f32::max: the non-NaN operand when one is NaN (fmath.rs relies on them).
inline float rmin(float a, float b) { if (a != a) return b; if (b != b) return a; return a < b ? a : b; }
inline float rmax(float a, float b) { if (a != a) return b; if (b != b) return a; return a > b ? a : b; }
// Rust f32::clamp (NaN stays NaN).
inline float rclamp(float x, float lo, float hi) { if (x < lo) x = lo; if (x > hi) x = hi; return x; }
// Rust `f32 as i64` / `as i32` / `as usize`: truncation toward zero, saturating, NaN -> 0.
inline int64_t f2i64(float x) {
    if (x != x) return 0;
    if (x >= 9.2233720368547758e18f) return INT64_MAX;
    if (x <= -9.2233720368547758e18f) return INT64_MIN;
    return (int64_t)x;
}
inline int32_t f2i32(float x) {
    if (x != x) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}
inline uint64_t f2usize(float x) {
    if (x != x || x <= 0.0f) return 0;
    if (x >= 1.8446744073709552e19f) return UINT64_MAX;
    return (uint64_t)x;
}

// ---- fmath.rs -------------------------------------------------------------------------------
constexpr float PI = 3.14159265358979323846f;
constexpr float TAU = 6.28318530717958647692f;
constexpr float FRAC_PI_2 = 1.57079632679489661923f;
constexpr float FRAC_PI_4 = 0.785398163397448309616f;
constexpr float FRAC_1_PI = 0.318309886183790671538f;
constexpr float LN_2 = 0.693147180559945309417f;
constexpr float LOG2_E = 1.44269504088896340736f;
constexpr float SQRT_2 = 1.41421356237309504880f;
const float DEG_TO_RAD = PI / 180.0f;

// fmath.rs:34-37 Cody–Waite split of pi/2.
constexpr float PIO2_1 = 1.5703125f;
constexpr float PIO2_2 = 4.837513e-4f;
constexpr float PIO2_3 = 7.54979e-8f;

inline float sin_poly(float r) {  // fmath.rs:41
    float r2 = r * r;
    float p = 1.0f / 362880.0f;
    p = p * r2 - 1.0f / 5040.0f;
    p = p * r2 + 1.0f / 120.0f;
    p = p * r2 - 1.0f / 6.0f;
    return r + r * r2 * p;
}
inline float cos_poly(float r) {  // fmath.rs:52
    float r2 = r * r;
    float p = -1.0f / 3628800.0f;
    p = p * r2 + 1.0f / 40320.0f;
    p = p * r2 - 1.0f / 720.0f;
    p = p * r2 + 1.0f / 24.0f;
    p = p * r2 - 0.5f;
    return 1.0f + r2 * p;
}
inline void sin_cos(float x, float& s_out, float& c_out) {  // fmath.rs:64
    if (!finite(x)) { s_out = 0.0f; c_out = 1.0f; return; }
    float k = std::floor(x * (2.0f / PI) + 0.5f);
    float r = ((x - k * PIO2_1) - k * PIO2_2) - k * PIO2_3;
    float s = sin_poly(r), c = cos_poly(r);
    switch (f2i64(k) & 3) {
        case 0: s_out = s; c_out = c; break;
        case 1: s_out = c; c_out = -s; break;
        case 2: s_out = -s; c_out = -c; break;
        default: s_out = -c; c_out = s; break;
    }
}
inline float fsin(float x) { float s, c; sin_cos(x, s, c); return s; }
inline float fcos(float x) { float s, c; sin_cos(x, s, c); return c; }
inline float pow2i(int32_t n) { return bitsf(((uint32_t)(n + 127)) << 23); }
inline float exp2(float x) {  // fmath.rs:100
    if (x != x) return x;
    if (x >= 128.0f) return F_INF;
    if (x < -150.0f) return 0.0f;
    float k = std::floor(x + 0.5f);
    float t = (x - k) * LN_2;
    float p = 1.0f / 5040.0f;
    p = p * t + 1.0f / 720.0f;
    p = p * t + 1.0f / 120.0f;
    p = p * t + 1.0f / 24.0f;
    p = p * t + 1.0f / 6.0f;
    p = p * t + 0.5f;
    p = p * t + 1.0f;
    p = p * t + 1.0f;
    int32_t ki = f2i32(k);
    int32_t k1 = ki / 2;
    return p * pow2i(k1) * pow2i(ki - k1);
}
inline float log2(float x) {  // fmath.rs:128
    if (x != x) return x;
    if (x <= 0.0f) return -F_INF;
    if (x == F_INF) return x;
    int32_t e = 0;
    if (x < std::numeric_limits<float>::min()) { x *= 8388608.0f; e = -23; }
    uint32_t bits = fbits(x);
    e += (int32_t)((bits >> 23) & 0xff) - 127;
    float m = bitsf((bits & 0x007fffffu) | 0x3f800000u);
    if (m > SQRT_2) { m *= 0.5f; e += 1; }
    float s = (m - 1.0f) / (m + 1.0f);
    float s2 = s * s;
    float p = 1.0f / 11.0f;
    p = p * s2 + 1.0f / 9.0f;
    p = p * s2 + 1.0f / 7.0f;
    p = p * s2 + 1.0f / 5.0f;
    p = p * s2 + 1.0f / 3.0f;
    float ln_m = 2.0f * (s + s * s2 * p);
    return (float)e + ln_m * LOG2_E;
}
inline float fexp(float x) { return exp2(x * LOG2_E); }
inline float fln(float x) { return log2(x) * LN_2; }
inline float powf_(float x, float y) {  // fmath.rs:174
    if (y == 0.0f) return 1.0f;
    if (x <= 0.0f) return y > 0.0f ? 0.0f : F_INF;
    if (x == 1.0f) return 1.0f;
    return exp2(y * log2(x));
}
inline float atan_poly(float u) {  // fmath.rs:187
    float u2 = u * u;
    float p = 1.0f / 17.0f;
    p = -p * u2 + 1.0f / 15.0f;
    p = -p * u2 + 1.0f / 13.0f;
    p = -p * u2 + 1.0f / 11.0f;
    p = -p * u2 + 1.0f / 9.0f;
    p = -p * u2 + 1.0f / 7.0f;
    p = -p * u2 + 1.0f / 5.0f;
    p = -p * u2 + 1.0f / 3.0f;
    return u - u * u2 * p;
}
inline float fatan(float x) {  // fmath.rs:202
    if (x != x) return x;
    float a = std::fabs(x);
    bool flip = a > 1.0f;
    float t = flip ? 1.0f / a : a;
    float r = t > 0.41421357f ? FRAC_PI_4 + atan_poly((t - 1.0f) / (t + 1.0f)) : atan_poly(t);
    if (flip) r = FRAC_PI_2 - r;
    return x < 0.0f ? -r : r;
}
inline float fatan2(float y, float x) {  // fmath.rs:225
    if (x != x || y != y) return std::numeric_limits<float>::quiet_NaN();
    if (x == 0.0f) return y > 0.0f ? FRAC_PI_2 : (y < 0.0f ? -FRAC_PI_2 : 0.0f);
    if (std::fabs(y) <= std::fabs(x)) {
        float r = fatan(y / x);
        if (!(x < 0.0f)) return r;
        return y < 0.0f ? r - PI : r + PI;
    }
    return y > 0.0f ? FRAC_PI_2 - fatan(x / y) : -FRAC_PI_2 - fatan(x / y);
}
inline float facos(float x) { x = rclamp(x, -1.0f, 1.0f); return fatan2(std::sqrt((1.0f - x) * (1.0f + x)), x); }

// ---- math.rs --------------------------------------------------------------------------------
struct Vec3 {
    float x = 0, y = 0, z = 0;
    Vec3() = default;
    Vec3(float x_, float y_, float z_) : x(x_), y(y_), z(z_) {}
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline Vec3 operator+(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 operator-(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 operator*(Vec3 a, Vec3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline Vec3 operator*(Vec3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline Vec3 operator/(Vec3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline Vec3 operator-(Vec3 a) { return {-a.x, -a.y, -a.z}; }
inline bool operator==(Vec3 a, Vec3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline float dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vec3 cross(Vec3 a, Vec3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float length_squared(Vec3 a) { return dot(a, a); }
inline float length(Vec3 a) { return std::sqrt(length_squared(a)); }
inline Vec3 normalize(Vec3 a) {  // math.rs:64
    float len = length(a);
    if (len > 0.0f && finite(len)) return a / len;
    return a;
}
inline Vec3 vmin(Vec3 a, Vec3 b) { return {rmin(a.x, b.x), rmin(a.y, b.y), rmin(a.z, b.z)}; }
inline Vec3 vmax(Vec3 a, Vec3 b) { return {rmax(a.x, b.x), rmax(a.y, b.y), rmax(a.z, b.z)}; }
inline Vec3 vabs(Vec3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline float max_component(Vec3 a) { return rmax(rmax(a.x, a.y), a.z); }
inline bool vfinite(Vec3 a) { return finite(a.x) && finite(a.y) && finite(a.z); }

struct Ray {
    Vec3 origin, dir;
    float t_min = 1.0e-3f, t_max = F_INF;
    Ray() = default;
    Ray(Vec3 o, Vec3 d) : origin(o), dir(d), t_min(1.0e-3f), t_max(F_INF) {}
    Vec3 at(float t) const { return origin + dir * t; }
};
constexpr float RAY_EPSILON = 1.0e-3f;

struct Frame {
    Vec3 x, y, z;
    static Frame from_normal(Vec3 n) {  // math.rs:263 (Duff et al. 2017)
        float sign = std::copysign(1.0f, n.z);
        float a = -1.0f / (sign + n.z);
        float b = n.x * n.y * a;
        Frame f;
        f.x = Vec3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
        f.y = Vec3(b, sign + n.y * n.y * a, -n.y);
        f.z = n;
        return f;
    }
    Vec3 to_local(Vec3 v) const { return {dot(v, x), dot(v, y), dot(v, z)}; }
    Vec3 to_world(Vec3 v) const { return x * v.x + y * v.y + z * v.z; }
};

inline float offset_axis(float p, float n) {  // math.rs:293
    const float ORIGIN = 1.0f / 32.0f, FLOAT_SCALE = 1.0f / 65536.0f, INT_SCALE = 256.0f;
    if (std::fabs(p) < ORIGIN) return p + FLOAT_SCALE * n;
    int32_t of = f2i32(INT_SCALE * n);
    int32_t pb = (int32_t)fbits(p);
    int32_t moved = (int32_t)((uint32_t)pb + (uint32_t)(p < 0.0f ? -of : of));
    float q = bitsf((uint32_t)moved);
    return finite(q) ? q : p;
}
inline Vec3 offset_origin(Vec3 p, Vec3 n) {
    return {offset_axis(p.x, n.x), offset_axis(p.y, n.y), offset_axis(p.z, n.z)};
}

struct Aabb {
    Vec3 min{F_INF, F_INF, F_INF}, max{-F_INF, -F_INF, -F_INF};
    Aabb() = default;
    Aabb(Vec3 a, Vec3 b) : min(a), max(b) {}
    bool is_empty() const { return min.x > max.x || min.y > max.y || min.z > max.z; }
    Aabb uni(const Aabb& o) const { return {vmin(min, o.min), vmax(max, o.max)}; }
    Aabb extend(Vec3 p) const { return {vmin(min, p), vmax(max, p)}; }
    Vec3 centroid() const { return (min + max) * 0.5f; }
    float surface_area() const {
        if (is_empty()) return 0.0f;
        Vec3 d = max - min;
        return 2.0f * (d.x * d.y + d.y * d.z + d.z * d.x);
    }
};

// ---- color.rs -------------------------------------------------------------------------------
struct Rgb {
    float r = 0, g = 0, b = 0;
    Rgb() = default;
    Rgb(float r_, float g_, float b_) : r(r_), g(g_), b(b_) {}
    static Rgb splat(float v) { return {v, v, v}; }
    float luminance() const { return 0.2126f * r + 0.7152f * g + 0.0722f * b; }
};
inline Rgb operator+(Rgb a, Rgb b) { return {a.r + b.r, a.g + b.g, a.b + b.b}; }
inline Rgb operator*(Rgb a, Rgb b) { return {a.r * b.r, a.g * b.g, a.b * b.b}; }
inline Rgb operator*(Rgb a, float s) { return {a.r * s, a.g * s, a.b * s}; }
inline Rgb operator/(Rgb a, float s) { return {a.r / s, a.g / s, a.b / s}; }
inline bool operator==(Rgb a, Rgb b) { return a.r == b.r && a.g == b.g && a.b == b.b; }
inline float peak(Rgb c) { return rmax(rmax(c.r, c.g), c.b); }
const Rgb WHITE(1, 1, 1), BLACK(0, 0, 0);

// ---- rng.rs ---------------------------------------------------------------------------------
struct Pcg32 {
    uint64_t state = 0, inc = 1;
    static Pcg32 seeded(uint64_t seed, uint64_t stream) {  // rng.rs:21
        Pcg32 r;
        r.state = 0;
        r.inc = (stream << 1) | 1;
        r.next_u32();
        r.state += seed;
        r.next_u32();
        return r;
    }
    uint32_t next_u32() {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        uint32_t xorshifted = (uint32_t)(((old >> 18) ^ old) >> 27);
        uint32_t rot = (uint32_t)(old >> 59);
        return (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
    }
    float next_f32() { return (float)(next_u32() >> 8) * (1.0f / 16777216.0f); }
};
inline uint64_t mix64(uint64_t z) {  // rng.rs:51
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// ---- sampler.rs -----------------------------------------------------------------------------
// The logical -> Sobol dimension permutation of the reference (sampler.rs:83). The values are the
// reference's chosen pairing and must be identical for the random numbers to match.
constexpr uint8_t LAYOUT[64] = {
    0, 1, 11, 50, 19, 2, 15, 10, 13, 20, 21, 5, 27, 3, 59, 25, 26, 6, 57, 18, 47, 28,
    31, 24, 44, 22, 58, 34, 37, 49, 52, 4, 9, 39, 41, 7, 12, 16, 29, 42, 45, 8, 38, 14,
    46, 48, 51, 33, 36, 32, 56, 53, 54, 35, 63, 43, 62, 55, 60, 23, 30, 17, 40, 61};
constexpr uint32_t DIM_CAMERA = 0, DIM_LENS = 2, DIM_FIRST_BOUNCE = 4, DIMS_PER_BOUNCE = 6;
constexpr uint32_t OFFSET_LIGHT_SELECT = 0, OFFSET_LIGHT = 1, OFFSET_BSDF = 3, OFFSET_ROULETTE = 5;
inline uint32_t bounce_dim(uint32_t b) { return DIM_FIRST_BOUNCE + b * DIMS_PER_BOUNCE; }
// sampler.rs:127-135: the hashed dimension deciding whether the ray of vertex `bounce` passes its
// `crossing`-th cut-out.
constexpr uint32_t DIM_CUTOUT = 1u << 20;
inline uint32_t cutout_dim(uint32_t bounce, uint32_t crossing) { return DIM_CUTOUT + bounce * 64 + (crossing < 63 ? crossing : 63); }

// Joe & Kuo (2008) new-joe-kuo-6.21201, dimensions 2..64: degree s, coefficient a, m_1..m_s.
struct JoeKuo { uint32_t s, a, m[9]; };
extern const JoeKuo JOE_KUO[63];
// MATRICES[d][k]: the direction number XORed in for bit k of the index (Bratley–Fox recurrence).
extern uint32_t SOBOL_MATRICES[64][32];
void init_sobol();

inline uint32_t sobol(uint32_t dim, uint32_t index) {  // sampler.rs:293
    const uint32_t* col = SOBOL_MATRICES[dim % 64];
    uint32_t x = 0;
    while (index) {
        uint32_t k = (uint32_t)__builtin_ctz(index);
        x ^= col[k];
        index &= index - 1;
    }
    return x;
}
inline uint32_t reverse_bits(uint32_t v) {
    v = ((v >> 1) & 0x55555555u) | ((v & 0x55555555u) << 1);
    v = ((v >> 2) & 0x33333333u) | ((v & 0x33333333u) << 2);
    v = ((v >> 4) & 0x0F0F0F0Fu) | ((v & 0x0F0F0F0Fu) << 4);
    v = ((v >> 8) & 0x00FF00FFu) | ((v & 0x00FF00FFu) << 8);
    return (v >> 16) | (v << 16);
}
inline uint32_t owen_scramble(uint32_t x, uint32_t seed) {  // sampler.rs:310 (Burley 2020)
    uint32_t v = reverse_bits(x);
    v += seed;
    v ^= v * 0x6c50b47cu;
    v ^= v * 0xb82f1e52u;
    v ^= v * 0xc7afe638u;
    v ^= v * 0x8d22f6e6u;
    return reverse_bits(v);
}
inline float to_unit(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

struct PixelSampler {  // sampler.rs:331
    uint64_t key;
    uint32_t index;
    PixelSampler(uint32_t seed, uint32_t x, uint32_t y, uint32_t idx) {
        uint64_t pixel = ((uint64_t)y << 32) | (uint64_t)x;
        key = mix64(pixel ^ mix64((uint64_t)seed ^ 0x5851f42d4c957f2dULL));
        index = idx;
    }
    uint64_t dim_seed(uint32_t dim) const {
        return mix64(key ^ ((uint64_t)(dim + 1) * 0x9e3779b97f4a7c15ULL));
    }
    float get1(uint32_t dim) const {
        uint64_t seed = dim_seed(dim);
        if (dim < 64) {
            uint32_t x = sobol(LAYOUT[dim], index);
            return to_unit(owen_scramble(x, (uint32_t)(seed >> 32)));
        }
        return to_unit((uint32_t)(mix64(seed ^ (uint64_t)index) >> 32));
    }
    void get2(uint32_t dim, float& a, float& b) const { a = get1(dim); b = get1(dim + 1); }
};

// ---- warp.rs --------------------------------------------------------------------------------
inline void concentric_disk(float u0, float u1, float& ox, float& oy) {  // warp.rs:12
    float a = 2.0f * u0 - 1.0f;
    float b = 2.0f * u1 - 1.0f;
    if (a == 0.0f && b == 0.0f) { ox = 0.0f; oy = 0.0f; return; }
    float r, phi;
    if (std::fabs(a) > std::fabs(b)) { r = a; phi = FRAC_PI_4 * (b / a); }
    else { r = b; phi = FRAC_PI_2 - FRAC_PI_4 * (a / b); }
    float s, c;
    sin_cos(phi, s, c);
    ox = r * c;
    oy = r * s;
}
inline Vec3 cosine_hemisphere(float u0, float u1) {  // warp.rs:30
    float x, y;
    concentric_disk(u0, u1, x, y);
    float z = std::sqrt(rmax(1.0f - x * x - y * y, 0.0f));
    return {x, y, z};
}

}  // namespace orc
