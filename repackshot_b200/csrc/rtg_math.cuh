// Deterministic maths shared by the host preparation and the sm_100a kernels: the elementary
// functions, vectors, frames, the Owen-scrambled Sobol sampler and the warps of the Repackshot
// engine (engine/crates/rt-core/src/fmath.rs:35-270, math.rs:1-400, rng.rs:1-55,
// sampler.rs:83-368, warp.rs:12-41, color.rs:45-47).
//
// Every expression is written in the reference's operation order. The device code is built with
// -fmad=false -prec-div=true -prec-sqrt=true -ftz=false and the host code with
// -ffp-contract=off, so each operation is one IEEE round-to-nearest step and the results are the
// reference's bits.
#pragma once
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define RTG_HD __host__ __device__ __forceinline__
#define RTG_D __device__ __forceinline__
// Large functions called from several places of a kernel: kept out of line on the device so the
// shade kernel's code stays small enough for the instruction cache. Internal linkage, so that
// several translation units can include them.
#define RTG_HD_NI static __host__ __device__ __noinline__
#define RTG_D_NI static __device__ __noinline__
#else
#define RTG_HD inline
#define RTG_D inline
#define RTG_HD_NI inline
#define RTG_D_NI inline
#endif

namespace rtg {

#define RTG_INF __int_as_float(0x7f800000)

RTG_HD uint32_t fbits(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u; std::memcpy(&u, &f, 4); return u;
#endif
}
RTG_HD float bitsf(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f; std::memcpy(&f, &u, 4); return f;
#endif
}
RTG_HD float f_inf() { return bitsf(0x7f800000u); }
constexpr float F_MAX = 3.40282347e+38f;
RTG_HD bool finitef(float x) { return (fbits(x) & 0x7f800000u) != 0x7f800000u; }
RTG_HD float absf(float x) { return bitsf(fbits(x) & 0x7fffffffu); }
RTG_HD bool signbitf(float x) { return (fbits(x) >> 31) != 0; }
RTG_HD float copysign_(float m, float s) { return bitsf((fbits(m) & 0x7fffffffu) | (fbits(s) & 0x80000000u)); }
RTG_HD float sqrt_(float x) {
#ifdef __CUDA_ARCH__
    return __fsqrt_rn(x);
#else
    return __builtin_sqrtf(x);
#endif
}
RTG_HD float floor_(float x) {
#ifdef __CUDA_ARCH__
    return floorf(x);
#else
    return __builtin_floorf(x);
#endif
}
// f32::min / f32::max of the reference: the other operand when one is NaN.
RTG_HD float rmin(float a, float b) { if (a != a) return b; if (b != b) return a; return a < b ? a : b; }
RTG_HD float rmax(float a, float b) { if (a != a) return b; if (b != b) return a; return a > b ? a : b; }
RTG_HD float rclamp(float x, float lo, float hi) { if (x < lo) x = lo; if (x > hi) x = hi; return x; }
// `as i32` / `as i64` / `as usize` of the reference: truncation, saturating, NaN -> 0.
RTG_HD int32_t f2i32(float x) {
    if (x != x) return 0;
    if (x >= 2147483648.0f) return 2147483647;
    if (x <= -2147483648.0f) return (-2147483647 - 1);
    return (int32_t)x;
}
RTG_HD int64_t f2i64(float x) {
    if (x != x) return 0;
    if (x >= 9.2233720368547758e18f) return 9223372036854775807LL;
    if (x <= -9.2233720368547758e18f) return (-9223372036854775807LL - 1);
    return (int64_t)x;
}
RTG_HD uint32_t f2u32_floor_nonneg(float x) {  // `as usize` for values known below 2^32
    if (x != x || x <= 0.0f) return 0;
    if (x >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)x;
}

// ---- fmath.rs --------------------------------------------------------------------------------
constexpr float PI = 3.14159265358979323846f;
constexpr float TAU = 6.28318530717958647692f;
constexpr float FRAC_PI_2 = 1.57079632679489661923f;
constexpr float FRAC_PI_4 = 0.785398163397448309616f;
constexpr float FRAC_1_PI = 0.318309886183790671538f;
constexpr float LN_2 = 0.693147180559945309417f;
constexpr float LOG2_E = 1.44269504088896340736f;
constexpr float SQRT_2 = 1.41421356237309504880f;

RTG_HD void sin_cos(float x, float& so, float& co) {  // fmath.rs:64 (Cody–Waite + Taylor)
    if (!finitef(x)) { so = 0.0f; co = 1.0f; return; }
    const float P1 = 1.5703125f, P2 = 4.837513e-4f, P3 = 7.54979e-8f;
    float k = floor_(x * (2.0f / PI) + 0.5f);
    float r = ((x - k * P1) - k * P2) - k * P3;
    float r2 = r * r;
    float p = 1.0f / 362880.0f;
    p = p * r2 - 1.0f / 5040.0f;
    p = p * r2 + 1.0f / 120.0f;
    p = p * r2 - 1.0f / 6.0f;
    float s = r + r * r2 * p;
    float q = -1.0f / 3628800.0f;
    q = q * r2 + 1.0f / 40320.0f;
    q = q * r2 - 1.0f / 720.0f;
    q = q * r2 + 1.0f / 24.0f;
    q = q * r2 - 0.5f;
    float c = 1.0f + r2 * q;
    switch ((int)(f2i64(k) & 3)) {
        case 0: so = s; co = c; break;
        case 1: so = c; co = -s; break;
        case 2: so = -s; co = -c; break;
        default: so = -c; co = s; break;
    }
}
RTG_HD float fcos(float x) { float s, c; sin_cos(x, s, c); return c; }
RTG_HD float pow2i(int32_t n) { return bitsf(((uint32_t)(n + 127)) << 23); }
RTG_HD float fexp2(float x) {  // fmath.rs:100
    if (x != x) return x;
    if (x >= 128.0f) return f_inf();
    if (x < -150.0f) return 0.0f;
    float k = floor_(x + 0.5f);
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
RTG_HD float flog2(float x) {  // fmath.rs:128
    if (x != x) return x;
    if (x <= 0.0f) return -f_inf();
    if (x == f_inf()) return x;
    int32_t e = 0;
    if (x < 1.17549435e-38f) { x *= 8388608.0f; e = -23; }
    uint32_t bits = fbits(x);
    e += (int32_t)((bits >> 23) & 0xffu) - 127;
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
RTG_HD float fexp(float x) { return fexp2(x * LOG2_E); }
RTG_HD float fln(float x) { return flog2(x) * LN_2; }
RTG_HD float fpow(float x, float y) {  // fmath.rs:174
    if (y == 0.0f) return 1.0f;
    if (x <= 0.0f) return y > 0.0f ? 0.0f : f_inf();
    if (x == 1.0f) return 1.0f;
    return fexp2(y * flog2(x));
}
// atan(u) for |u| <= tan(pi/8): the Taylor series to u^17 (fmath.rs:191).
RTG_HD float atan_taylor(float u) {
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
// Arctangent in [-pi/2, pi/2]: reduced to [0, 1] by atan(a) = pi/2 - atan(1/a), then below
// tan(pi/8) by atan(t) = pi/4 + atan((t - 1)/(t + 1)) (fmath.rs:206).
RTG_HD float fatan(float x) {
    if (x != x) return x;
    float a = absf(x);
    bool flip = a > 1.0f;
    float t = flip ? 1.0f / a : a;
    float r = t > 0.41421357f ? FRAC_PI_4 + atan_taylor((t - 1.0f) / (t + 1.0f)) : atan_taylor(t);
    if (flip) r = FRAC_PI_2 - r;
    return x < 0.0f ? -r : r;
}
// Four-quadrant arctangent of y / x in [-pi, pi]; atan2(0, 0) = 0 (fmath.rs:227).
RTG_HD float fatan2(float y, float x) {
    if (x != x || y != y) return bitsf(0x7fc00000u);
    if (x == 0.0f) return y > 0.0f ? FRAC_PI_2 : (y < 0.0f ? -FRAC_PI_2 : 0.0f);
    if (absf(y) <= absf(x)) {
        float r = fatan(y / x);
        if (!(x < 0.0f)) return r;
        return y < 0.0f ? r - PI : r + PI;
    }
    return y > 0.0f ? FRAC_PI_2 - fatan(x / y) : -FRAC_PI_2 - fatan(x / y);
}
// Arccosine in [0, pi] of x clamped to [-1, 1] (fmath.rs:253).
RTG_HD float facos(float x) {
    x = rclamp(x, -1.0f, 1.0f);
    return fatan2(sqrt_((1.0f - x) * (1.0f + x)), x);
}

// ---- math.rs / color.rs ------------------------------------------------------------------------
struct V3 { float x, y, z; };
RTG_HD V3 v3(float x, float y, float z) { V3 v; v.x = x; v.y = y; v.z = z; return v; }
RTG_HD V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
RTG_HD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
RTG_HD V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
RTG_HD V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
RTG_HD V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
RTG_HD V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
RTG_HD bool veq(V3 a, V3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
RTG_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
RTG_HD V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
RTG_HD float len2(V3 a) { return dot(a, a); }
RTG_HD float len(V3 a) { return sqrt_(len2(a)); }
RTG_HD V3 normalize(V3 a) { float l = len(a); return (l > 0.0f && finitef(l)) ? a / l : a; }
RTG_HD bool vfinite(V3 a) { return finitef(a.x) && finitef(a.y) && finitef(a.z); }
RTG_HD float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

struct Rgb { float r, g, b; };
RTG_HD Rgb rgb(float r, float g, float b) { Rgb c; c.r = r; c.g = g; c.b = b; return c; }
RTG_HD Rgb splat(float v) { return rgb(v, v, v); }
RTG_HD Rgb operator+(Rgb a, Rgb b) { return rgb(a.r + b.r, a.g + b.g, a.b + b.b); }
RTG_HD Rgb operator*(Rgb a, Rgb b) { return rgb(a.r * b.r, a.g * b.g, a.b * b.b); }
RTG_HD Rgb operator*(Rgb a, float s) { return rgb(a.r * s, a.g * s, a.b * s); }
RTG_HD Rgb operator/(Rgb a, float s) { return rgb(a.r / s, a.g / s, a.b / s); }
RTG_HD float luminance(Rgb c) { return 0.2126f * c.r + 0.7152f * c.g + 0.0722f * c.b; }
RTG_HD float peak(Rgb c) { return rmax(rmax(c.r, c.g), c.b); }

struct Frame { V3 x, y, z; };
RTG_HD Frame frame_from_normal(V3 n) {  // math.rs:263 (Duff et al. 2017)
    float sign = copysign_(1.0f, n.z);
    float a = -1.0f / (sign + n.z);
    float b = n.x * n.y * a;
    Frame f;
    f.x = v3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    f.y = v3(b, sign + n.y * n.y * a, -n.y);
    f.z = n;
    return f;
}
RTG_HD V3 to_local(const Frame& f, V3 v) { return v3(dot(v, f.x), dot(v, f.y), dot(v, f.z)); }
RTG_HD V3 to_world(const Frame& f, V3 v) { return f.x * v.x + f.y * v.y + f.z * v.z; }

RTG_HD float offset_axis(float p, float n) {  // math.rs:293 (Wächter & Binder 2019)
    if (absf(p) < 1.0f / 32.0f) return p + (1.0f / 65536.0f) * n;
    int32_t of = f2i32(256.0f * n);
    uint32_t moved = fbits(p) + (uint32_t)(p < 0.0f ? -of : of);
    float q = bitsf(moved);
    return finitef(q) ? q : p;
}
RTG_HD V3 offset_origin(V3 p, V3 n) { return v3(offset_axis(p.x, n.x), offset_axis(p.y, n.y), offset_axis(p.z, n.z)); }

// ---- rng.rs / sampler.rs -------------------------------------------------------------------------
RTG_HD uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
RTG_HD uint32_t brev(uint32_t v) {
#ifdef __CUDA_ARCH__
    return __brev(v);
#else
    v = ((v >> 1) & 0x55555555u) | ((v & 0x55555555u) << 1);
    v = ((v >> 2) & 0x33333333u) | ((v & 0x33333333u) << 2);
    v = ((v >> 4) & 0x0F0F0F0Fu) | ((v & 0x0F0F0F0Fu) << 4);
    v = ((v >> 8) & 0x00FF00FFu) | ((v & 0x00FF00FFu) << 8);
    return (v >> 16) | (v << 16);
#endif
}
RTG_HD int ctz32(uint32_t v) {
#ifdef __CUDA_ARCH__
    return __ffs((int)v) - 1;
#else
    return __builtin_ctz(v);
#endif
}
RTG_HD uint32_t owen_scramble(uint32_t x, uint32_t seed) {  // sampler.rs:310 (Burley 2020)
    uint32_t v = brev(x);
    v += seed;
    v ^= v * 0x6c50b47cu;
    v ^= v * 0xb82f1e52u;
    v ^= v * 0xc7afe638u;
    v ^= v * 0x8d22f6e6u;
    return brev(v);
}
RTG_HD float to_unit(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

constexpr uint32_t DIM_CAMERA = 0, DIM_LENS = 2;
RTG_HD uint32_t bounce_dim(uint32_t b) { return 4u + b * 6u; }
constexpr uint32_t OFF_LIGHT_SELECT = 0, OFF_LIGHT = 1, OFF_BSDF = 3, OFF_ROULETTE = 5;

// The sampler reads the generator matrices (64 dims x 32 columns) and the logical->Sobol layout
// from a table the caller provides (constant memory on the device).
struct SobolTable { uint32_t m[64][32]; uint32_t layout[64]; };

RTG_HD uint64_t pixel_key(uint32_t seed, uint32_t x, uint32_t y) {  // sampler.rs:339
    uint64_t pixel = ((uint64_t)y << 32) | (uint64_t)x;
    return mix64(pixel ^ mix64((uint64_t)seed ^ 0x5851f42d4c957f2dULL));
}
RTG_HD float sample1(const SobolTable& T, uint64_t key, uint32_t index, uint32_t dim) {  // sampler.rs:353
    uint64_t seed = mix64(key ^ ((uint64_t)(dim + 1) * 0x9e3779b97f4a7c15ULL));
    if (dim < 64) {
        const uint32_t* col = T.m[T.layout[dim]];
        uint32_t bits = index, x = 0;
        while (bits) { x ^= col[ctz32(bits)]; bits &= bits - 1; }
        return to_unit(owen_scramble(x, (uint32_t)(seed >> 32)));
    }
    return to_unit((uint32_t)(mix64(seed ^ (uint64_t)index) >> 32));
}

// ---- warp.rs ------------------------------------------------------------------------------------
RTG_HD void concentric_disk(float u0, float u1, float& ox, float& oy) {
    float a = 2.0f * u0 - 1.0f;
    float b = 2.0f * u1 - 1.0f;
    if (a == 0.0f && b == 0.0f) { ox = 0.0f; oy = 0.0f; return; }
    float r, phi;
    if (absf(a) > absf(b)) { r = a; phi = FRAC_PI_4 * (b / a); }
    else { r = b; phi = FRAC_PI_2 - FRAC_PI_4 * (a / b); }
    float s, c;
    sin_cos(phi, s, c);
    ox = r * c;
    oy = r * s;
}
RTG_HD V3 cosine_hemisphere(float u0, float u1) {
    float x, y;
    concentric_disk(u0, u1, x, y);
    return v3(x, y, sqrt_(rmax(1.0f - x * x - y * y, 0.0f)));
}

}  // namespace rtg

namespace rtg {
// PCG-XSH-RR 64/32 (rng.rs:21-44), used by the host-side energy-table generator.
struct Pcg32 {
    uint64_t state, inc;
};
RTG_HD uint32_t pcg_next(Pcg32& r) {
    uint64_t old = r.state;
    r.state = old * 6364136223846793005ULL + r.inc;
    uint32_t xorshifted = (uint32_t)(((old >> 18) ^ old) >> 27);
    uint32_t rot = (uint32_t)(old >> 59);
    return (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
}
RTG_HD Pcg32 pcg_seeded(uint64_t seed, uint64_t stream) {
    Pcg32 r;
    r.state = 0;
    r.inc = (stream << 1) | 1;
    pcg_next(r);
    r.state += seed;
    pcg_next(r);
    return r;
}
RTG_HD float pcg_f32(Pcg32& r) { return (float)(pcg_next(r) >> 8) * (1.0f / 16777216.0f); }
}  // namespace rtg

#if !defined(__CUDACC__)
// Host builds of the device headers (the CPU-side checks of the traversal): the CUDA intrinsics
// the kernels use, with their documented results.
#include <vector_types.h>
template <class T>
inline T __ldg(const T* p) { return *p; }
inline int __ffs(int x) { return __builtin_ffs(x); }
inline int __popc(uint32_t x) { return __builtin_popcount(x); }
inline uint32_t __float_as_uint(float f) { return rtg::fbits(f); }
inline float __uint_as_float(uint32_t u) { return rtg::bitsf(u); }
#endif
