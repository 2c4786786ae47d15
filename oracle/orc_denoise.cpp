// Test infrastructure: the CPU restatement the CUDA path is checked against, never shipped.
//
// The denoiser (engine/crates/rt-post/src/denoise.rs:44-788): an edge-avoiding a-trous wavelet
// filter guided by the exact passes and each pixel's sample variance, in f32 and in the
// reference's order of operations, and its input format (rt-wasm/src/lib.rs:420-475).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr uint32_t LEVELS = 5;                  // denoise.rs:48
constexpr float SIGMA_LUMINANCE = 4.0f;         // denoise.rs:50
constexpr float SIGMA_DEPTH = 1.0f;             // denoise.rs:54
constexpr float SIGMA_ALBEDO = 0.1f;            // denoise.rs:56
constexpr uint32_t MIN_SAMPLES_FOR_VARIANCE = 4;  // denoise.rs:58
constexpr float MIN_ALBEDO = 0.01f;             // denoise.rs:121
constexpr float FIREFLY_RATIO = 4.0f;           // denoise.rs:123
constexpr float FIREFLY_FLOOR = 0.05f;          // denoise.rs:125
constexpr float KERNEL[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
constexpr float GAUSS3[3] = {0.25f, 0.5f, 0.25f};

struct Preset {  // denoise.rs:66-119
    uint32_t levels, variance_radius;
    uint32_t halo() const { return (2u << levels) + 8u; }
};

// Rust's f32::max and min: a NaN operand gives the other one.
float fmax_rs(float a, float b) { return a != a ? b : (b != b ? a : (a > b ? a : b)); }
float luminance(float r, float g, float b) { return 0.2126f * r + 0.7152f * g + 0.0722f * b; }
float pow128(float x) {
    float v = x;
    for (int i = 0; i < 7; ++i) v *= v;
    return v;
}
float falloff(float x) {  // denoise.rs:770
    float t = 1.0f - x * (1.0f / 16.0f);
    if (std::isnan(t) || t <= 0.0f) return 0.0f;
    t = t * t;
    t = t * t;
    t = t * t;
    return t * t;
}

struct Guide {
    uint32_t part, material;
    float n[3], z, dz[2], a[3];
    bool foreground() const { return part != 0; }
    bool same_surface(const Guide& o) const { return part == o.part && material == o.material; }
};
float dot3(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
float depth_term(const Guide& g, const Guide& q, float dx, float dy) {  // denoise.rs:751
    if (!(std::isfinite(g.z) && std::isfinite(q.z))) return g.z == q.z ? 0.0f : INFINITY;
    const float expected = std::fabs(g.dz[0] * dx + g.dz[1] * dy);
    const float eps = 1.0e-3f * std::fabs(g.z) + 1.0e-6f;
    return std::fabs(g.z - q.z) / (SIGMA_DEPTH * expected + eps);
}
float albedo_term(const Guide& g, const Guide& q) {
    return (std::fabs(g.a[0] - q.a[0]) + std::fabs(g.a[1] - q.a[1]) + std::fabs(g.a[2] - q.a[2])) / SIGMA_ALBEDO;
}
float surface_weight(const Guide& g, const Guide& q, float dx, float dy) {
    return pow128(fmax_rs(dot3(g.n, q.n), 0.0f)) * falloff(depth_term(g, q, dx, dy));
}

struct Input {
    uint32_t width, height, origin_y, rows, samples;
    const float *sums, *lum2, *albedo, *normal, *depth, *counts;
    const uint32_t *part, *material;
};

// filter_band (denoise.rs:435): RGBA sums of the whole band.
std::vector<float> filter_band(const Input& in, Preset preset) {
    const size_t w = in.width, h = in.rows, n = w * h;
    const uint32_t samples = in.samples > 1 ? in.samples : 1;
    const float inv = 1.0f / (float)samples;
    std::vector<float> out(in.sums, in.sums + n * 4);
    std::vector<Guide> guides(n);
    auto finite = [](float v) { return std::isfinite(v) ? v : 0.0f; };
    for (size_t p = 0; p < n; ++p) {
        Guide& g = guides[p];
        g.part = in.part[p];
        g.material = in.material[p];
        for (int k = 0; k < 3; ++k) {
            g.n[k] = finite(in.normal[p * 3 + k]);
            g.a[k] = finite(in.albedo[p * 3 + k]);
        }
        g.z = in.depth[p];
        g.dz[0] = g.dz[1] = 0.0f;
    }
    for (size_t y = 0; y < h; ++y)
        for (size_t x = 0; x < w; ++x) {
            const size_t p = y * w + x;
            const Guide g = guides[p];
            if (!g.foreground() || !std::isfinite(g.z)) continue;
            auto zq = [&](bool has, size_t q, float& z) {
                if (!has || !guides[q].same_surface(g) || !std::isfinite(guides[q].z)) return false;
                z = guides[q].z;
                return true;
            };
            auto grad = [&](bool ha, size_t a, bool hb, size_t b) {
                float za = 0, zb = 0;
                const bool sa = zq(ha, a, za), sb = zq(hb, b, zb);
                if (sa && sb) return 0.5f * (zb - za);
                if (sa) return g.z - za;
                if (sb) return zb - g.z;
                return 0.0f;
            };
            guides[p].dz[0] = grad(x > 0, p - 1, x + 1 < w, p + 1);
            guides[p].dz[1] = grad(y > 0, p - w, y + 1 < h, p + w);
        }
    std::vector<float> divisor(n * 3, 1.0f), light(n * 3, 0.0f), var(n, 0.0f);
    for (size_t p = 0; p < n; ++p) {
        const Guide& g = guides[p];
        if (!g.foreground()) continue;
        const float c[3] = {in.sums[p * 4] * inv, in.sums[p * 4 + 1] * inv, in.sums[p * 4 + 2] * inv};
        for (int k = 0; k < 3; ++k) {
            const float d = fmax_rs(g.a[k], MIN_ALBEDO);
            divisor[p * 3 + k] = d;
            light[p * 3 + k] = c[k] / d;
        }
        const bool own = in.counts != nullptr;
        const bool enough = own ? in.counts[p] >= (float)MIN_SAMPLES_FOR_VARIANCE : samples >= MIN_SAMPLES_FOR_VARIANCE;
        if (enough) {
            const float l = luminance(c[0], c[1], c[2]);
            const float m2 = in.lum2[p] * inv;
            const float dof = own ? in.counts[p] - 1.0f : (float)(samples - 1);
            const float v = fmax_rs(m2 - l * l, 0.0f) / dof;
            const float ld = luminance(divisor[p * 3], divisor[p * 3 + 1], divisor[p * 3 + 2]);
            var[p] = v / (ld * ld);
        }
    }
    auto lum_of = [](const std::vector<float>& li, size_t p) { return luminance(li[p * 3], li[p * 3 + 1], li[p * 3 + 2]); };
    std::vector<float> before(n);
    for (size_t p = 0; p < n; ++p) before[p] = lum_of(light, p);
    for (size_t y = 0; y < h; ++y)
        for (size_t x = 0; x < w; ++x) {
            const size_t p = y * w + x;
            const Guide& g = guides[p];
            if (!g.foreground()) continue;
            float brightest = 0.0f, vmax = 0.0f;
            uint32_t count = 0;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const long qx = (long)x + dx, qy = (long)y + dy;
                    if ((dx == 0 && dy == 0) || qx < 0 || qy < 0 || qx >= (long)w || qy >= (long)h) continue;
                    const size_t q = (size_t)qy * w + (size_t)qx;
                    if (!g.same_surface(guides[q])) continue;
                    brightest = fmax_rs(brightest, before[q]);
                    vmax = fmax_rs(vmax, var[q]);  // the raster order's earlier pixels already clamped
                    ++count;
                }
            const float limit = FIREFLY_RATIO * brightest + FIREFLY_FLOOR;
            if (count >= 3 && before[p] > limit) {
                const float k = limit / before[p];
                for (int c = 0; c < 3; ++c) light[p * 3 + c] *= k;
                var[p] = vmax;
            }
        }
    auto few = [&](size_t p) {
        return in.counts ? in.counts[p] < (float)MIN_SAMPLES_FOR_VARIANCE : samples < MIN_SAMPLES_FOR_VARIANCE;
    };
    bool any_few = false;
    for (size_t p = 0; p < n && !any_few; ++p) any_few = few(p);
    if (any_few) {
        const int r = (int)preset.variance_radius;
        for (size_t y = 0; y < h; ++y)
            for (size_t x = 0; x < w; ++x) {
                const size_t p = y * w + x;
                const Guide& g = guides[p];
                if (!g.foreground() || !few(p)) continue;
                float sw = 0.0f, m1 = 0.0f, m2 = 0.0f;
                for (int dy = -r; dy <= r; ++dy) {
                    const long qy = (long)y + dy;
                    if (qy < 0 || qy >= (long)h) continue;
                    for (int dx = -r; dx <= r; ++dx) {
                        const long qx = (long)x + dx;
                        if (qx < 0 || qx >= (long)w) continue;
                        const size_t q = (size_t)qy * w + (size_t)qx;
                        const Guide& gq = guides[q];
                        if (!g.same_surface(gq)) continue;
                        const float wgt = surface_weight(g, gq, (float)dx, (float)dy);
                        const float l = lum_of(light, q);
                        sw += wgt;
                        m1 += wgt * l;
                        m2 += wgt * l * l;
                    }
                }
                if (sw > 0.0f) {
                    m1 /= sw;
                    m2 /= sw;
                    var[p] = fmax_rs(m2 - m1 * m1, 0.0f);
                }
            }
    }
    std::vector<float> next_light = light, next_var = var, gvar(n, 0.0f), lum(n, 0.0f);
    for (uint32_t level = 0; level < preset.levels; ++level) {
        const int step = 1 << level;
        for (size_t p = 0; p < n; ++p) lum[p] = lum_of(light, p);
        for (size_t y = 0; y < h; ++y)
            for (size_t x = 0; x < w; ++x) {
                const size_t p = y * w + x;
                const Guide& g = guides[p];
                if (!g.foreground()) continue;
                float sw = 0.0f, sv = 0.0f;
                for (int j = 0; j < 3; ++j) {
                    const long qy = (long)y + j - 1;
                    if (qy < 0 || qy >= (long)h) continue;
                    for (int i = 0; i < 3; ++i) {
                        const long qx = (long)x + i - 1;
                        if (qx < 0 || qx >= (long)w) continue;
                        const size_t q = (size_t)qy * w + (size_t)qx;
                        if (!g.same_surface(guides[q])) continue;
                        const float k = GAUSS3[j] * GAUSS3[i];
                        sw += k;
                        sv += k * var[q];
                    }
                }
                gvar[p] = sw > 0.0f ? sv / sw : var[p];
            }
        for (size_t y = 0; y < h; ++y)
            for (size_t x = 0; x < w; ++x) {
                const size_t p = y * w + x;
                const Guide& g = guides[p];
                if (!g.foreground()) continue;
                const float lp = lum[p];
                const float inv_sigma_l = 1.0f / (SIGMA_LUMINANCE * std::sqrt(fmax_rs(gvar[p], 0.0f) + 1.0e-10f));
                float sw = 0.0f, sv = 0.0f, sc[3] = {0.0f, 0.0f, 0.0f};
                for (int j = 0; j < 5; ++j) {
                    const int dy = (j - 2) * step;
                    const long qy = (long)y + dy;
                    if (qy < 0 || qy >= (long)h) continue;
                    for (int i = 0; i < 5; ++i) {
                        const int dx = (i - 2) * step;
                        const long qx = (long)x + dx;
                        if (qx < 0 || qx >= (long)w) continue;
                        const size_t q = (size_t)qy * w + (size_t)qx;
                        const Guide& gq = guides[q];
                        if (!g.same_surface(gq)) continue;
                        const float wn = q == p ? 1.0f : pow128(fmax_rs(dot3(g.n, gq.n), 0.0f));
                        if (wn <= 0.0f) continue;
                        const float exponent = std::fabs(lp - lum[q]) * inv_sigma_l + depth_term(g, gq, (float)dx, (float)dy) + albedo_term(g, gq);
                        const float wgt = KERNEL[j] * KERNEL[i] * wn * falloff(exponent);
                        sw += wgt;
                        sv += wgt * wgt * var[q];
                        for (int k = 0; k < 3; ++k) sc[k] += wgt * light[q * 3 + k];
                    }
                }
                const float inv_w = 1.0f / sw;
                for (int k = 0; k < 3; ++k) next_light[p * 3 + k] = sc[k] * inv_w;
                next_var[p] = sv * inv_w * inv_w;
            }
        std::swap(light, next_light);
        std::swap(var, next_var);
    }
    const float count = (float)samples;
    for (size_t p = 0; p < n; ++p) {
        if (!guides[p].foreground()) continue;
        for (int k = 0; k < 3; ++k) {
            const float c = light[p * 3 + k] * divisor[p * 3 + k];
            out[p * 4 + k] = std::isfinite(c) ? c * count : in.sums[p * 4 + k];
        }
    }
    return out;
}

}  // namespace

extern "C" {

// rt_denoise_with (rt-wasm/src/ffi.rs:642, lib.rs:420): preset 0 (full) or 1 (viewport), strength,
// a band of `rows` rows from `origin_y` of a width x height image of `samples` samples; `words`
// holds the planes sums (4), lum2, albedo (3), normal (3), depth, part id, material id (14 words
// a pixel) and, with 15, each pixel's own count. Writes the RGBA sums of rows y0 .. y1. 0, 3 for a
// null pointer, 5 when the preset, the sizes, the band or its halo do not fit.
uint32_t orc_denoise(uint32_t preset_id, float strength, uint32_t width, uint32_t height, uint32_t origin_y, uint32_t rows,
                     uint32_t samples, uint32_t y0, uint32_t y1, const uint32_t* words, uint32_t words_per_pixel, float* out) {
    if (!words || !out) return 3;
    if (preset_id > 1 || (words_per_pixel != 14 && words_per_pixel != 15)) return 5;
    const Preset preset = preset_id == 0 ? Preset{LEVELS, 3} : Preset{3, 1};
    const size_t n = (size_t)width * rows;
    auto f = [&](size_t from) { return reinterpret_cast<const float*>(words + from); };
    Input in{width, height, origin_y, rows, samples, f(0), f(n * 4), f(n * 5), f(n * 8), f(n * 11),
             words_per_pixel == 15 ? f(n * 14) : nullptr, words + n * 12, words + n * 13};
    // check (denoise.rs:274) and check_rows (denoise.rs:347)
    if (width == 0 || (uint64_t)origin_y + rows > height) return 5;
    const uint32_t halo = preset.halo(), band_end = origin_y + rows;
    const uint32_t low = y0 > halo ? y0 - halo : 0;
    const uint64_t high = std::min<uint64_t>((uint64_t)y1 + halo, height);
    if (y0 > y1 || y0 < origin_y || y1 > band_end || origin_y > low || band_end < high) return 5;
    const float s = std::isnan(strength) ? 1.0f : (strength < 0.0f ? 0.0f : (strength > 1.0f ? 1.0f : strength));
    const size_t a = (size_t)(y0 - origin_y) * width * 4, b = (size_t)(y1 - origin_y) * width * 4;
    if (s <= 0.0f) {
        std::memcpy(out, in.sums + a, (b - a) * 4);
        return 0;
    }
    const std::vector<float> band = filter_band(in, preset);
    std::memcpy(out, band.data() + a, (b - a) * 4);
    if (s < 1.0f) {  // blend (denoise.rs:396)
        const float k = 1.0f - s;
        for (size_t i = 0; i < b - a; ++i)
            if (i % 4 != 3) out[i] = in.sums[a + i] * k + out[i] * s;
    }
    return 0;
}

uint32_t orc_denoise_halo(uint32_t preset_id) { return preset_id == 0 ? Preset{LEVELS, 3}.halo() : (preset_id == 1 ? Preset{3, 1}.halo() : 0); }

}  // extern "C"
