// ORACLE (test infrastructure only). Film output restated from engine/crates/rt-core/src/
// color.rs:90-270 (exposure, the tone curves, sRGB encoding) and image.rs:156-214 (resolve and the
// 8- and 16-bit encoders), with the same f32 operations in the same order. Nothing in the product
// links this file.
#include <cstdint>

#include "orc_core.h"

namespace orc {
namespace {

// color.rs:152 aces_tonemap: Narkowicz's ACES fit, per channel, then clamped.
float aces1(float x) {
    x = rmax(x, 0.0f);
    return rclamp((x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f), 0.0f, 1.0f);
}

// color.rs:162-176: the log2 shaper over [min EV, max EV].
constexpr float SHAPER_MIN = -12.473931f, SHAPER_MAX = 4.026069f;
float shaper(float x) {
    float ev = log2(rmax(x, 1.0e-10f));
    return rclamp((ev - SHAPER_MIN) / (SHAPER_MAX - SHAPER_MIN), 0.0f, 1.0f);
}

// color.rs:181 base_contrast: the sixth-order fit, evaluated left to right as written.
float contrast(float x) {
    float x2 = x * x, x4 = x2 * x2;
    return 15.5f * x4 * x2 - 40.14f * x4 * x + 31.96f * x4 - 6.868f * x2 * x + 0.4298f * x2 + 0.1191f * x - 0.00232f;
}

// color.rs:191: back to display-linear with the 2.2 power.
float display(float y) { return powf_(rclamp(y, 0.0f, 1.0f), 2.2f); }

// color.rs:206-214: the AgX inset rows.
constexpr float INSET[3][3] = {{0.84247906f, 0.0784336f, 0.079223745f},
                               {0.042328242f, 0.8784686f, 0.07916613f},
                               {0.042375655f, 0.0784336f, 0.879143f}};

// color.rs:217 invert3: the inverse by cofactors, in f32.
void invert3(const float m[3][3], float o[3][3]) {
    float c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
    float c01 = m[1][2] * m[2][0] - m[1][0] * m[2][2];
    float c02 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
    float det = m[0][0] * c00 + m[0][1] * c01 + m[0][2] * c02;
    float inv = 1.0f / det;
    o[0][0] = c00 * inv;
    o[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * inv;
    o[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * inv;
    o[1][0] = c01 * inv;
    o[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * inv;
    o[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * inv;
    o[2][0] = c02 * inv;
    o[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * inv;
    o[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * inv;
}

Rgb mul3(const float m[3][3], Rgb c) {
    return Rgb(m[0][0] * c.r + m[0][1] * c.g + m[0][2] * c.b, m[1][0] * c.r + m[1][1] * c.g + m[1][2] * c.b,
               m[2][0] * c.r + m[2][1] * c.g + m[2][2] * c.b);
}

// color.rs:137 Tonemap::apply; unknown values are ACES (color.rs:112).
Rgb tonemap(uint32_t kind, Rgb c) {
    switch (kind) {
        case 0: return c;
        case 2: return Rgb(display(contrast(shaper(c.r))), display(contrast(shaper(c.g))), display(contrast(shaper(c.b))));
        case 3: {
            float outset[3][3];
            invert3(INSET, outset);
            Rgb in = mul3(INSET, Rgb(rmax(c.r, 0.0f), rmax(c.g, 0.0f), rmax(c.b, 0.0f)));
            Rgb curved(contrast(shaper(in.r)), contrast(shaper(in.g)), contrast(shaper(in.b)));
            Rgb out = mul3(outset, curved);
            return Rgb(display(out.r), display(out.g), display(out.b));
        }
        case 4: return Rgb(rclamp(c.r, 0.0f, 1.0f), rclamp(c.g, 0.0f, 1.0f), rclamp(c.b, 0.0f, 1.0f));
        default: return Rgb(aces1(c.r), aces1(c.g), aces1(c.b));
    }
}

// color.rs:255 srgb_encode.
float srgb(float linear) {
    float l = rclamp(linear, 0.0f, 1.0f);
    if (l <= 0.0031308f) return l * 12.92f;
    return 1.055f * powf_(l, 1.0f / 2.4f) - 0.055f;
}

// Rust's `as u8` / `as u16`: truncation, saturating, NaN to 0.
uint32_t sat(float v, float top) {
    if (!(v > 0.0f)) return 0;
    if (v >= top) return (uint32_t)top;
    return (uint32_t)v;
}

}  // namespace
}  // namespace orc

using namespace orc;

extern "C" {

// image.rs:186 to_srgb8_tonemapped / image.rs:200 to_srgb16_tonemapped over film sums (rgb 3n,
// weight n): out8 (3n bytes) and out16 (3n words), either may be null.
void orc_film_encode(const float* rgb, const float* weight, uint32_t n, float ev, uint32_t kind, uint8_t* out8, uint16_t* out16) {
    float gain = exp2(ev);
    for (uint32_t i = 0; i < n; ++i) {
        float w = weight[i];
        Rgb px(0.0f, 0.0f, 0.0f);
        if (w > 0.0f) {
            float inv = 1.0f / w;
            px = Rgb(rgb[3 * i] * inv, rgb[3 * i + 1] * inv, rgb[3 * i + 2] * inv);
        }
        Rgb mapped = tonemap(kind, Rgb(px.r * gain, px.g * gain, px.b * gain));
        float v[3] = {mapped.r, mapped.g, mapped.b};
        for (int c = 0; c < 3; ++c) {
            float e = srgb(v[c]);
            if (out8) out8[3 * i + c] = (uint8_t)sat(e * 255.0f + 0.5f, 255.0f);
            if (out16) out16[3 * i + c] = (uint16_t)sat(e * 65535.0f + 0.5f, 65535.0f);
        }
    }
}

// Film::to_linear_exposed (image.rs:218-221): the resolved film times exposure(ev), no curve, no clamp.
void orc_film_linear(const float* rgb, const float* weight, uint32_t n, float ev, float* out) {
    float gain = exp2(ev);
    for (uint32_t i = 0; i < n; ++i) {
        float w = weight[i];
        float inv = w > 0.0f ? 1.0f / w : 0.0f;
        for (int c = 0; c < 3; ++c) out[3 * i + c] = (w > 0.0f ? rgb[3 * i + c] * inv : 0.0f) * gain;
    }
}

// The single-value functions for the reference's known answers: which 0 exposure, 1 ACES (one
// channel), 2 sRGB encode; 3..7 Tonemap::apply with kind which - 3 on the grey (x, x, x), giving
// its green channel.
void orc_color(uint32_t which, const float* in, uint32_t n, float* out) {
    for (uint32_t i = 0; i < n; ++i) {
        float x = in[i];
        switch (which) {
            case 0: out[i] = exp2(x); break;
            case 1: out[i] = aces1(x); break;
            case 2: out[i] = srgb(x); break;
            default: out[i] = tonemap(which - 3, Rgb(x, x, x)).g; break;
        }
    }
}

// AgX's outset matrix (the inverse of the inset) times the inset, row major: the identity up to
// rounding (color.rs's test of the pair).
void orc_agx_identity(float* out9) {
    float o[3][3];
    invert3(INSET, o);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) out9[3 * r + c] = o[r][0] * INSET[0][c] + o[r][1] * INSET[1][c] + o[r][2] * INSET[2][c];
}

}  // extern "C"
