// Film output on the device: resolve, exposure, the tone curves and sRGB encoding of the
// Repackshot engine (engine/crates/rt-core/src/color.rs:90-270, image.rs:156-214), each in the
// reference's f32 operations and order, so the 8- and 16-bit images have its bytes.
#pragma once
#include "rtg_math.cuh"

namespace rtg {

// Tone curve values of the RSB RNDR section (color.rs:95-117); any other value is ACES.
constexpr uint32_t TONEMAP_LINEAR = 0, TONEMAP_ACES = 1, TONEMAP_FILMIC = 2, TONEMAP_AGX = 3, TONEMAP_STANDARD = 4;

// AgX's inset and outset matrices, rows (color.rs:206-246). The outset is the inset's inverse by
// cofactors in f32 (agx_matrices), computed once on the host and passed to the kernel.
struct AgxMatrices { float inset[9], outset[9]; };

RTG_HD AgxMatrices agx_matrices() {
    AgxMatrices a;
    const float m[9] = {0.84247906f, 0.0784336f, 0.079223745f, 0.042328242f, 0.8784686f, 0.07916613f, 0.042375655f, 0.0784336f, 0.879143f};
    for (int k = 0; k < 9; ++k) a.inset[k] = m[k];
    float c00 = m[4] * m[8] - m[5] * m[7];
    float c01 = m[5] * m[6] - m[3] * m[8];
    float c02 = m[3] * m[7] - m[4] * m[6];
    float det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    float inv = 1.0f / det;
    a.outset[0] = c00 * inv;
    a.outset[1] = (m[2] * m[7] - m[1] * m[8]) * inv;
    a.outset[2] = (m[1] * m[5] - m[2] * m[4]) * inv;
    a.outset[3] = c01 * inv;
    a.outset[4] = (m[0] * m[8] - m[2] * m[6]) * inv;
    a.outset[5] = (m[2] * m[3] - m[0] * m[5]) * inv;
    a.outset[6] = c02 * inv;
    a.outset[7] = (m[1] * m[6] - m[0] * m[7]) * inv;
    a.outset[8] = (m[0] * m[4] - m[1] * m[3]) * inv;
    return a;
}

RTG_HD float tone_aces(float x) {  // Narkowicz's ACES fit, clamped
    x = rmax(x, 0.0f);
    return rclamp((x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f), 0.0f, 1.0f);
}
RTG_HD float tone_shaper(float x) {  // log2 over [-12.473931, 4.026069] EV to [0, 1]
    const float lo = -12.473931f, hi = 4.026069f;
    float ev = flog2(rmax(x, 1.0e-10f));
    return rclamp((ev - lo) / (hi - lo), 0.0f, 1.0f);
}
RTG_HD float tone_contrast(float x) {  // the sixth-order base-contrast fit, left to right
    float x2 = x * x, x4 = x2 * x2;
    return 15.5f * x4 * x2 - 40.14f * x4 * x + 31.96f * x4 - 6.868f * x2 * x + 0.4298f * x2 + 0.1191f * x - 0.00232f;
}
RTG_HD float tone_display(float y) { return fpow(rclamp(y, 0.0f, 1.0f), 2.2f); }

RTG_HD Rgb tonemap_apply(uint32_t kind, Rgb c, const AgxMatrices& agx) {
    if (kind == TONEMAP_LINEAR) return c;
    if (kind == TONEMAP_FILMIC)
        return rgb(tone_display(tone_contrast(tone_shaper(c.r))), tone_display(tone_contrast(tone_shaper(c.g))),
                   tone_display(tone_contrast(tone_shaper(c.b))));
    if (kind == TONEMAP_AGX) {
        const float* m = agx.inset;
        float r = rmax(c.r, 0.0f), g = rmax(c.g, 0.0f), b = rmax(c.b, 0.0f);
        float i0 = m[0] * r + m[1] * g + m[2] * b, i1 = m[3] * r + m[4] * g + m[5] * b, i2 = m[6] * r + m[7] * g + m[8] * b;
        float k0 = tone_contrast(tone_shaper(i0)), k1 = tone_contrast(tone_shaper(i1)), k2 = tone_contrast(tone_shaper(i2));
        const float* o = agx.outset;
        return rgb(tone_display(o[0] * k0 + o[1] * k1 + o[2] * k2), tone_display(o[3] * k0 + o[4] * k1 + o[5] * k2),
                   tone_display(o[6] * k0 + o[7] * k1 + o[8] * k2));
    }
    if (kind == TONEMAP_STANDARD) return rgb(rclamp(c.r, 0.0f, 1.0f), rclamp(c.g, 0.0f, 1.0f), rclamp(c.b, 0.0f, 1.0f));
    return rgb(tone_aces(c.r), tone_aces(c.g), tone_aces(c.b));
}

RTG_HD float srgb_encode(float linear) {
    float l = rclamp(linear, 0.0f, 1.0f);
    if (l <= 0.0031308f) return l * 12.92f;
    return 1.055f * fpow(l, 1.0f / 2.4f) - 0.055f;
}

// Rust's `as u8` / `as u16` of a float: truncation, saturating, NaN to 0.
RTG_HD uint32_t saturate_cast(float v, float top) {
    if (!(v > 0.0f)) return 0u;
    if (v >= top) return (uint32_t)top;
    return (uint32_t)v;
}

}  // namespace rtg
