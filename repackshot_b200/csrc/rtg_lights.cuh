// The shapes of the lights (engine/crates/rt-core/src/light.rs:140-470, warp.rs:38): area lights,
// suns and sphere lights (points and spots), host and device alike. The host uses the sphere's
// mask for the static selection weights, the device everything.
#pragma once
#include "rtg_dev.h"

namespace rtg {

RTG_HD V3 ld3(const float* p) { return v3(p[0], p[1], p[2]); }

// ---- area lights --------------------------------------------------------------------------------
RTG_HD float orientation_bound(V3 v, float d2, V3 axis, float bound) {  // light.rs:260 with θo = 0
    if (d2 <= bound * bound) return 1.0f;
    const float cos_o = 1.0f, sin_o = 0.0f;
    float inv_d = 1.0f / sqrt_(d2);
    float sin_u = bound * inv_d;
    float cos_u = sqrt_(rmax(1.0f - sin_u * sin_u, 0.0f));
    float cos_s = cos_o * cos_u - sin_o * sin_u;
    float sin_s = sin_o * cos_u + cos_o * sin_u;
    if (sin_s < 0.0f) return 1.0f;
    float cos_t = dot(v, axis) * inv_d;
    if (cos_t >= cos_s) return 1.0f;
    float sin_t = sqrt_(rmax(1.0f - cos_t * cos_t, 0.0f));
    return rmax(cos_t * cos_s + sin_t * sin_s, 0.0f);
}
RTG_HD float area_weight(const LightDev& a, V3 x) {
    V3 v = x - ld3(a.centre);
    float d2 = len2(v);
    float o = orientation_bound(v, d2, ld3(a.fz), a.bound);
    if (o <= 0.0f) return 0.0f;
    return a.base * o / (rmax(d2, a.area) * 1.0e-6f);
}
RTG_HD Rgb area_radiance(const LightDev& a, float cos) {
    Rgb r = rgb(a.radiance[0], a.radiance[1], a.radiance[2]);
    return a.exponent == 0.0f ? r : r * fpow(cos, a.exponent);
}
RTG_HD bool area_intersect(const LightDev& a, V3 o, V3 d, float tmin, float tmax, float& t, float& cos) {
    V3 n = ld3(a.fz);
    float denom = dot(d, n);
    if (denom >= 0.0f) return false;
    t = dot(ld3(a.centre) - o, n) / denom;
    if (!(t > tmin && t < tmax)) return false;
    V3 q = (o + d * t) - ld3(a.centre);
    float x = dot(q, ld3(a.fx)), y = dot(q, ld3(a.fy));
    bool inside = a.rect ? (absf(x) <= a.half_x && absf(y) <= a.half_y) : (x * x + y * y <= a.radius * a.radius);
    if (!inside) return false;
    cos = -denom;
    return true;
}

// ---- suns ---------------------------------------------------------------------------------------
// A direction inside the disc of a sun that is not a delta (light.rs:319).
RTG_HD bool sun_contains(const LightDev& s, V3 dir) { return !s.delta && dot(dir, ld3(s.fz)) >= s.cos_max; }

// Uniform direction in the cone about +z with 1 - cos θmax = one_minus_cos_max (warp.rs:38).
RTG_HD V3 uniform_cone(float u0, float u1, float one_minus_cos_max) {
    float one_minus_cos = u0 * one_minus_cos_max;
    float cos = 1.0f - one_minus_cos;
    float sin = sqrt_(rmax(one_minus_cos * (2.0f - one_minus_cos), 0.0f));
    float sp, cp;
    sin_cos(TAU * u1, sp, cp);
    return v3(sin * cp, sin * sp, cos);
}

// ---- sphere lights (points and spots) -------------------------------------------------------------
// How much of its light reaches x: 1 for a point light; for a spot a smoothstep from 0 at the
// edge of its cone to 1 at its inner cone, by the direction from its centre (light.rs:368).
RTG_HD float sphere_mask(const LightDev& l, V3 x) {
    if (l.cos_outer < -1.0f) return 1.0f;
    V3 d = x - ld3(l.centre);
    float n2 = len2(d);
    if (!(n2 > 0.0f)) return 0.0f;
    float c = dot(d, ld3(l.fz)) / sqrt_(n2);
    if (c <= l.cos_outer) return 0.0f;
    if (c >= l.cos_inner) return 1.0f;
    float t = (c - l.cos_outer) / (l.cos_inner - l.cos_outer);
    return t * t * (3.0f - 2.0f * t);
}
// 1 - cos θmax of the cone the sphere fills seen from dist2 (mm²) away; false from inside it; 0
// below 1e-7, where it is a point (light.rs:398).
RTG_HD bool sphere_cone(const LightDev& l, float dist2, float& omc) {
    float r2 = l.radius * l.radius;
    if (!(dist2 - r2 > 0.0f)) return false;
    float sin2 = r2 / dist2;
    omc = sin2 / (1.0f + sqrt_(rmax(1.0f - sin2, 0.0f)));
    if (omc < 1.0e-7f) omc = 0.0f;
    return true;
}
// Where a ray of unit direction meets the sphere from outside in (tmin, tmax) (light.rs:409).
RTG_HD bool sphere_intersect(const LightDev& l, V3 o, V3 d, float tmin, float tmax, float& t) {
    if (!(l.radius > 0.0f)) return false;
    V3 oc = o - ld3(l.centre);
    float r2 = l.radius * l.radius;
    if (len2(oc) <= r2) return false;
    float b = dot(oc, d);
    float disc = r2 - len2(oc - d * b);
    if (disc < 0.0f) return false;
    t = -b - sqrt_(disc);
    return t > tmin && t < tmax;
}
// Selection weight at x: lum(I) mask(x) / max(d², r²) in m² (light.rs:430).
RTG_HD float sphere_weight(const LightDev& l, V3 x) {
    float m = sphere_mask(l, x);
    if (m <= 0.0f) return 0.0f;
    float d2 = len2(x - ld3(l.centre)) * 1.0e-6f;
    return l.base * m / rmax(d2, l.near2);
}

}  // namespace rtg
