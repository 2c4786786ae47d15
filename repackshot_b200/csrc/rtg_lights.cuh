// The shapes of the lights (engine/crates/rt-core/src/light.rs:140-470, warp.rs:38): area lights,
// suns and sphere lights (points and spots), host and device alike. The host uses the sphere's
// mask for the static selection weights, the device everything.
#pragma once
#include "rtg_dev.h"

namespace rtg {

RTG_HD V3 ld3(const float* p) { return v3(p[0], p[1], p[2]); }

// ---- area lights --------------------------------------------------------------------------------
// light.rs:212: the largest cosine between a normal in the cone (axis, half-angle θo) of a light
// bounded by a sphere of radius `bound` and the direction towards a point at v from its centre.
RTG_HD float orientation_bound_cone(V3 v, float d2, V3 axis, float cos_o, float sin_o, float bound) {
    if (d2 <= bound * bound) return 1.0f;
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
RTG_HD float orientation_bound(V3 v, float d2, V3 axis, float bound) {  // θo = 0: a flat light
    return orientation_bound_cone(v, d2, axis, 1.0f, 0.0f, bound);
}
RTG_HD float area_weight(const LightDev& a, V3 x) {
    V3 v = x - ld3(a.centre);
    float d2 = len2(v);
    float o = orientation_bound(v, d2, ld3(a.fz), a.bound);
    if (o <= 0.0f) return 0.0f;
    return a.base * o / (rmax(d2, a.area) * 1.0e-6f);
}
// light.rs:468 MeshEmitter::weight: lum(L) A cos' / max(d^2, A) from its centroid.
RTG_HD float mesh_weight(const LightDev& a, V3 x) {
    V3 v = x - ld3(a.centre);
    float d2 = len2(v);
    float o = a.cos_o <= -1.0f ? 1.0f : orientation_bound_cone(v, d2, ld3(a.fz), a.cos_o, a.sin_o, a.bound);
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

// ---- IES profiles (ies.rs:350-430) ----------------------------------------------------------------
// The cell of an increasing list of n >= 2 angles that holds x: the last one at or below x, at
// most the second last (partition_point(a <= x) - 1, saturating).
RTG_HD uint32_t ies_cell(const float* a, uint32_t n, float x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1;
        else hi = mid;
    }
    const uint32_t i = lo ? lo - 1 : 0;
    return i < n - 2 ? i : n - 2;
}
// phi (degrees) folded into the stored range by the table's symmetry (0 rotational, 1 quadrant,
// 2 bilateral 0-180, 3 bilateral 90-270, 4 full).
RTG_HD float ies_fold(uint32_t sym, float phi) {
    const float p = phi - 360.0f * floor_(phi / 360.0f);
    if (sym == 2) return p > 180.0f ? 360.0f - p : p;
    if (sym == 1) {
        const float q = p > 180.0f ? 360.0f - p : p;
        return q > 90.0f ? 180.0f - q : q;
    }
    if (sym == 3) {
        if (p >= 90.0f && p <= 270.0f) return p;
        const float q = 180.0f - p;
        return q < 0.0f ? q + 360.0f : q;
    }
    return p;
}
// The share of its peak an IES light sends towards the unit direction `local` of its own frame
// (+z its axis, phi = 0 along +y, increasing towards +x): the candela interpolated bilinearly in
// gamma and phi, 0 outside the vertical range, over the peak, at most 1.
RTG_HD float ies_shape(const LightDev& l, V3 local) {
    constexpr float kRad = 180.0f / PI;
    const float* v = l.ies;
    const float* hz = l.ies + l.ies_nv;
    const float* cd = hz + l.ies_nh;
    const uint32_t nv = l.ies_nv, nh = l.ies_nh;
    const float rho = sqrt_(local.x * local.x + local.y * local.y);
    const float gamma = fatan2(rho, local.z) * kRad;
    float intensity = 0.0f;
    if (gamma >= v[0] && gamma <= v[nv - 1]) {
        const uint32_t i = ies_cell(v, nv, gamma);
        const float t = (gamma - v[i]) / (v[i + 1] - v[i]);
        auto along = [&](uint32_t row) {
            const float a = cd[row * nv + i], b = cd[row * nv + i + 1];
            return a + (b - a) * t;
        };
        if (nh == 1) {
            intensity = along(0);
        } else {
            const float p = ies_fold(l.ies_sym, fatan2(local.x, local.y) * kRad);
            const uint32_t j = ies_cell(hz, nh, p);
            const float s = (p - hz[j]) / (hz[j + 1] - hz[j]);
            const float a = along(j), b = along(j + 1);
            intensity = a + (b - a) * s;
        }
    }
    return rmin(intensity / l.ies_peak, 1.0f);
}

// ---- sphere lights (points, spots and IES lights) --------------------------------------------------
// How much of its light reaches x: 1 for a point light; for a spot a smoothstep from 0 at the
// edge of its cone to 1 at its inner cone, by the direction from its centre (light.rs:368).
RTG_HD float sphere_mask(const LightDev& l, V3 x) {
    if (l.ies) {  // L5: the profile's share of its peak towards x, seen from the centre
        const V3 d = x - ld3(l.centre);
        const float n2 = len2(d);
        if (!(n2 > 0.0f)) return 0.0f;
        const V3 u = d / sqrt_(n2);
        return ies_shape(l, v3(dot(u, ld3(l.fx)), dot(u, ld3(l.fy)), dot(u, ld3(l.fz))));
    }
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
