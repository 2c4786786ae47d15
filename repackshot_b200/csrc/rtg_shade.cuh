// Lights, environment and camera on the device (engine/crates/rt-core/src/light.rs:120-1552,
// environment.rs:275-441, scene/mod.rs:280-359, render.rs:79-97, pixel_filter.rs:103-130).
#pragma once
#include "rtg_trace.cuh"

namespace rtg {

RTG_D V3 ld3(const float* p) { return v3(p[0], p[1], p[2]); }

// ---- environment ramp ---------------------------------------------------------------------------
RTG_D float env_value(const LightsDev& L, float z) {
    z = rclamp(z, -1.0f, 1.0f);
    if (z < 0.0f) return L.env_floor * -z + L.env_horizon * (1.0f + z);
    return L.env_horizon * (1.0f - z) + L.env_zenith * z;
}
RTG_D float env_pdf(const LightsDev& L, V3 dir) {
    if (L.env_total <= 0.0f) return 0.0f;
    return env_value(L, dir.z) / (TAU * L.env_total);
}
RTG_D float invert_linear(float a, float b, float u) {
    float c = u * 0.5f * (a + b);
    float denom = a + sqrt_(rmax(a * a + 2.0f * (b - a) * c, 0.0f));
    return denom > 0.0f ? rclamp(2.0f * c / denom, 0.0f, 1.0f) : 0.0f;
}
RTG_D bool env_sample(const LightsDev& L, float u0, float u1, V3& dir, float& pdf) {
    if (L.env_total <= 0.0f) return false;
    float target = u0 * L.env_total;
    float z;
    if (target < L.env_lower) {
        z = -1.0f + invert_linear(L.env_floor, L.env_horizon, target / L.env_lower);
    } else {
        float upper = L.env_total - L.env_lower;
        z = invert_linear(L.env_horizon, L.env_zenith, rclamp((target - L.env_lower) / upper, 0.0f, 1.0f));
    }
    z = rclamp(z, -1.0f, 1.0f);
    float r = sqrt_(rmax((1.0f - z) * (1.0f + z), 0.0f));
    float s, c;
    sin_cos(TAU * u1, s, c);
    dir = v3(r * c, r * s, z);
    pdf = env_pdf(L, dir);
    return pdf > 0.0f;
}

// ---- area lights --------------------------------------------------------------------------------
RTG_D float orientation_bound(V3 v, float d2, V3 axis, float bound) {  // light.rs:260 with θo = 0
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
RTG_D float area_weight(const AreaLightDev& a, V3 x) {
    V3 v = x - ld3(a.centre);
    float d2 = len2(v);
    float o = orientation_bound(v, d2, ld3(a.fz), a.bound);
    if (o <= 0.0f) return 0.0f;
    return a.base * o / (rmax(d2, a.area) * 1.0e-6f);
}
RTG_D Rgb area_radiance(const AreaLightDev& a, float cos) {
    Rgb r = rgb(a.radiance[0], a.radiance[1], a.radiance[2]);
    return a.exponent == 0.0f ? r : r * fpow(cos, a.exponent);
}
RTG_D bool area_intersect(const AreaLightDev& a, V3 o, V3 d, float tmin, float tmax, float& t, float& cos) {
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

// The selection at a vertex (light.rs:495): its point, the sum of the weights there and whether
// it is the static one. Weights are recomputed from the point with the same operations.
struct Sel { V3 p; float total; bool by_flux; };
RTG_D float entry_weight(const LightsDev& L, int e, V3 x) {
    int a = L.entries[e];
    return a >= 0 ? area_weight(L.areas[a], x) : L.env_base;
}
RTG_D Sel select_at(const LightsDev& L, V3 x) {
    Sel s;
    s.p = x;
    s.total = 0.0f;
    s.by_flux = !(L.per_point && L.n_entries > 0);
    if (!s.by_flux)
        for (int e = 0; e < L.n_entries; ++e) s.total += entry_weight(L, e, x);
    return s;
}
RTG_D float pmf_of(const LightsDev& L, uint32_t entry, const Sel& s) {
    if ((int)entry >= L.n_entries) return 0.0f;
    if (s.by_flux) return L.flux_pmf[entry];
    if (!(s.total > 0.0f && finitef(s.total))) return 0.0f;
    return entry_weight(L, (int)entry, s.p) / s.total;
}
RTG_D float power_heuristic(float pa, float pb) {
    if (!(pa > 0.0f)) return 0.0f;
    float r = pb / pa;
    return 1.0f / (1.0f + r * r);
}

struct LightSample { V3 wi; float distance; Rgb radiance; float pdf; bool glossy, shadow; int area; };  // area: -1 environment

RTG_D_NI bool sample_light(const LightsDev& L, const Sel& s, float u_select, float u0, float u1, LightSample& out) {  // light.rs:1150
    int n = L.n_entries;
    if (n == 0) return false;
    int index = 0;
    float pmf = 0.0f;
    if (s.by_flux) {
        int k = 0;
        while (k < n && L.cdf[k] <= u_select) ++k;
        index = k < n - 1 ? k : n - 1;
        pmf = pmf_of(L, (uint32_t)index, s);
    } else {
        if (!(s.total > 0.0f && finitef(s.total))) return false;
        float acc = 0.0f, lo = 0.0f;
        int last = n - 1;
        for (int e = 0; e <= last; ++e) {
            float w = entry_weight(L, e, s.p);
            acc += w;
            float hi = e == last ? 1.0f : acc / s.total;
            if (hi > u_select || e == last) { index = e; pmf = w / s.total; break; }
            lo = hi;
        }
        (void)lo;
    }
    if (!(pmf > 0.0f)) return false;
    int a = L.entries[index];
    out.area = a;
    if (a >= 0) {
        const AreaLightDev& l = L.areas[a];
        float x, y;
        if (l.rect) { x = (2.0f * u0 - 1.0f) * l.half_x; y = (2.0f * u1 - 1.0f) * l.half_y; }
        else { concentric_disk(u0, u1, x, y); x = x * l.radius; y = y * l.radius; }
        V3 p = ld3(l.centre) + ld3(l.fx) * x + ld3(l.fy) * y;
        V3 d = p - s.p;
        float dist2 = len2(d);
        float distance = sqrt_(dist2);
        V3 wi = d / distance;
        float cos = -dot(wi, ld3(l.fz));
        if (!(cos > 0.0f && distance > 0.0f)) return false;
        out.wi = wi;
        out.distance = distance;
        out.radiance = area_radiance(l, cos);
        out.pdf = pmf * dist2 / (l.area * cos);
        out.glossy = l.glossy != 0;
        out.shadow = l.shadow != 0;
    } else {
        V3 wi;
        float p;
        if (!env_sample(L, u0, u1, wi, p)) return false;
        out.wi = wi;
        out.distance = f_inf();
        out.radiance = splat(env_value(L, wi.z));
        out.pdf = pmf * p;
        out.glossy = true;
        out.shadow = true;
    }
    return out.pdf > 0.0f && finitef(out.pdf) && luminance(out.radiance) > 0.0f;
}

// Lights::crossed_from (light.rs:1350): area lights a ray crosses before t_max.
RTG_D_NI Rgb crossed_from(const LightsDev& L, V3 o, V3 d, float tmin, float tmax, bool has_pdf, float pdf, const Sel& from, float offset) {
    Rgb sum = splat(0.0f);
    for (int i = 0; i < L.n_areas; ++i) {
        const AreaLightDev& l = L.areas[i];
        if (!(has_pdf ? l.glossy : l.camera)) continue;
        float t, cos;
        if (!area_intersect(l, o, d, tmin, tmax, t, cos)) continue;
        float w = 1.0f;
        if (has_pdf) {
            float dd = offset + t;
            float light_pdf = pmf_of(L, l.entry, from) * dd * dd / (l.area * cos);
            w = power_heuristic(pdf, light_pdf);
        }
        sum = sum + area_radiance(l, cos) * w;
    }
    return sum;
}
// Lights::escaped (light.rs:1502) for the ramp environment.
RTG_D Rgb escaped(const LightsDev& L, V3 dir, bool has_pdf, float pdf, const Sel& from) {
    Rgb e = splat(env_value(L, dir.z));
    if (!has_pdf || !L.env_is_entry) return e;
    return e * power_heuristic(pdf, pmf_of(L, L.env_entry, from) * env_pdf(L, dir));
}

// ---- camera (render.rs:79, scene/mod.rs:280) -------------------------------------------------------
RTG_D float filter_offset(uint32_t filter, float u) {
    if (filter == 1) return 0.5f;
    if (filter == 2) return 0.5f + (u < 0.5f ? sqrt_(2.0f * u) - 1.0f : 1.0f - sqrt_(2.0f - 2.0f * u));
    return u;
}
RTG_D void camera_ray(const SceneDev& S, const SobolTable& T, uint32_t x, uint32_t y, uint32_t index, V3& o, V3& d) {
    uint32_t width = S.width ? S.width : 1, height = S.height ? S.height : 1;
    float aspect = (float)width / (float)height;
    uint64_t key = pixel_key(S.seed, x, y);
    float du = filter_offset(S.pixel_filter, sample1(T, key, index, DIM_CAMERA));
    float dv = filter_offset(S.pixel_filter, sample1(T, key, index, DIM_CAMERA + 1));
    float u = ((float)x + du) / (float)width;
    float v = ((float)y + dv) / (float)height;
    V3 pos = ld3(S.cam_pos), fwd = ld3(S.cam_fwd), right = ld3(S.cam_right), up = ld3(S.cam_up);
    if (S.ortho) {
        float w = S.ortho_width;
        o = pos + right * ((u - 0.5f) * w) + up * ((0.5f - v) * w / aspect);
        d = fwd;
        return;
    }
    float sw, sh;
    if (aspect >= 1.0f) { sw = S.sensor_mm; sh = S.sensor_mm / aspect; }
    else { sw = S.sensor_mm * aspect; sh = S.sensor_mm; }
    float px = (u - 0.5f) * sw;
    float py = (0.5f - v) * sh;
    V3 dir = normalize(fwd * S.focal_mm + right * px + up * py);
    if (S.lens_radius == 0.0f) { o = pos; d = dir; return; }
    float lx = 0.0f, ly = 0.0f;
    if (S.lens_radius > 0.0f) concentric_disk(sample1(T, key, index, DIM_LENS), sample1(T, key, index, DIM_LENS + 1), lx, ly);
    V3 focus = pos + dir * (S.focus_dist / dot(dir, fwd));
    o = pos + (right * lx + up * ly) * S.lens_radius;
    d = normalize(focus - o);
}

}  // namespace rtg
