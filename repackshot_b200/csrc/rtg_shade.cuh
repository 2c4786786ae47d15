// Lights, environment and camera on the device (engine/crates/rt-core/src/light.rs:120-1552,
// environment.rs:275-441, scene/mod.rs:280-359, render.rs:79-97, pixel_filter.rs:103-130).
#pragma once
#include "rtg_lights.cuh"
#include "rtg_trace.cuh"

namespace rtg {

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

// The selection at a vertex (light.rs:495): its point, the sum of the weights there and whether
// it is the static one. Weights are recomputed from the point with the same operations.
struct Sel { V3 p; float total; bool by_flux; };
RTG_D float entry_weight(const LightsDev& L, int e, V3 x) {  // light.rs:1014
    int a = L.entries[e];
    if (a < 0) return L.env_base;
    const LightDev& l = L.lights[a];
    if (l.kind == LIGHT_AREA) return area_weight(l, x);
    if (l.kind == LIGHT_SUN) return l.base;
    return sphere_weight(l, x);
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

// light: index into lights[], -1 the environment; delta: no other technique finds it
struct LightSample { V3 wi; float distance; Rgb radiance; float pdf; bool glossy, shadow, delta; int light; };

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
    out.light = a;
    out.delta = false;
    if (a >= 0 && L.lights[a].kind == LIGHT_SUN) {  // light.rs:1197
        const LightDev& l = L.lights[a];
        out.distance = f_inf();
        out.radiance = rgb(l.radiance[0], l.radiance[1], l.radiance[2]);
        out.glossy = l.glossy != 0;
        out.shadow = l.shadow != 0;
        if (l.delta) {
            out.wi = ld3(l.fz);
            out.pdf = pmf;
            out.delta = true;
        } else {
            Frame f;
            f.x = ld3(l.fx); f.y = ld3(l.fy); f.z = ld3(l.fz);
            out.wi = normalize(to_world(f, uniform_cone(u0, u1, l.one_minus_cos_max)));
            out.pdf = pmf / l.solid_angle;
        }
    } else if (a >= 0 && L.lights[a].kind == LIGHT_SPHERE) {  // light.rs:1224
        const LightDev& l = L.lights[a];
        float m = sphere_mask(l, s.p);
        V3 d = ld3(l.centre) - s.p;
        float dist2 = len2(d);
        if (!(m > 0.0f && dist2 > 0.0f)) return false;
        float dist = sqrt_(dist2);
        V3 towards = d / dist;
        float omc = 0.0f;
        if (l.radius > 0.0f && !sphere_cone(l, dist2, omc)) return false;
        out.glossy = l.glossy != 0;
        out.shadow = l.shadow != 0;
        if (omc == 0.0f) {
            out.wi = towards;
            out.distance = dist;
            out.radiance = rgb(l.intensity[0], l.intensity[1], l.intensity[2]) * (m / (dist2 * 1.0e-6f));
            out.pdf = pmf;
            out.delta = true;
        } else {
            V3 wi = normalize(to_world(frame_from_normal(towards), uniform_cone(u0, u1, omc)));
            float b = dot(wi, d);
            float r2 = l.radius * l.radius;
            float near = b - sqrt_(rmax(r2 - len2(d - wi * b), 0.0f));
            out.wi = wi;
            out.distance = rmax(near, 0.0f);
            out.radiance = rgb(l.radiance[0], l.radiance[1], l.radiance[2]) * m;
            out.pdf = pmf / (TAU * omc);
        }
    } else if (a >= 0) {
        const LightDev& l = L.lights[a];
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

// The light of one sphere a ray crosses before t_max (light.rs:1387), seen from the vertex the
// ray left offset earlier; false when it adds nothing.
RTG_D bool sphere_crossed(const LightsDev& L, const LightDev& l, V3 o, V3 d, float tmin, float tmax, bool has_pdf, float pdf,
                          const Sel& from, float offset, Rgb& out) {
    if (!(has_pdf ? l.glossy : l.camera)) return false;
    float t;
    if (!sphere_intersect(l, o, d, tmin, tmax, t)) return false;
    V3 vertex = o - d * offset;
    float m = sphere_mask(l, vertex);
    if (!(m > 0.0f)) return false;
    float w = 1.0f;
    if (has_pdf) {
        float omc;
        if (sphere_cone(l, len2(ld3(l.centre) - vertex), omc) && omc > 0.0f)
            w = power_heuristic(pdf, pmf_of(L, l.entry, from) / (TAU * omc));
        else
            w = 0.0f;
    }
    out = rgb(l.radiance[0], l.radiance[1], l.radiance[2]) * (m * w);
    return true;
}
// The light of one sun an escaping ray sees (light.rs:1507); false when it adds nothing.
RTG_D bool sun_seen(const LightsDev& L, const LightDev& l, V3 dir, bool has_pdf, float pdf, const Sel& from, Rgb& out) {
    if (!((has_pdf ? l.glossy : l.camera) && sun_contains(l, dir))) return false;
    float w = has_pdf ? power_heuristic(pdf, pmf_of(L, l.entry, from) / l.solid_angle) : 1.0f;
    out = rgb(l.radiance[0], l.radiance[1], l.radiance[2]) * w;
    return true;
}

// Lights::crossed_from (light.rs:1329): the area lights, then the spheres, a ray crosses before t_max.
RTG_D_NI Rgb crossed_from(const LightsDev& L, V3 o, V3 d, float tmin, float tmax, bool has_pdf, float pdf, const Sel& from, float offset) {
    Rgb sum = splat(0.0f);
    for (int i = 0; i < L.n_areas; ++i) {
        const LightDev& l = L.lights[i];
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
    const int first_sphere = L.n_areas + (int)L.n_suns;
    for (int i = first_sphere; i < first_sphere + (int)L.n_spheres; ++i) {
        Rgb c;
        if (sphere_crossed(L, L.lights[i], o, d, tmin, tmax, has_pdf, pdf, from, offset, c)) sum = sum + c;
    }
    return sum;
}
// sum plus the sun discs an escaping ray sees, in their order.
RTG_D_NI Rgb add_suns(const LightsDev& L, Rgb sum, V3 dir, bool has_pdf, float pdf, const Sel& from) {
    for (int i = L.n_areas; i < L.n_areas + (int)L.n_suns; ++i) {
        Rgb c;
        if (sun_seen(L, L.lights[i], dir, has_pdf, pdf, from, c)) sum = sum + c;
    }
    return sum;
}
// Lights::escaped (light.rs:1502): the ramp environment, then the sun discs.
RTG_D Rgb escaped(const LightsDev& L, V3 dir, bool has_pdf, float pdf, const Sel& from) {
    Rgb sum = splat(env_value(L, dir.z));
    if (has_pdf && L.env_is_entry) sum = sum * power_heuristic(pdf, pmf_of(L, L.env_entry, from) * env_pdf(L, dir));
    return L.n_suns ? add_suns(L, sum, dir, has_pdf, pdf, from) : sum;
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
