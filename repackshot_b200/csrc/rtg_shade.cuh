// Lights, environment and camera on the device (engine/crates/rt-core/src/light.rs:120-1552,
// environment.rs:275-441, scene/mod.rs:280-359, render.rs:79-97, pixel_filter.rs:103-130).
#pragma once
#include "rtg_lights.cuh"
#include "rtg_trace.cuh"

namespace rtg {

// ---- images (bitmap.rs:127-175) --------------------------------------------------------------------
// f32 to u32 as Rust's `as` converts: NaN and negatives to 0, saturating above.
RTG_D uint32_t sat_u32(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)x;
}
RTG_D Rgb texel(const float* tex, uint32_t w, uint32_t h, uint32_t x, uint32_t y) {
    x = x < w - 1 ? x : w - 1;
    y = y < h - 1 ? y : h - 1;
    const float* p = tex + 3 * ((size_t)y * w + x);
    return rgb(p[0], p[1], p[2]);
}
// Bilinear lookup at (u, v), pixel centres at (i + 1/2) / n; wrap_u wraps the columns.
RTG_D Rgb bilinear(const float* tex, uint32_t width, uint32_t height, float u, float v, bool wrap_u) {
    float w = (float)width, h = (float)height;
    float fx = u * w - 0.5f;
    float fy = rclamp(v * h - 0.5f, 0.0f, h - 1.0f);
    float x0f = floorf(fx), y0f = floorf(fy);
    float tx = fx - x0f, ty = fy - y0f;
    uint32_t x0, x1;
    if (wrap_u) {
        float r0 = fmodf(x0f, w), r1 = fmodf(x0f + 1.0f, w);
        if (r0 < 0.0f) r0 = r0 + absf(w);
        if (r1 < 0.0f) r1 = r1 + absf(w);
        x0 = min(sat_u32(r0), width - 1);
        x1 = min(sat_u32(r1), width - 1);
    } else {
        x0 = sat_u32(rclamp(x0f, 0.0f, w - 1.0f));
        x1 = sat_u32(rclamp(x0f + 1.0f, 0.0f, w - 1.0f));
    }
    uint32_t y0 = sat_u32(y0f);
    uint32_t y1 = y0 + 1 < height - 1 ? y0 + 1 : height - 1;
    Rgb top = texel(tex, width, height, x0, y0) * (1.0f - tx) + texel(tex, width, height, x1, y0) * tx;
    Rgb bottom = texel(tex, width, height, x0, y1) * (1.0f - tx) + texel(tex, width, height, x1, y1) * tx;
    return top * (1.0f - ty) + bottom * ty;
}

// ---- environment map (environment.rs:40-130, bitmap.rs:312-408) -----------------------------------
RTG_D void dir_to_uv(V3 d, float& u, float& v) {
    float uu = 0.5f + fatan2(-d.y, d.x) * (0.5f * FRAC_1_PI);
    u = uu - floorf(uu);
    v = rclamp(facos(d.z) * FRAC_1_PI, 0.0f, 1.0f);
}
RTG_D V3 map_to_image(const EnvMapDev& m, V3 d) { return v3(m.rot_c * d.x + m.rot_s * d.y, -m.rot_s * d.x + m.rot_c * d.y, d.z); }
RTG_D V3 map_to_world(const EnvMapDev& m, V3 d) { return v3(m.rot_c * d.x - m.rot_s * d.y, m.rot_s * d.x + m.rot_c * d.y, d.z); }
RTG_D Rgb map_radiance(const EnvMapDev& m, V3 dir) {
    float u, v;
    dir_to_uv(map_to_image(m, dir), u, v);
    return bilinear(m.texels, m.width, m.height, u, v, true) * m.scale;
}
// The bucket of a normalised CDF that holds u (the first entry above u), and u rescaled into it.
RTG_D void cdf_search(const float* cdf, uint32_t n, float u, uint32_t& i, float& rest) {
    uint32_t lo = 0, hi = n;  // partition point of cdf[k] <= u
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (cdf[mid] <= u) lo = mid + 1;
        else hi = mid;
    }
    i = lo < n - 1 ? lo : n - 1;
    float below = i == 0 ? 0.0f : cdf[i - 1];
    float width = cdf[i] - below;
    rest = width > 0.0f ? rclamp((u - below) / width, 0.0f, 0.99999994f) : 0.5f;
}
RTG_D float map_cell_pdf(const EnvMapDev& m, float u, float v) {
    uint32_t x = min(sat_u32(u * (float)m.gw), m.gw - 1), y = min(sat_u32(v * (float)m.gh), m.gh - 1);
    return m.weights[y * m.gw + x] / m.mean;
}
RTG_D float map_pdf(const EnvMapDev& m, V3 dir) {
    V3 local = map_to_image(m, dir);
    float sin_theta = sqrt_(rmax((1.0f - local.z) * (1.0f + local.z), 0.0f));
    if (sin_theta <= 0.0f) return 0.0f;
    float u, v;
    dir_to_uv(local, u, v);
    return map_cell_pdf(m, u, v) / (2.0f * PI * PI * sin_theta);
}
RTG_D bool map_sample(const EnvMapDev& m, float s0, float s1, V3& dir, float& pdf) {
    uint32_t y, x;
    float fy, fx;
    cdf_search(m.marginal, m.gh, s1, y, fy);
    cdf_search(m.conditional + (size_t)y * m.gw, m.gw, s0, x, fx);
    float u = ((float)x + fx) / (float)m.gw, v = ((float)y + fy) / (float)m.gh;
    float pdf_uv = m.weights[y * m.gw + x] / m.mean;
    float st, ct, sp, cp;
    sin_cos(PI * v, st, ct);
    sin_cos(TAU * (u - 0.5f), sp, cp);
    if (!(st > 0.0f && pdf_uv > 0.0f)) return false;
    dir = normalize(map_to_world(m, v3(st * cp, -st * sp, ct)));
    pdf = map_pdf(m, dir);
    return pdf > 0.0f;
}

// ---- environment ramp ---------------------------------------------------------------------------
RTG_D float env_value(const LightsDev& L, float z) {
    z = rclamp(z, -1.0f, 1.0f);
    if (z < 0.0f) return L.env_floor * -z + L.env_horizon * (1.0f + z);
    return L.env_horizon * (1.0f - z) + L.env_zenith * z;
}
RTG_D float ramp_pdf(const LightsDev& L, V3 dir) {
    if (L.env_total <= 0.0f) return 0.0f;
    return env_value(L, dir.z) / (TAU * L.env_total);
}
RTG_D float invert_linear(float a, float b, float u) {
    float c = u * 0.5f * (a + b);
    float denom = a + sqrt_(rmax(a * a + 2.0f * (b - a) * c, 0.0f));
    return denom > 0.0f ? rclamp(2.0f * c / denom, 0.0f, 1.0f) : 0.0f;
}
RTG_D bool ramp_sample(const LightsDev& L, float u0, float u1, V3& dir, float& pdf) {
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
    pdf = ramp_pdf(L, dir);
    return pdf > 0.0f;
}
// EnvLight (environment.rs:333): the map or the ramp.
RTG_D Rgb env_radiance(const LightsDev& L, V3 dir) { return L.env_is_map ? map_radiance(L.env_map, dir) : splat(env_value(L, dir.z)); }
RTG_D float env_pdf(const LightsDev& L, V3 dir) { return L.env_is_map ? map_pdf(L.env_map, dir) : ramp_pdf(L, dir); }
RTG_D bool env_sample(const LightsDev& L, float u0, float u1, V3& dir, float& pdf) {
    return L.env_is_map ? map_sample(L.env_map, u0, u1, dir, pdf) : ramp_sample(L, u0, u1, dir, pdf);
}

// ---- background image (integrator/mod.rs:199-232) -----------------------------------------------------
// What a camera ray that escapes shows at screen position (su, sv): the fitted image, or the
// background colour outside a fitted image.
RTG_D Rgb backdrop(const SceneDev& S, float su, float sv) {
    const Rgb colour = rgb(S.background_color[0], S.background_color[1], S.background_color[2]);
    if (S.background != 3) return colour;
    float u = (su - S.plate_rect[0]) / (S.plate_rect[2] - S.plate_rect[0]);
    float v = (sv - S.plate_rect[1]) / (S.plate_rect[3] - S.plate_rect[1]);
    if (S.plate_fit != 2) {
        const bool fit = S.plate_fit == 1;
        const float k = S.frame_aspect / S.image_aspect;
        if (S.image_aspect > S.frame_aspect) {
            if (fit) v = 0.5f + (v - 0.5f) * (1.0f / k);
            else u = 0.5f + (u - 0.5f) * k;
        } else if (fit) {
            u = 0.5f + (u - 0.5f) * k;
        } else {
            v = 0.5f + (v - 0.5f) * (S.image_aspect / S.frame_aspect);
        }
    }
    if (S.plate_fit == 1 && !(u >= 0.0f && u <= 1.0f && v >= 0.0f && v <= 1.0f)) return colour;
    return bilinear(S.plate, S.plate_w, S.plate_h, rclamp(u, 0.0f, 1.0f), rclamp(v, 0.0f, 1.0f), false);
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
    if (l.kind == LIGHT_MESH) return mesh_weight(l, x);
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

// light.rs:1543 emitter_weight: for a BSDF-sampled ray (density pdf, selection `from`) that hit an
// emissive instance at distance t with `cos` between the ray and the geometric normal, the MIS
// weight of its emission against its mesh light's next-event sample (1 without a mesh light).
RTG_D float emitter_weight(const LightsDev& L, uint32_t emitter, float pdf, const Sel& from, float t, float cos) {
    if (emitter == 0) return 1.0f;
    const LightDev& l = L.lights[emitter - 1];
    const float light_pdf = pmf_of(L, l.entry, from) * t * t / (l.area * rmax(absf(cos), 1.0e-7f));
    return power_heuristic(pdf, light_pdf);
}

// light: index into lights[], -1 the environment; delta: no other technique finds it
struct LightSample { V3 wi; float distance; Rgb radiance; float pdf; bool glossy, shadow, delta; int light; };

RTG_D_NI bool sample_light(const LightsDev& L, const Sel& s, float u_select, float u0, float u1, LightSample& out) {  // light.rs:1150
    int n = L.n_entries;
    if (n == 0) return false;
    int index = 0;
    float pmf = 0.0f, rest = 0.0f;  // rest: where u_select falls within its bucket (a mesh light's triangle)
    if (s.by_flux) {  // pick (light.rs:634)
        int k = 0;
        while (k < n && L.cdf[k] <= u_select) ++k;
        index = k < n - 1 ? k : n - 1;
        pmf = pmf_of(L, (uint32_t)index, s);
        const float lo = index == 0 ? 0.0f : L.cdf[index - 1], width = L.cdf[index] - lo;
        rest = width > 0.0f ? rclamp((u_select - lo) / width, 0.0f, 0.99999994f) : 0.0f;
    } else {
        if (!(s.total > 0.0f && finitef(s.total))) return false;
        // pick_at (light.rs:1118): the first bucket whose end passes u_select
        float acc = 0.0f, lo = 0.0f;
        int last = n - 1;
        for (int e = 0; e <= last; ++e) {
            float w = entry_weight(L, e, s.p);
            acc += w;
            float hi = e == last ? 1.0f : acc / s.total;
            if (hi > u_select || e == last) {
                index = e;
                pmf = w / s.total;
                const float width = hi - lo;
                rest = width > 0.0f ? rclamp((u_select - lo) / width, 0.0f, 0.99999994f) : 0.0f;
                break;
            }
            lo = hi;
        }
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
    } else if (a >= 0 && L.lights[a].kind == LIGHT_MESH) {  // light.rs:1270: a triangle by area, a point uniformly
        const LightDev& l = L.lights[a];
        uint32_t k = 0;
        while (k < l.n_tris && __ldg(&l.tris[4 * k].w) <= rest) ++k;
        const uint32_t t = k < l.n_tris - 1 ? k : l.n_tris - 1;
        const float4 ca = __ldg(&l.tris[4 * t]), cb = __ldg(&l.tris[4 * t + 1]), cc = __ldg(&l.tris[4 * t + 2]), nn = __ldg(&l.tris[4 * t + 3]);
        const float su = sqrt_(u0);  // warp.rs:57 uniform_triangle
        const float b0 = 1.0f - su, b1 = u1 * su, b2 = 1.0f - b0 - b1;
        const V3 p = v3(ca.x, ca.y, ca.z) * b0 + v3(cb.x, cb.y, cb.z) * b1 + v3(cc.x, cc.y, cc.z) * b2;
        const V3 d = p - s.p;
        const float dist2 = len2(d);
        const float distance = sqrt_(dist2);
        const V3 wi = d / distance;
        const float facing = -dot(wi, v3(nn.x, nn.y, nn.z));
        if (!(distance > 0.0f) || (!l.two_sided && facing <= 0.0f)) return false;
        const float cos = absf(facing);
        if (!(cos > 0.0f)) return false;
        out.wi = wi;
        out.distance = distance;
        out.radiance = rgb(l.radiance[0], l.radiance[1], l.radiance[2]);
        out.pdf = pmf * dist2 / (l.area * cos);
        out.glossy = true;
        out.shadow = true;
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
        out.radiance = env_radiance(L, wi);
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
// Lights::camera_sees_panel (light.rs:1490): a camera ray meets a light it sees (an area light
// flagged camera, or a sphere flagged camera that lights the ray's origin) before t_max.
RTG_D bool camera_sees_panel(const LightsDev& L, V3 o, V3 d, float t_max) {
    for (int i = 0; i < L.n_areas; ++i) {
        float t, cos;
        if (L.lights[i].camera && area_intersect(L.lights[i], o, d, 1.0e-3f, t_max, t, cos)) return true;
    }
    const int first = L.n_areas + (int)L.n_suns;
    for (int i = first; i < first + (int)L.n_spheres; ++i) {
        float t;
        const LightDev& l = L.lights[i];
        if (l.camera && sphere_intersect(l, o, d, 1.0e-3f, t_max, t) && sphere_mask(l, o) > 0.0f) return true;
    }
    return false;
}
// Lights::escaped (light.rs:1502): the ramp environment, then the sun discs.
RTG_D Rgb escaped(const LightsDev& L, V3 dir, bool has_pdf, float pdf, const Sel& from) {
    Rgb sum = env_radiance(L, dir);
    if (has_pdf && L.env_is_entry) sum = sum * power_heuristic(pdf, pmf_of(L, L.env_entry, from) * env_pdf(L, dir));
    return L.n_suns ? add_suns(L, sum, dir, has_pdf, pdf, from) : sum;
}

// ---- camera (render.rs:79, scene/mod.rs:280) -------------------------------------------------------
// pixel_filter.rs:103: where a uniform number puts a camera sample on one axis, in pixels from
// the pixel's side: the standard box (u), none (the centre), the tent, or Blackman-Harris (its
// tabulated inverse CDF, linear between the points s = q^-1(u)).
RTG_D float filter_offset(const SceneDev& S, float u) {
    const uint32_t filter = S.pixel_filter;
    if (filter == 1) return 0.5f;
    if (filter == 2) return 0.5f + (u < 0.5f ? sqrt_(2.0f * u) - 1.0f : 1.0f - sqrt_(2.0f - 2.0f * u));
    if (filter == 3) {
        const float s = u < 0.5f ? sqrt_(0.5f * u) : 1.0f - sqrt_(0.5f - 0.5f * u);
        const float f = rclamp(s * 255.0f, 0.0f, 255.0f);
        const uint32_t i = min((uint32_t)f, 254u);
        const float t = f - (float)i, a = S.filter_table[i], b = S.filter_table[i + 1];
        return 0.5f + (a + (b - a) * t);
    }
    return u;
}
// The scramble key of a pixel's sample (sampler.rs:339 with the render's seed): indices from
// S.split_b on take S.seed_b. Every render has split_b = 0xffffffff, so its keys are the seed's.
RTG_D uint64_t sample_key(const SceneDev& S, uint32_t x, uint32_t y, uint32_t index) {
    return pixel_key(index >= S.split_b ? S.seed_b : S.seed, x, y);
}
// The screen position (u, v) in [0, 1]^2 of a camera sample (render.rs:96).
RTG_D void screen_of(const SceneDev& S, const SobolTable& T, uint32_t x, uint32_t y, uint32_t index, float& su, float& sv) {
    uint32_t width = S.width ? S.width : 1, height = S.height ? S.height : 1;
    uint64_t key = sample_key(S, x, y, index);
    float du = filter_offset(S, sample1(T, key, index, DIM_CAMERA));
    float dv = filter_offset(S, sample1(T, key, index, DIM_CAMERA + 1));
    su = rclamp(((float)x + du) / (float)width, 0.0f, 1.0f);
    sv = rclamp(((float)y + dv) / (float)height, 0.0f, 1.0f);
}
// Camera::generate_ray (scene/mod.rs:294) through the image point (u, v) and the lens point
// (lx, ly) of the unit disc. False where a panoramic camera sees nothing (a fisheye beyond 180
// degrees from its axis: scene/mod.rs:227 gives a ray along the axis with an empty interval, whose
// sample weighs black); the ray is then (position, axis).
RTG_D bool camera_ray_at(const SceneDev& S, float u, float v, float lx, float ly, V3& o, V3& d) {
    uint32_t width = S.width ? S.width : 1, height = S.height ? S.height : 1;
    float aspect = (float)width / (float)height;
    V3 pos = ld3(S.cam_pos), fwd = ld3(S.cam_fwd), right = ld3(S.cam_right), up = ld3(S.cam_up);
    if (S.projection == 1) {  // scene/mod.rs:200: longitude across the width, latitude across the height
        const float lon = (u - 0.5f) * (S.fov_x_deg * (PI / 180.0f));
        const float lat = (0.5f - v) * (S.fov_y_deg * (PI / 180.0f));
        float s_lat, c_lat, s_lon, c_lon;
        sin_cos(lat, s_lat, c_lat);
        sin_cos(lon, s_lon, c_lon);
        o = pos;
        d = fwd * (c_lat * c_lon) + right * (c_lat * s_lon) + up * s_lat;
        return true;
    }
    if (S.projection == 2) {  // scene/mod.rs:207: the equidistant fisheye
        const float k = S.fov_x_deg * (PI / 180.0f);
        const float x = (u - 0.5f) * k;
        const float y = (0.5f - v) * k / rmax(aspect, 1.0e-6f);
        const float theta = sqrt_(x * x + y * y);
        o = pos;
        d = fwd;
        if (theta != theta || theta > PI) return false;
        if (theta == 0.0f) return true;
        float s, c;
        sin_cos(theta, s, c);
        d = fwd * c + (right * x + up * y) * (s / theta);
        return true;
    }
    if (S.ortho) {
        float w = S.ortho_width;
        o = pos + right * ((u - 0.5f) * w) + up * ((0.5f - v) * w / aspect);
        d = fwd;
        return true;
    }
    float sw, sh;
    if (aspect >= 1.0f) { sw = S.sensor_mm; sh = S.sensor_mm / aspect; }
    else { sw = S.sensor_mm * aspect; sh = S.sensor_mm; }
    float px = (u - 0.5f) * sw;
    float py = (0.5f - v) * sh;
    V3 dir = normalize(fwd * S.focal_mm + right * px + up * py);
    if (S.lens_radius == 0.0f) { o = pos; d = dir; return true; }
    V3 focus = pos + dir * (S.focus_dist / dot(dir, fwd));
    o = pos + (right * lx + up * ly) * S.lens_radius;
    d = normalize(focus - o);
    return true;
}
// The camera sample of (pixel, index): camera_sample_weighted (render.rs:79) with the plain thin
// lens; false for a panoramic camera's sample that sees nothing (its weight is black).
RTG_D bool camera_ray(const SceneDev& S, const SobolTable& T, uint32_t x, uint32_t y, uint32_t index, V3& o, V3& d) {
    uint32_t width = S.width ? S.width : 1, height = S.height ? S.height : 1;
    uint64_t key = sample_key(S, x, y, index);
    float du = filter_offset(S, sample1(T, key, index, DIM_CAMERA));
    float dv = filter_offset(S, sample1(T, key, index, DIM_CAMERA + 1));
    float u = ((float)x + du) / (float)width;
    float v = ((float)y + dv) / (float)height;
    float lx = 0.0f, ly = 0.0f;
    if (!S.ortho && S.lens_radius > 0.0f)
        concentric_disk(sample1(T, key, index, DIM_LENS), sample1(T, key, index, DIM_LENS + 1), lx, ly);
    return camera_ray_at(S, u, v, lx, ly, o, d);
}

}  // namespace rtg
