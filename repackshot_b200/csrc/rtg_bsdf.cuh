// The principled BSDF of the Repackshot engine on the device: GGX conductor, dielectric (opaque
// and clear, with refraction) and Lambert lobes, Kulla–Conty / Turquin energy compensation from
// the 16-bit tables, lobe-mixture sampling and pdf (engine/crates/rt-core/src/bsdf.rs:113-993,
// bsdf/energy.rs:305-554). The particle forward lobe and the scattering-medium exit lobe of the
// reference are not part of this path.
#pragma once
#include "rtg_math.cuh"

namespace rtg {

constexpr float MIN_ALPHA = 1.0e-3f;
constexpr float COAT_F0 = 0.04f;
constexpr float MAX_REFLECT_PROBABILITY = 0.99f;
constexpr float MIN_COMPENSATED_ALPHA = 2.0e-3f;
constexpr int NODES_MU = 32, NODES_ROUGHNESS = 32, NODES_IOR = 17;

// Device addresses of the six energy tables (u16 fractions and their f32 cosine-weighted means).
struct EnergyTables {
    const uint16_t* albedo;
    const uint16_t* schlick;
    const uint16_t* clear_in;
    const uint16_t* clear_out;
    const float* albedo_avg;
    const float* schlick_avg;
};

// Material as the kernels read it: the MATL fields the BSDF and the integrator use.
struct DevMaterial {
    uint32_t kind, flags;
    float base[3];
    float metallic, roughness, ior, transmission, coat, coat_roughness, anisotropy, absorption_mm;
    float emission[3];  // radiance of an emitter (emission * emission_power, clamped at 0)
    float sigma[3];     // Beer–Lambert coefficients per mm inside a clear solid
    uint32_t has_medium;
    float opacity;  // below 1: a cut-out
};
constexpr uint32_t MATERIAL_GLASS = 1, MATERIAL_EMISSIVE = 2, MATERIAL_FLAG_THIN = 2;

RTG_HD float ggx_d(V3 h, float a2) {
    float t = a2 * h.z * h.z + (h.x * h.x + h.y * h.y);
    if (t <= 0.0f) return 0.0f;
    return a2 / (PI * t * t);
}
RTG_HD float ggx_lambda(V3 w, float a2) {
    float cos2 = w.z * w.z;
    if (cos2 <= 0.0f) return f_inf();
    float tan2 = (w.x * w.x + w.y * w.y) / cos2;
    return (sqrt_(1.0f + a2 * tan2) - 1.0f) * 0.5f;
}
struct Ggx {
    float ax, ay, a2;
    bool iso;
};
RTG_HD Ggx make_ggx(float alpha, float anisotropy) {
    Ggx g;
    if (anisotropy > 0.0f) {
        float s = sqrt_(1.0f - 0.9f * anisotropy);
        g.ax = rmax(alpha / s, MIN_ALPHA);
        g.ay = rmax(alpha * s, MIN_ALPHA);
        g.a2 = alpha * alpha;
        g.iso = false;
    } else {
        g.ax = alpha; g.ay = alpha; g.a2 = alpha * alpha; g.iso = true;
    }
    return g;
}
RTG_HD float ggx_D(const Ggx& g, V3 h) {
    if (g.iso) return ggx_d(h, g.a2);
    float x = h.x / g.ax, y = h.y / g.ay;
    float t = x * x + y * y + h.z * h.z;
    if (t <= 0.0f) return 0.0f;
    return 1.0f / (PI * g.ax * g.ay * t * t);
}
RTG_HD float ggx_L(const Ggx& g, V3 w) {
    if (g.iso) return ggx_lambda(w, g.a2);
    float cos2 = w.z * w.z;
    if (cos2 <= 0.0f) return f_inf();
    float x = g.ax * w.x, y = g.ay * w.y;
    return (sqrt_(1.0f + (x * x + y * y) / cos2) - 1.0f) * 0.5f;
}
RTG_HD float ggx_reflection_pdf(const Ggx& g, V3 wo, V3 h) {
    float g1 = 1.0f / (1.0f + ggx_L(g, wo));
    return g1 * ggx_D(g, h) / (4.0f * wo.z);
}
RTG_HD float ggx_microfacet(const Ggx& g, V3 wo, V3 wi, V3 h) {
    float g2 = 1.0f / (1.0f + ggx_L(g, wo) + ggx_L(g, wi));
    return ggx_D(g, h) * g2 / (4.0f * wo.z * wi.z);
}
RTG_HD float schlick(float f0, float f90, float cos) {
    float m = rclamp(1.0f - cos, 0.0f, 1.0f);
    float m2 = m * m;
    return f0 + (f90 - f0) * (m2 * m2 * m);
}
RTG_HD float fresnel_dielectric(float cos_i, float eta) {
    cos_i = rclamp(cos_i, 0.0f, 1.0f);
    float sin2_t = (1.0f - cos_i * cos_i) / (eta * eta);
    if (sin2_t >= 1.0f) return 1.0f;
    float cos_t = sqrt_(1.0f - sin2_t);
    float rs = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    float rp = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    return 0.5f * (rs * rs + rp * rp);
}
RTG_HD float thin_reflectance(float cos, float eta) {
    float r = fresnel_dielectric(cos, eta);
    return 2.0f * r / (1.0f + r);
}
RTG_HD bool refract(V3 wo, V3 h, float eta, V3& out) {
    float cos_i = dot(wo, h);
    float sin2_t = (1.0f - cos_i * cos_i) / (eta * eta);
    if (sin2_t >= 1.0f) return false;
    float cos_t = sqrt_(1.0f - sin2_t);
    out = normalize(h * (cos_i / eta - cos_t) - wo / eta);
    return true;
}
RTG_HD V3 sample_vndf(V3 wo, float ax, float ay, float u0, float u1) {  // Heitz 2018
    V3 vh = normalize(v3(ax * wo.x, ay * wo.y, wo.z));
    float lensq = vh.x * vh.x + vh.y * vh.y;
    V3 t1 = lensq > 0.0f ? v3(-vh.y, vh.x, 0.0f) / sqrt_(lensq) : v3(1.0f, 0.0f, 0.0f);
    V3 t2 = cross(vh, t1);
    float r = sqrt_(u0);
    float sp, cp;
    sin_cos(TAU * u1, sp, cp);
    float p1 = r * cp;
    float s = 0.5f * (1.0f + vh.z);
    float p2 = (1.0f - s) * sqrt_(rmax(1.0f - p1 * p1, 0.0f)) + s * (r * sp);
    V3 nh = t1 * p1 + t2 * p2 + vh * sqrt_(rmax(1.0f - p1 * p1 - p2 * p2, 0.0f));
    return normalize(v3(ax * nh.x, ay * nh.y, rmax(nh.z, 1.0e-7f)));
}

// ---- energy table lookups ------------------------------------------------------------------------
RTG_HD void locate(float x, int n, int& i, float& w) {
    float t = rclamp(x, 0.0f, 1.0f) * (float)(n - 1);
    uint32_t ti = f2u32_floor_nonneg(t);
    i = (int)(ti < (uint32_t)(n - 2) ? ti : (uint32_t)(n - 2));
    w = t - (float)i;
}
RTG_HD float tab(const uint16_t* t, int idx) {
#ifdef __CUDA_ARCH__
    return (float)__ldg(t + idx) * (1.0f / 65535.0f);
#else
    return (float)t[idx] * (1.0f / 65535.0f);
#endif
}
RTG_HD float table_lookup(const uint16_t* table, float mu, float alpha) {
    int i, j;
    float u, v;
    locate(sqrt_(rmax(mu, 0.0f)), NODES_MU, i, u);
    locate(sqrt_(rmax(alpha, 0.0f)), NODES_ROUGHNESS, j, v);
    float a00 = tab(table, j * NODES_MU + i), a01 = tab(table, j * NODES_MU + i + 1);
    float a10 = tab(table, (j + 1) * NODES_MU + i), a11 = tab(table, (j + 1) * NODES_MU + i + 1);
    float low = a00 + (a01 - a00) * u;
    float high = a10 + (a11 - a10) * u;
    return low + (high - low) * v;
}
RTG_HD float avg_lookup(const float* t, float alpha) {
    int j; float v;
    locate(sqrt_(rmax(alpha, 0.0f)), NODES_ROUGHNESS, j, v);
    return t[j] + (t[j + 1] - t[j]) * v;
}
RTG_HD float schlick_average(float f0, float f90) { return f0 + (f90 - f0) * (1.0f / 21.0f); }
RTG_HD float multiple_fresnel(float f_avg, float e_avg) {
    float d = 1.0f - f_avg * (1.0f - e_avg);
    return d > 0.0f ? f_avg * f_avg * e_avg / d : 0.0f;
}
RTG_HD float clear_albedo(const EnergyTables& E, float mu, float alpha, float eta) {
    const uint16_t* table = eta >= 1.0f ? E.clear_in : E.clear_out;
    float ior = eta >= 1.0f ? eta : 1.0f / eta;
    const float MAX_X = (3.0f - 1.0f) / (3.0f + 1.0f);
    float x = (ior - 1.0f) / (ior + 1.0f);
    int k; float w;
    locate(x / MAX_X, NODES_IOR, k, w);
    const int slice = NODES_MU * NODES_ROUGHNESS;
    float a = table_lookup(table + k * slice, mu, alpha);
    float b = table_lookup(table + (k + 1) * slice, mu, alpha);
    return a + (b - a) * w;
}

struct Layer {
    float f0, f90, strength, alpha, ms, norm;
    bool rough;
};
RTG_HD Layer layer_clear() { Layer l; l.f0 = 0; l.f90 = 0; l.strength = 0; l.alpha = 0; l.ms = 0; l.norm = 1.0f; l.rough = false; return l; }
RTG_HD Layer make_layer(const EnergyTables& E, float f0, float f90, float strength, float alpha, float ms) {
    if (strength != strength || strength <= 0.0f || (f90 <= 0.0f && f0 <= 0.0f)) return layer_clear();
    Layer l;
    l.f0 = f0; l.f90 = f90; l.strength = strength; l.alpha = alpha; l.ms = ms;
    l.rough = alpha >= MIN_COMPENSATED_ALPHA;
    float avg;
    if (l.rough) {
        float e_avg = avg_lookup(E.albedo_avg, alpha);
        avg = f0 * e_avg + (f90 - f0) * avg_lookup(E.schlick_avg, alpha) + ms * (1.0f - e_avg);
    } else {
        avg = schlick_average(f0, f90);
    }
    avg = avg * strength;
    l.norm = 1.0f / (1.0f - rmin(avg, 0.999f));
    return l;
}
RTG_HD float layer_passes(const EnergyTables& E, const Layer& l, float mu) {
    float e;
    if (l.rough) {
        float ee = table_lookup(E.albedo, mu, l.alpha);
        e = l.f0 * ee + (l.f90 - l.f0) * table_lookup(E.schlick, mu, l.alpha) + l.ms * (1.0f - ee);
    } else {
        float m = rclamp(1.0f - mu, 0.0f, 1.0f);
        float m2 = m * m;
        e = l.f0 + (l.f90 - l.f0) * (m2 * m2 * m);
    }
    return 1.0f - rclamp(e * l.strength, 0.0f, 1.0f);
}
struct MsLobe { float alpha, norm, e_avg; bool on; };
RTG_HD MsLobe make_lobe(const EnergyTables& E, float alpha) {
    MsLobe l; l.on = false; l.alpha = 0; l.norm = 0; l.e_avg = 0;
    if (alpha != alpha || alpha < MIN_COMPENSATED_ALPHA) return l;
    float e_avg = avg_lookup(E.albedo_avg, alpha);
    float lost = 1.0f - e_avg;
    if (!(lost > 1.0e-6f)) return l;
    l.on = true; l.alpha = alpha; l.norm = FRAC_1_PI / lost; l.e_avg = e_avg;
    return l;
}
RTG_HD float lobe_lost(const EnergyTables& E, const MsLobe& l, float mu) { return rmax(1.0f - table_lookup(E.albedo, mu, l.alpha), 0.0f); }

enum LobesSel { LOBES_ALL = 0, LOBES_DIFFUSE = 1 };
struct BsdfSample { V3 wi; Rgb weight; float pdf; bool straight; };
struct LobeWeights { float coat, specular, diffuse, clear, ms; };

struct Bsdf {
    Rgb diffuse, metal_f0, metal_f90;
    float metallic, dielectric, f0, f90;
    Ggx spec;
    float coat;
    Ggx coat_ggx;
    float clear, eta;
    Rgb tint;
    bool thin;
    bool ms_spec_on; MsLobe ms_spec_lobe; Rgb ms_spec_colour;
    bool ms_coat_on; MsLobe ms_coat_lobe; float ms_coat_c;
    bool ms_clear_on; float ms_clear_alpha;
    Layer base_layer, coat_layer;
    float diffuse_norm;
};

RTG_HD bool has_specular(const Bsdf& b) { return (b.f90 > 0.0f && b.dielectric > 0.0f) || b.metallic > 0.0f; }
RTG_HD float joint_norm(const EnergyTables& E, const Layer& below, const Layer& above) {
    if (above.strength <= 0.0f) return below.norm;
    if (below.strength <= 0.0f) return above.norm;
    const float G[8][2] = {{0.019855072f, 0.05061427f}, {0.10166676f, 0.11119052f}, {0.2372338f, 0.15685332f},
                           {0.40828268f, 0.18134189f},  {0.5917173f, 0.18134189f},  {0.7627662f, 0.15685332f},
                           {0.8983332f, 0.11119052f},   {0.9801449f, 0.05061427f}};
    float sum = 0.0f;
    for (int i = 0; i < 8; ++i) sum = sum + G[i][1] * 2.0f * G[i][0] * layer_passes(E, below, G[i][0]) * layer_passes(E, above, G[i][0]);
    return 1.0f / rmax(sum, 0.001f);
}

RTG_HD Bsdf bsdf_lambert(Rgb a) {
    Bsdf b;
    b.diffuse = rgb(rclamp(a.r, 0.0f, 1.0f), rclamp(a.g, 0.0f, 1.0f), rclamp(a.b, 0.0f, 1.0f));
    b.metal_f0 = splat(0.0f); b.metal_f90 = splat(0.0f);
    b.metallic = 0.0f; b.dielectric = 1.0f; b.f0 = 0.0f; b.f90 = 0.0f;
    b.spec = make_ggx(1.0f, 0.0f);
    b.coat = 0.0f;
    b.coat_ggx = make_ggx(1.0f, 0.0f);
    b.clear = 0.0f; b.eta = 1.0f; b.tint = splat(1.0f); b.thin = false;
    b.ms_spec_on = false; b.ms_coat_on = false; b.ms_clear_on = false;
    b.ms_spec_lobe.on = false; b.ms_coat_lobe.on = false;
    b.ms_spec_colour = splat(0.0f); b.ms_coat_c = 0.0f; b.ms_clear_alpha = 0.0f;
    b.base_layer = layer_clear(); b.coat_layer = layer_clear();
    b.diffuse_norm = 1.0f;
    return b;
}

// Bsdf::surface_at (bsdf.rs:382) with multiple_scattering (bsdf.rs:445) and layers (bsdf.rs:423).
RTG_HD Bsdf bsdf_surface(const EnergyTables& E, const DevMaterial& m, bool entering) {
    Rgb base = rgb(rclamp(m.base[0], 0.0f, 1.0f), rclamp(m.base[1], 0.0f, 1.0f), rclamp(m.base[2], 0.0f, 1.0f));
    float metallic = m.kind == MATERIAL_GLASS ? 0.0f : rclamp(m.metallic, 0.0f, 1.0f);
    float transmission = rclamp(m.transmission, 0.0f, 1.0f);
    float ior = rmax(m.ior, 1.0f);
    float f0 = ((ior - 1.0f) / (ior + 1.0f)) * ((ior - 1.0f) / (ior + 1.0f));
    float roughness = rclamp(m.roughness, 0.0f, 1.0f);
    float coat_roughness = rclamp(m.coat_roughness, 0.0f, 1.0f);
    float anisotropy = rclamp(m.anisotropy, 0.0f, 1.0f);
    float clear = (1.0f - metallic) * transmission;
    bool thin = (m.flags & MATERIAL_FLAG_THIN) != 0 || ior < 1.0001f;
    Bsdf b;
    b.eta = (thin || entering) ? ior : 1.0f / ior;
    if (thin) b.tint = base;
    else if (m.absorption_mm > 0.0f) b.tint = splat(1.0f);
    else b.tint = rgb(sqrt_(base.r), sqrt_(base.g), sqrt_(base.b));
    b.coat = (clear > 0.0f && !thin && !entering) ? 0.0f : rclamp(m.coat, 0.0f, 1.0f);
    b.diffuse = base * ((1.0f - metallic) * (1.0f - transmission));
    b.metal_f0 = base;
    b.metal_f90 = rgb(rmin(50.0f * base.r, 1.0f), rmin(50.0f * base.g, 1.0f), rmin(50.0f * base.b, 1.0f));
    b.metallic = metallic;
    b.dielectric = (1.0f - metallic) * (1.0f - transmission);
    b.f0 = f0;
    b.f90 = rmin(50.0f * f0, 1.0f);
    b.spec = make_ggx(rmax(roughness * roughness, MIN_ALPHA), anisotropy);
    b.coat_ggx = make_ggx(rmax(coat_roughness * coat_roughness, MIN_ALPHA), 0.0f);
    b.clear = clear;
    b.thin = thin;
    // multiple_scattering
    float alpha = b.spec.iso ? b.spec.ax : sqrt_(b.spec.ax * b.spec.ay);
    b.ms_spec_on = false; b.ms_coat_on = false; b.ms_clear_on = false;
    b.ms_spec_colour = splat(0.0f); b.ms_coat_c = 0.0f; b.ms_clear_alpha = 0.0f;
    b.ms_spec_lobe.on = false; b.ms_coat_lobe.on = false;
    MsLobe lobe = make_lobe(E, alpha);
    if (lobe.on && has_specular(b)) {
        float diel = b.dielectric > 0.0f ? b.dielectric * multiple_fresnel(schlick_average(b.f0, b.f90), lobe.e_avg) : 0.0f;
        Rgb colour;
        if (b.metallic > 0.0f) {
            colour = rgb(multiple_fresnel(schlick_average(b.metal_f0.r, b.metal_f90.r), lobe.e_avg),
                         multiple_fresnel(schlick_average(b.metal_f0.g, b.metal_f90.g), lobe.e_avg),
                         multiple_fresnel(schlick_average(b.metal_f0.b, b.metal_f90.b), lobe.e_avg)) *
                         b.metallic +
                     splat(diel);
        } else {
            colour = splat(diel);
        }
        if (peak(colour) > 0.0f) { b.ms_spec_on = true; b.ms_spec_lobe = lobe; b.ms_spec_colour = colour; }
    }
    if (b.coat > 0.0f) {
        MsLobe cl = make_lobe(E, b.coat_ggx.ax);
        if (cl.on) {
            float c = b.coat * multiple_fresnel(schlick_average(COAT_F0, 1.0f), cl.e_avg);
            if (c > 0.0f) { b.ms_coat_on = true; b.ms_coat_lobe = cl; b.ms_coat_c = c; }
        }
    }
    if (clear > 0.0f && !thin && alpha >= MIN_COMPENSATED_ALPHA) { b.ms_clear_on = true; b.ms_clear_alpha = alpha; }
    // layers
    b.base_layer = layer_clear();
    b.coat_layer = layer_clear();
    if (b.diffuse.r > 0.0f || b.diffuse.g > 0.0f || b.diffuse.b > 0.0f) {
        float ms = b.ms_spec_on ? multiple_fresnel(schlick_average(b.f0, b.f90), b.ms_spec_lobe.e_avg) : 0.0f;
        b.base_layer = make_layer(E, b.f0, b.f90, 1.0f, alpha, ms);
    }
    if (b.coat > 0.0f) {
        float ms = b.ms_coat_on ? multiple_fresnel(schlick_average(COAT_F0, 1.0f), b.ms_coat_lobe.e_avg) : 0.0f;
        b.coat_layer = make_layer(E, COAT_F0, 1.0f, b.coat, b.coat_ggx.ax, ms);
    }
    b.diffuse_norm = joint_norm(E, b.base_layer, b.coat_layer);
    return b;
}

RTG_HD Rgb specular_fresnel(const Bsdf& b, float cos) {
    float d = schlick(b.f0, b.f90, cos);
    if (b.metallic <= 0.0f && b.clear <= 0.0f) return splat(d);
    Rgb metal = rgb(schlick(b.metal_f0.r, b.metal_f90.r, cos), schlick(b.metal_f0.g, b.metal_f90.g, cos),
                    schlick(b.metal_f0.b, b.metal_f90.b, cos));
    return splat(d) * b.dielectric + metal * b.metallic;
}
RTG_HD float coat_fresnel(const Bsdf& b, float cos) { return b.coat <= 0.0f ? 0.0f : b.coat * schlick(COAT_F0, 1.0f, cos); }
RTG_HD float clear_fresnel(const Bsdf& b, float cos) { return b.thin ? thin_reflectance(cos, b.eta) : fresnel_dielectric(cos, b.eta); }
RTG_HD float reflect_probability(const Bsdf& b, float cos) { return rmin(clear_fresnel(b, cos), MAX_REFLECT_PROBABILITY); }
RTG_HD float reflect_chance(const Bsdf& b, float mu_o, float cos_h) {
    return b.ms_clear_on ? clear_fresnel(b, cos_h) : reflect_probability(b, mu_o);
}
RTG_HD bool clear_compensation(const EnergyTables& E, const Bsdf& b, float mu_o, float& k) {
    if (!b.ms_clear_on) return false;
    float e = clear_albedo(E, mu_o, b.ms_clear_alpha, b.eta);
    k = 1.0f / rmax(e, 0.05f);
    return true;
}
RTG_HD Rgb straight_transmittance(const Bsdf& b, float cos) {
    if (!(b.thin && b.clear > 0.0f)) return splat(0.0f);
    cos = rmin(absf(cos), 1.0f);
    float t = 1.0f - thin_reflectance(cos, b.eta);
    return b.tint * (b.clear * (1.0f - coat_fresnel(b, cos)) * t);
}

RTG_HD LobeWeights lobe_weights(const EnergyTables& E, const Bsdf& b, V3 wo) {
    float c = coat_fresnel(b, wo.z);
    float below = 1.0f - c;
    float specular = has_specular(b) ? below * rmax(luminance(specular_fresnel(b, wo.z)), 0.0f) : 0.0f;
    float diff = below * luminance(b.diffuse) * layer_passes(E, b.base_layer, wo.z);
    float cl = below * b.clear;
    float ms = 0.0f;
    if (b.ms_spec_on) ms += below * rmax(luminance(b.ms_spec_colour), 0.0f) * lobe_lost(E, b.ms_spec_lobe, wo.z);
    if (b.ms_coat_on) ms += b.ms_coat_c * lobe_lost(E, b.ms_coat_lobe, wo.z);
    float total = c + specular + diff + cl + ms;
    LobeWeights w;
    if (total > 0.0f) {
        float inv = 1.0f / total;
        w.coat = c * inv; w.specular = specular * inv; w.diffuse = diff * inv; w.clear = cl * inv; w.ms = ms * inv;
    } else {
        w.coat = 0; w.specular = 0; w.diffuse = 0; w.clear = 0; w.ms = 0;
    }
    return w;
}

RTG_HD bool refraction_half(const Bsdf& b, V3 wo, V3 wi, V3& h, float& co, float& ci) {
    h = normalize(wo + wi * b.eta);
    if (h.z < 0.0f) h = -h;
    co = dot(wo, h);
    ci = dot(wi, h);
    return co > 0.0f && ci < 0.0f && len2(h) > 0.5f;
}
RTG_HD Rgb eval_refraction(const EnergyTables& E, const Bsdf& b, V3 wo, V3 wi) {
    V3 h; float co, ci;
    if (!refraction_half(b, wo, wi, h, co, ci)) return splat(0.0f);
    float f = fresnel_dielectric(co, b.eta);
    float denom = co + b.eta * ci;
    float g2 = 1.0f / (1.0f + ggx_L(b.spec, wo) + ggx_L(b.spec, wi));
    float value = (1.0f - f) * ggx_D(b.spec, h) * g2 * (-ci) * co / (-wi.z * wo.z * denom * denom);
    float k;
    if (clear_compensation(E, b, wo.z, k)) value *= k;
    float attenuation = layer_passes(E, b.coat_layer, wo.z);
    return b.tint * (b.clear * attenuation * value);
}
RTG_HD_NI Rgb bsdf_eval(const EnergyTables& E, const Bsdf& b, V3 wo, V3 wi, int lobes) {
    if (wo.z <= 0.0f) return splat(0.0f);
    if (wi.z <= 0.0f) {
        if (wi.z < 0.0f && lobes == LOBES_ALL && b.clear > 0.0f && !b.thin) return eval_refraction(E, b, wo, wi);
        return splat(0.0f);
    }
    float attenuation = layer_passes(E, b.coat_layer, wo.z) * layer_passes(E, b.coat_layer, wi.z);
    Rgb diff = b.diffuse * (FRAC_1_PI * layer_passes(E, b.base_layer, wo.z) * layer_passes(E, b.base_layer, wi.z) * b.diffuse_norm);
    if (lobes == LOBES_DIFFUSE) return diff * attenuation;
    V3 h = normalize(wo + wi);
    float cos_h = rmax(dot(wo, h), 0.0f);
    Rgb below = diff;
    if (has_specular(b)) below = below + specular_fresnel(b, cos_h) * ggx_microfacet(b.spec, wo, wi, h);
    if (b.ms_spec_on) below = below + b.ms_spec_colour * (lobe_lost(E, b.ms_spec_lobe, wo.z) * lobe_lost(E, b.ms_spec_lobe, wi.z) * b.ms_spec_lobe.norm);
    if (b.clear > 0.0f) {
        float cl = b.clear * clear_fresnel(b, cos_h) * ggx_microfacet(b.spec, wo, wi, h);
        float k;
        if (clear_compensation(E, b, wo.z, k)) cl *= k;
        below = below + splat(cl);
    }
    Rgb f = below * attenuation;
    if (b.coat > 0.0f) f = f + splat(coat_fresnel(b, cos_h) * ggx_microfacet(b.coat_ggx, wo, wi, h));
    if (b.ms_coat_on) f = f + splat(b.ms_coat_c * (lobe_lost(E, b.ms_coat_lobe, wo.z) * lobe_lost(E, b.ms_coat_lobe, wi.z) * b.ms_coat_lobe.norm));
    return f;
}
RTG_HD float pdf_with(const Bsdf& b, const LobeWeights& w, V3 wo, V3 wi) {
    float p = (w.diffuse + w.ms) * wi.z * FRAC_1_PI;
    if (w.specular > 0.0f || w.coat > 0.0f || w.clear > 0.0f) {
        V3 h = normalize(wo + wi);
        if (dot(wo, h) > 0.0f) {
            if (w.specular > 0.0f) p += w.specular * ggx_reflection_pdf(b.spec, wo, h);
            if (w.coat > 0.0f) p += w.coat * ggx_reflection_pdf(b.coat_ggx, wo, h);
            if (w.clear > 0.0f) p += w.clear * reflect_chance(b, wo.z, dot(wo, h)) * ggx_reflection_pdf(b.spec, wo, h);
        }
    }
    return p;
}
RTG_HD float refraction_pdf(const Bsdf& b, const LobeWeights& w, V3 wo, V3 wi) {
    if (w.clear != w.clear || w.clear <= 0.0f) return 0.0f;
    V3 h; float co, ci;
    if (!refraction_half(b, wo, wi, h, co, ci)) return 0.0f;
    float g1 = 1.0f / (1.0f + ggx_L(b.spec, wo));
    float visible = g1 * ggx_D(b.spec, h) * co / wo.z;
    float denom = co + b.eta * ci;
    float jacobian = b.eta * b.eta * (-ci) / (denom * denom);
    return w.clear * (1.0f - reflect_chance(b, wo.z, co)) * visible * jacobian;
}
RTG_HD_NI float bsdf_pdf(const EnergyTables& E, const Bsdf& b, V3 wo, V3 wi) {
    if (wo.z <= 0.0f) return 0.0f;
    if (wi.z <= 0.0f) {
        if (wi.z < 0.0f && b.clear > 0.0f && !b.thin) return refraction_pdf(b, lobe_weights(E, b, wo), wo, wi);
        return 0.0f;
    }
    return pdf_with(b, lobe_weights(E, b, wo), wo, wi);
}

RTG_HD bool finish_reflection(const EnergyTables& E, const Bsdf& b, const LobeWeights& w, V3 wo, V3 wi, BsdfSample& out) {
    if (wi.z <= 0.0f) return false;
    float p = pdf_with(b, w, wo, wi);
    if (!(p > 0.0f && finitef(p))) return false;
    out.weight = bsdf_eval(E, b, wo, wi, LOBES_ALL) * (wi.z / p);
    out.wi = wi; out.pdf = p; out.straight = false;
    return true;
}
RTG_HD bool finish_refraction(const EnergyTables& E, const Bsdf& b, const LobeWeights& w, V3 wo, V3 h, BsdfSample& out) {
    V3 wi;
    if (!refract(wo, h, b.eta, wi)) return false;
    if (wi.z >= 0.0f) return false;
    float p = refraction_pdf(b, w, wo, wi);
    if (!(p > 0.0f && finitef(p))) return false;
    out.weight = eval_refraction(E, b, wo, wi) * (-wi.z / p);
    out.wi = wi; out.pdf = p; out.straight = false;
    return true;
}
RTG_HD_NI bool bsdf_sample(const EnergyTables& E, const Bsdf& b, V3 wo, float u0, float u1, BsdfSample& out) {  // bsdf.rs:833
    if (wo.z <= 0.0f) return false;
    LobeWeights w = lobe_weights(E, b, wo);
    V3 wi;
    if (u0 < w.coat) {
        V3 h = sample_vndf(wo, b.coat_ggx.ax, b.coat_ggx.ay, u0 / w.coat, u1);
        wi = h * (2.0f * dot(wo, h)) - wo;
    } else if (u0 < w.coat + w.specular) {
        V3 h = sample_vndf(wo, b.spec.ax, b.spec.ay, (u0 - w.coat) / w.specular, u1);
        wi = h * (2.0f * dot(wo, h)) - wo;
    } else if (w.diffuse + w.ms > 0.0f && (w.clear <= 0.0f || u0 < w.coat + w.specular + (w.diffuse + w.ms))) {
        float start = w.coat + w.specular;
        float uu = rclamp((u0 - start) / (w.diffuse + w.ms), 0.0f, 0.99999994f);
        wi = cosine_hemisphere(uu, u1);
    } else if (w.clear > 0.0f) {
        // sample_clear (bsdf.rs:889)
        float start = w.coat + w.specular + (w.diffuse + w.ms);
        float uc = rclamp((u0 - start) / w.clear, 0.0f, 0.99999994f);
        if (b.ms_clear_on) {
            // sample_rough_clear (bsdf.rs:947)
            V3 h = sample_vndf(wo, b.spec.ax, b.spec.ay, uc, u1);
            float fr = clear_fresnel(b, dot(wo, h));
            uint64_t key = ((uint64_t)fbits(uc) << 32) | (uint64_t)fbits(u1);
            float choice = (float)(mix64(key ^ 0x9e3779b97f4a7c15ULL) >> 40) * (1.0f / 16777216.0f);
            if (choice < fr) return finish_reflection(E, b, w, wo, h * (2.0f * dot(wo, h)) - wo, out);
            return finish_refraction(E, b, w, wo, h, out);
        }
        float pr = reflect_probability(b, wo.z);
        if (uc < pr) {
            V3 h = sample_vndf(wo, b.spec.ax, b.spec.ay, uc / pr, u1);
            return finish_reflection(E, b, w, wo, h * (2.0f * dot(wo, h)) - wo, out);
        }
        if (b.thin) {
            float chance = w.clear * (1.0f - pr);
            if (chance != chance || chance <= 0.0f) return false;
            out.weight = straight_transmittance(b, wo.z) / chance;
            out.wi = -wo; out.pdf = chance; out.straight = true;
            return true;
        }
        float ut = rclamp((uc - pr) / (1.0f - pr), 0.0f, 0.99999994f);
        V3 h = sample_vndf(wo, b.spec.ax, b.spec.ay, ut, u1);
        return finish_refraction(E, b, w, wo, h, out);
    } else {
        return false;
    }
    return finish_reflection(E, b, w, wo, wi, out);
}

}  // namespace rtg
