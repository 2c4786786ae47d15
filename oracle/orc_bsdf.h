// ORACLE (test infrastructure only). Restatement of the reference's principled BSDF and its
// multiple-scattering energy compensation (engine/crates/rt-core/src/bsdf.rs,
// bsdf/energy.rs, bsdf/forward.rs:138-200 without the particle forward lobe).
#pragma once
#include <cstdint>
#include <vector>

#include "orc_core.h"

namespace orc {

constexpr float MIN_ALPHA = 1.0e-3f;                 // bsdf.rs:91
constexpr float COAT_F0 = 0.04f;                     // bsdf.rs:93
constexpr float MAX_REFLECT_PROBABILITY = 0.99f;     // bsdf.rs:95
constexpr float MIN_COMPENSATED_ALPHA = 2.0e-3f;     // energy.rs:58
constexpr int NODES_MU = 32, NODES_ROUGHNESS = 32, NODES_IOR = 17;  // energy.rs:60-64
constexpr float MAX_IOR = 3.0f;
constexpr uint64_t ENERGY_SEED = 0xe9ae9aULL;        // energy.rs:68
constexpr uint32_t ENERGY_STRATA = 64;

// The six energy tables of energy_table.rs, generated by `generate_energy_tables` with the
// reference's recipe (energy.rs:130-300): Monte Carlo with a fixed seed.
struct EnergyTables {
    std::vector<uint16_t> albedo, schlick, clear_in, clear_out;  // 1024, 1024, 17408, 17408
    std::vector<float> albedo_avg, schlick_avg;                   // 32, 32
};
const EnergyTables& energy_tables();  // generated once, multithreaded
void generate_energy_tables(EnergyTables& out, int threads);

// ---- GGX (bsdf.rs:118-205) -------------------------------------------------------------------
inline float ggx_d(Vec3 h, float a2) {  // bsdf.rs:248
    float t = a2 * h.z * h.z + (h.x * h.x + h.y * h.y);
    if (t <= 0.0f) return 0.0f;
    return a2 / (PI * t * t);
}
inline float ggx_lambda(Vec3 w, float a2) {  // bsdf.rs:258
    float cos2 = w.z * w.z;
    if (cos2 <= 0.0f) return F_INF;
    float tan2 = (w.x * w.x + w.y * w.y) / cos2;
    return (std::sqrt(1.0f + a2 * tan2) - 1.0f) * 0.5f;
}
struct Ggx {
    float ax = 1, ay = 1, a2 = 1;
    bool iso = true;
    static Ggx make(float alpha, float anisotropy) {
        Ggx g;
        if (anisotropy > 0.0f) {
            float s = std::sqrt(1.0f - 0.9f * anisotropy);
            g.ax = rmax(alpha / s, MIN_ALPHA);
            g.ay = rmax(alpha * s, MIN_ALPHA);
            g.a2 = alpha * alpha;
            g.iso = false;
        } else {
            g.ax = alpha; g.ay = alpha; g.a2 = alpha * alpha; g.iso = true;
        }
        return g;
    }
    float d(Vec3 h) const {
        if (iso) return ggx_d(h, a2);
        float x = h.x / ax, y = h.y / ay;
        float t = x * x + y * y + h.z * h.z;
        if (t <= 0.0f) return 0.0f;
        return 1.0f / (PI * ax * ay * t * t);
    }
    float lambda(Vec3 w) const {
        if (iso) return ggx_lambda(w, a2);
        float cos2 = w.z * w.z;
        if (cos2 <= 0.0f) return F_INF;
        float x = ax * w.x, y = ay * w.y;
        return (std::sqrt(1.0f + (x * x + y * y) / cos2) - 1.0f) * 0.5f;
    }
    float reflection_pdf(Vec3 wo, Vec3 h) const {
        float g1 = 1.0f / (1.0f + lambda(wo));
        return g1 * d(h) / (4.0f * wo.z);
    }
    float microfacet(Vec3 wo, Vec3 wi, Vec3 h) const {
        float g2 = 1.0f / (1.0f + lambda(wo) + lambda(wi));
        return d(h) * g2 / (4.0f * wo.z * wi.z);
    }
};

inline float schlick(float f0, float f90, float cos) {  // bsdf.rs:213
    float m = rclamp(1.0f - cos, 0.0f, 1.0f);
    float m2 = m * m;
    return f0 + (f90 - f0) * (m2 * m2 * m);
}
inline float fresnel_dielectric(float cos_i, float eta) {  // bsdf.rs:222
    cos_i = rclamp(cos_i, 0.0f, 1.0f);
    float sin2_t = (1.0f - cos_i * cos_i) / (eta * eta);
    if (sin2_t >= 1.0f) return 1.0f;
    float cos_t = std::sqrt(1.0f - sin2_t);
    float rs = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    float rp = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    return 0.5f * (rs * rs + rp * rp);
}
inline float thin_reflectance(float cos, float eta) {
    float r = fresnel_dielectric(cos, eta);
    return 2.0f * r / (1.0f + r);
}
inline bool refract(Vec3 wo, Vec3 h, float eta, Vec3& out) {  // bsdf.rs:237
    float cos_i = dot(wo, h);
    float sin2_t = (1.0f - cos_i * cos_i) / (eta * eta);
    if (sin2_t >= 1.0f) return false;
    float cos_t = std::sqrt(1.0f - sin2_t);
    out = normalize(h * (cos_i / eta - cos_t) - wo / eta);
    return true;
}
inline Vec3 sample_vndf(Vec3 wo, float ax, float ay, float u0, float u1) {  // bsdf.rs:269
    Vec3 vh = normalize(Vec3(ax * wo.x, ay * wo.y, wo.z));
    float lensq = vh.x * vh.x + vh.y * vh.y;
    Vec3 t1 = lensq > 0.0f ? Vec3(-vh.y, vh.x, 0.0f) / std::sqrt(lensq) : Vec3(1.0f, 0.0f, 0.0f);
    Vec3 t2 = cross(vh, t1);
    float r = std::sqrt(u0);
    float sp, cp;
    sin_cos(TAU * u1, sp, cp);
    float p1 = r * cp;
    float s = 0.5f * (1.0f + vh.z);
    float p2 = (1.0f - s) * std::sqrt(rmax(1.0f - p1 * p1, 0.0f)) + s * (r * sp);
    Vec3 nh = t1 * p1 + t2 * p2 + vh * std::sqrt(rmax(1.0f - p1 * p1 - p2 * p2, 0.0f));
    return normalize(Vec3(ax * nh.x, ay * nh.y, rmax(nh.z, 1.0e-7f)));
}

// ---- energy.rs lookups ------------------------------------------------------------------------
inline void locate(float x, int n, int& i, float& w) {  // energy.rs:305
    float t = rclamp(x, 0.0f, 1.0f) * (float)(n - 1);
    uint64_t ti = f2usize(t);
    i = (int)(ti < (uint64_t)(n - 2) ? ti : (uint64_t)(n - 2));
    w = t - (float)i;
}
inline float table_lookup(const uint16_t* table, float mu, float alpha) {  // energy.rs:313
    const float UNIT = 1.0f / 65535.0f;
    int i, j;
    float u, v;
    locate(std::sqrt(rmax(mu, 0.0f)), NODES_MU, i, u);
    locate(std::sqrt(rmax(alpha, 0.0f)), NODES_ROUGHNESS, j, v);
    auto at = [&](int jj, int ii) { return (float)table[jj * NODES_MU + ii] * UNIT; };
    float low = at(j, i) + (at(j, i + 1) - at(j, i)) * u;
    float high = at(j + 1, i) + (at(j + 1, i + 1) - at(j + 1, i)) * u;
    return low + (high - low) * v;
}
inline float albedo(float mu, float alpha) { return table_lookup(energy_tables().albedo.data(), mu, alpha); }
inline float schlick_albedo(float mu, float alpha) { return table_lookup(energy_tables().schlick.data(), mu, alpha); }
inline float avg_lookup(const std::vector<float>& t, float alpha) {
    int j; float v;
    locate(std::sqrt(rmax(alpha, 0.0f)), NODES_ROUGHNESS, j, v);
    return t[j] + (t[j + 1] - t[j]) * v;
}
inline float albedo_avg(float alpha) { return avg_lookup(energy_tables().albedo_avg, alpha); }
inline float schlick_avg(float alpha) { return avg_lookup(energy_tables().schlick_avg, alpha); }
inline float schlick_average(float f0, float f90) { return f0 + (f90 - f0) * (1.0f / 21.0f); }
inline float multiple_fresnel(float f_avg, float e_avg) {
    float d = 1.0f - f_avg * (1.0f - e_avg);
    return d > 0.0f ? f_avg * f_avg * e_avg / d : 0.0f;
}
inline float clear_albedo(float mu, float alpha, float eta) {  // energy.rs:482
    const EnergyTables& t = energy_tables();
    const std::vector<uint16_t>& table = eta >= 1.0f ? t.clear_in : t.clear_out;
    float ior = eta >= 1.0f ? eta : 1.0f / eta;
    const float MAX_X = (MAX_IOR - 1.0f) / (MAX_IOR + 1.0f);
    float x = (ior - 1.0f) / (ior + 1.0f);
    int k; float w;
    locate(x / MAX_X, NODES_IOR, k, w);
    int slice = NODES_MU * NODES_ROUGHNESS;
    float a = table_lookup(table.data() + k * slice, mu, alpha);
    float b = table_lookup(table.data() + (k + 1) * slice, mu, alpha);
    return a + (b - a) * w;
}

struct Layer {  // energy.rs:368
    float f0 = 0, f90 = 0, strength = 0;
    bool rough = false;
    float r_alpha = 0, r_ms = 0;
    float norm = 1.0f;
    static Layer clear() { return Layer(); }
    static Layer make(float f0, float f90, float strength, float alpha, float ms) {
        if (strength != strength || strength <= 0.0f || (f90 <= 0.0f && f0 <= 0.0f)) return Layer();
        Layer l;
        l.f0 = f0; l.f90 = f90; l.strength = strength;
        l.rough = alpha >= MIN_COMPENSATED_ALPHA;
        l.r_alpha = alpha; l.r_ms = ms;
        float avg;
        if (l.rough) {
            float e_avg = albedo_avg(alpha);
            avg = f0 * e_avg + (f90 - f0) * schlick_avg(alpha) + ms * (1.0f - e_avg);
        } else {
            avg = schlick_average(f0, f90);
        }
        avg = avg * strength;
        l.norm = 1.0f / (1.0f - rmin(avg, 0.999f));
        return l;
    }
    float albedo_at(float mu) const {
        float e;
        if (rough) {
            float ee = albedo(mu, r_alpha);
            e = f0 * ee + (f90 - f0) * schlick_albedo(mu, r_alpha) + r_ms * (1.0f - ee);
        } else {
            float m = rclamp(1.0f - mu, 0.0f, 1.0f);
            float m2 = m * m;
            e = f0 + (f90 - f0) * (m2 * m2 * m);
        }
        return rclamp(e * strength, 0.0f, 1.0f);
    }
    float passes(float mu) const { return 1.0f - albedo_at(mu); }
    bool is_clear() const { return strength <= 0.0f; }
};
// 8-point Gauss–Legendre on [0, 1] (energy.rs:454): the textbook nodes and weights.
constexpr float GAUSS_8[8][2] = {
    {0.019855072f, 0.05061427f}, {0.10166676f, 0.11119052f}, {0.2372338f, 0.15685332f},
    {0.40828268f, 0.18134189f},  {0.5917173f, 0.18134189f},  {0.7627662f, 0.15685332f},
    {0.8983332f, 0.11119052f},   {0.9801449f, 0.05061427f}};
inline float joint_norm(const Layer& below, const Layer& above) {  // energy.rs:472
    if (above.is_clear()) return below.norm;
    if (below.is_clear()) return above.norm;
    float sum = 0.0f;
    for (int i = 0; i < 8; ++i) {
        float mu = GAUSS_8[i][0], w = GAUSS_8[i][1];
        sum = sum + w * 2.0f * mu * below.passes(mu) * above.passes(mu);
    }
    return 1.0f / rmax(sum, 0.001f);
}
struct Lobe {  // energy.rs:520
    bool on = false;
    float alpha = 0, norm = 0, e_avg = 0;
    static Lobe make(float alpha) {
        Lobe l;
        if (alpha != alpha || alpha < MIN_COMPENSATED_ALPHA) return l;
        float e_avg = albedo_avg(alpha);
        float lost = 1.0f - e_avg;
        if (!(lost > 1.0e-6f)) return l;
        l.on = true; l.alpha = alpha; l.norm = FRAC_1_PI / lost; l.e_avg = e_avg;
        return l;
    }
    float lost(float mu) const { return rmax(1.0f - albedo(mu, alpha), 0.0f); }
    float shape(float mu_o, float mu_i) const { return lost(mu_o) * lost(mu_i) * norm; }
};

// ---- Material (scene/mod.rs:365-466) -----------------------------------------------------------
constexpr uint32_t MATERIAL_PRINCIPLED = 0, MATERIAL_GLASS = 1, MATERIAL_EMISSIVE = 2;
constexpr uint32_t MATERIAL_FLAG_LIGHT = 1, MATERIAL_FLAG_THIN = 2;
struct Material {
    uint32_t kind = MATERIAL_PRINCIPLED;
    Rgb base_color = Rgb::splat(0.8f);
    float metallic = 0.0f, roughness = 0.5f, ior = 1.5f, transmission = 0.0f;
    float coat = 0.0f, coat_roughness = 0.0f;
    Rgb emission = BLACK;
    float emission_power = 0.0f;
    uint32_t flags = 0;
    float opacity = 1.0f, anisotropy = 0.0f, absorption_mm = 0.0f, bevel_mm = 0.0f;
    float scatter_mm = 0.0f;
    Rgb scatter_color = WHITE;
    float scatter_g = 0.0f, abbe = 0.0f;
    bool is_emissive() const { return kind == MATERIAL_EMISSIVE; }
    Rgb radiance() const {
        if (!is_emissive()) return BLACK;
        Rgb e = emission * emission_power;
        return {rmax(e.r, 0.0f), rmax(e.g, 0.0f), rmax(e.b, 0.0f)};
    }
};

enum class Lobes { All, Diffuse };
struct BsdfSample { Vec3 wi; Rgb weight; float pdf; bool straight; };

struct Bsdf {  // bsdf.rs:309
    Rgb diffuse, metal_f0, metal_f90;
    float metallic = 0, dielectric = 0, f0 = 0, f90 = 0;
    Ggx spec;
    float coat = 0;
    Ggx coat_ggx;
    float clear = 0, eta = 1;
    Rgb tint = WHITE;
    bool thin = false;
    // MultiScatter
    bool ms_spec_on = false; Lobe ms_spec_lobe; Rgb ms_spec_colour;
    bool ms_coat_on = false; Lobe ms_coat_lobe; float ms_coat_c = 0;
    bool ms_clear_on = false; float ms_clear_alpha = 0;
    Layer base_layer, coat_layer;
    float diffuse_norm = 1.0f;

    static Bsdf surface_at(const Material& m, bool entering, float ior_in);
    static Bsdf surface(const Material& m, bool entering) { return surface_at(m, entering, m.ior); }
    static Bsdf lambert(Rgb albedo_);

    bool has_specular() const { return (f90 > 0.0f && dielectric > 0.0f) || metallic > 0.0f; }
    Rgb specular_fresnel(float cos) const;
    float coat_fresnel(float cos) const { return coat <= 0.0f ? 0.0f : coat * schlick(COAT_F0, 1.0f, cos); }
    float clear_fresnel(float cos) const { return thin ? thin_reflectance(cos, eta) : fresnel_dielectric(cos, eta); }
    float reflect_probability(float cos) const { return rmin(clear_fresnel(cos), MAX_REFLECT_PROBABILITY); }
    float reflect_chance(float mu_o, float cos_h) const {
        return ms_clear_on ? clear_fresnel(cos_h) : reflect_probability(mu_o);
    }
    bool clear_compensation(float mu_o, float& k) const {
        if (!ms_clear_on) return false;
        float e = clear_albedo(mu_o, ms_clear_alpha, eta);
        k = 1.0f / rmax(e, 0.05f);
        return true;
    }
    Rgb straight_transmittance(float cos) const;

    struct LobeWeights { float coat, specular, diffuse, clear, ms; };
    LobeWeights lobe_weights(Vec3 wo) const;
    Rgb eval(Vec3 wo, Vec3 wi, Lobes lobes) const;
    bool refraction_half(Vec3 wo, Vec3 wi, Vec3& h, float& co, float& ci) const;
    Rgb eval_refraction(Vec3 wo, Vec3 wi) const;
    float pdf(Vec3 wo, Vec3 wi) const;
    float pdf_with(const LobeWeights& w, Vec3 wo, Vec3 wi) const;
    float refraction_pdf(const LobeWeights& w, Vec3 wo, Vec3 wi) const;
    bool sample(Vec3 wo, float u0, float u1, BsdfSample& out) const;
    bool sample_clear(const LobeWeights& w, Vec3 wo, float u0, float u1, BsdfSample& out) const;
    bool sample_rough_clear(const LobeWeights& w, Vec3 wo, float u0, float u1, BsdfSample& out) const;

   private:
    void multiple_scattering();
    void layers();
};

}  // namespace orc
