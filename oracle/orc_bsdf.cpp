// ORACLE (test infrastructure only). Principled BSDF (bsdf.rs:360-993) and the energy-table
// generator (bsdf/energy.rs:107-300), restated from the reference.
#include "orc_bsdf.h"

#include <atomic>
#include <mutex>
#include <thread>

namespace orc {

// ---- energy table generator (energy.rs:73-300) -------------------------------------------------
static float node_mu(int i) {
    float t = (float)i / (float)(NODES_MU - 1);
    return rmax(t * t, 1.0f / 2048.0f);
}
static float node_alpha(int j) {
    float r = (float)j / (float)(NODES_ROUGHNESS - 1);
    return r * r;
}
static float node_ior(int k) {
    const float MAX_X = (MAX_IOR - 1.0f) / (MAX_IOR + 1.0f);
    float x = MAX_X * (float)k / (float)(NODES_IOR - 1);
    return (1.0f + x) / (1.0f - x);
}
static Vec3 outgoing(float mu) { return {std::sqrt(rmax(1.0f - mu * mu, 0.0f)), 0.0f, mu}; }
static void jitter(Pcg32& rng, uint32_t s, uint32_t strata, float& a, float& b) {
    uint32_t i = s % strata, j = s / strata;
    float inv = 1.0f / (float)strata;
    float r0 = rng.next_f32();
    float r1 = rng.next_f32();
    a = rmin(((float)i + r0) * inv, 0.99999994f);
    b = rmin(((float)j + r1) * inv, 0.99999994f);
}
static double g2_over_g1(const Ggx& g, Vec3 wo, Vec3 wi) {
    float lo = g.lambda(wo), li = g.lambda(wi);
    return (double)((1.0f + lo) / (1.0f + lo + li));
}
static double integrate_albedo(float mu, float alpha, uint32_t strata, uint64_t stream) {
    if (alpha <= 0.0f) return 1.0;
    Ggx g = Ggx::make(alpha, 0.0f);
    Vec3 wo = outgoing(mu);
    Pcg32 rng = Pcg32::seeded(ENERGY_SEED, stream);
    double sum = 0.0;
    uint32_t n = strata * strata;
    for (uint32_t s = 0; s < n; ++s) {
        float a, b;
        jitter(rng, s, strata, a, b);
        Vec3 h = sample_vndf(wo, alpha, alpha, a, b);
        Vec3 wi = h * (2.0f * dot(wo, h)) - wo;
        if (wi.z > 0.0f) sum += g2_over_g1(g, wo, wi);
    }
    return sum / (double)n;
}
static double integrate_schlick(float mu, float alpha, uint32_t strata, uint64_t stream) {
    if (alpha <= 0.0f) {
        double m = (double)(1.0f - mu);
        return m * m * m * m * m;
    }
    Ggx g = Ggx::make(alpha, 0.0f);
    Vec3 wo = outgoing(mu);
    Pcg32 rng = Pcg32::seeded(ENERGY_SEED ^ 0x5c41ULL, stream);
    double sum = 0.0;
    uint32_t n = strata * strata;
    for (uint32_t s = 0; s < n; ++s) {
        float a, b;
        jitter(rng, s, strata, a, b);
        Vec3 h = sample_vndf(wo, alpha, alpha, a, b);
        float c = dot(wo, h);
        Vec3 wi = h * (2.0f * c) - wo;
        if (wi.z > 0.0f) {
            double m = (double)rclamp(1.0f - c, 0.0f, 1.0f);
            sum += m * m * m * m * m * g2_over_g1(g, wo, wi);
        }
    }
    return sum / (double)n;
}
static double integrate_clear(float mu, float alpha, float eta, uint32_t strata, uint64_t stream) {
    if (alpha <= 0.0f || std::fabs(eta - 1.0f) < 1.0e-6f) return 1.0;
    Ggx g = Ggx::make(alpha, 0.0f);
    Vec3 wo = outgoing(mu);
    Pcg32 rng = Pcg32::seeded(ENERGY_SEED ^ 0xc1eaULL, stream);
    double sum = 0.0;
    uint32_t n = strata * strata;
    for (uint32_t s = 0; s < n; ++s) {
        float a, b;
        jitter(rng, s, strata, a, b);
        Vec3 h = sample_vndf(wo, alpha, alpha, a, b);
        float cos = dot(wo, h);
        float f = fresnel_dielectric(cos, eta);
        Vec3 wr = h * (2.0f * cos) - wo;
        if (wr.z > 0.0f) sum += (double)f * g2_over_g1(g, wo, wr);
        if (f < 1.0f) {
            Vec3 wt;
            if (refract(wo, h, eta, wt) && wt.z < 0.0f) sum += (double)(1.0f - f) * g2_over_g1(g, wo, wt);
        }
    }
    return sum / (double)n;
}
static uint16_t quantise(double v) {
    double c = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
    return (uint16_t)std::round(c * 65535.0);
}
static std::vector<float> generate_avg(const std::vector<uint16_t>& table) {
    std::vector<float> out(NODES_ROUGHNESS);
    const uint32_t AVG_STEPS = 4096;
    for (int j = 0; j < NODES_ROUGHNESS; ++j) {
        float alpha = node_alpha(j);
        double sum = 0.0;
        for (uint32_t m = 0; m < AVG_STEPS; ++m) {
            float mu = ((float)m + 0.5f) / (float)AVG_STEPS;
            sum += (double)table_lookup(table.data(), mu, alpha) * (double)mu;
        }
        out[j] = (float)(2.0 * sum / (double)AVG_STEPS);
    }
    return out;
}

void generate_energy_tables(EnergyTables& t, int threads) {
    const int slice = NODES_MU * NODES_ROUGHNESS;
    t.albedo.assign(slice, 0);
    t.schlick.assign(slice, 0);
    t.clear_in.assign(slice * NODES_IOR, 0);
    t.clear_out.assign(slice * NODES_IOR, 0);
    // Work items: albedo nodes, schlick nodes, then clear-in and clear-out nodes.
    const int total = 2 * slice + 2 * slice * NODES_IOR;
    std::atomic<int> next(0);
    auto worker = [&]() {
        for (;;) {
            int w = next.fetch_add(64);
            if (w >= total) break;
            int end = w + 64 < total ? w + 64 : total;
            for (int item = w; item < end; ++item) {
                if (item < slice) {
                    int j = item / NODES_MU, i = item % NODES_MU;
                    uint64_t stream = (uint64_t)(j * NODES_MU + i);
                    t.albedo[item] = quantise(integrate_albedo(node_mu(i), node_alpha(j), ENERGY_STRATA, stream));
                } else if (item < 2 * slice) {
                    int k = item - slice;
                    int j = k / NODES_MU, i = k % NODES_MU;
                    uint64_t stream = (uint64_t)(j * NODES_MU + i) + (1ULL << 24);
                    t.schlick[k] = quantise(integrate_schlick(node_mu(i), node_alpha(j), ENERGY_STRATA, stream));
                } else {
                    int c = item - 2 * slice;
                    bool entering = c < slice * NODES_IOR;
                    int idx = entering ? c : c - slice * NODES_IOR;
                    int k = idx / slice, rem = idx % slice;
                    int j = rem / NODES_MU, i = rem % NODES_MU;
                    float ior = node_ior(k);
                    float eta = entering ? ior : 1.0f / ior;
                    uint64_t stream = (uint64_t)((k * NODES_ROUGHNESS + j) * NODES_MU + i) + (entering ? 0ULL : (1ULL << 20));
                    uint16_t v = quantise(integrate_clear(node_mu(i), node_alpha(j), eta, ENERGY_STRATA, stream));
                    (entering ? t.clear_in : t.clear_out)[idx] = v;
                }
            }
        }
    };
    if (threads < 1) threads = 1;
    std::vector<std::thread> pool;
    for (int i = 0; i < threads; ++i) pool.emplace_back(worker);
    for (auto& th : pool) th.join();
    t.albedo_avg = generate_avg(t.albedo);
    t.schlick_avg = generate_avg(t.schlick);
}

static EnergyTables* g_tables = nullptr;
static std::once_flag g_tables_once;
const EnergyTables& energy_tables() {
    std::call_once(g_tables_once, []() {
        g_tables = new EnergyTables();
        unsigned hw = std::thread::hardware_concurrency();
        generate_energy_tables(*g_tables, hw ? (int)hw : 4);
    });
    return *g_tables;
}

// ---- Bsdf (bsdf.rs:360-993) ----------------------------------------------------------------------
static Rgb rgb_clamp01(Rgb c) { return {rclamp(c.r, 0.0f, 1.0f), rclamp(c.g, 0.0f, 1.0f), rclamp(c.b, 0.0f, 1.0f)}; }

Bsdf Bsdf::surface_at(const Material& m, bool entering, float ior_in) {
    Rgb base = rgb_clamp01(m.base_color);
    float metallic = m.kind == MATERIAL_GLASS ? 0.0f : rclamp(m.metallic, 0.0f, 1.0f);
    float transmission = rclamp(m.transmission, 0.0f, 1.0f);
    float ior = rmax(ior_in, 1.0f);
    float f0 = ((ior - 1.0f) / (ior + 1.0f)) * ((ior - 1.0f) / (ior + 1.0f));
    float roughness = rclamp(m.roughness, 0.0f, 1.0f);
    float coat_roughness = rclamp(m.coat_roughness, 0.0f, 1.0f);
    float anisotropy = rclamp(m.anisotropy, 0.0f, 1.0f);
    float clear = (1.0f - metallic) * transmission;
    bool thin = (m.flags & MATERIAL_FLAG_THIN) != 0 || ior < 1.0001f;
    float eta = (thin || entering) ? ior : 1.0f / ior;
    Rgb tint;
    if (thin) tint = base;
    else if (m.absorption_mm > 0.0f) tint = WHITE;
    else tint = Rgb(std::sqrt(base.r), std::sqrt(base.g), std::sqrt(base.b));
    float coat = (clear > 0.0f && !thin && !entering) ? 0.0f : rclamp(m.coat, 0.0f, 1.0f);
    Bsdf b;
    b.diffuse = base * ((1.0f - metallic) * (1.0f - transmission));
    b.metal_f0 = base;
    b.metal_f90 = Rgb(rmin(50.0f * base.r, 1.0f), rmin(50.0f * base.g, 1.0f), rmin(50.0f * base.b, 1.0f));
    b.metallic = metallic;
    b.dielectric = (1.0f - metallic) * (1.0f - transmission);
    b.f0 = f0;
    b.f90 = rmin(50.0f * f0, 1.0f);
    b.spec = Ggx::make(rmax(roughness * roughness, MIN_ALPHA), anisotropy);
    b.coat = coat;
    b.coat_ggx = Ggx::make(rmax(coat_roughness * coat_roughness, MIN_ALPHA), 0.0f);
    b.clear = clear;
    b.eta = eta;
    b.tint = tint;
    b.thin = thin;
    b.multiple_scattering();
    b.layers();
    return b;
}

Bsdf Bsdf::lambert(Rgb a) {  // bsdf.rs:502
    Bsdf b;
    b.diffuse = rgb_clamp01(a);
    b.metal_f0 = BLACK;
    b.metal_f90 = BLACK;
    b.metallic = 0.0f;
    b.dielectric = 1.0f;
    b.f0 = 0.0f;
    b.f90 = 0.0f;
    b.spec = Ggx::make(1.0f, 0.0f);
    b.coat = 0.0f;
    b.coat_ggx = Ggx::make(1.0f, 0.0f);
    b.clear = 0.0f;
    b.eta = 1.0f;
    b.tint = WHITE;
    b.thin = false;
    return b;
}

void Bsdf::layers() {  // bsdf.rs:423
    float alpha = spec.iso ? spec.ax : std::sqrt(spec.ax * spec.ay);
    if (diffuse.r > 0.0f || diffuse.g > 0.0f || diffuse.b > 0.0f) {
        float ms = ms_spec_on ? multiple_fresnel(schlick_average(f0, f90), ms_spec_lobe.e_avg) : 0.0f;
        base_layer = Layer::make(f0, f90, 1.0f, alpha, ms);
    }
    if (coat > 0.0f) {
        float ms = ms_coat_on ? multiple_fresnel(schlick_average(COAT_F0, 1.0f), ms_coat_lobe.e_avg) : 0.0f;
        coat_layer = Layer::make(COAT_F0, 1.0f, coat, coat_ggx.ax, ms);
    }
    diffuse_norm = joint_norm(base_layer, coat_layer);
}

void Bsdf::multiple_scattering() {  // bsdf.rs:445
    float alpha = spec.iso ? spec.ax : std::sqrt(spec.ax * spec.ay);
    Lobe lobe = Lobe::make(alpha);
    if (lobe.on && has_specular()) {
        auto ms = [&](float a0, float a90) { return multiple_fresnel(schlick_average(a0, a90), lobe.e_avg); };
        float diel = dielectric > 0.0f ? dielectric * ms(f0, f90) : 0.0f;
        Rgb colour;
        if (metallic > 0.0f) {
            colour = Rgb(ms(metal_f0.r, metal_f90.r), ms(metal_f0.g, metal_f90.g), ms(metal_f0.b, metal_f90.b)) * metallic +
                     Rgb::splat(diel);
        } else {
            colour = Rgb::splat(diel);
        }
        if (peak(colour) > 0.0f) { ms_spec_on = true; ms_spec_lobe = lobe; ms_spec_colour = colour; }
    }
    if (coat > 0.0f) {
        Lobe cl = Lobe::make(coat_ggx.ax);
        if (cl.on) {
            float c = coat * multiple_fresnel(schlick_average(COAT_F0, 1.0f), cl.e_avg);
            if (c > 0.0f) { ms_coat_on = true; ms_coat_lobe = cl; ms_coat_c = c; }
        }
    }
    if (clear > 0.0f && !thin && alpha >= MIN_COMPENSATED_ALPHA) { ms_clear_on = true; ms_clear_alpha = alpha; }
}

Rgb Bsdf::straight_transmittance(float cos) const {  // bsdf.rs:572
    if (!(thin && clear > 0.0f)) return BLACK;
    cos = rmin(std::fabs(cos), 1.0f);
    float t = 1.0f - thin_reflectance(cos, eta);
    return tint * (clear * (1.0f - coat_fresnel(cos)) * t);
}

Rgb Bsdf::specular_fresnel(float cos) const {  // bsdf.rs:594
    float d = schlick(f0, f90, cos);
    if (metallic <= 0.0f && clear <= 0.0f) return Rgb::splat(d);
    Rgb metal(schlick(metal_f0.r, metal_f90.r, cos), schlick(metal_f0.g, metal_f90.g, cos), schlick(metal_f0.b, metal_f90.b, cos));
    return Rgb::splat(d) * dielectric + metal * metallic;
}

Bsdf::LobeWeights Bsdf::lobe_weights(Vec3 wo) const {  // bsdf.rs:648
    float c = coat_fresnel(wo.z);
    float below = 1.0f - c;
    float specular = has_specular() ? below * rmax(specular_fresnel(wo.z).luminance(), 0.0f) : 0.0f;
    float diff = below * diffuse.luminance() * base_layer.passes(wo.z);
    float cl = below * clear;
    float ms = 0.0f;
    if (ms_spec_on) ms += below * rmax(ms_spec_colour.luminance(), 0.0f) * ms_spec_lobe.lost(wo.z);
    if (ms_coat_on) ms += ms_coat_c * ms_coat_lobe.lost(wo.z);
    float total = c + specular + diff + cl + ms;
    if (total > 0.0f) {
        float inv = 1.0f / total;
        return {c * inv, specular * inv, diff * inv, cl * inv, ms * inv};
    }
    return {0, 0, 0, 0, 0};
}

Rgb Bsdf::eval(Vec3 wo, Vec3 wi, Lobes lobes) const {  // bsdf.rs:693 (eval_surface)
    if (wo.z <= 0.0f) return BLACK;
    if (wi.z <= 0.0f) {
        if (wi.z < 0.0f && lobes == Lobes::All && clear > 0.0f && !thin) return eval_refraction(wo, wi);
        return BLACK;
    }
    float attenuation = coat_layer.passes(wo.z) * coat_layer.passes(wi.z);
    Rgb diff = diffuse * (FRAC_1_PI * base_layer.passes(wo.z) * base_layer.passes(wi.z) * diffuse_norm);
    if (lobes == Lobes::Diffuse) return diff * attenuation;
    Vec3 h = normalize(wo + wi);
    float cos_h = rmax(dot(wo, h), 0.0f);
    Rgb below = diff;
    if (has_specular()) below = below + specular_fresnel(cos_h) * spec.microfacet(wo, wi, h);
    if (ms_spec_on) below = below + ms_spec_colour * ms_spec_lobe.shape(wo.z, wi.z);
    if (clear > 0.0f) {
        float cl = clear * clear_fresnel(cos_h) * spec.microfacet(wo, wi, h);
        float k;
        if (clear_compensation(wo.z, k)) cl *= k;
        below = below + Rgb::splat(cl);
    }
    Rgb f = below * attenuation;
    if (coat > 0.0f) f = f + Rgb::splat(coat_fresnel(cos_h) * coat_ggx.microfacet(wo, wi, h));
    if (ms_coat_on) f = f + Rgb::splat(ms_coat_c * ms_coat_lobe.shape(wo.z, wi.z));
    return f;
}

bool Bsdf::refraction_half(Vec3 wo, Vec3 wi, Vec3& h, float& co, float& ci) const {  // bsdf.rs:750
    h = normalize(wo + wi * eta);
    if (h.z < 0.0f) h = -h;
    co = dot(wo, h);
    ci = dot(wi, h);
    return co > 0.0f && ci < 0.0f && length_squared(h) > 0.5f;
}

Rgb Bsdf::eval_refraction(Vec3 wo, Vec3 wi) const {  // bsdf.rs:761
    Vec3 h; float co, ci;
    if (!refraction_half(wo, wi, h, co, ci)) return BLACK;
    float f = fresnel_dielectric(co, eta);
    float denom = co + eta * ci;
    float g2 = 1.0f / (1.0f + spec.lambda(wo) + spec.lambda(wi));
    float value = (1.0f - f) * spec.d(h) * g2 * (-ci) * co / (-wi.z * wo.z * denom * denom);
    float k;
    if (clear_compensation(wo.z, k)) value *= k;
    float attenuation = coat_layer.passes(wo.z);
    return tint * (clear * attenuation * value);
}

float Bsdf::pdf(Vec3 wo, Vec3 wi) const {  // bsdf.rs:780 (pdf_surface)
    if (wo.z <= 0.0f) return 0.0f;
    if (wi.z <= 0.0f) {
        if (wi.z < 0.0f && clear > 0.0f && !thin) return refraction_pdf(lobe_weights(wo), wo, wi);
        return 0.0f;
    }
    return pdf_with(lobe_weights(wo), wo, wi);
}

float Bsdf::pdf_with(const LobeWeights& w, Vec3 wo, Vec3 wi) const {  // bsdf.rs:797
    float p = (w.diffuse + w.ms) * wi.z * FRAC_1_PI;
    if (w.specular > 0.0f || w.coat > 0.0f || w.clear > 0.0f) {
        Vec3 h = normalize(wo + wi);
        if (dot(wo, h) > 0.0f) {
            if (w.specular > 0.0f) p += w.specular * spec.reflection_pdf(wo, h);
            if (w.coat > 0.0f) p += w.coat * coat_ggx.reflection_pdf(wo, h);
            if (w.clear > 0.0f) p += w.clear * reflect_chance(wo.z, dot(wo, h)) * spec.reflection_pdf(wo, h);
        }
    }
    return p;
}

float Bsdf::refraction_pdf(const LobeWeights& w, Vec3 wo, Vec3 wi) const {  // bsdf.rs:819
    if (w.clear != w.clear || w.clear <= 0.0f) return 0.0f;
    Vec3 h; float co, ci;
    if (!refraction_half(wo, wi, h, co, ci)) return 0.0f;
    float g1 = 1.0f / (1.0f + spec.lambda(wo));
    float visible = g1 * spec.d(h) * co / wo.z;
    float denom = co + eta * ci;
    float jacobian = eta * eta * (-ci) / (denom * denom);
    return w.clear * (1.0f - reflect_chance(wo.z, co)) * visible * jacobian;
}

bool Bsdf::sample(Vec3 wo, float u0, float u1, BsdfSample& out) const {  // bsdf.rs:833
    if (wo.z <= 0.0f) return false;
    LobeWeights w = lobe_weights(wo);
    Vec3 wi;
    if (u0 < w.coat) {
        Vec3 h = sample_vndf(wo, coat_ggx.ax, coat_ggx.ay, u0 / w.coat, u1);
        wi = h * (2.0f * dot(wo, h)) - wo;
    } else if (u0 < w.coat + w.specular) {
        Vec3 h = sample_vndf(wo, spec.ax, spec.ay, (u0 - w.coat) / w.specular, u1);
        wi = h * (2.0f * dot(wo, h)) - wo;
    } else if (w.diffuse + w.ms > 0.0f && (w.clear <= 0.0f || u0 < w.coat + w.specular + (w.diffuse + w.ms))) {
        float start = w.coat + w.specular;
        float uu = rclamp((u0 - start) / (w.diffuse + w.ms), 0.0f, 0.99999994f);
        wi = cosine_hemisphere(uu, u1);
    } else if (w.clear > 0.0f) {
        return sample_clear(w, wo, u0, u1, out);
    } else {
        return false;
    }
    if (wi.z <= 0.0f) return false;
    float p = pdf_with(w, wo, wi);
    if (!(p > 0.0f && finite(p))) return false;
    out.weight = eval(wo, wi, Lobes::All) * (wi.z / p);
    out.wi = wi;
    out.pdf = p;
    out.straight = false;
    return true;
}

bool Bsdf::sample_clear(const LobeWeights& w, Vec3 wo, float u0, float u1, BsdfSample& out) const {  // bsdf.rs:889
    float start = w.coat + w.specular + (w.diffuse + w.ms);
    float uc = rclamp((u0 - start) / w.clear, 0.0f, 0.99999994f);
    if (ms_clear_on) return sample_rough_clear(w, wo, uc, u1, out);
    float pr = reflect_probability(wo.z);
    if (uc < pr) {
        Vec3 h = sample_vndf(wo, spec.ax, spec.ay, uc / pr, u1);
        Vec3 wi = h * (2.0f * dot(wo, h)) - wo;
        if (wi.z <= 0.0f) return false;
        float p = pdf_with(w, wo, wi);
        if (!(p > 0.0f && finite(p))) return false;
        out.weight = eval(wo, wi, Lobes::All) * (wi.z / p);
        out.wi = wi; out.pdf = p; out.straight = false;
        return true;
    }
    if (thin) {
        float chance = w.clear * (1.0f - pr);
        if (chance != chance || chance <= 0.0f) return false;
        out.weight = straight_transmittance(wo.z) / chance;
        out.wi = -wo; out.pdf = chance; out.straight = true;
        return true;
    }
    float ut = rclamp((uc - pr) / (1.0f - pr), 0.0f, 0.99999994f);
    Vec3 h = sample_vndf(wo, spec.ax, spec.ay, ut, u1);
    Vec3 wi;
    if (!refract(wo, h, eta, wi)) return false;
    if (wi.z >= 0.0f) return false;
    float p = refraction_pdf(w, wo, wi);
    if (!(p > 0.0f && finite(p))) return false;
    out.weight = eval_refraction(wo, wi) * (-wi.z / p);
    out.wi = wi; out.pdf = p; out.straight = false;
    return true;
}

bool Bsdf::sample_rough_clear(const LobeWeights& w, Vec3 wo, float u0, float u1, BsdfSample& out) const {  // bsdf.rs:947
    Vec3 h = sample_vndf(wo, spec.ax, spec.ay, u0, u1);
    float fresnel = clear_fresnel(dot(wo, h));
    uint64_t key = ((uint64_t)fbits(u0) << 32) | (uint64_t)fbits(u1);
    float choice = (float)(mix64(key ^ 0x9e3779b97f4a7c15ULL) >> 40) * (1.0f / 16777216.0f);
    if (choice < fresnel) {
        Vec3 wi = h * (2.0f * dot(wo, h)) - wo;
        if (wi.z <= 0.0f) return false;
        float p = pdf_with(w, wo, wi);
        if (!(p > 0.0f && finite(p))) return false;
        out.weight = eval(wo, wi, Lobes::All) * (wi.z / p);
        out.wi = wi; out.pdf = p; out.straight = false;
        return true;
    }
    Vec3 wi;
    if (!refract(wo, h, eta, wi)) return false;
    if (wi.z >= 0.0f) return false;
    float p = refraction_pdf(w, wo, wi);
    if (!(p > 0.0f && finite(p))) return false;
    out.weight = eval_refraction(wo, wi) * (-wi.z / p);
    out.wi = wi; out.pdf = p; out.straight = false;
    return true;
}

}  // namespace orc
