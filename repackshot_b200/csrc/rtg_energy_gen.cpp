// Build-time generator of the multiple-scattering energy tables of the BSDF, by the Monte Carlo
// recipe of engine/crates/rt-core/src/bsdf/energy.rs:73-300: per node 64 x 64 jittered visible
// normals (Heitz 2018) with a PCG32 stream per node and seed 0xe9ae9a, f64 sums, values stored
// as 16-bit fractions; the cosine-weighted means by a 4096-step midpoint rule over the table's
// own lookup. The same recipe gives the same bits on every machine.
//
// Usage: rtg_energy_gen OUT.inc   (writes the C arrays the library includes)
#include <atomic>
#include <cmath>
#include <cstdio>
#include <thread>
#include <vector>

#include "rtg_bsdf.cuh"

using namespace rtg;

namespace {
constexpr uint64_t SEED = 0xe9ae9aULL;
constexpr uint32_t STRATA = 64;

float node_mu(int i) { float t = (float)i / (float)(NODES_MU - 1); return rmax(t * t, 1.0f / 2048.0f); }
float node_alpha(int j) { float r = (float)j / (float)(NODES_ROUGHNESS - 1); return r * r; }
float node_ior(int k) {
    const float MAX_X = (3.0f - 1.0f) / (3.0f + 1.0f);
    float x = MAX_X * (float)k / (float)(NODES_IOR - 1);
    return (1.0f + x) / (1.0f - x);
}
V3 outgoing(float mu) { return v3(sqrt_(rmax(1.0f - mu * mu, 0.0f)), 0.0f, mu); }
void jitter(Pcg32& rng, uint32_t s, float& a, float& b) {
    uint32_t i = s % STRATA, j = s / STRATA;
    float inv = 1.0f / (float)STRATA;
    float r0 = pcg_f32(rng);
    float r1 = pcg_f32(rng);
    a = rmin(((float)i + r0) * inv, 0.99999994f);
    b = rmin(((float)j + r1) * inv, 0.99999994f);
}
double g2_over_g1(const Ggx& g, V3 wo, V3 wi) {
    float lo = ggx_L(g, wo), li = ggx_L(g, wi);
    return (double)((1.0f + lo) / (1.0f + lo + li));
}
// kind 0: albedo, 1: Schlick moment, 2: clear lobe power albedo at `eta`.
double integrate(int kind, float mu, float alpha, float eta, uint64_t stream) {
    if (kind == 1 && alpha <= 0.0f) {
        double m = (double)(1.0f - mu);
        return m * m * m * m * m;
    }
    if (alpha <= 0.0f) return 1.0;
    if (kind == 2 && std::fabs(eta - 1.0f) < 1.0e-6f) return 1.0;
    Ggx g = make_ggx(alpha, 0.0f);
    V3 wo = outgoing(mu);
    uint64_t seed = kind == 0 ? SEED : (kind == 1 ? (SEED ^ 0x5c41ULL) : (SEED ^ 0xc1eaULL));
    Pcg32 rng = pcg_seeded(seed, stream);
    double sum = 0.0;
    const uint32_t n = STRATA * STRATA;
    for (uint32_t s = 0; s < n; ++s) {
        float a, b;
        jitter(rng, s, a, b);
        V3 h = sample_vndf(wo, alpha, alpha, a, b);
        float c = dot(wo, h);
        V3 wr = h * (2.0f * c) - wo;
        if (kind == 0) {
            if (wr.z > 0.0f) sum += g2_over_g1(g, wo, wr);
        } else if (kind == 1) {
            if (wr.z > 0.0f) {
                double m = (double)rclamp(1.0f - c, 0.0f, 1.0f);
                sum += m * m * m * m * m * g2_over_g1(g, wo, wr);
            }
        } else {
            float f = fresnel_dielectric(c, eta);
            if (wr.z > 0.0f) sum += (double)f * g2_over_g1(g, wo, wr);
            if (f < 1.0f) {
                V3 wt;
                if (refract(wo, h, eta, wt) && wt.z < 0.0f) sum += (double)(1.0f - f) * g2_over_g1(g, wo, wt);
            }
        }
    }
    return sum / (double)n;
}
uint16_t quantise(double v) { double c = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v); return (uint16_t)std::round(c * 65535.0); }
std::vector<float> averages(const std::vector<uint16_t>& table) {
    std::vector<float> out(NODES_ROUGHNESS);
    for (int j = 0; j < NODES_ROUGHNESS; ++j) {
        float alpha = node_alpha(j);
        double sum = 0.0;
        for (uint32_t m = 0; m < 4096; ++m) {
            float mu = ((float)m + 0.5f) / 4096.0f;
            sum += (double)table_lookup(table.data(), mu, alpha) * (double)mu;
        }
        out[j] = (float)(2.0 * sum / 4096.0);
    }
    return out;
}
void dump_u16(FILE* f, const char* name, const std::vector<uint16_t>& v) {
    fprintf(f, "static const uint16_t %s[%zu] = {", name, v.size());
    for (size_t i = 0; i < v.size(); ++i) fprintf(f, "%s%u,", i % 24 ? "" : "\n", v[i]);
    fprintf(f, "\n};\n");
}
void dump_f32(FILE* f, const char* name, const std::vector<float>& v) {
    fprintf(f, "static const uint32_t %s[%zu] = {", name, v.size());
    for (size_t i = 0; i < v.size(); ++i) fprintf(f, "%s0x%08xu,", i % 8 ? "" : "\n", fbits(v[i]));
    fprintf(f, "\n};\n");
}
}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) { fprintf(stderr, "usage: rtg_energy_gen OUT.inc\n"); return 2; }
    const int slice = NODES_MU * NODES_ROUGHNESS;
    std::vector<uint16_t> albedo(slice), schlick(slice), clear_in(slice * NODES_IOR), clear_out(slice * NODES_IOR);
    const int total = 2 * slice + 2 * slice * NODES_IOR;
    std::atomic<int> next(0);
    auto worker = [&]() {
        for (;;) {
            int item = next.fetch_add(1);
            if (item >= total) break;
            if (item < slice) {
                int j = item / NODES_MU, i = item % NODES_MU;
                albedo[item] = quantise(integrate(0, node_mu(i), node_alpha(j), 1.0f, (uint64_t)(j * NODES_MU + i)));
            } else if (item < 2 * slice) {
                int k = item - slice, j = k / NODES_MU, i = k % NODES_MU;
                schlick[k] = quantise(integrate(1, node_mu(i), node_alpha(j), 1.0f, (uint64_t)(j * NODES_MU + i) + (1ULL << 24)));
            } else {
                int c = item - 2 * slice;
                bool entering = c < slice * NODES_IOR;
                int idx = entering ? c : c - slice * NODES_IOR;
                int k = idx / slice, rem = idx % slice, j = rem / NODES_MU, i = rem % NODES_MU;
                float ior = node_ior(k);
                uint64_t stream = (uint64_t)((k * NODES_ROUGHNESS + j) * NODES_MU + i) + (entering ? 0ULL : (1ULL << 20));
                uint16_t v = quantise(integrate(2, node_mu(i), node_alpha(j), entering ? ior : 1.0f / ior, stream));
                (entering ? clear_in : clear_out)[idx] = v;
            }
        }
    };
    unsigned hw = std::thread::hardware_concurrency();
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < (hw ? hw : 4); ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    FILE* f = fopen(argv[1], "w");
    if (!f) { perror(argv[1]); return 1; }
    fprintf(f, "// Generated by rtg_energy_gen (the recipe of bsdf/energy.rs); do not edit.\n");
    dump_u16(f, "E_ALBEDO", albedo);
    dump_u16(f, "E_SCHLICK", schlick);
    dump_u16(f, "E_CLEAR_IN", clear_in);
    dump_u16(f, "E_CLEAR_OUT", clear_out);
    dump_f32(f, "E_ALBEDO_AVG", averages(albedo));
    dump_f32(f, "E_SCHLICK_AVG", averages(schlick));
    fclose(f);
    return 0;
}
