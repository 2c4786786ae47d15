// The denoiser's kernels (engine/crates/rt-post/src/denoise.rs:435-788); see rtg_denoise.h.
#include <cuda_runtime.h>

#include "rtg_denoise.h"
#include "rtg_math.cuh"

namespace rtg {
namespace {

constexpr float SIGMA_LUMINANCE = 4.0f;  // denoise.rs:50
constexpr float SIGMA_DEPTH = 1.0f;      // denoise.rs:54
constexpr float SIGMA_ALBEDO = 0.1f;     // denoise.rs:56
constexpr float MIN_SAMPLES = 4.0f;      // denoise.rs:58
constexpr float MIN_ALBEDO = 0.01f;      // denoise.rs:121
constexpr float FIREFLY_RATIO = 4.0f;    // denoise.rs:123
constexpr float FIREFLY_FLOOR = 0.05f;   // denoise.rs:125
__constant__ float c_kernel[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
__constant__ float c_gauss3[3] = {0.25f, 0.5f, 0.25f};

// Rust's f32::max: a NaN operand gives the other one.
__device__ __forceinline__ float max_rs(float a, float b) { return a != a ? b : (b != b ? a : (a > b ? a : b)); }
__device__ __forceinline__ float lum3(float r, float g, float b) { return 0.2126f * r + 0.7152f * g + 0.0722f * b; }
__device__ __forceinline__ float fin(float v) { return finitef(v) ? v : 0.0f; }
__device__ __forceinline__ float pow128(float x) {
    float v = x;
#pragma unroll
    for (int i = 0; i < 7; ++i) v = v * v;
    return v;
}
__device__ __forceinline__ float falloff(float x) {  // denoise.rs:770: (1 - x/16)^16
    float t = 1.0f - x * (1.0f / 16.0f);
    if (t != t || t <= 0.0f) return 0.0f;
    t = t * t;
    t = t * t;
    t = t * t;
    return t * t;
}

// One pixel's guides, as three float4: {part, material, z, dz.x}, {dz.y, n}, {a, 0}.
struct G {
    uint32_t part, material;
    float z, dzx, dzy, n[3], a[3];
    __device__ bool fg() const { return part != 0; }
    __device__ bool same(const G& o) const { return part == o.part && material == o.material; }
};
struct Guides {
    float4 *g0, *g1, *g2;
    __device__ G load(size_t p) const {
        const float4 a = g0[p], b = g1[p], c = g2[p];
        G g;
        g.part = __float_as_uint(a.x);
        g.material = __float_as_uint(a.y);
        g.z = a.z;
        g.dzx = a.w;
        g.dzy = b.x;
        g.n[0] = b.y; g.n[1] = b.z; g.n[2] = b.w;
        g.a[0] = c.x; g.a[1] = c.y; g.a[2] = c.z;
        return g;
    }
    __device__ uint2 ids(size_t p) const {
        const float4 a = g0[p];
        return make_uint2(__float_as_uint(a.x), __float_as_uint(a.y));
    }
};
__device__ __forceinline__ float dot3(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ float depth_term(const G& g, const G& q, float dx, float dy) {  // denoise.rs:751
    if (!(finitef(g.z) && finitef(q.z))) return g.z == q.z ? 0.0f : f_inf();
    const float expected = fabsf(g.dzx * dx + g.dzy * dy);
    const float eps = 1.0e-3f * fabsf(g.z) + 1.0e-6f;
    return fabsf(g.z - q.z) / (SIGMA_DEPTH * expected + eps);
}
__device__ __forceinline__ float albedo_term(const G& g, const G& q) {
    return (fabsf(g.a[0] - q.a[0]) + fabsf(g.a[1] - q.a[1]) + fabsf(g.a[2] - q.a[2])) / SIGMA_ALBEDO;
}

#define DN_LOOP(n) for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < (n); p += (size_t)gridDim.x * blockDim.x)

// The guides with the depth gradient, the albedo divisor, the illumination, its variance and its
// luminance (denoise.rs:440-528).
__global__ void k_dn_prep(DnSrc src, uint32_t w, uint32_t h, uint32_t samples, Guides G_, float* divisor, float* light, float* var,
                          float* before) {
    const size_t n = (size_t)w * h;
    const float inv = 1.0f / (float)samples;
    DN_LOOP(n) {
        const uint32_t x = (uint32_t)(p % w), y = (uint32_t)(p / w);
        const uint32_t part = src.part[p], material = src.material[p];
        const float z = src.depth[p];
        float a[3], nn[3];
        const float aw = src.albedo_weight ? src.albedo_weight[p] : 1.0f;
        for (int k = 0; k < 3; ++k) {
            float av = src.albedo[3 * p + k];
            if (src.albedo_weight) av = aw > 0.0f ? av * (1.0f / aw) : 0.0f;  // passes.rs:364 resolve
            a[k] = fin(av);
            nn[k] = fin(src.normal[3 * p + k]);
        }
        float dz[2] = {0.0f, 0.0f};
        if (part != 0 && finitef(z)) {
            auto zq = [&](bool has, size_t q, float& out) {
                if (!has || src.part[q] != part || src.material[q] != material || !finitef(src.depth[q])) return false;
                out = src.depth[q];
                return true;
            };
            auto grad = [&](bool ha, size_t qa, bool hb, size_t qb) {
                float za = 0.0f, zb = 0.0f;
                const bool sa = zq(ha, qa, za), sb = zq(hb, qb, zb);
                if (sa && sb) return 0.5f * (zb - za);
                if (sa) return z - za;
                if (sb) return zb - z;
                return 0.0f;
            };
            dz[0] = grad(x > 0, p - 1, x + 1 < w, p + 1);
            dz[1] = grad(y > 0, p - w, y + 1 < h, p + w);
        }
        G_.g0[p] = make_float4(__uint_as_float(part), __uint_as_float(material), z, dz[0]);
        G_.g1[p] = make_float4(dz[1], nn[0], nn[1], nn[2]);
        G_.g2[p] = make_float4(a[0], a[1], a[2], 0.0f);
        float d[3] = {1.0f, 1.0f, 1.0f}, li[3] = {0.0f, 0.0f, 0.0f}, v = 0.0f;
        if (part != 0) {
            const float* s = src.rgb + p * src.rgb_stride;
            const float c[3] = {s[0] * inv, s[1] * inv, s[2] * inv};
            for (int k = 0; k < 3; ++k) {
                d[k] = max_rs(a[k], MIN_ALBEDO);
                li[k] = c[k] / d[k];
            }
            const bool own = src.counts != nullptr;
            const float cnt = own ? src.counts[p] : 0.0f;
            const bool enough = own ? cnt >= MIN_SAMPLES : (float)samples >= MIN_SAMPLES;
            if (enough) {
                const float l = lum3(c[0], c[1], c[2]);
                const float m2 = src.lum2[p] * inv;
                const float dof = own ? cnt - 1.0f : (float)(samples - 1);
                const float vv = max_rs(m2 - l * l, 0.0f) / dof;
                const float ld = lum3(d[0], d[1], d[2]);
                v = vv / (ld * ld);
            }
        }
        for (int k = 0; k < 3; ++k) {
            divisor[3 * p + k] = d[k];
            light[3 * p + k] = li[k];
        }
        var[p] = v;
        before[p] = lum3(li[0], li[1], li[2]);
    }
}

// The firefly clamp (denoise.rs:533-567): the set of fireflies depends on the luminances before the
// clamp only, so this pass finds it, scales each firefly's light, and gives it the largest
// variance of its neighbours as they were (the first Jacobi sweep).
__global__ void k_dn_firefly(uint32_t w, uint32_t h, Guides G_, const float* before, float* light, const float* var, float* var_out,
                             uint32_t* ffly) {
    const size_t n = (size_t)w * h;
    DN_LOOP(n) {
        const uint2 id = G_.ids(p);
        uint32_t is = 0;
        float vo = var[p];
        if (id.x != 0) {
            const int x = (int)(p % w), y = (int)(p / w);
            float brightest = 0.0f, vmax = 0.0f;
            uint32_t count = 0;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int qx = x + dx, qy = y + dy;
                    if ((dx == 0 && dy == 0) || qx < 0 || qy < 0 || qx >= (int)w || qy >= (int)h) continue;
                    const size_t q = (size_t)qy * w + (size_t)qx;
                    const uint2 iq = G_.ids(q);
                    if (iq.x != id.x || iq.y != id.y) continue;
                    brightest = max_rs(brightest, before[q]);
                    vmax = max_rs(vmax, var[q]);
                    ++count;
                }
            const float limit = FIREFLY_RATIO * brightest + FIREFLY_FLOOR;
            if (count >= 3 && before[p] > limit) {
                const float k = limit / before[p];
                for (int c = 0; c < 3; ++c) light[3 * p + c] = light[3 * p + c] * k;
                vo = vmax;
                is = 1;
            }
        }
        ffly[p] = is;
        var_out[p] = vo;
    }
}

// A Jacobi sweep of the fireflies' variances: the raster order's earlier firefly neighbours give
// their swept value, the others their own (denoise.rs:549 reads var as the loop has left it).
__global__ void k_dn_firefly_sweep(uint32_t w, uint32_t h, Guides G_, const uint32_t* ffly, const float* var, const float* cur, float* next,
                                   uint32_t* changed) {
    const size_t n = (size_t)w * h;
    DN_LOOP(n) {
        float v = cur[p];
        if (ffly[p]) {
            const uint2 id = G_.ids(p);
            const int x = (int)(p % w), y = (int)(p / w);
            float vmax = 0.0f;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int qx = x + dx, qy = y + dy;
                    if ((dx == 0 && dy == 0) || qx < 0 || qy < 0 || qx >= (int)w || qy >= (int)h) continue;
                    const size_t q = (size_t)qy * w + (size_t)qx;
                    const uint2 iq = G_.ids(q);
                    if (iq.x != id.x || iq.y != id.y) continue;
                    vmax = max_rs(vmax, (ffly[q] && q < p) ? cur[q] : var[q]);
                }
            if (__float_as_uint(vmax) != __float_as_uint(v)) *changed = 1u;
            v = vmax;
        }
        next[p] = v;
    }
}

// The spatial variance of a pixel with too few samples (denoise.rs:577-618).
__global__ void k_dn_spatial(uint32_t w, uint32_t h, Guides G_, const float* counts, uint32_t samples, int r, const float* light, float* var) {
    const size_t n = (size_t)w * h;
    DN_LOOP(n) {
        const bool few = counts ? counts[p] < MIN_SAMPLES : (float)samples < MIN_SAMPLES;
        if (!few) continue;
        const G g = G_.load(p);
        if (!g.fg()) continue;
        const int x = (int)(p % w), y = (int)(p / w);
        float sw = 0.0f, m1 = 0.0f, m2 = 0.0f;
        for (int dy = -r; dy <= r; ++dy) {
            const int qy = y + dy;
            if (qy < 0 || qy >= (int)h) continue;
            for (int dx = -r; dx <= r; ++dx) {
                const int qx = x + dx;
                if (qx < 0 || qx >= (int)w) continue;
                const size_t q = (size_t)qy * w + (size_t)qx;
                const G gq = G_.load(q);
                if (!g.same(gq)) continue;
                const float wgt = pow128(max_rs(dot3(g.n, gq.n), 0.0f)) * falloff(depth_term(g, gq, (float)dx, (float)dy));
                const float l = lum3(light[3 * q], light[3 * q + 1], light[3 * q + 2]);
                sw = sw + wgt;
                m1 = m1 + wgt * l;
                m2 = m2 + wgt * l * l;
            }
        }
        if (sw > 0.0f) {
            m1 = m1 / sw;
            m2 = m2 / sw;
            var[p] = max_rs(m2 - m1 * m1, 0.0f);
        }
    }
}

__global__ void k_dn_lum(size_t n, const float* light, float* lum) {
    DN_LOOP(n) lum[p] = lum3(light[3 * p], light[3 * p + 1], light[3 * p + 2]);
}

// The variance of pixel p blurred by a 3 x 3 Gaussian on the same surface (denoise.rs:628-654).
// Only the a-trous pass of the same level reads it, for its own pixel, so the pass computes it.
__device__ __forceinline__ float gauss_var(uint32_t w, uint32_t h, const Guides& G_, const float* var, size_t p, uint2 id) {
    const int x = (int)(p % w), y = (int)(p / w);
    float sw = 0.0f, sv = 0.0f;
    {
        for (int j = 0; j < 3; ++j) {
            const int qy = y + j - 1;
            if (qy < 0 || qy >= (int)h) continue;
            for (int i = 0; i < 3; ++i) {
                const int qx = x + i - 1;
                if (qx < 0 || qx >= (int)w) continue;
                const size_t q = (size_t)qy * w + (size_t)qx;
                const uint2 iq = G_.ids(q);
                if (iq.x != id.x || iq.y != id.y) continue;
                const float k = c_gauss3[j] * c_gauss3[i];
                sw = sw + k;
                sv = sv + k * var[q];
            }
        }
    }
    return sw > 0.0f ? sv / sw : var[p];
}

// One a-trous pass, taps `step` pixels apart (denoise.rs:655-708), and the luminance of its result.
__global__ void k_dn_atrous(uint32_t w, uint32_t h, int step, Guides G_, const float* light, const float* var, const float* lum,
                            float* light_next, float* var_next, float* lum_next) {
    const size_t n = (size_t)w * h;
    DN_LOOP(n) {
        const G g = G_.load(p);
        if (!g.fg()) continue;
        const int x = (int)(p % w), y = (int)(p / w);
        const float lp = lum[p];
        const float gv = gauss_var(w, h, G_, var, p, make_uint2(g.part, g.material));
        const float inv_sigma_l = 1.0f / (SIGMA_LUMINANCE * sqrt_(max_rs(gv, 0.0f) + 1.0e-10f));
        float sw = 0.0f, sv = 0.0f, sc0 = 0.0f, sc1 = 0.0f, sc2 = 0.0f;
        for (int j = 0; j < 5; ++j) {
            const int dy = (j - 2) * step;
            const int qy = y + dy;
            if (qy < 0 || qy >= (int)h) continue;
            for (int i = 0; i < 5; ++i) {
                const int dx = (i - 2) * step;
                const int qx = x + dx;
                if (qx < 0 || qx >= (int)w) continue;
                const size_t q = (size_t)qy * w + (size_t)qx;
                const G gq = G_.load(q);
                if (!g.same(gq)) continue;
                const float wn = q == p ? 1.0f : pow128(max_rs(dot3(g.n, gq.n), 0.0f));
                if (wn <= 0.0f) continue;
                const float exponent = fabsf(lp - lum[q]) * inv_sigma_l + depth_term(g, gq, (float)dx, (float)dy) + albedo_term(g, gq);
                const float wgt = c_kernel[j] * c_kernel[i] * wn * falloff(exponent);
                sw = sw + wgt;
                sv = sv + wgt * wgt * var[q];
                sc0 = sc0 + wgt * light[3 * q];
                sc1 = sc1 + wgt * light[3 * q + 1];
                sc2 = sc2 + wgt * light[3 * q + 2];
            }
        }
        const float inv_w = 1.0f / sw;
        const float l0 = sc0 * inv_w, l1 = sc1 * inv_w, l2 = sc2 * inv_w;
        light_next[3 * p] = l0;
        light_next[3 * p + 1] = l1;
        light_next[3 * p + 2] = l2;
        var_next[p] = sv * inv_w * inv_w;
        lum_next[p] = lum3(l0, l1, l2);
    }
}

// The albedo multiplied back, as sums of `samples` samples (denoise.rs:716-730), RGBA.
__global__ void k_dn_final(DnSrc src, uint32_t w, uint32_t h, uint32_t samples, Guides G_, const float* light, const float* divisor,
                           float* out) {
    const size_t n = (size_t)w * h;
    const float count = (float)samples;
    DN_LOOP(n) {
        const float* s = src.rgb + p * src.rgb_stride;
        const bool fg = G_.ids(p).x != 0;
        for (int k = 0; k < 3; ++k) {
            float o = s[k];
            if (fg) {
                const float c = light[3 * p + k] * divisor[3 * p + k];
                if (finitef(c)) o = c * count;
            }
            out[4 * p + k] = o;
        }
        out[4 * p + 3] = src.alpha[p * src.alpha_stride];
    }
}

// adaptive.rs:260 rescale: a pixel's sums of n samples as sums of s, RGBA interleaved, and its
// squared-luminance sum (the film of a uniform render keeps its bits: n == s).
__device__ __forceinline__ float rescale(float sum, float n, float s) { return n == s ? sum : (n > 0.0f ? sum * (1.0f / n) * s : 0.0f); }
__global__ void k_dn_rescale(const float* rgb, const float* alpha, const float* lum2, const float* weight, size_t n, float s, float* rgba,
                             float* lum2_out) {
    DN_LOOP(n) {
        const float w = weight[p];
        for (int k = 0; k < 3; ++k) rgba[4 * p + k] = rescale(rgb[3 * p + k], w, s);
        rgba[4 * p + 3] = rescale(alpha[p], w, s);
        lum2_out[p] = rescale(lum2[p], w, s);
    }
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

cudaError_t launch_dn_rescale(const float* rgb, const float* alpha, const float* lum2, const float* weight, size_t n, uint32_t samples, float* rgba,
                              float* lum2_out, cudaStream_t st, int grid) {
    k_dn_rescale<<<grid, 256, 0, st>>>(rgb, alpha, lum2, weight, n, (float)samples, rgba, lum2_out);
    return cudaGetLastError();
}

size_t dn_scratch_bytes(size_t n) {
    // 3 guide float4 planes; divisor and two light planes (3 floats); var x 3, lum x 2, before
    // (floats); firefly flags; two counters.
    return 3 * align256(n * 16) + 3 * align256(n * 12) + 6 * align256(n * 4) + align256(n * 4) + 256;
}

cudaError_t denoise_band(const DnSrc& src, uint32_t width, uint32_t rows, uint32_t samples, DnPreset preset, void* scratch, float* out,
                         cudaStream_t st, int grid, uint64_t& launches) {
    const size_t n = (size_t)width * rows;
    samples = samples > 1 ? samples : 1;
    uint8_t* p = (uint8_t*)scratch;
    auto take = [&](size_t bytes) { uint8_t* r = p; p += align256(bytes); return r; };
    Guides G_{(float4*)take(n * 16), (float4*)take(n * 16), (float4*)take(n * 16)};
    float* divisor = (float*)take(n * 12);
    float* light[2] = {(float*)take(n * 12), (float*)take(n * 12)};
    float* var[2] = {(float*)take(n * 4), (float*)take(n * 4)};
    float* var0 = (float*)take(n * 4);
    float* lum[2] = {(float*)take(n * 4), (float*)take(n * 4)};
    float* before = (float*)take(n * 4);
    uint32_t* ffly = (uint32_t*)take(n * 4);
    uint32_t* changed = (uint32_t*)take(256);
    cudaError_t e;
    if ((e = cudaMemsetAsync(light[1], 0, n * 12, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(lum[1], 0, n * 4, st)) != cudaSuccess) return e;
    k_dn_prep<<<grid, 256, 0, st>>>(src, width, rows, samples, G_, divisor, light[0], var0, before);
    k_dn_firefly<<<grid, 256, 0, st>>>(width, rows, G_, before, light[0], var0, var[0], ffly);
    launches += 2;
    // Jacobi sweeps until the fireflies' variances stop changing (at most one per firefly in a
    // chain of neighbours; in practice one or two).
    int cur = 0;
    for (size_t sweep = 0; sweep <= n; ++sweep) {
        uint32_t moved = 0;
        if ((e = cudaMemsetAsync(changed, 0, 4, st)) != cudaSuccess) return e;
        k_dn_firefly_sweep<<<grid, 256, 0, st>>>(width, rows, G_, ffly, var0, var[cur], var[cur ^ 1], changed);
        launches += 1;
        if ((e = cudaMemcpyAsync(&moved, changed, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
        cur ^= 1;
        if (!moved) break;
    }
    k_dn_spatial<<<grid, 256, 0, st>>>(width, rows, G_, src.counts, samples, (int)preset.variance_radius, light[0], var[cur]);
    k_dn_lum<<<grid, 256, 0, st>>>(n, light[0], lum[0]);
    launches += 2;
    // var[cur ^ 1] holds the variances before the last sweep: the fireflies' only, so copy the
    // final plane over it to keep the background's and the others' equal in both.
    if ((e = cudaMemcpyAsync(var[cur ^ 1], var[cur], n * 4, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
    int l = 0;
    for (uint32_t level = 0; level < preset.levels; ++level) {
        k_dn_atrous<<<grid, 256, 0, st>>>(width, rows, 1 << level, G_, light[l], var[cur], lum[l], light[l ^ 1], var[cur ^ 1], lum[l ^ 1]);
        launches += 1;
        l ^= 1;
        cur ^= 1;
    }
    k_dn_final<<<grid, 256, 0, st>>>(src, width, rows, samples, G_, light[l], divisor, out);
    launches += 1;
    return cudaGetLastError();
}

}  // namespace rtg
