// Bitmaps of a scene on the host: decoding of the BMAP formats into linear RGB texels
// (engine/crates/rt-core/src/bitmap.rs:100-300, hdr.rs:30-240) and the importance-sampling grid
// of an environment map (environment.rs:60-95, bitmap.rs:312-372). The device reads the texels and
// the grid's CDFs (rtg_shade.cuh).
#include <cctype>
#include <cmath>
#include <cstring>

#include "rtg_scene.h"

namespace rtg {
namespace {

// The sRGB decoding of every byte value with the reference's powf (bitmap.rs:108).
const float* srgb_to_linear() {
    static float t[256];
    static bool done = false;
    if (!done) {
        for (int i = 0; i < 256; ++i) {
            float c = (float)i / 255.0f;
            t[i] = c <= 0.04045f ? c / 12.92f : fpow((c + 0.055f) / 1.055f, 2.4f);
        }
        done = true;
    }
    return t;
}

// Cleans linear floats (non-finite and negative to 0) and halves the image (2 x 2 box, an odd
// last row or column averaged with itself) until it is at most 4096 wide (bitmap.rs:182-216).
void to_linear(uint32_t width, uint32_t height, std::vector<float> rgb, HImage& out) {
    for (float& v : rgb)
        if (!(finitef(v) && v > 0.0f)) v = 0.0f;
    size_t w = width, h = height;
    while (w > 4096) {
        size_t nw = (w + 1) / 2, nh = (h + 1) / 2;
        std::vector<float> half(3 * nw * nh);
        for (size_t y = 0; y < nh; ++y) {
            size_t ya = 2 * y, yb = std::min(2 * y + 1, h - 1);
            for (size_t x = 0; x < nw; ++x) {
                size_t xa = 2 * x, xb = std::min(2 * x + 1, w - 1);
                for (int c = 0; c < 3; ++c) {
                    float a = rgb[3 * (ya * w + xa) + c] + rgb[3 * (ya * w + xb) + c];
                    float b = rgb[3 * (yb * w + xa) + c] + rgb[3 * (yb * w + xb) + c];
                    half[3 * (y * nw + x) + c] = (a + b) * 0.25f;
                }
            }
        }
        rgb.swap(half);
        w = nw;
        h = nh;
    }
    out.width = (uint32_t)w;
    out.height = (uint32_t)h;
    out.texels = std::move(rgb);
}

// Radiance RGBE files (hdr.rs): a header ending in an empty line, "-Y h +X w" or "+Y h +X w",
// then scanlines, flat (with old-style repeat markers) or in the newer per-channel run-length code.
struct HdrReader {
    const uint8_t* b;
    size_t n, pos = 0;
    bool line(size_t& start, size_t& end) {
        size_t k = pos;
        while (k < n && b[k] != '\n') ++k;
        if (k >= n) return false;
        start = pos;
        end = k;
        pos = k + 1;
        return true;
    }
    bool scanline(std::vector<uint8_t>& row, size_t width) {
        if (width >= 8 && width <= 0x7fff && pos + 4 <= n && b[pos] == 2 && b[pos + 1] == 2 && (b[pos + 2] & 0x80) == 0) {
            if ((((size_t)b[pos + 2] << 8) | b[pos + 3]) != width) return false;
            pos += 4;
            for (int ch = 0; ch < 4; ++ch)
                for (size_t x = 0; x < width;) {
                    if (pos >= n) return false;
                    size_t count = b[pos++];
                    if (count > 128) {
                        count -= 128;
                        if (pos >= n || x + count > width) return false;
                        const uint8_t value = b[pos++];
                        for (size_t j = 0; j < count; ++j) row[4 * (x + j) + ch] = value;
                    } else {
                        if (count == 0 || x + count > width || pos + count > n) return false;
                        for (size_t j = 0; j < count; ++j) row[4 * (x + j) + ch] = b[pos + j];
                        pos += count;
                    }
                    x += count;
                }
            return true;
        }
        unsigned shift = 0;
        for (size_t x = 0; x < width;) {
            if (pos + 4 > n) return false;
            const uint8_t* p = b + pos;
            pos += 4;
            if (p[0] == 1 && p[1] == 1 && p[2] == 1) {
                size_t count = (size_t)p[3] << shift;
                if (x == 0 || x + count > width) return false;
                for (size_t j = 0; j < count; ++j) std::memcpy(&row[4 * (x + j)], &row[4 * (x - 1)], 4);
                x += count;
                shift += 8;
            } else {
                std::memcpy(&row[4 * x], p, 4);
                x += 1;
                shift = 0;
            }
        }
        return true;
    }
};

bool decode_hdr(const uint8_t* bytes, size_t n, uint32_t& width, uint32_t& height, std::vector<float>& rgb) {
    auto starts = [&](const char* s) { size_t k = std::strlen(s); return n >= k && std::memcmp(bytes, s, k) == 0; };
    if (!(starts("#?RADIANCE") || starts("#?RGBE"))) return false;
    HdrReader r{bytes, n};
    size_t a, z;
    if (!r.line(a, z)) return false;
    for (;;) {
        if (!r.line(a, z)) return false;
        if (a == z) break;
        if (z - a >= 7 && std::memcmp(bytes + a, "FORMAT=", 7) == 0) {
            size_t s = a + 7, e = z;
            auto blank = [](uint8_t c) { return c == ' ' || c == '\t' || c == '\r' || c == '\f' || c == '\n'; };
            while (s < e && blank(bytes[s])) ++s;
            while (e > s && blank(bytes[e - 1])) --e;
            if (!(e - s == 15 && std::memcmp(bytes + s, "32-bit_rle_rgbe", 15) == 0)) return false;
        }
    }
    if (!r.line(a, z)) return false;
    std::vector<std::string> words;
    for (size_t i = a; i < z;) {
        while (i < z && std::isspace(bytes[i])) ++i;
        size_t j = i;
        while (j < z && !std::isspace(bytes[j])) ++j;
        if (j > i) words.emplace_back((const char*)bytes + i, j - i);
        i = j;
    }
    if (words.size() != 4 || words[2] != "+X" || (words[0] != "-Y" && words[0] != "+Y")) return false;
    const bool top_down = words[0] == "-Y";
    auto number = [](const std::string& t, uint32_t& v) {
        if (t.empty() || t.size() > 10) return false;
        uint64_t x = 0;
        for (char c : t) {
            if (c < '0' || c > '9') return false;
            x = 10 * x + (uint64_t)(c - '0');
        }
        if (x > 0xffffffffull) return false;
        v = (uint32_t)x;
        return true;
    };
    if (!number(words[1], height) || !number(words[3], width) || width == 0 || height == 0) return false;
    if ((uint64_t)width * height > (1ull << 28)) return false;
    rgb.assign(3 * (size_t)width * height, 0.0f);
    std::vector<uint8_t> row(4 * (size_t)width);
    for (size_t y = 0; y < height; ++y) {
        if (!r.scanline(row, width)) return false;
        float* out = rgb.data() + 3 * (top_down ? y : height - 1 - y) * (size_t)width;
        for (size_t x = 0; x < width; ++x) {
            const uint8_t* p = &row[4 * x];
            if (p[3] == 0) continue;  // zero
            // 2^(e - 136): the mantissa bytes scaled by the shared exponent (hdr.rs:40-56)
            const int e = (int)p[3] - 136;
            const float f = e >= -126 ? bitsf((uint32_t)(e + 127) << 23) : (e >= -149 ? bitsf(1u << (e + 149)) : 0.0f);
            out[3 * x] = (float)p[0] * f;
            out[3 * x + 1] = (float)p[1] * f;
            out[3 * x + 2] = (float)p[2] * f;
        }
    }
    return true;
}

// The bucket boundaries of a row of weights, normalised (the last exactly 1 when the row has
// weight), and the row's sum.
float cumulative(const float* w, size_t n, float* cdf) {
    float acc = 0.0f;
    for (size_t i = 0; i < n; ++i) {
        acc += w[i];
        cdf[i] = acc;
    }
    if (acc > 0.0f) {
        for (size_t i = 0; i < n; ++i) cdf[i] /= acc;
        cdf[n - 1] = 1.0f;
    }
    return acc;
}

}  // namespace

bool decode_bitmap(uint32_t format, uint32_t width, uint32_t height, const uint8_t* data, size_t len, HImage& out, std::string& reason,
                   bool& unsupported) {
    unsupported = false;
    const uint64_t px = (uint64_t)width * height;
    auto raw = [&](uint64_t bytes_per_pixel) {
        if (width == 0 || height == 0 || width > 65536 || height > 65536 || px > (1ull << 28) || px * bytes_per_pixel != len) {
            reason = "bitmap size does not match its data";
            return false;
        }
        return true;
    };
    const float* srgb = srgb_to_linear();
    switch (format) {
        case 0:
        case 1: {  // 8-bit sRGB RGB or RGBA (alpha ignored)
            const size_t stride = format == 0 ? 3 : 4;
            if (!raw(stride)) return false;
            out.width = width;
            out.height = height;
            out.texels.resize(3 * px);
            for (size_t i = 0; i < px; ++i)
                for (int c = 0; c < 3; ++c) out.texels[3 * i + c] = srgb[data[stride * i + c]];
            return true;
        }
        case 2: {  // little-endian linear f32 RGB
            if (!raw(12)) return false;
            std::vector<float> rgb(3 * px);
            std::memcpy(rgb.data(), data, len);
            to_linear(width, height, std::move(rgb), out);
            return true;
        }
        case 16: {  // a Radiance file
            uint32_t w = 0, h = 0;
            std::vector<float> rgb;
            if (!decode_hdr(data, len, w, h, rgb)) {
                reason = "unreadable Radiance HDR image";
                return false;
            }
            if (!(width == 0 && height == 0) && !(width == w && height == h)) {
                reason = "bitmap size does not match its data";
                return false;
            }
            to_linear(w, h, std::move(rgb), out);
            return true;
        }
        case 17:
            unsupported = true;
            reason = "unsupported: OpenEXR bitmap";
            return false;
        default:
            reason = "unknown bitmap format";
            return false;
    }
}

bool build_env_map(const HImage& img, float scale, float rotation_deg, HEnvMap& out) {
    const size_t w = img.width, h = img.height;
    const size_t fx = std::max<size_t>((w + 511) / 512, 1), fy = std::max<size_t>((h + 255) / 256, 1);
    const size_t gw = (w + fx - 1) / fx, gh = (h + fy - 1) / fy;
    out.gw = (uint32_t)gw;
    out.gh = (uint32_t)gh;
    out.weights.assign(gw * gh, 0.0f);
    float mean = 0.0f;
    for (size_t gy = 0; gy < gh; ++gy) {
        float s = 0.0f, cth;
        sin_cos(PI * ((float)gy + 0.5f) / (float)gh, s, cth);
        float row_sum = 0.0f;
        for (size_t gx = 0; gx < gw; ++gx) {
            float lum = 0.0f;
            uint32_t count = 0;
            for (size_t y = gy * fy; y < std::min((gy + 1) * fy, h); ++y)
                for (size_t x = gx * fx; x < std::min((gx + 1) * fx, w); ++x) {
                    const float* t = &img.texels[3 * (y * w + x)];
                    lum += rmax(luminance(rgb(t[0], t[1], t[2])), 0.0f);
                    count += 1;
                }
            lum = lum / (float)std::max(count, 1u);
            out.weights[gy * gw + gx] = lum * s;
            row_sum += lum * s;
        }
        mean += row_sum / (float)gw;
    }
    out.mean_luminance = scale * (mean / (float)gh) * (0.5f * PI);
    // Distribution2D::new (bitmap.rs:343): per-row conditional CDFs, the marginal over rows.
    out.conditional.assign(gw * gh, 0.0f);
    std::vector<float> row_sums(gh);
    for (size_t y = 0; y < gh; ++y) row_sums[y] = cumulative(&out.weights[y * gw], gw, &out.conditional[y * gw]);
    out.marginal.assign(gh, 0.0f);
    float acc = 0.0f;
    for (size_t y = 0; y < gh; ++y) {
        acc += row_sums[y];
        out.marginal[y] = acc;
    }
    if (!(acc > 0.0f && finitef(acc))) return false;
    for (float& m : out.marginal) m /= acc;
    out.marginal[gh - 1] = 1.0f;
    out.mean = acc / (float)(gw * gh);
    out.scale = scale;
    sin_cos(rotation_deg * (PI / 180.0f), out.rot_s, out.rot_c);
    return true;
}

// ---- the classic sky (sky.rs:200-348): Preetham, Shirley and Smits 1999 -----------------------------
namespace {
// The Perez coefficients A..E as (slope, intercept) in the turbidity for the luminance Y and the
// chromaticities x, y, and the zenith chromaticity fits in (T^2, T, 1) x (theta^3, theta^2,
// theta, 1): the paper's Appendix A.2.
constexpr float kPerez[3][5][2] = {
    {{0.1787f, -1.4630f}, {-0.3554f, 0.4275f}, {-0.0227f, 5.3251f}, {0.1206f, -2.5771f}, {-0.0670f, 0.3703f}},
    {{-0.0193f, -0.2592f}, {-0.0665f, 0.0008f}, {-0.0004f, 0.2125f}, {-0.0641f, -0.8989f}, {-0.0033f, 0.0452f}},
    {{-0.0167f, -0.2608f}, {-0.0950f, 0.0092f}, {-0.0079f, 0.2102f}, {-0.0441f, -1.6537f}, {-0.0109f, 0.0529f}}};
constexpr float kZenithX[3][4] = {{0.00166f, -0.00375f, 0.00209f, 0.0f}, {-0.02903f, 0.06377f, -0.03202f, 0.00394f},
                                  {0.11693f, -0.21196f, 0.06052f, 0.25886f}};
constexpr float kZenithY[3][4] = {{0.00275f, -0.00610f, 0.00317f, 0.0f}, {-0.04214f, 0.08970f, -0.04153f, 0.00516f},
                                  {0.15346f, -0.26756f, 0.06670f, 0.26688f}};

float clamped_exp(float x) { return fexp(rclamp(x, -80.0f, 80.0f)); }
// The Perez distribution F(theta, gamma) from cos theta, gamma and cos gamma.
float perez_f(const float* c, float cos_theta, float gamma, float cos_gamma) {
    return (1.0f + c[0] * clamped_exp(c[1] / cos_theta)) * (1.0f + c[2] * clamped_exp(c[3] * gamma) + c[4] * cos_gamma * cos_gamma);
}

struct ClassicSky {
    V3 sun;
    float coef[3][5], zenith_over_perez[3];
    ClassicSky(float azimuth_deg, float elevation_deg, float turbidity) {
        const float t = finitef(turbidity) ? rclamp(turbidity, 1.7f, 10.0f) : 3.0f;
        const float elevation = finitef(elevation_deg) ? rclamp(elevation_deg, 1.0f, 90.0f) : 45.0f;
        const float azimuth = finitef(azimuth_deg) ? azimuth_deg : 0.0f;
        float se, ce, sa, ca;
        sin_cos(elevation * (PI / 180.0f), se, ce);
        sin_cos(azimuth * (PI / 180.0f), sa, ca);
        sun = v3(ce * ca, ce * sa, se);
        const float theta_s = (90.0f - elevation) * (PI / 180.0f);
        for (int q = 0; q < 3; ++q)
            for (int k = 0; k < 5; ++k) coef[q][k] = kPerez[q][k][0] * t + kPerez[q][k][1];
        // zenith luminance (kcd/m^2) and chromaticity
        const float chi = (4.0f / 9.0f - t / 120.0f) * (PI - 2.0f * theta_s);
        float sc, cc;
        sin_cos(chi, sc, cc);
        const float y_z = (4.0453f * t - 4.9710f) * (sc / cc) - 0.2155f * t + 2.4192f;
        const float th[4] = {theta_s * theta_s * theta_s, theta_s * theta_s, theta_s, 1.0f};
        const float tt[3] = {t * t, t, 1.0f};
        auto fit = [&](const float (*m)[4]) {
            float sum = 0.0f;
            for (int i = 0; i < 3; ++i) {
                float r = 0.0f;
                for (int j = 0; j < 4; ++j) r += m[i][j] * th[j];
                sum += tt[i] * r;
            }
            return sum;
        };
        const float zenith[3] = {rmax(y_z, 1.0e-3f), fit(kZenithX), fit(kZenithY)};
        const float cs = fcos(theta_s);
        for (int q = 0; q < 3; ++q) zenith_over_perez[q] = zenith[q] / perez_f(coef[q], 1.0f, theta_s, cs);
    }
    // Linear Rec. 709 radiance in a unit direction above the horizon; black below.
    Rgb radiance(V3 dir) const {
        if (dir.z <= 0.0f) return rgb(0.0f, 0.0f, 0.0f);
        const float cos_gamma = rclamp(dot(dir, sun), -1.0f, 1.0f);
        const float gamma = facos(cos_gamma);
        const float cos_theta = rmax(dir.z, 1.0e-3f);
        float v[3];
        for (int q = 0; q < 3; ++q) v[q] = zenith_over_perez[q] * perez_f(coef[q], cos_theta, gamma, cos_gamma);
        const float lum = rmax(v[0], 0.0f), x = v[1], y = rmax(v[2], 1.0e-4f);
        // CIE xyY to XYZ to linear Rec. 709 (IEC 61966-2-1, D65), negatives clamped
        const float bx = x / y * lum, bz = (1.0f - x - y) / y * lum;
        const float r = 3.2404542f * bx - 1.5371385f * lum - 0.4985314f * bz;
        const float g = -0.969266f * bx + 1.8760108f * lum + 0.041556f * bz;
        const float b = 0.0556434f * bx - 0.2040259f * lum + 1.0572252f * bz;
        return rgb(rmax(r, 0.0f), rmax(g, 0.0f), rmax(b, 0.0f));
    }
};
}  // namespace

// ---- the physical sky (sky.rs:96-198): the Hosek-Wilkie functional form with the Repackshot fit ----
namespace {
// The fitted table (data/sky_table.f32, embedded at build time): 3240 coefficients
// [turbidity 1..10][ground albedo 0, 1][R, G, B][control point 0..5][A..I], then 360 radiances
// [turbidity][albedo][R, G, B][control point].
constexpr float kSkyTable[] = {
#include "_gen/rtg_sky_table.inc"
};
constexpr int kSkyParams = 9, kSkyControl = 6, kSkyCoefficients = 3240;
static_assert(sizeof(kSkyTable) / sizeof(float) == kSkyCoefficients + 360, "sky table size");
constexpr float kGroundAlbedo = 0.2f;  // sky.rs:68 GROUND_ALBEDO

struct SkyKnot {
    float weight, coef[3][kSkyParams], radiance[3];
};

// The sky for one sun position, turbidity and albedo: up to four knots (two turbidities times two
// albedos), each the table's quintic Bezier curves at x = (elevation / 90)^(1/3); radiances blended.
struct PhysicalSky {
    V3 sun;
    SkyKnot knots[4];
    int n = 0;
    PhysicalSky(float azimuth_deg, float elevation_deg, float turbidity, float albedo) {
        const float t = finitef(turbidity) ? rclamp(turbidity, 1.0f, 10.0f) : 3.0f;
        const float elevation = finitef(elevation_deg) ? rclamp(elevation_deg, 0.0f, 90.0f) : 45.0f;
        const float azimuth = finitef(azimuth_deg) ? azimuth_deg : 0.0f;
        const float a = finitef(albedo) ? rclamp(albedo, 0.0f, 1.0f) : kGroundAlbedo;
        float se, ce, sa, ca;
        sin_cos(elevation * (PI / 180.0f), se, ce);
        sin_cos(azimuth * (PI / 180.0f), sa, ca);
        sun = v3(ce * ca, ce * sa, se);
        const float x = fpow(elevation / 90.0f, 1.0f / 3.0f);
        // the six quintic Bernstein polynomials at x
        const float y = 1.0f - x, x2 = x * x, y2 = y * y, x3 = x2 * x, y3 = y2 * y;
        const float b[kSkyControl] = {y3 * y2, 5.0f * x * y2 * y2, 10.0f * x2 * y3, 10.0f * x3 * y2, 5.0f * x2 * x2 * y, x3 * x2};
        const float tt = t - 1.0f;
        const int i = std::min((int)std::floor(tt), 8);
        const float f = tt - (float)i;
        const int ti[2] = {i, i + 1};
        const float wt[2] = {1.0f - f, f}, wa[2] = {1.0f - a, a};
        for (int p = 0; p < 2; ++p)
            for (int q = 0; q < 2; ++q) {
                const float weight = wt[p] * wa[q];
                if (weight <= 0.0f) continue;
                SkyKnot& k = knots[n++];
                k = SkyKnot{};
                k.weight = weight;
                for (int c = 0; c < 3; ++c) {
                    const int base = (ti[p] * 2 + q) * 3 + c;
                    for (int m = 0; m < kSkyControl; ++m) {
                        for (int j = 0; j < kSkyParams; ++j) k.coef[c][j] += b[m] * kSkyTable[(base * kSkyControl + m) * kSkyParams + j];
                        k.radiance[c] += b[m] * kSkyTable[kSkyCoefficients + base * kSkyControl + m];
                    }
                }
            }
    }
    // Linear Rec. 709 radiance in a unit direction above the horizon, in the model's units; black
    // below. 1 + H^2 - 2 H cos gamma as (1 - H)^2 + H |v - s|^2 and gamma as atan2(|v x s|, v . s).
    Rgb radiance(V3 dir) const {
        if (dir.z <= 0.0f) return rgb(0.0f, 0.0f, 0.0f);
        const float cos_theta = dir.z;
        const float cos_gamma = rclamp(dot(dir, sun), -1.0f, 1.0f);
        const float gamma = fatan2(len(cross(dir, sun)), dot(dir, sun));
        const V3 chord = dir - sun;
        const float chord2 = dot(chord, chord);
        const float cg2 = cos_gamma * cos_gamma;
        const float horizon = 1.0f / (cos_theta + 0.01f);
        const float sq = sqrt_(cos_theta);
        float out[3] = {0.0f, 0.0f, 0.0f};
        for (int k = 0; k < n; ++k)
            for (int c = 0; c < 3; ++c) {
                const float* q = knots[k].coef[c];
                const float den = (1.0f - q[7]) * (1.0f - q[7]) + q[7] * chord2;
                const float chi = (1.0f + cg2) / (den * sqrt_(den));
                const float value = (1.0f + q[0] * clamped_exp(q[1] * horizon)) *
                                    (q[2] + q[3] * clamped_exp(q[4] * gamma) + q[5] * cg2 + q[6] * chi + q[8] * sq);
                out[c] += knots[k].weight * value * knots[k].radiance[c];
            }
        return rgb(rmax(out[0], 0.0f), rmax(out[1], 0.0f), rmax(out[2], 0.0f));
    }
};

// sum += x with Neumaier's compensation c (environment.rs:204): the total is sum + c.
inline void add_compensated(float& sum, float& c, float x) {
    const float t = sum + x;
    if (absf(sum) >= absf(x)) c += (sum - t) + x;
    else c += (x - t) + sum;
    sum = t;
}
}  // namespace

// environment.rs:216 tabulate_sky: the sky's upper half from the model, scaled so that a horizontal
// surface gets the dome's irradiance 2 pi (horizon / 6 + zenith / 3) strength; the lower half the
// ground, floor * strength. The physical sky sums the irradiance with compensation, the classic
// one plainly.
template <class Sky>
static HImage tabulate_sky(const HScene& s, const Sky& sky, bool compensated) {
    const uint32_t w = 256, h = 128;
    HImage img;
    img.width = w;
    img.height = h;
    img.texels.assign(3 * (size_t)w * h, 0.0f);
    float irradiance = 0.0f, irradiance_c = 0.0f;
    const float cell = (PI / (float)h) * (TAU / (float)w);
    for (uint32_t y = 0; y < h / 2; ++y) {
        const float v = ((float)y + 0.5f) / (float)h;
        float st, ct;
        sin_cos(PI * v, st, ct);
        float row = 0.0f, row_c = 0.0f;
        for (uint32_t x = 0; x < w; ++x) {
            const float u = ((float)x + 0.5f) / (float)w;
            float sp, cp;
            sin_cos(TAU * (u - 0.5f), sp, cp);
            const V3 d = v3(st * cp, -st * sp, ct);  // uv_to_direction (environment.rs:53)
            const Rgb c = sky.radiance(d);
            float* o = &img.texels[3 * ((size_t)y * w + x)];
            o[0] = c.r; o[1] = c.g; o[2] = c.b;
            const float term = luminance(c) * d.z * st;
            if (compensated) add_compensated(row, row_c, term);
            else row += term;
        }
        if (compensated) add_compensated(irradiance, irradiance_c, (row + row_c) * cell);
        else irradiance += row * cell;
    }
    irradiance = irradiance + irradiance_c;
    const float strength = rmax(s.env_strength, 0.0f);
    const float target = strength * TAU * (rmax(s.env_horizon, 0.0f) / 6.0f + rmax(s.env_zenith, 0.0f) / 3.0f);
    const float scale = irradiance > 0.0f ? target / irradiance : 0.0f;
    const float ground = rmax(s.env_floor * strength, 0.0f);
    for (size_t i = 0; i < img.texels.size(); ++i)
        img.texels[i] = i / (3 * (size_t)w) < h / 2 ? img.texels[i] * scale : ground;
    return img;
}

HImage sky_image(const HScene& s) {
    if (s.sky_model == 1) return tabulate_sky(s, ClassicSky(s.sun_azimuth_deg, s.sun_elevation_deg, s.sky_turbidity), false);
    return tabulate_sky(s, PhysicalSky(s.sun_azimuth_deg, s.sun_elevation_deg, s.sky_turbidity, kGroundAlbedo), true);
}

}  // namespace rtg
