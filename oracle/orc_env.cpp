// ORACLE (test infrastructure only). Bitmaps, Radiance HDR decoding, the 2-D sampling
// distribution and the HDRI environment, restated from engine/crates/rt-core/src/bitmap.rs:100-410,
// hdr.rs:30-240 and environment.rs:40-420.
#include <cctype>
#include <cstring>

#include "orc_scene.h"

namespace orc {

// ---- bitmap.rs ---------------------------------------------------------------------------------
const float* srgb_table() {  // bitmap.rs:108
    static float table[256];
    static bool ready = false;
    if (!ready) {
        for (int i = 0; i < 256; ++i) {
            float c = (float)i / 255.0f;
            table[i] = c <= 0.04045f ? c / 12.92f : powf_((c + 0.055f) / 1.055f, 2.4f);
        }
        ready = true;
    }
    return table;
}

Rgb Image::texel(uint32_t x, uint32_t y) const {  // bitmap.rs:127
    x = x < width - 1 ? x : width - 1;
    y = y < height - 1 ? y : height - 1;
    size_t i = 3 * ((size_t)y * width + x);
    if (!srgb8) return Rgb(linear[i], linear[i + 1], linear[i + 2]);
    const float* t = srgb_table();
    return Rgb(t[bytes[i]], t[bytes[i + 1]], t[bytes[i + 2]]);
}

// f32 as u32, saturating (Rust `as`): NaN and negatives to 0.
static uint32_t to_u32(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)x;
}

Rgb Image::bilinear(float u, float v, bool wrap_u) const {  // bitmap.rs:147
    float w = (float)width, h = (float)height;
    float fx = u * w - 0.5f;
    float fy = rclamp(v * h - 0.5f, 0.0f, h - 1.0f);
    float x0f = std::floor(fx);
    float y0f = std::floor(fy);
    float tx = fx - x0f, ty = fy - y0f;
    auto column = [&](float x) -> uint32_t {
        if (wrap_u) {
            float r = std::fmod(x, w);
            if (r < 0.0f) r = r + std::fabs(w);  // rem_euclid
            uint32_t c = to_u32(r);
            return c < width - 1 ? c : width - 1;
        }
        return to_u32(rclamp(x, 0.0f, w - 1.0f));
    };
    uint32_t x0 = column(x0f), x1 = column(x0f + 1.0f);
    uint32_t y0 = to_u32(y0f);
    uint32_t y1 = y0 + 1 < height - 1 ? y0 + 1 : height - 1;
    Rgb top = texel(x0, y0) * (1.0f - tx) + texel(x1, y0) * tx;
    Rgb bottom = texel(x0, y1) * (1.0f - tx) + texel(x1, y1) * tx;
    return top * (1.0f - ty) + bottom * ty;
}

static void halve(size_t& w, size_t& h, std::vector<float>& rgb) {  // bitmap.rs:182
    size_t nw = (w + 1) / 2, nh = (h + 1) / 2;
    std::vector<float> out(3 * nw * nh, 0.0f);
    for (size_t y = 0; y < nh; ++y) {
        size_t ya = 2 * y, yb = 2 * y + 1 < h - 1 ? 2 * y + 1 : h - 1;
        for (size_t x = 0; x < nw; ++x) {
            size_t xa = 2 * x, xb = 2 * x + 1 < w - 1 ? 2 * x + 1 : w - 1;
            for (int c = 0; c < 3; ++c) {
                float a = rgb[3 * (ya * w + xa) + c] + rgb[3 * (ya * w + xb) + c];
                float b = rgb[3 * (yb * w + xa) + c] + rgb[3 * (yb * w + xb) + c];
                out[3 * (y * nw + x) + c] = (a + b) * 0.25f;
            }
        }
    }
    w = nw;
    h = nh;
    rgb.swap(out);
}

static void linear_image(uint32_t width, uint32_t height, std::vector<float> rgb, Image& out) {  // bitmap.rs:201
    for (float& v : rgb)
        if (!(finite(v) && v > 0.0f)) v = 0.0f;
    size_t w = width, h = height;
    while (w > 4096) halve(w, h, rgb);  // MAX_LINEAR_WIDTH
    out = Image();
    out.width = (uint32_t)w;
    out.height = (uint32_t)h;
    out.srgb8 = false;
    out.linear = std::move(rgb);
}

// ---- hdr.rs ------------------------------------------------------------------------------------
static float hdr_pow2(int e) {  // hdr.rs:40
    if (e >= -126) return bitsf((uint32_t)(e + 127) << 23);
    if (e >= -149) return bitsf(1u << (e + 149));
    return 0.0f;
}
static bool hdr_line(const uint8_t* b, size_t n, size_t& pos, size_t& start, size_t& end) {
    start = pos;
    size_t k = pos;
    while (k < n && b[k] != '\n') ++k;
    if (k >= n) return false;
    end = k;
    pos = k + 1;
    return true;
}
static bool hdr_scanline(const uint8_t* b, size_t n, size_t& pos, std::vector<uint8_t>& row, size_t width) {  // hdr.rs:120
    bool new_rle = width >= 8 && width <= 0x7fff && n >= pos + 4 && b[pos] == 2 && b[pos + 1] == 2 && (b[pos + 2] & 0x80) == 0;
    if (new_rle) {
        size_t declared = ((size_t)b[pos + 2] << 8) | (size_t)b[pos + 3];
        if (declared != width) return false;
        pos += 4;
        for (int ch = 0; ch < 4; ++ch) {
            size_t x = 0;
            while (x < width) {
                if (pos >= n) return false;
                size_t count = b[pos++];
                if (count > 128) {
                    size_t k = count - 128;
                    if (pos >= n) return false;
                    uint8_t value = b[pos++];
                    if (x + k > width) return false;
                    for (size_t j = 0; j < k; ++j) row[(x + j) * 4 + ch] = value;
                    x += k;
                } else {
                    if (count == 0 || x + count > width || pos + count > n) return false;
                    for (size_t j = 0; j < count; ++j) row[(x + j) * 4 + ch] = b[pos + j];
                    pos += count;
                    x += count;
                }
            }
        }
        return true;
    }
    size_t x = 0;
    unsigned shift = 0;
    while (x < width) {
        if (pos + 4 > n) return false;
        const uint8_t* p = b + pos;
        pos += 4;
        if (p[0] == 1 && p[1] == 1 && p[2] == 1) {
            if (x == 0) return false;
            size_t k = (size_t)p[3] << shift;
            if (x + k > width) return false;
            for (size_t j = 0; j < k; ++j) std::memcpy(&row[(x + j) * 4], &row[(x - 1) * 4], 4);
            x += k;
            shift += 8;
        } else {
            std::memcpy(&row[x * 4], p, 4);
            x += 1;
            shift = 0;
        }
    }
    return true;
}
// hdr.rs:203 decode: header lines up to an empty one, the resolution line, then the scanlines.
static bool hdr_decode(const uint8_t* b, size_t n, uint32_t& width, uint32_t& height, std::vector<float>& rgb, std::string& reason) {
    auto starts = [&](const char* s) { size_t k = std::strlen(s); return n >= k && std::memcmp(b, s, k) == 0; };
    if (!(starts("#?RADIANCE") || starts("#?RGBE"))) { reason = "unreadable Radiance HDR image"; return false; }
    reason = "unreadable Radiance HDR image";
    size_t pos = 0, s0, e0;
    if (!hdr_line(b, n, pos, s0, e0)) return false;
    for (;;) {
        if (!hdr_line(b, n, pos, s0, e0)) return false;
        if (e0 == s0) break;
        const char* fmt = "FORMAT=";
        if (e0 - s0 >= 7 && std::memcmp(b + s0, fmt, 7) == 0) {
            size_t a = s0 + 7, z = e0;
            while (a < z && (b[a] == ' ' || b[a] == '\t' || b[a] == '\r' || b[a] == '\f')) ++a;
            while (z > a && (b[z - 1] == ' ' || b[z - 1] == '\t' || b[z - 1] == '\r' || b[z - 1] == '\f')) --z;
            const char* want = "32-bit_rle_rgbe";
            if (!(z - a == std::strlen(want) && std::memcmp(b + a, want, z - a) == 0)) return false;
        }
    }
    if (!hdr_line(b, n, pos, s0, e0)) return false;
    std::string res((const char*)b + s0, e0 - s0);
    std::vector<std::string> parts;
    {
        size_t i = 0;
        while (i < res.size()) {
            while (i < res.size() && std::isspace((unsigned char)res[i])) ++i;
            size_t j = i;
            while (j < res.size() && !std::isspace((unsigned char)res[j])) ++j;
            if (j > i) parts.push_back(res.substr(i, j - i));
            i = j;
        }
    }
    if (parts.size() != 4 || parts[2] != "+X") return false;
    bool top_down;
    if (parts[0] == "-Y") top_down = true;
    else if (parts[0] == "+Y") top_down = false;
    else return false;
    auto parse = [](const std::string& t, uint32_t& v) {
        if (t.empty() || t.size() > 10) return false;
        uint64_t x = 0;
        for (char c : t) {
            if (c < '0' || c > '9') return false;
            x = x * 10 + (uint64_t)(c - '0');
        }
        if (x > 0xffffffffull) return false;
        v = (uint32_t)x;
        return true;
    };
    uint32_t h, w;
    if (!(parse(parts[1], h) && parse(parts[3], w)) || w == 0 || h == 0) return false;
    if ((uint64_t)w * h > (1ull << 28)) return false;
    width = w;
    height = h;
    rgb.assign(3 * (size_t)w * h, 0.0f);
    std::vector<uint8_t> row(4 * (size_t)w, 0);
    for (size_t y = 0; y < h; ++y) {
        if (!hdr_scanline(b, n, pos, row, w)) return false;
        size_t dst = top_down ? y : h - 1 - y;
        for (size_t x = 0; x < w; ++x) {
            const uint8_t* p = &row[x * 4];
            float* o = &rgb[3 * (dst * w + x)];
            if (p[3] == 0) { o[0] = o[1] = o[2] = 0.0f; continue; }
            float f = hdr_pow2((int)p[3] - 136);
            o[0] = (float)p[0] * f;
            o[1] = (float)p[1] * f;
            o[2] = (float)p[2] * f;
        }
    }
    return true;
}

bool decode_bitmap(uint32_t format, uint32_t width, uint32_t height, const uint8_t* data, size_t len, Image& out,
                   std::string& reason, bool& unsupported) {  // bitmap.rs:236
    unsupported = false;
    auto raw_size = [&](uint64_t bpp) {
        uint64_t px = (uint64_t)width * height;
        if (width == 0 || height == 0 || width > 65536 || height > 65536 || px > (1ull << 28) || px * bpp != (uint64_t)len) {
            reason = "bitmap size does not match its data";
            return false;
        }
        return true;
    };
    switch (format) {
        case 0:
            if (!raw_size(3)) return false;
            out = Image();
            out.width = width;
            out.height = height;
            out.srgb8 = true;
            out.bytes.assign(data, data + len);
            return true;
        case 1:
            if (!raw_size(4)) return false;
            out = Image();
            out.width = width;
            out.height = height;
            out.srgb8 = true;
            for (size_t i = 0; i + 3 < len; i += 4) out.bytes.insert(out.bytes.end(), data + i, data + i + 3);
            return true;
        case 2: {
            if (!raw_size(12)) return false;
            std::vector<float> rgb(len / 4);
            std::memcpy(rgb.data(), data, len / 4 * 4);
            linear_image(width, height, std::move(rgb), out);
            return true;
        }
        case 16: {
            uint32_t w, h;
            std::vector<float> rgb;
            if (!hdr_decode(data, len, w, h, rgb, reason)) return false;
            if (!(width == 0 && height == 0) && !(width == w && height == h)) {
                reason = "bitmap size does not match its data";
                return false;
            }
            linear_image(w, h, std::move(rgb), out);
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

// ---- bitmap.rs:312-408 Distribution2D -----------------------------------------------------------
static void search(const float* cdf, size_t n, float u, size_t& i, float& rest) {  // bitmap.rs:314
    size_t k = 0;
    while (k < n && cdf[k] <= u) ++k;
    i = k < n - 1 ? k : n - 1;
    float lo = i == 0 ? 0.0f : cdf[i - 1];
    float width = cdf[i] - lo;
    rest = width > 0.0f ? rclamp((u - lo) / width, 0.0f, 0.99999994f) : 0.5f;
}
bool Distribution2D::make(size_t w, size_t h, std::vector<float> wts, Distribution2D& out) {
    Distribution2D d;
    d.width = w;
    d.height = h;
    d.conditional.assign(w * h, 0.0f);
    std::vector<float> row_sums(h, 0.0f);
    for (size_t y = 0; y < h; ++y) {
        float acc = 0.0f;
        for (size_t x = 0; x < w; ++x) {
            acc += wts[y * w + x];
            d.conditional[y * w + x] = acc;
        }
        row_sums[y] = acc;
        if (acc > 0.0f) {
            for (size_t x = 0; x < w; ++x) d.conditional[y * w + x] /= acc;
            d.conditional[(y + 1) * w - 1] = 1.0f;
        }
    }
    d.marginal.assign(h, 0.0f);
    float acc = 0.0f;
    for (size_t y = 0; y < h; ++y) {
        acc += row_sums[y];
        d.marginal[y] = acc;
    }
    if (!(acc > 0.0f && finite(acc))) return false;
    for (float& m : d.marginal) m /= acc;
    d.marginal[h - 1] = 1.0f;
    d.mean = acc / (float)(w * h);
    d.weights = std::move(wts);
    out = std::move(d);
    return true;
}
void Distribution2D::sample(float s0, float s1, float& u, float& v, float& pdf_out) const {
    size_t y, x;
    float fy, fx;
    search(marginal.data(), height, s1, y, fy);
    search(conditional.data() + y * width, width, s0, x, fx);
    u = ((float)x + fx) / (float)width;
    v = ((float)y + fy) / (float)height;
    pdf_out = weights[y * width + x] / mean;
}
static size_t to_usize(float x) {
    if (!(x > 0.0f)) return 0;
    if (x >= 1.8446744e19f) return SIZE_MAX;
    return (size_t)x;
}
float Distribution2D::pdf(float u, float v) const {
    size_t x = to_usize(u * (float)width), y = to_usize(v * (float)height);
    x = x < width - 1 ? x : width - 1;
    y = y < height - 1 ? y : height - 1;
    return weights[y * width + x] / mean;
}

// ---- environment.rs:40-130 ---------------------------------------------------------------------
static void direction_to_uv(Vec3 d, float& u, float& v) {
    float uu = 0.5f + fatan2(-d.y, d.x) * (0.5f * FRAC_1_PI);
    float vv = facos(d.z) * FRAC_1_PI;
    u = uu - std::floor(uu);
    v = rclamp(vv, 0.0f, 1.0f);
}
static Vec3 uv_to_direction(float u, float v, float& sin_theta) {
    float st, ct, sp, cp;
    sin_cos(PI * v, st, ct);
    sin_cos(TAU * (u - 0.5f), sp, cp);
    sin_theta = st;
    return Vec3(st * cp, -st * sp, ct);
}
bool EnvMap::make(const Image* image, float scale, float rotation_deg, EnvMap& out) {
    size_t w = image->width, h = image->height;
    size_t fx = (w + 511) / 512, fy = (h + 255) / 256;
    fx = fx > 1 ? fx : 1;
    fy = fy > 1 ? fy : 1;
    size_t gw = (w + fx - 1) / fx, gh = (h + fy - 1) / fy;
    std::vector<float> weights(gw * gh, 0.0f);
    float mean = 0.0f;
    for (size_t gy = 0; gy < gh; ++gy) {
        float theta = PI * ((float)gy + 0.5f) / (float)gh;
        float s = fsin(theta);
        float row_sum = 0.0f;
        for (size_t gx = 0; gx < gw; ++gx) {
            float lum = 0.0f;
            uint32_t n = 0;
            size_t y1 = (gy + 1) * fy < h ? (gy + 1) * fy : h, x1 = (gx + 1) * fx < w ? (gx + 1) * fx : w;
            for (size_t y = gy * fy; y < y1; ++y)
                for (size_t x = gx * fx; x < x1; ++x) {
                    lum += rmax(image->texel((uint32_t)x, (uint32_t)y).luminance(), 0.0f);
                    n += 1;
                }
            lum = lum / (float)(n > 1 ? n : 1);
            weights[gy * gw + gx] = lum * s;
            row_sum += lum * s;
        }
        mean += row_sum / (float)gw;
    }
    EnvMap m;
    m.image = image;
    m.scale = scale;
    m.mean_luminance = scale * (mean / (float)gh) * (0.5f * PI);
    if (!Distribution2D::make(gw, gh, std::move(weights), m.dist)) return false;
    sin_cos(rotation_deg * DEG_TO_RAD, m.rot_s, m.rot_c);
    out = std::move(m);
    return true;
}
Rgb EnvMap::radiance(Vec3 dir) const {
    float u, v;
    direction_to_uv(to_image(dir), u, v);
    return image->bilinear(u, v, true) * scale;
}
float EnvMap::pdf(Vec3 dir) const {
    Vec3 local = to_image(dir);
    float sin_theta = std::sqrt(rmax((1.0f - local.z) * (1.0f + local.z), 0.0f));
    if (sin_theta <= 0.0f) return 0.0f;
    float u, v;
    direction_to_uv(local, u, v);
    return dist.pdf(u, v) / (2.0f * PI * PI * sin_theta);
}
bool EnvMap::sample(float u0, float u1, Vec3& dir, float& pdf_out) const {
    float u, v, pdf_uv, sin_theta;
    dist.sample(u0, u1, u, v, pdf_uv);
    Vec3 local = uv_to_direction(u, v, sin_theta);
    if (!(sin_theta > 0.0f && pdf_uv > 0.0f)) return false;
    dir = normalize(to_world(local));
    pdf_out = pdf(dir);
    return pdf_out > 0.0f;
}
// ---- sky.rs:200-348 the classic sky ----------------------------------------------------------------
// The Perez coefficients A..E as (slope, intercept) in the turbidity for Y, x and y, and the zenith
// chromaticity fits: Preetham et al. 1999, Appendix A.2.
static const float PEREZ_TABLE[3][5][2] = {
    {{0.1787f, -1.4630f}, {-0.3554f, 0.4275f}, {-0.0227f, 5.3251f}, {0.1206f, -2.5771f}, {-0.0670f, 0.3703f}},
    {{-0.0193f, -0.2592f}, {-0.0665f, 0.0008f}, {-0.0004f, 0.2125f}, {-0.0641f, -0.8989f}, {-0.0033f, 0.0452f}},
    {{-0.0167f, -0.2608f}, {-0.0950f, 0.0092f}, {-0.0079f, 0.2102f}, {-0.0441f, -1.6537f}, {-0.0109f, 0.0529f}},
};
static const float ZENITH_XC[3][4] = {{0.00166f, -0.00375f, 0.00209f, 0.0f}, {-0.02903f, 0.06377f, -0.03202f, 0.00394f},
                                      {0.11693f, -0.21196f, 0.06052f, 0.25886f}};
static const float ZENITH_YC[3][4] = {{0.00275f, -0.00610f, 0.00317f, 0.0f}, {-0.04214f, 0.08970f, -0.04153f, 0.00516f},
                                      {0.15346f, -0.26756f, 0.06670f, 0.26688f}};
static float sky_exp(float x) { return fexp(rclamp(x, -80.0f, 80.0f)); }
static float perez(const float* c, float cos_theta, float gamma, float cos_gamma) {
    return (1.0f + c[0] * sky_exp(c[1] / cos_theta)) * (1.0f + c[2] * sky_exp(c[3] * gamma) + c[4] * cos_gamma * cos_gamma);
}
static Rgb xyy_to_rgb(float x, float y, float lum) {  // sky.rs:341 (IEC 61966-2-1, D65)
    float bx = x / y * lum;
    float bz = (1.0f - x - y) / y * lum;
    float r = 3.2404542f * bx - 1.5371385f * lum - 0.4985314f * bz;
    float g = -0.969266f * bx + 1.8760108f * lum + 0.041556f * bz;
    float b = 0.0556434f * bx - 0.2040259f * lum + 1.0572252f * bz;
    return Rgb(rmax(r, 0.0f), rmax(g, 0.0f), rmax(b, 0.0f));
}
Preetham Preetham::make(float azimuth_deg, float elevation_deg, float turbidity) {
    Preetham p;
    float t = finite(turbidity) ? rclamp(turbidity, 1.7f, 10.0f) : 3.0f;
    float elevation = finite(elevation_deg) ? rclamp(elevation_deg, 1.0f, 90.0f) : 45.0f;
    float azimuth = finite(azimuth_deg) ? azimuth_deg : 0.0f;
    float se, ce, sa, ca;
    sin_cos(elevation * DEG_TO_RAD, se, ce);
    sin_cos(azimuth * DEG_TO_RAD, sa, ca);
    p.sun = Vec3(ce * ca, ce * sa, se);
    float theta_s = (90.0f - elevation) * DEG_TO_RAD;
    for (int q = 0; q < 3; ++q)
        for (int k = 0; k < 5; ++k) p.coefficients[q][k] = PEREZ_TABLE[q][k][0] * t + PEREZ_TABLE[q][k][1];
    float chi = (4.0f / 9.0f - t / 120.0f) * (PI - 2.0f * theta_s);
    float sc, cc;
    sin_cos(chi, sc, cc);
    float y_z = (4.0453f * t - 4.9710f) * (sc / cc) - 0.2155f * t + 2.4192f;
    float th[4] = {theta_s * theta_s * theta_s, theta_s * theta_s, theta_s, 1.0f};
    auto poly = [&](const float (*m)[4]) {
        float tt[3] = {t * t, t, 1.0f};
        float sum = 0.0f;
        for (int i = 0; i < 3; ++i) {
            float r = 0.0f;
            for (int j = 0; j < 4; ++j) r += m[i][j] * th[j];
            sum += tt[i] * r;
        }
        return sum;
    };
    float zenith[3] = {rmax(y_z, 1.0e-3f), poly(ZENITH_XC), poly(ZENITH_YC)};
    float cs = fcos(theta_s);
    for (int q = 0; q < 3; ++q) p.zenith_over_perez[q] = zenith[q] / perez(p.coefficients[q], 1.0f, theta_s, cs);
    return p;
}
Rgb Preetham::radiance(Vec3 dir) const {
    if (dir.z <= 0.0f) return BLACK;
    float cos_gamma = rclamp(dot(dir, sun), -1.0f, 1.0f);
    float gamma = facos(cos_gamma);
    float cos_theta = rmax(dir.z, 1.0e-3f);
    float v[3];
    for (int q = 0; q < 3; ++q) v[q] = zenith_over_perez[q] * perez(coefficients[q], cos_theta, gamma, cos_gamma);
    return xyy_to_rgb(v[1], rmax(v[2], 1.0e-4f), rmax(v[0], 0.0f));
}
// ---- sky.rs:96-198 the physical sky: the Hosek-Wilkie form, coefficients from the fitted table ----
// The table (set by orc_set_sky_table): 3240 coefficients [turbidity 1..10][albedo 0, 1][R, G, B]
// [control point 0..5][A..I], then 360 radiances [turbidity][albedo][R, G, B][control point].
static std::vector<float> g_sky_table;
PhysicalSky PhysicalSky::make(float azimuth_deg, float elevation_deg, float turbidity, float albedo) {  // sky.rs:113
    PhysicalSky p;
    float t = finite(turbidity) ? rclamp(turbidity, 1.0f, 10.0f) : 3.0f;
    float elevation = finite(elevation_deg) ? rclamp(elevation_deg, 0.0f, 90.0f) : 45.0f;
    float azimuth = finite(azimuth_deg) ? azimuth_deg : 0.0f;
    float a = finite(albedo) ? rclamp(albedo, 0.0f, 1.0f) : 0.2f;
    float se, ce, sa, ca;
    sin_cos(elevation * DEG_TO_RAD, se, ce);
    sin_cos(azimuth * DEG_TO_RAD, sa, ca);
    p.sun = Vec3(ce * ca, ce * sa, se);
    float x = powf_(elevation / 90.0f, 1.0f / 3.0f);
    float y = 1.0f - x, x2 = x * x, y2 = y * y, x3 = x2 * x, y3 = y2 * y;
    float bern[6] = {y3 * y2, 5.0f * x * y2 * y2, 10.0f * x2 * y3, 10.0f * x3 * y2, 5.0f * x2 * x2 * y, x3 * x2};  // sky.rs:91
    float tt = t - 1.0f;
    int i = std::min((int)std::floor(tt), 8);
    float f = tt - (float)i;
    int tis[2] = {i, i + 1};
    float wts[2] = {1.0f - f, f}, was[2] = {1.0f - a, a};
    p.n = 0;
    if (g_sky_table.size() != 3600) return p;
    for (int u = 0; u < 2; ++u)
        for (int ai = 0; ai < 2; ++ai) {
            float weight = wts[u] * was[ai];
            if (weight <= 0.0f) continue;
            Knot& k = p.knots[p.n++];
            k = Knot{};
            k.weight = weight;
            for (int c = 0; c < 3; ++c) {
                int base = (tis[u] * 2 + ai) * 3 + c;
                for (int m = 0; m < 6; ++m) {
                    for (int j = 0; j < 9; ++j) k.coefficients[c][j] += bern[m] * g_sky_table[(base * 6 + m) * 9 + j];
                    k.radiance[c] += bern[m] * g_sky_table[3240 + base * 6 + m];
                }
            }
        }
    return p;
}
Rgb PhysicalSky::radiance(Vec3 dir) const {  // sky.rs:170
    if (dir.z <= 0.0f) return BLACK;
    float cos_theta = dir.z;
    float cos_gamma = rclamp(dot(dir, sun), -1.0f, 1.0f);
    float gamma = fatan2(length(cross(dir, sun)), dot(dir, sun));
    Vec3 chord = dir - sun;
    float chord2 = dot(chord, chord);
    float cg2 = cos_gamma * cos_gamma;
    float horizon = 1.0f / (cos_theta + 0.01f);
    float sq = std::sqrt(cos_theta);
    float out[3] = {0.0f, 0.0f, 0.0f};
    for (int k = 0; k < n; ++k)
        for (int c = 0; c < 3; ++c) {
            const float* q = knots[k].coefficients[c];
            float den = (1.0f - q[7]) * (1.0f - q[7]) + q[7] * chord2;
            float chi = (1.0f + cg2) / (den * std::sqrt(den));
            float value = (1.0f + q[0] * sky_exp(q[1] * horizon)) * (q[2] + q[3] * sky_exp(q[4] * gamma) + q[5] * cg2 + q[6] * chi + q[8] * sq);
            out[c] += knots[k].weight * value * knots[k].radiance[c];
        }
    return Rgb(rmax(out[0], 0.0f), rmax(out[1], 0.0f), rmax(out[2], 0.0f));
}

// environment.rs:204 add_compensated: sum += x with Neumaier's compensation c.
static void add_compensated(float& sum, float& c, float x) {
    float t = sum + x;
    if (std::fabs(sum) >= std::fabs(x)) c += (sum - t) + x;
    else c += (x - t) + sum;
    sum = t;
}

// environment.rs:216 tabulate_sky: the upper half from the model, scaled so that a horizontal
// surface gets the dome's irradiance 2 pi (horizon / 6 + zenith / 3) strength; the lower half the
// ground, floor * strength. The physical sky sums with compensation, the classic one plainly.
template <class Sky>
static Image tabulate_sky(const Environment& env, const Sky& sky, bool compensated) {
    const uint32_t w = 256, h = 128;
    std::vector<float> rgb(3 * (size_t)w * h, 0.0f);
    float irradiance = 0.0f, irradiance_c = 0.0f;
    const float cell = (PI / (float)h) * (TAU / (float)w);
    for (uint32_t y = 0; y < h / 2; ++y) {
        float v = ((float)y + 0.5f) / (float)h;
        float row = 0.0f, row_c = 0.0f;
        for (uint32_t x = 0; x < w; ++x) {
            float u = ((float)x + 0.5f) / (float)w, sin_theta;
            Vec3 d = uv_to_direction(u, v, sin_theta);
            Rgb c = sky.radiance(d);
            float* o = &rgb[3 * ((size_t)y * w + x)];
            o[0] = c.r; o[1] = c.g; o[2] = c.b;
            float term = c.luminance() * d.z * sin_theta;
            if (compensated) add_compensated(row, row_c, term);
            else row += term;
        }
        if (compensated) add_compensated(irradiance, irradiance_c, (row + row_c) * cell);
        else irradiance += row * cell;
    }
    irradiance = irradiance + irradiance_c;
    float strength = rmax(env.strength, 0.0f);
    float target = strength * TAU * (rmax(env.horizon, 0.0f) / 6.0f + rmax(env.zenith, 0.0f) / 3.0f);
    float scale = irradiance > 0.0f ? target / irradiance : 0.0f;
    float ground = rmax(env.floor * strength, 0.0f);
    for (size_t i = 0; i < rgb.size(); ++i) rgb[i] = i / (3 * (size_t)w) < h / 2 ? rgb[i] * scale : ground;
    Image img;
    img.width = w;
    img.height = h;
    img.linear = std::move(rgb);
    return img;
}

// environment.rs:178 sky_image: the scene's sky model tabulated.
Image sky_image(const Environment& env) {
    if (env.sky_model == 1)
        return tabulate_sky(env, Preetham::make(env.sun_azimuth_deg, env.sun_elevation_deg, env.sky_turbidity), false);
    return tabulate_sky(env, PhysicalSky::make(env.sun_azimuth_deg, env.sun_elevation_deg, env.sky_turbidity, 0.2f), true);
}

}  // namespace orc

extern "C" {
// The physical sky's fitted table: n = 3600 floats (3240 coefficients, then 360 radiances).
void orc_set_sky_table(const float* values, uint32_t n) { orc::g_sky_table.assign(values, values + n); }
}

namespace orc {

EnvLight EnvLight::make(const Environment& env, const std::vector<Image>& bitmaps) {  // environment.rs:335
    EnvLight e;
    float strength = rmax(env.strength, 0.0f);
    if (env.kind == 1) { e.ramp = Ramp::make(env.horizon, env.horizon, env.horizon, strength); return e; }
    if (env.kind == 2) {
        e.owned = std::make_shared<Image>(sky_image(env));
        if (EnvMap::make(e.owned.get(), 1.0f, 0.0f, e.map)) e.is_map = true;
        else e.ramp = Ramp::make(0.0f, 0.0f, 0.0f, strength);
        return e;
    }
    if (env.kind == 3 && env.hdri_map != NO_BITMAP && env.hdri_map < bitmaps.size()) {
        if (EnvMap::make(&bitmaps[env.hdri_map], strength, env.rotation_deg, e.map)) e.is_map = true;
        else e.ramp = Ramp::make(0.0f, 0.0f, 0.0f, strength);
        return e;
    }
    e.ramp = Ramp::make(env.floor, env.horizon, env.zenith, strength);
    return e;
}

}  // namespace orc
