// ORACLE (test infrastructure only). IES LM-63 type C photometric profiles, restated from
// engine/crates/rt-core/src/ies.rs:207-629: the reader, the bilinear intensity by the table's
// symmetry, and the closed-form flux of that interpolant.
#include <cctype>
#include <cstdlib>
#include <cstring>

#include "orc_scene.h"

namespace orc {
namespace {
const float DEG = DEG_TO_RAD;
const float RAD = 180.0f / PI;
bool same(float a, float b) { return std::fabs(a - b) < 1.0e-3f; }
bool increasing(const std::vector<float>& a) {
    for (size_t i = 1; i < a.size(); ++i)
        if (!(a[i - 1] < a[i])) return false;
    return true;
}
// The cell of an increasing list that holds x (the last for the top angle).
size_t cell(const std::vector<float>& a, float x) {
    size_t k = 0;
    while (k < a.size() && a[k] <= x) ++k;
    size_t i = k ? k - 1 : 0;
    return i < a.size() - 2 ? i : a.size() - 2;
}
float sin_minus_x_cos(float x) {  // ies.rs:468
    if (x < 0.05f) {
        float x2 = x * x;
        return x * x2 * (1.0f / 3.0f - x2 * (1.0f / 30.0f - x2 * (1.0f / 840.0f)));
    }
    return fsin(x) - x * fcos(x);
}
// A decimal number as Rust's f32 parser takes it: [+-] digits [. digits] [e [+-] digits], or inf,
// infinity, nan (rejected later as not finite).
bool number(const char* t, size_t n, float& out) {
    std::string s(t, n);
    size_t i = 0;
    if (i < n && (s[i] == '+' || s[i] == '-')) ++i;
    std::string rest;
    for (size_t k = i; k < n; ++k) rest += (char)std::tolower((unsigned char)s[k]);
    if (rest == "inf" || rest == "infinity" || rest == "nan") { out = F_INF; return true; }
    size_t digits = 0;
    while (i < n && std::isdigit((unsigned char)s[i])) { ++i; ++digits; }
    if (i < n && s[i] == '.') {
        ++i;
        while (i < n && std::isdigit((unsigned char)s[i])) { ++i; ++digits; }
    }
    if (digits == 0) return false;
    if (i < n && (s[i] == 'e' || s[i] == 'E')) {
        ++i;
        if (i < n && (s[i] == '+' || s[i] == '-')) ++i;
        size_t e = 0;
        while (i < n && std::isdigit((unsigned char)s[i])) { ++i; ++e; }
        if (e == 0) return false;
    }
    if (i != n) return false;
    out = std::strtof(s.c_str(), nullptr);
    return true;
}
}  // namespace

bool IesProfile::parse(const uint8_t* b, size_t len, IesProfile& out, std::string& reason) {
    if (len > 2u * 1024u * 1024u) { reason = "the IES file is too large"; return false; }
    // read_header (ies.rs:550): lines up to TILT=
    size_t pos = 0, data_at = 0;
    bool tilt = false;
    while (pos < len) {
        size_t end = pos;
        while (end < len && b[end] != '\n' && b[end] != '\r') ++end;
        size_t s = pos, e = end;
        while (s < e && std::isspace(b[s])) ++s;
        while (e > s && std::isspace(b[e - 1])) --e;
        pos = end;
        if (pos < len) pos += (b[pos] == '\r' && pos + 1 < len && b[pos + 1] == '\n') ? 2 : 1;
        if (e - s >= 5 && std::toupper(b[s]) == 'T' && std::toupper(b[s + 1]) == 'I' && std::toupper(b[s + 2]) == 'L' &&
            std::toupper(b[s + 3]) == 'T' && b[s + 4] == '=') {
            size_t vs = s + 5;
            while (vs < e && std::isspace(b[vs])) ++vs;
            std::string v;
            for (size_t k = vs; k < e; ++k) v += (char)std::toupper(b[k]);
            if (v == "NONE") { tilt = true; data_at = pos; break; }
            reason = v == "INCLUDE" ? "TILT=INCLUDE is not supported: export the profile with TILT=NONE"
                                    : "a TILT file is not supported: the profile needs TILT=NONE";
            return false;
        }
    }
    if (!tilt) { reason = "the IES file has no TILT= line"; return false; }
    // read_numbers (ies.rs:601): numbers separated by ASCII white space or commas
    std::vector<float> nums;
    for (size_t i = data_at; i < len;) {
        while (i < len && (std::isspace(b[i]) || b[i] == ',')) ++i;
        size_t j = i;
        while (j < len && !(std::isspace(b[j]) || b[j] == ',')) ++j;
        if (j > i) {
            float v;
            if (!number((const char*)b + i, j - i, v) || !finite(v)) { reason = "the IES table holds a value that is not a number"; return false; }
            nums.push_back(v);
        }
        i = j;
    }
    if (nums.size() < 13) { reason = "the IES file ends inside the thirteen numbers of its header"; return false; }
    auto whole = [](float x, uint32_t& v) {
        if (!(x >= 0.0f && x <= 1.0e9f) || x != std::floor(x)) return false;
        v = (uint32_t)x;
        return true;
    };
    uint32_t nv, nh, type;
    if (!whole(nums[3], nv) || nv < 1 || !whole(nums[4], nh) || nh < 1) { reason = "the IES angle counts must be whole numbers of at least one"; return false; }
    if (nv > 4096 || nh > 4096) { reason = "the IES file declares too many angles"; return false; }
    if (!whole(nums[5], type) || type < 1 || type > 3) { reason = "the IES photometric type is not 1, 2 or 3"; return false; }
    if (type != 1) { reason = "only photometric type C is supported, not type A or B"; return false; }
    float multiplier = nums[2];
    if (multiplier <= 0.0f) { reason = "the IES candela multiplier must be positive"; return false; }
    size_t expected = 13 + (size_t)nv + nh + (size_t)nv * nh;
    if (nums.size() < expected) { reason = "the IES file has fewer values than its counts declare"; return false; }
    if (nums.size() > expected) { reason = "the IES file has more values than its counts declare"; return false; }
    IesProfile p;
    p.vertical.assign(nums.begin() + 13, nums.begin() + 13 + nv);
    p.horizontal.assign(nums.begin() + 13 + nv, nums.begin() + 13 + nv + nh);
    const std::vector<float>& v = p.vertical;
    bool vok = v.size() >= 2 && increasing(v) &&
               ((same(v[0], 0.0f) && (same(v.back(), 90.0f) || same(v.back(), 180.0f))) || (same(v[0], 90.0f) && same(v.back(), 180.0f)));
    if (!vok) { reason = "the IES vertical angles must increase and run 0-90, 0-180 or 90-180"; return false; }
    const std::vector<float>& h = p.horizontal;
    const char* hbad = "the IES horizontal angles must increase and be one angle, 0-90, 0-180, 90-270 or 0-360";
    if (h.size() == 1) {
        if (!(h[0] >= 0.0f && h[0] <= 360.0f)) { reason = hbad; return false; }
        p.symmetry = Rotational;
    } else {
        if (!increasing(h)) { reason = hbad; return false; }
        float f = h[0], l = h.back();
        if (same(f, 0.0f) && same(l, 90.0f)) p.symmetry = Quadrant;
        else if (same(f, 0.0f) && same(l, 180.0f)) p.symmetry = Bilateral0;
        else if (same(f, 90.0f) && same(l, 270.0f)) p.symmetry = Bilateral90;
        else if (same(f, 0.0f) && same(l, 360.0f)) p.symmetry = Full;
        else { reason = hbad; return false; }
    }
    for (size_t k = 13 + nv + nh; k < expected; ++k)
        if (nums[k] < 0.0f) { reason = "the IES table has a negative candela value"; return false; }
    for (size_t k = 13 + nv + nh; k < expected; ++k) p.candela.push_back(nums[k] * multiplier);
    float peak = 0.0f;
    for (float c : p.candela) peak = rmax(peak, c);
    if (!(peak > 0.0f && finite(peak))) { reason = "the IES table is all zeros: it gives no light"; return false; }
    p.peak = peak;
    p.flux = p.integrate();
    out = std::move(p);
    return true;
}

float IesProfile::fold(float phi) const {  // ies.rs:395
    float p = phi - 360.0f * std::floor(phi / 360.0f);
    switch (symmetry) {
        case Bilateral0: return p > 180.0f ? 360.0f - p : p;
        case Quadrant: {
            float q = p > 180.0f ? 360.0f - p : p;
            return q > 90.0f ? 180.0f - q : q;
        }
        case Bilateral90: {
            if (p >= 90.0f && p <= 270.0f) return p;
            float q = 180.0f - p;
            return q < 0.0f ? q + 360.0f : q;
        }
        default: return p;
    }
}
float IesProfile::intensity(float gamma, float phi) const {  // ies.rs:350
    const std::vector<float>& v = vertical;
    size_t last = v.size() - 1;
    if (!(gamma >= v[0] && gamma <= v[last])) return 0.0f;
    size_t i = cell(v, gamma);
    float t = (gamma - v[i]) / (v[i + 1] - v[i]);
    size_t n = v.size();
    auto along = [&](size_t row) {
        float a = candela[row * n + i], b = candela[row * n + i + 1];
        return a + (b - a) * t;
    };
    if (horizontal.size() == 1) return along(0);
    float p = fold(phi);
    size_t j = cell(horizontal, p);
    float s = (p - horizontal[j]) / (horizontal[j + 1] - horizontal[j]);
    float a = along(j), b2 = along(j + 1);
    return a + (b2 - a) * s;
}
float IesProfile::shape(Vec3 local) const {  // ies.rs:378-392
    float rho = std::sqrt(local.x * local.x + local.y * local.y);
    float gamma = fatan2(rho, local.z) * RAD;
    float phi = horizontal.size() == 1 ? 0.0f : fatan2(local.x, local.y) * RAD;
    return rmin(intensity(gamma, phi) / peak, 1.0f);
}
float IesProfile::row_integral(size_t row) const {  // ies.rs:431
    size_t n = vertical.size();
    float sum = 0.0f;
    for (size_t i = 0; i + 1 < n; ++i) {
        float g0 = vertical[i] * DEG, g1 = vertical[i + 1] * DEG;
        float a = candela[row * n + i], b = candela[row * n + i + 1];
        float half = 0.5f * (g1 - g0), mid = 0.5f * (g0 + g1);
        float mean = 0.5f * (a + b), slope = (b - a) / (g1 - g0);
        sum += mean * 2.0f * fsin(mid) * fsin(half) + slope * fcos(mid) * 2.0f * sin_minus_x_cos(half);
    }
    return sum;
}
float IesProfile::integrate() const {  // ies.rs:451
    size_t rows = horizontal.size();
    if (rows == 1) return TAU * row_integral(0);
    std::vector<float> columns(rows);
    for (size_t j = 0; j < rows; ++j) columns[j] = row_integral(j);
    float sum = 0.0f;
    for (size_t j = 0; j + 1 < rows; ++j) {
        float width = (horizontal[j + 1] - horizontal[j]) * DEG;
        sum += width * 0.5f * (columns[j] + columns[j + 1]);
    }
    float copies = (symmetry == Rotational || symmetry == Full) ? 1.0f : ((symmetry == Quadrant) ? 4.0f : 2.0f);
    return sum * copies;
}

}  // namespace orc
