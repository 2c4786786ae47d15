// IES LM-63 photometric profiles on the host (engine/crates/rt-core/src/ies.rs:207-629): the
// reader of type C files and the flux of the bilinear interpolant, in closed form per cell. The
// device evaluates the interpolant itself (ies_shape, rtg_lights.cuh) from the flattened table.
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "rtg_scene.h"

namespace rtg {
namespace {

const float kDeg = PI / 180.0f;
bool same_angle(float a, float b) { return absf(a - b) < 1.0e-3f; }
bool strictly_increasing(const std::vector<float>& a) {
    for (size_t i = 1; i < a.size(); ++i)
        if (!(a[i - 1] < a[i])) return false;
    return true;
}
// sin x - x cos x without its cancellation for small x (ies.rs:468).
float sin_less_x_cos(float x) {
    if (x < 0.05f) {
        const float x2 = x * x;
        return x * x2 * (1.0f / 3.0f - x2 * (1.0f / 30.0f - x2 * (1.0f / 840.0f)));
    }
    float s, c;
    sin_cos(x, s, c);
    return s - x * c;
}
// The integral of sin(gamma) times the intensity along one row of the table (ies.rs:431): per cell
// the intensity is linear in gamma, and the integral is closed-form.
float row_integral(const HIes& p, size_t row) {
    const size_t n = p.vertical.size();
    float sum = 0.0f;
    for (size_t i = 0; i + 1 < n; ++i) {
        const float g0 = p.vertical[i] * kDeg, g1 = p.vertical[i + 1] * kDeg;
        const float a = p.candela[row * n + i], b = p.candela[row * n + i + 1];
        const float half = 0.5f * (g1 - g0), mid = 0.5f * (g0 + g1);
        const float mean = 0.5f * (a + b), slope = (b - a) / (g1 - g0);
        float sm, cm, sh, ch;
        sin_cos(mid, sm, cm);
        sin_cos(half, sh, ch);
        sum += mean * 2.0f * sm * sh + slope * cm * 2.0f * sin_less_x_cos(half);
    }
    return sum;
}
// A number token as Rust's f32 parser reads it: [+-] digits [. digits] [e [+-] digits], or
// inf / infinity / nan (which are not finite, so refused).
bool read_number(const uint8_t* t, size_t n, float& out) {
    std::string s((const char*)t, n), low;
    size_t i = (n && (s[0] == '+' || s[0] == '-')) ? 1 : 0;
    for (size_t k = i; k < n; ++k) low += (char)std::tolower((unsigned char)s[k]);
    if (low == "inf" || low == "infinity" || low == "nan") return false;
    size_t digits = 0;
    while (i < n && std::isdigit((unsigned char)s[i])) { ++i; ++digits; }
    if (i < n && s[i] == '.') {
        for (++i; i < n && std::isdigit((unsigned char)s[i]); ++i) ++digits;
    }
    if (!digits) return false;
    if (i < n && (s[i] == 'e' || s[i] == 'E')) {
        ++i;
        if (i < n && (s[i] == '+' || s[i] == '-')) ++i;
        size_t e = 0;
        for (; i < n && std::isdigit((unsigned char)s[i]); ++i) ++e;
        if (!e) return false;
    }
    if (i != n) return false;
    out = std::strtof(s.c_str(), nullptr);  // correctly rounded, as the reference's parser
    return finitef(out);
}

}  // namespace

bool parse_ies(const uint8_t* b, size_t len, HIes& out, std::string& reason) {
    if (len > 2u * 1024u * 1024u) { reason = "the IES file is too large"; return false; }
    // The header: lines (a CR LF is one break) up to TILT=, which must be NONE.
    size_t pos = 0, data_at = 0;
    bool tilt = false;
    while (pos < len && !tilt) {
        size_t end = pos;
        while (end < len && b[end] != '\n' && b[end] != '\r') ++end;
        size_t s = pos, e = end;
        while (s < e && std::isspace(b[s])) ++s;
        while (e > s && std::isspace(b[e - 1])) --e;
        pos = end;
        if (pos < len) pos += (b[pos] == '\r' && pos + 1 < len && b[pos + 1] == '\n') ? 2 : 1;
        if (e - s >= 5) {
            std::string head((const char*)b + s, 5);
            for (char& c : head) c = (char)std::toupper((unsigned char)c);
            if (head == "TILT=") {
                size_t vs = s + 5;
                while (vs < e && std::isspace(b[vs])) ++vs;
                std::string v((const char*)b + vs, e - vs);
                for (char& c : v) c = (char)std::toupper((unsigned char)c);
                if (v != "NONE") {
                    reason = v == "INCLUDE" ? "TILT=INCLUDE is not supported: export the profile with TILT=NONE"
                                            : "a TILT file is not supported: the profile needs TILT=NONE";
                    return false;
                }
                tilt = true;
                data_at = pos;
            }
        }
    }
    if (!tilt) { reason = "the IES file has no TILT= line"; return false; }
    std::vector<float> nums;
    for (size_t i = data_at; i < len;) {
        while (i < len && (std::isspace(b[i]) || b[i] == ',')) ++i;
        size_t j = i;
        while (j < len && !(std::isspace(b[j]) || b[j] == ',')) ++j;
        if (j > i) {
            float v;
            if (!read_number(b + i, j - i, v)) { reason = "the IES table holds a value that is not a number"; return false; }
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
    uint32_t nv = 0, nh = 0, type = 0;
    if (!whole(nums[3], nv) || nv < 1 || !whole(nums[4], nh) || nh < 1) {
        reason = "the IES angle counts must be whole numbers of at least one";
        return false;
    }
    if (nv > 4096 || nh > 4096) { reason = "the IES file declares too many angles"; return false; }
    if (!whole(nums[5], type) || type < 1 || type > 3) { reason = "the IES photometric type is not 1, 2 or 3"; return false; }
    if (type != 1) { reason = "only photometric type C is supported, not type A or B"; return false; }
    const float multiplier = nums[2];
    if (multiplier <= 0.0f) { reason = "the IES candela multiplier must be positive"; return false; }
    const size_t expected = 13 + (size_t)nv + nh + (size_t)nv * nh;
    if (nums.size() != expected) {
        reason = nums.size() < expected ? "the IES file has fewer values than its counts declare"
                                        : "the IES file has more values than its counts declare";
        return false;
    }
    HIes p;
    p.vertical.assign(nums.begin() + 13, nums.begin() + 13 + nv);
    p.horizontal.assign(nums.begin() + 13 + nv, nums.begin() + 13 + nv + nh);
    const std::vector<float>& v = p.vertical;
    const bool vertical_ok = v.size() >= 2 && strictly_increasing(v) &&
                             ((same_angle(v[0], 0.0f) && (same_angle(v.back(), 90.0f) || same_angle(v.back(), 180.0f))) ||
                              (same_angle(v[0], 90.0f) && same_angle(v.back(), 180.0f)));
    if (!vertical_ok) { reason = "the IES vertical angles must increase and run 0-90, 0-180 or 90-180"; return false; }
    const std::vector<float>& h = p.horizontal;
    const char* bad_h = "the IES horizontal angles must increase and be one angle, 0-90, 0-180, 90-270 or 0-360";
    if (h.size() == 1) {
        if (!(h[0] >= 0.0f && h[0] <= 360.0f)) { reason = bad_h; return false; }
        p.symmetry = IES_ROTATIONAL;
    } else {
        if (!strictly_increasing(h)) { reason = bad_h; return false; }
        const float f = h[0], l = h.back();
        if (same_angle(f, 0.0f) && same_angle(l, 90.0f)) p.symmetry = IES_QUADRANT;
        else if (same_angle(f, 0.0f) && same_angle(l, 180.0f)) p.symmetry = IES_BILATERAL0;
        else if (same_angle(f, 90.0f) && same_angle(l, 270.0f)) p.symmetry = IES_BILATERAL90;
        else if (same_angle(f, 0.0f) && same_angle(l, 360.0f)) p.symmetry = IES_FULL;
        else { reason = bad_h; return false; }
    }
    for (size_t k = 13 + nv + nh; k < expected; ++k)
        if (nums[k] < 0.0f) { reason = "the IES table has a negative candela value"; return false; }
    for (size_t k = 13 + nv + nh; k < expected; ++k) p.candela.push_back(nums[k] * multiplier);
    for (float c : p.candela) p.peak = rmax(p.peak, c);
    if (!(p.peak > 0.0f && finitef(p.peak))) { reason = "the IES table is all zeros: it gives no light"; return false; }
    // The flux of the interpolant over the sphere (ies.rs:451): rows linear in phi between them.
    if (h.size() == 1) {
        p.flux = TAU * row_integral(p, 0);
    } else {
        float sum = 0.0f, prev = row_integral(p, 0);
        for (size_t j = 0; j + 1 < h.size(); ++j) {
            const float next = row_integral(p, j + 1);
            sum += (h[j + 1] - h[j]) * kDeg * 0.5f * (prev + next);
            prev = next;
        }
        const float copies = p.symmetry == IES_QUADRANT ? 4.0f : (p.symmetry == IES_FULL ? 1.0f : 2.0f);
        p.flux = sum * copies;
    }
    out = std::move(p);
    return true;
}

}  // namespace rtg
