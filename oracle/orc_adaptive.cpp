// Test infrastructure: the CPU restatement the CUDA path is checked against, never shipped.
//
// Adaptive sampling, restated from engine/crates/rt-core/src/adaptive.rs in f32 and in the
// reference's order of operations (the decision is bit-exact by design: the reference ports it to
// TypeScript and pins its bits).
#include "orc_adaptive.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "orc_core.h"

namespace orc {

float ad_floor_for(float ev) { return AD_EPSILON / exp2(ev); }  // adaptive.rs:85, color.rs:146

float ad_pixel_error(float r, float g, float b, float lum2, uint32_t n, float floor) {  // adaptive.rs:93
    if (n < 2) return AD_UNMEASURED;
    const float nf = (float)n;
    const float inv = 1.0f / nf;
    const float l = 0.2126f * (r * inv) + 0.7152f * (g * inv) + 0.0722f * (b * inv);
    const float m2 = lum2 * inv;
    if (!(std::isfinite(l) && std::isfinite(m2))) return AD_UNMEASURED;
    const float d = m2 - l * l;
    const float spread = d > 0.0f ? d : 0.0f;
    const float var = spread / (nf - 1.0f);
    const float mean = l > 0.0f ? l : 0.0f;
    const float e = std::sqrt(var) / (mean + floor);
    return (std::isfinite(e) && e < AD_UNMEASURED) ? e : AD_UNMEASURED;
}

Decision ad_decide(uint32_t width, uint32_t height, const uint32_t* counts, const float* sums, size_t stride,
                   const float* lum2, float floor, float target, uint32_t cap, std::vector<uint8_t>& active) {  // adaptive.rs:132
    const size_t w = width, h = height;
    const size_t cols = (width + AD_BLOCK - 1) / AD_BLOCK, rows = (height + AD_BLOCK - 1) / AD_BLOCK;
    const size_t blocks = cols * rows;
    auto block_of = [&](size_t x, size_t y) { return (y / AD_BLOCK) * cols + x / AD_BLOCK; };
    std::vector<float> error(w * h);
    for (size_t y = 0; y < h; ++y)
        for (size_t x = 0; x < w; ++x) {
            const size_t p = y * w + x, i = p * stride;
            error[p] = ad_pixel_error(sums[i], sums[i + 1], sums[i + 2], lum2[p], counts[block_of(x, y)], floor);
        }
    std::vector<float> block_error(blocks, 0.0f);
    for (size_t y = 0; y < h; ++y) {
        const size_t y0 = y ? y - 1 : 0, y1 = std::min(y + 2, h);
        for (size_t x = 0; x < w; ++x) {
            const size_t x0 = x ? x - 1 : 0, x1 = std::min(x + 2, w);
            float sum = 0.0f;
            for (size_t ny = y0; ny < y1; ++ny)
                for (size_t nx = x0; nx < x1; ++nx) sum += error[ny * w + nx];
            const float s = sum / (float)((y1 - y0) * (x1 - x0));
            const size_t b = block_of(x, y);
            if (s > block_error[b]) block_error[b] = s;
        }
    }
    const float floor_target = target > 0.0f ? target : 0.0f;
    auto candidate = [&](size_t b) { return block_error[b] > floor_target && (cap == 0 || counts[b] < cap); };
    std::vector<float> errors;
    for (size_t b = 0; b < blocks; ++b)
        if (candidate(b)) errors.push_back(block_error[b]);
    Decision d;
    d.blocks = (uint32_t)blocks;
    for (float e : block_error)
        if (e > d.max_error) d.max_error = e;
    if (floor_target > 0.0f) {
        for (size_t b = 0; b < blocks; ++b) {
            if (!candidate(b)) continue;
            const float ratio = block_error[b] / floor_target;
            const float n = (float)counts[b];
            float need = n * (ratio * ratio - 1.0f);
            if (cap > 0) {
                const float room = (float)(cap - counts[b]);
                if (need > room) need = room;
            }
            const size_t bx = b % cols, by = b / cols;
            const size_t bw = std::min<size_t>(w - bx * AD_BLOCK, AD_BLOCK), bh = std::min<size_t>(h - by * AD_BLOCK, AD_BLOCK);
            d.remaining += need * (float)(bw * bh);
        }
    }
    active.assign(blocks, 0);
    if (errors.empty()) return d;
    // The 50 % quantile of the candidates' errors (all finite and positive: one value whatever the
    // sort).
    const size_t mid = (errors.size() - 1) / 2;
    std::nth_element(errors.begin(), errors.begin() + mid, errors.end());
    d.threshold = errors[mid];
    uint32_t count = 0, least = UINT32_MAX;
    for (size_t b = 0; b < blocks; ++b)
        if (candidate(b) && block_error[b] >= d.threshold) {
            active[b] = 1;
            ++count;
            least = std::min(least, counts[b]);
        }
    const uint32_t factor = std::min(std::max((uint32_t)blocks / (4 * count), 1u), AD_MAX_FACTOR);
    d.round = std::min(AD_ROUND * factor, std::max(least, AD_ROUND));
    d.active = count;
    return d;
}

Adaptive::Adaptive(uint32_t w, uint32_t h, float exposure_ev, float noise_threshold, uint32_t c)  // adaptive.rs:349
    : width(w), height(h), cols((w + AD_BLOCK - 1) / AD_BLOCK), rows((h + AD_BLOCK - 1) / AD_BLOCK), cap(c) {
    counts.assign((size_t)cols * rows, 0);
    active.assign((size_t)cols * rows, 1);
    round = cap > 0 ? std::min(AD_WARMUP, cap) : AD_WARMUP;
    target = noise_threshold > 0.0f ? noise_threshold : 0.0f;  // f32::max(x, 0) (NaN gives 0)
    floor = ad_floor_for(exposure_ev);
}

uint32_t Adaptive::quota(size_t b) const {  // adaptive.rs:409
    if (!active[b]) return 0;
    if (cap > 0) return std::min(round, cap > counts[b] ? cap - counts[b] : 0u);
    return round;
}

uint32_t Adaptive::samples_of(size_t b) const { return counts[b] + std::min(quota(b), done); }

void Adaptive::min_max(uint32_t& lo, uint32_t& hi) const {  // adaptive.rs:426
    lo = UINT32_MAX;
    hi = 0;
    for (size_t b = 0; b < counts.size(); ++b) {
        const uint32_t n = samples_of(b);
        lo = std::min(lo, n);
        hi = std::max(hi, n);
    }
    if (lo == UINT32_MAX) lo = hi = 0;
}

void Adaptive::work(uint32_t tx, uint32_t ty, uint32_t tw, uint32_t th, uint32_t count, std::vector<BlockWork>& out) const {  // adaptive.rs:471
    out.clear();
    const uint32_t x_end = (uint32_t)std::min<uint64_t>((uint64_t)tx + tw, width);
    const uint32_t y_end = (uint32_t)std::min<uint64_t>((uint64_t)ty + th, height);
    if (tx >= x_end || ty >= y_end || count == 0) return;
    for (uint32_t by = ty / AD_BLOCK; by <= (y_end - 1) / AD_BLOCK; ++by)
        for (uint32_t bx = tx / AD_BLOCK; bx <= (x_end - 1) / AD_BLOCK; ++bx) {
            const size_t b = (size_t)by * cols + bx;
            const uint32_t q = quota(b);
            if (q <= done) continue;
            const uint32_t x0 = std::max(bx * AD_BLOCK, tx), y0 = std::max(by * AD_BLOCK, ty);
            const uint32_t x1 = std::min((bx + 1) * AD_BLOCK, x_end), y1 = std::min((by + 1) * AD_BLOCK, y_end);
            out.push_back(BlockWork{x0, y0, x1 - x0, y1 - y0, counts[b] + done, std::min(q - done, count)});
        }
}

void Adaptive::advance(uint32_t count) { done = std::min(done + count, round); }  // adaptive.rs:502

Decision Adaptive::decide(const float* sums, size_t stride, const float* lum2) {  // adaptive.rs:513
    for (size_t b = 0; b < counts.size(); ++b) counts[b] += quota(b);
    iteration += round;
    done = 0;
    const Decision d = ad_decide(width, height, counts.data(), sums, stride, lum2, floor, target, cap, active);
    round = d.round;
    last = d;
    decided = true;
    return d;
}

}  // namespace orc

using namespace orc;

extern "C" {

// rt_adaptive_decide (rt-wasm/src/ffi.rs:237, lib.rs:660): the decision of a width x height image
// from its block counts, RGBA sums (4 floats per pixel) and squared-luminance sums. Writes one byte
// per block and six words (round, active, blocks, then the bits of threshold, max_error and
// remaining). 0, 2 for an empty image, 3 for a null pointer.
uint32_t orc_adaptive_decide(uint32_t width, uint32_t height, float ev, float target, uint32_t cap, const uint32_t* counts,
                             const float* sums, const float* lum2, uint8_t* active, uint32_t* words6) {
    if (!counts || !sums || !lum2 || !active || !words6) return 3;
    if (width == 0 || height == 0) return 2;
    std::vector<uint8_t> act;
    const Decision d = ad_decide(width, height, counts, sums, 4, lum2, ad_floor_for(ev), target, cap, act);
    std::memcpy(active, act.data(), act.size());
    words6[0] = d.round;
    words6[1] = d.active;
    words6[2] = d.blocks;
    std::memcpy(&words6[3], &d.threshold, 4);
    std::memcpy(&words6[4], &d.max_error, 4);
    std::memcpy(&words6[5], &d.remaining, 4);
    return 0;
}

float orc_pixel_error(float r, float g, float b, float lum2, uint32_t n, float floor) {
    return ad_pixel_error(r, g, b, lum2, n, floor);
}

}  // extern "C"
