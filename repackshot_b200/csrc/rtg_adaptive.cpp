// The per-block half of the adaptive decision on the host (engine/crates/rt-core/src/adaptive.rs:
// 184-253): a few thousand block errors, read in the reference's order and in f32, so that the
// threshold, the remaining work and the round's size have its bits.
#include <algorithm>

#include "rtg_adaptive.h"
#include "rtg_math.cuh"

namespace rtg {

float ad_floor_for(float ev) { return AD_EPSILON / fexp2(ev); }  // adaptive.rs:85, color.rs:146

AdDecision ad_decide_blocks(uint32_t width, uint32_t height, const uint32_t* counts, const float* block_error, float target,
                            uint32_t cap, std::vector<uint8_t>& active) {
    const size_t w = width, h = height, cols = ad_cols(width), blocks = cols * ad_rows(height);
    const float floor_target = target > 0.0f ? target : 0.0f;
    auto candidate = [&](size_t b) { return block_error[b] > floor_target && (cap == 0 || counts[b] < cap); };
    std::vector<float> errors;
    for (size_t b = 0; b < blocks; ++b)
        if (candidate(b)) errors.push_back(block_error[b]);
    AdDecision d;
    d.blocks = (uint32_t)blocks;
    for (size_t b = 0; b < blocks; ++b)
        if (block_error[b] > d.max_error) d.max_error = block_error[b];
    // What is still needed to reach the target, each block at most to the cap (adaptive.rs:198).
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
            d.remaining = d.remaining + need * (float)(bw * bh);
        }
    }
    active.assign(blocks, 0);
    if (errors.empty()) return d;
    // The 50 % quantile of the candidates' errors: positive and finite, so one value whatever the
    // order of equal ones.
    const size_t mid = (errors.size() - 1) / 2;
    std::nth_element(errors.begin(), errors.begin() + (ptrdiff_t)mid, errors.end());
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

}  // namespace rtg
