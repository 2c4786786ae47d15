// Test infrastructure: the CPU restatement the CUDA path is checked against, never shipped.
//
// Adaptive sampling (engine/crates/rt-core/src/adaptive.rs:44-551): the per-pixel relative error
// of the mean, its 3 x 3 smoothing, the per-block maximum, the candidates, the threshold of the
// moment and the size of the next round (`decide`), and the round state (`Adaptive`).
#pragma once
#include <cstdint>
#include <vector>

namespace orc {

constexpr uint32_t AD_BLOCK = 8;          // adaptive.rs:47
constexpr uint32_t AD_WARMUP = 16;        // adaptive.rs:49
constexpr uint32_t AD_ROUND = 16;         // adaptive.rs:51
constexpr uint32_t AD_MAX_FACTOR = 16;    // adaptive.rs:53
constexpr float AD_EPSILON = 0.01f;       // adaptive.rs:56
constexpr float AD_UNMEASURED = 1.0e30f;  // adaptive.rs:59

struct Decision {  // adaptive.rs:65
    uint32_t round = 0, active = 0, blocks = 0;
    float threshold = 0, max_error = 0, remaining = 0;
};

float ad_floor_for(float ev);
float ad_pixel_error(float r, float g, float b, float lum2, uint32_t n, float floor);
Decision ad_decide(uint32_t width, uint32_t height, const uint32_t* counts, const float* sums, size_t stride,
                   const float* lum2, float floor, float target, uint32_t cap, std::vector<uint8_t>& active);

// One active block's share of a pass (adaptive.rs:304 BlockWork).
struct BlockWork {
    uint32_t x, y, w, h, first, count;
};

// The round state of an adaptive render (adaptive.rs:318-551).
struct Adaptive {
    uint32_t width = 0, height = 0, cols = 0, rows = 0;
    std::vector<uint32_t> counts;
    std::vector<uint8_t> active;
    uint32_t round = 0, done = 0, iteration = 0, cap = 0;
    float target = 0, floor = 0;
    bool decided = false;
    Decision last;

    Adaptive(uint32_t w, uint32_t h, float exposure_ev, float noise_threshold, uint32_t cap);
    uint32_t left() const { return round - done; }
    bool converged() const { return round == 0; }
    bool warming_up() const { return !decided; }
    uint32_t next_iteration() const { return iteration + done; }
    uint32_t quota(size_t b) const;
    uint32_t samples_of(size_t b) const;
    void min_max(uint32_t& lo, uint32_t& hi) const;
    // The work of a pass of `count` samples in the tile (tx, ty, tw, th).
    void work(uint32_t tx, uint32_t ty, uint32_t tw, uint32_t th, uint32_t count, std::vector<BlockWork>& out) const;
    void advance(uint32_t count);
    Decision decide(const float* sums, size_t stride, const float* lum2);
};

}  // namespace orc
