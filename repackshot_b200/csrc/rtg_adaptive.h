// Adaptive sampling (E10, engine/crates/rt-core/src/adaptive.rs:1-551): the image decides, at the
// end of every round, which 8 x 8 blocks of pixels get the next one and how many samples it has.
//
// On the device, the per-pixel part (steps 1-3: the relative error of every pixel's mean, its
// 3 x 3 smoothing and the largest per block) reads the film where it lies, one CTA per block with
// its 10 x 10 halo staged in shared memory; the host takes the per-block part (steps 4-5: the
// candidates, the median of their errors, the round's size), a few thousand floats, in the
// reference's order. An adaptive pass renders the pixels of its active blocks from two packed
// lists (plain pixels, and edge pixels that take k samples a sample index), expanded on the device
// from the host's list of blocks, each entry carrying its block's first sample index.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace rtg {

constexpr uint32_t AD_BLOCK = 8;          // adaptive.rs:47
constexpr uint32_t AD_WARMUP = 16;        // adaptive.rs:49
constexpr uint32_t AD_ROUND = 16;         // adaptive.rs:51
constexpr uint32_t AD_MAX_FACTOR = 16;    // adaptive.rs:53
constexpr float AD_EPSILON = 0.01f;       // adaptive.rs:56
constexpr float AD_UNMEASURED = 1.0e30f;  // adaptive.rs:59

struct AdDecision {  // adaptive.rs:65
    uint32_t round = 0, active = 0, blocks = 0;
    float threshold = 0, max_error = 0, remaining = 0;
};

// One active block of a pass: its index, its first sample index (the samples it had when the
// round began) and where its pixels start in the plain and in the edge list.
struct AdEntry {
    uint32_t block, base, off_plain, off_edge;
};

#ifdef __CUDACC__
#define RTG_AD_HD __host__ __device__ __forceinline__
#else
#define RTG_AD_HD inline
#endif
RTG_AD_HD uint32_t ad_cols(uint32_t width) { return (width + AD_BLOCK - 1) / AD_BLOCK; }
RTG_AD_HD uint32_t ad_rows(uint32_t height) { return (height + AD_BLOCK - 1) / AD_BLOCK; }

// The floor of the mean in the relative error for an exposure of `ev` stops (adaptive.rs:85).
float ad_floor_for(float ev);

// Steps 4 and 5 of adaptive.rs:132 from the block errors: the candidates, the threshold of the
// moment, the blocks of the next round (into `active`) and its size.
AdDecision ad_decide_blocks(uint32_t width, uint32_t height, const uint32_t* counts, const float* block_error, float target,
                            uint32_t cap, std::vector<uint8_t>& active);

// Steps 1-3 on the device: block_error[b] = the largest 3 x 3-smoothed relative error of block b's
// pixels, from the radiance sums (`stride` floats a pixel, red green blue first), the
// squared-luminance sums and the samples of every block.
cudaError_t launch_block_error(const float* sums, uint32_t stride, const float* lum2, const uint32_t* counts, uint32_t width,
                               uint32_t height, float floor, float* block_error, cudaStream_t st, int grid);
// Per block: its image pixels that are not edge pixels and those that are (counts2[2 b], [2 b + 1]);
// `edge` (one byte a pixel) may be null: no edge pixels.
cudaError_t launch_block_pixels(const uint8_t* edge, uint32_t width, uint32_t height, uint32_t* counts2, cudaStream_t st, int grid);
// The pixels of `n` entries into the plain and the edge list (packed x | y << 16, row-major within
// a block), each with its block's first sample index.
cudaError_t launch_block_expand(const AdEntry* entries, uint32_t n, const uint8_t* edge, uint32_t width, uint32_t height,
                                uint32_t* plain, uint32_t* plain_base, uint32_t* edges, uint32_t* edge_base, cudaStream_t st, int grid);

}  // namespace rtg
