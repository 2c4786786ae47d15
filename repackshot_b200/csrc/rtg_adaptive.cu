// Adaptive sampling on the device (engine/crates/rt-core/src/adaptive.rs:93-183): the error of
// every pixel, its 3 x 3 smoothing and the largest per block, plus the expansion of a pass's
// active blocks into pixel lists. Compiled, as every kernel here, without contraction into FMA and
// with IEEE division and square root, so that each error has the reference's bits.
#include <cuda_runtime.h>

#include "rtg_adaptive.h"
#include "rtg_math.cuh"

namespace rtg {
namespace {

constexpr int HALO = AD_BLOCK + 2;

// The relative error of the mean of one pixel (adaptive.rs:93).
__device__ __forceinline__ float pixel_error(float r, float g, float b, float lum2, uint32_t n, float floor) {
    if (n < 2) return AD_UNMEASURED;
    const float nf = (float)n;
    const float inv = 1.0f / nf;
    const float l = 0.2126f * (r * inv) + 0.7152f * (g * inv) + 0.0722f * (b * inv);
    const float m2 = lum2 * inv;
    if (!(finitef(l) && finitef(m2))) return AD_UNMEASURED;
    const float d = m2 - l * l;
    const float spread = d > 0.0f ? d : 0.0f;
    const float var = spread / (nf - 1.0f);
    const float mean = l > 0.0f ? l : 0.0f;
    const float e = sqrt_(var) / (mean + floor);
    return (finitef(e) && e < AD_UNMEASURED) ? e : AD_UNMEASURED;
}

// One CTA of 64 threads per block (grid-stride over blocks): the errors of the block's 10 x 10
// neighbourhood into shared memory, then each pixel's 3 x 3 mean (clipped to the image, summed row
// by row as adaptive.rs:171 does) and the block's maximum. Every error is finite and not negative,
// so the maximum is that of the bit patterns as unsigned integers.
__global__ void __launch_bounds__(64) k_block_error(const float* __restrict__ sums, uint32_t stride, const float* __restrict__ lum2,
                                                    const uint32_t* __restrict__ counts, uint32_t width, uint32_t height, float floor,
                                                    float* __restrict__ block_error) {
    __shared__ float e[HALO][HALO];
    __shared__ uint32_t warp_max[2];
    const uint32_t cols = ad_cols(width), blocks = cols * ad_rows(height);
    const uint32_t t = threadIdx.x;
    for (uint32_t b = blockIdx.x; b < blocks; b += gridDim.x) {
        const int bx = (int)(b % cols) * (int)AD_BLOCK, by = (int)(b / cols) * (int)AD_BLOCK;
        for (uint32_t i = t; i < HALO * HALO; i += blockDim.x) {
            const int x = bx - 1 + (int)(i % HALO), y = by - 1 + (int)(i / HALO);
            float v = 0.0f;
            if (x >= 0 && y >= 0 && x < (int)width && y < (int)height) {
                const size_t p = (size_t)y * width + (size_t)x;
                const float* s = sums + p * stride;
                const uint32_t n = __ldg(&counts[(uint32_t)y / AD_BLOCK * cols + (uint32_t)x / AD_BLOCK]);
                v = pixel_error(__ldg(s), __ldg(s + 1), __ldg(s + 2), __ldg(&lum2[p]), n, floor);
            }
            e[i / HALO][i % HALO] = v;
        }
        __syncthreads();
        const int x = bx + (int)(t % AD_BLOCK), y = by + (int)(t / AD_BLOCK);
        uint32_t bits = 0;
        if (x < (int)width && y < (int)height) {
            const int y0 = y > 0 ? y - 1 : 0, y1 = y + 2 < (int)height ? y + 2 : (int)height;
            const int x0 = x > 0 ? x - 1 : 0, x1 = x + 2 < (int)width ? x + 2 : (int)width;
            float sum = 0.0f;
            for (int ny = y0; ny < y1; ++ny)
                for (int nx = x0; nx < x1; ++nx) sum = sum + e[ny - by + 1][nx - bx + 1];
            bits = __float_as_uint(sum / (float)((y1 - y0) * (x1 - x0)));
        }
        bits = __reduce_max_sync(0xffffffffu, bits);
        if ((t & 31) == 0) warp_max[t >> 5] = bits;
        __syncthreads();
        if (t == 0) block_error[b] = __uint_as_float(warp_max[0] > warp_max[1] ? warp_max[0] : warp_max[1]);
        __syncthreads();
    }
}

// Per block, its plain and its edge pixels inside the image.
__global__ void k_block_pixels(const uint8_t* __restrict__ edge, uint32_t width, uint32_t height, uint32_t* __restrict__ counts2) {
    const uint32_t cols = ad_cols(width), blocks = cols * ad_rows(height);
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < blocks; b += gridDim.x * blockDim.x) {
        const uint32_t bx = b % cols * AD_BLOCK, by = b / cols * AD_BLOCK;
        const uint32_t x1 = bx + AD_BLOCK < width ? bx + AD_BLOCK : width, y1 = by + AD_BLOCK < height ? by + AD_BLOCK : height;
        uint32_t plain = 0, edges = 0;
        for (uint32_t y = by; y < y1; ++y)
            for (uint32_t x = bx; x < x1; ++x) {
                if (edge && edge[(size_t)y * width + x]) ++edges;
                else ++plain;
            }
        counts2[2 * b] = plain;
        counts2[2 * b + 1] = edges;
    }
}

// One CTA of 64 threads per entry: thread t is pixel t of the block (row-major); a pixel's place
// in its list is the entry's offset plus the pixels of its kind before it in the block.
__global__ void __launch_bounds__(64) k_block_expand(const AdEntry* __restrict__ entries, uint32_t n, const uint8_t* __restrict__ edge,
                                                     uint32_t width, uint32_t height, uint32_t* __restrict__ plain,
                                                     uint32_t* __restrict__ plain_base, uint32_t* __restrict__ edges,
                                                     uint32_t* __restrict__ edge_base) {
    __shared__ uint32_t lower[2];  // the plain and the edge pixels of warp 0
    const uint32_t cols = ad_cols(width);
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const AdEntry en = entries[i];
        const uint32_t x = en.block % cols * AD_BLOCK + t % AD_BLOCK, y = en.block / cols * AD_BLOCK + t / AD_BLOCK;
        const bool inside = x < width && y < height;
        const bool is_edge = inside && edge && edge[(size_t)y * width + x];
        const bool is_plain = inside && !is_edge;
        const uint32_t pm = __ballot_sync(0xffffffffu, is_plain), em = __ballot_sync(0xffffffffu, is_edge);
        if (warp == 0 && lane == 0) {
            lower[0] = (uint32_t)__popc(pm);
            lower[1] = (uint32_t)__popc(em);
        }
        __syncthreads();
        const uint32_t below = (1u << lane) - 1u;
        const uint32_t packed = x | (y << 16);
        if (is_plain) {
            const uint32_t k = en.off_plain + (warp ? lower[0] : 0u) + (uint32_t)__popc(pm & below);
            plain[k] = packed;
            plain_base[k] = en.base;
        }
        if (is_edge) {
            const uint32_t k = en.off_edge + (warp ? lower[1] : 0u) + (uint32_t)__popc(em & below);
            edges[k] = packed;
            edge_base[k] = en.base;
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_block_error(const float* sums, uint32_t stride, const float* lum2, const uint32_t* counts, uint32_t width,
                               uint32_t height, float floor, float* block_error, cudaStream_t st, int grid) {
    k_block_error<<<grid, 64, 0, st>>>(sums, stride, lum2, counts, width, height, floor, block_error);
    return cudaGetLastError();
}

cudaError_t launch_block_pixels(const uint8_t* edge, uint32_t width, uint32_t height, uint32_t* counts2, cudaStream_t st, int grid) {
    k_block_pixels<<<grid, 128, 0, st>>>(edge, width, height, counts2);
    return cudaGetLastError();
}

cudaError_t launch_block_expand(const AdEntry* entries, uint32_t n, const uint8_t* edge, uint32_t width, uint32_t height,
                                uint32_t* plain, uint32_t* plain_base, uint32_t* edges, uint32_t* edge_base, cudaStream_t st, int grid) {
    k_block_expand<<<grid, 64, 0, st>>>(entries, n, edge, width, height, plain, plain_base, edges, edge_base);
    return cudaGetLastError();
}

}  // namespace rtg
