// The denoiser on the device (engine/crates/rt-post/src/denoise.rs): the edge-avoiding a-trous
// wavelet filter guided by the exact passes and each pixel's sample variance, bit-exact with the
// reference (every step in f32 in its order of operations; no FMA contraction).
//
// Each step of the reference's filter_band is one data-parallel kernel over the band's pixels:
// the guides (with the depth gradient), the albedo divisor, the illumination and its variance;
// the firefly clamp; the spatial variance where a pixel has too few samples; per level the 3 x 3
// Gaussian of the variance and the 5 x 5 dilated a-trous pass (which also writes the next level's
// luminance); and the albedo multiplied back. The one order dependence of the reference (a
// firefly takes the largest variance of its neighbours, the raster order's earlier ones already
// clamped) is resolved by Jacobi sweeps over the fireflies until nothing changes: the dependence
// runs from earlier to later pixels only, so the sweeps reach the sequential result.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace rtg {

// Where a band's input lies (device pointers; `width` x `rows` pixels, rows from the top).
struct DnSrc {
    const float* rgb;  // radiance sums, red green blue first, `rgb_stride` floats a pixel
    uint32_t rgb_stride;
    const float* alpha;  // coverage sums, `alpha_stride` floats a pixel
    uint32_t alpha_stride;
    const float* lum2;           // squared-luminance sums
    const float* albedo;         // albedo, 3 a pixel: the resolved pass, or sums when `albedo_weight` is set
    const float* albedo_weight;  // samples of each albedo sum (null: `albedo` is resolved)
    const float* normal;         // 3 a pixel
    const float* depth;
    const uint32_t* part;
    const uint32_t* material;
    const float* counts;  // each pixel's own samples (null: `samples` for all)
};

struct DnPreset {
    uint32_t levels, variance_radius;
};
inline DnPreset dn_preset(uint32_t id) { return id == 0 ? DnPreset{5, 3} : DnPreset{3, 1}; }  // denoise.rs:73-89
inline uint32_t dn_halo(DnPreset p) { return (2u << p.levels) + 8u; }                        // denoise.rs:96

// Device scratch bytes for a band of n pixels.
size_t dn_scratch_bytes(size_t n);
// Denoises the band: RGBA sums of all its pixels into `out` (device, 4 floats a pixel). `scratch`
// holds dn_scratch_bytes(width * rows) bytes. Returns the CUDA error, if any; `launches` counts
// the kernels launched.
cudaError_t denoise_band(const DnSrc& src, uint32_t width, uint32_t rows, uint32_t samples, DnPreset preset, void* scratch, float* out,
                         cudaStream_t st, int grid, uint64_t& launches);

// The sums of a film whose pixels have their own sample counts (`weight`) as sums of `samples`
// samples (adaptive.rs:260 rescale; rt-cli/src/lib.rs:104 denoise_film_at): RGBA interleaved and
// the squared-luminance sums. A pixel with `samples` samples keeps its bits.
cudaError_t launch_dn_rescale(const float* rgb, const float* alpha, const float* lum2, const float* weight, size_t n, uint32_t samples, float* rgba,
                              float* lum2_out, cudaStream_t st, int grid);

}  // namespace rtg
