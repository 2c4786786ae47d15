// Host interface of rtg_noalloc.cu: the progressive render whose path state sits in a fixed
// device array instead of memory allocated per scene.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "rtg_kernels.h"

namespace rtg {

struct NoallocJob {
    const SceneDev* S;
    const LightsDev* lights;
    FilmDev film;
    uint32_t width, height;  // the image; the film's rectangle is clipped to it
    uint32_t first, count;   // samples first .. first + count - 1
    cudaStream_t stream;
    int sms;
    float* guide_sum = nullptr;     // a film with fused guides: its albedo sums (3 a pixel) ...
    float* guide_weight = nullptr;  // ... and weights, which every wave adds to; else null
};

struct NoallocResult {
    uint64_t waves = 0, extend_rays = 0, shadow_rays = 0;
};

// The fixed array's address on the current device; looked up on the first call per device.
uint32_t noalloc_scratch(void** out, const char** why);

// Renders the job's samples into its film and waits for them. On failure *why names the cause.
uint32_t noalloc_render(const NoallocJob& job, NoallocResult& res, const char** why);

}  // namespace rtg
