// Progressive render with its path state in a fixed device array: the allocation-free variant of
// the wavefront render behind rtg_render_progressive_noalloc.
//
// The ordinary entry point sizes its path buffers to the wave with cudaMalloc (160-odd bytes per
// path, up to 16 Mi paths). Callers that cannot allocate device memory at render time -- a host
// whose device memory is all handed to its own pool allocator, or a render server that must not
// meet an out-of-memory error in the middle of a frame -- use this variant instead. It runs the
// same kernels in the same order; only the path buffers differ, so the film receives the same bits.
//
// The array is RTG_NOALLOC_SCRATCH_BYTES (12 MiB) of device memory in this file's module. Every
// GPU that loads the module holds it until the process exits, whether or not this variant is
// called. It holds one wave of at most RTG_NOALLOC_MAX_PATHS (65,536) paths.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "../../include/repackshot_b200.h"
#include "rtg_kernels.h"
#include "rtg_noalloc.h"

namespace rtg {
namespace {

// Bytes per path of the structure-of-arrays state (PathBuffers): o, d, thr, sum, sel, hit, sh_o,
// sh_d, sh_c (16 each), flags, medium, queue[0], queue[1], sorted, key (4 each); then the
// first-hit albedo of each path (16), which a film with fused guides adds to its guide sums.
constexpr size_t kBytesPerPath = 10 * 16 + 6 * 4;
constexpr size_t kPaths = RTG_NOALLOC_MAX_PATHS;
constexpr size_t kBinsBytes = 512 * 4;
constexpr size_t kCountersBytes = 64;  // [0], [1] queue lengths, [2] shadow queue, [3] error bits
constexpr size_t kRaysBytes = 64;      // [0] camera + extension rays, [1] shadow rays
constexpr size_t kLayoutBytes = kPaths * kBytesPerPath + kBinsBytes + kCountersBytes + kRaysBytes;
static_assert(kPaths % 64 == 0, "every array must keep 256-byte alignment");
static_assert(kLayoutBytes <= RTG_NOALLOC_SCRATCH_BYTES, "the fixed array must hold one full wave");

static __device__ __align__(256) unsigned char g_path_scratch[RTG_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
void* g_scratch_ptr[kMaxDevices] = {};  // the array's address on each device, once looked up

// Carves one wave's path buffers out of the array, in the order of PathBuffers; *albedo gets the
// per-path albedo slice after them.
PathBuffers carve(void* base, float4** albedo) {
    unsigned char* p = static_cast<unsigned char*>(base);
    auto take = [&](size_t each) { unsigned char* r = p; p += kPaths * each; return r; };
    PathBuffers P{};
    P.o = (float4*)take(16);
    P.d = (float4*)take(16);
    P.thr = (float4*)take(16);
    P.sum = (float4*)take(16);
    P.sel = (float4*)take(16);
    P.flags = (uint32_t*)take(4);
    P.medium = (uint32_t*)take(4);
    P.hit = (uint4*)take(16);
    P.queue[0] = (uint32_t*)take(4);
    P.queue[1] = (uint32_t*)take(4);
    P.sorted = (uint32_t*)take(4);
    P.key = (uint32_t*)take(4);
    P.bins = (uint32_t*)p;
    p += kBinsBytes;
    P.sh_o = (float4*)take(16);
    P.sh_d = (float4*)take(16);
    P.sh_c = (float4*)take(16);
    P.counters = (uint32_t*)p;
    p += kCountersBytes;
    P.rays = (unsigned long long*)p;
    p += kRaysBytes;
    *albedo = (float4*)take(16);
    return P;
}

int grid_for(uint32_t n, int per_block, int sms) {
    long g = ((long)n + per_block - 1) / per_block;
    long cap = (long)sms * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

}  // namespace

uint32_t noalloc_scratch(void** out, const char** why) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { *why = cudaGetErrorString(e); return RTG_STATUS_CUDA_ERROR; }
    if (dev < 0 || dev >= kMaxDevices) { *why = "device index beyond the 64 this library tracks"; return RTG_STATUS_CUDA_ERROR; }
    // A cached address is checked against the device's mappings: after cudaDeviceReset the array
    // is loaded again, possibly elsewhere, and the lookup is redone.
    if (g_scratch_ptr[dev]) {
        cudaPointerAttributes a{};
        if (cudaPointerGetAttributes(&a, g_scratch_ptr[dev]) != cudaSuccess || a.type != cudaMemoryTypeDevice || a.device != dev) {
            cudaGetLastError();
            g_scratch_ptr[dev] = nullptr;
        }
    }
    if (!g_scratch_ptr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress((void**)&ptr, g_path_scratch);
        if (e != cudaSuccess || !ptr) { *why = cudaGetErrorString(e); return RTG_STATUS_CUDA_ERROR; }
        g_scratch_ptr[dev] = ptr;
    }
    *out = g_scratch_ptr[dev];
    return RTG_STATUS_OK;
}

uint32_t noalloc_render(const NoallocJob& job, NoallocResult& res, const char** why) {
    res = NoallocResult{};
    const uint64_t x_end = job.film.ox + (uint64_t)job.film.w < job.width ? job.film.ox + (uint64_t)job.film.w : job.width;
    const uint64_t y_end = job.film.oy + (uint64_t)job.film.h < job.height ? job.film.oy + (uint64_t)job.film.h : job.height;
    if (job.film.ox >= x_end || job.film.oy >= y_end || job.count == 0) return RTG_STATUS_OK;
    const uint32_t cw = (uint32_t)(x_end - job.film.ox), ch = (uint32_t)(y_end - job.film.oy);
    if (cw > kPaths) {
        *why = "film wider than RTG_NOALLOC_MAX_PATHS (65536) pixels: one row does not fit the fixed path array";
        return RTG_STATUS_BAD_FILM;
    }
    void* base = nullptr;
    uint32_t st = noalloc_scratch(&base, why);
    if (st) return st;
    float4* albedo = nullptr;
    const PathBuffers P = carve(base, &albedo);
    // Rows per band so that one band of one sample fits the array, then samples per wave.
    const uint64_t npix = (uint64_t)cw * ch;
    const uint32_t band_rows = npix > kPaths ? (uint32_t)(kPaths / cw) : ch;
    for (uint32_t by = 0; by < ch; by += band_rows) {
        const uint32_t bh = band_rows < ch - by ? band_rows : ch - by;
        const uint64_t bpix = (uint64_t)cw * bh;
        uint64_t per = kPaths / bpix;
        if (per > job.count) per = job.count;
        const uint32_t per_wave = (uint32_t)per;
        // The counters and ray counts are the only part of the array that must start at zero;
        // the camera kernel writes every path slot of a wave before anything reads it.
        cudaError_t e = cudaMemsetAsync(P.counters, 0, kCountersBytes + kRaysBytes, job.stream);
        if (e != cudaSuccess) { *why = cudaGetErrorString(e); return RTG_STATUS_CUDA_ERROR; }
        for (uint32_t s = 0; s < job.count; s += per_wave) {
            const uint32_t ns = per_wave < job.count - s ? per_wave : job.count - s;
            WaveDesc wd{job.film.ox, job.film.oy + by, cw, bh, job.first + s, (uint32_t)(bpix * ns), nullptr};
            if (job.guide_sum) {  // fused guides: every wave's first hits add their albedo too
                wd.alb = albedo;
                wd.guide_sum = job.guide_sum;
                wd.guide_weight = job.guide_weight;
            }
            launch_wave(*job.S, job.lights, wd, P, &job.film, job.stream, grid_for(wd.n, 128, job.sms), nullptr);
            e = cudaGetLastError();
            if (e != cudaSuccess) { *why = cudaGetErrorString(e); return RTG_STATUS_CUDA_ERROR; }
            res.waves += 1;
        }
        uint32_t counters[4];
        unsigned long long rays[2];
        e = cudaMemcpyAsync(counters, P.counters, sizeof(counters), cudaMemcpyDeviceToHost, job.stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(rays, P.rays, sizeof(rays), cudaMemcpyDeviceToHost, job.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(job.stream);
        if (e != cudaSuccess) { *why = cudaGetErrorString(e); return RTG_STATUS_CUDA_ERROR; }
        if (counters[3] & 1u) { *why = "traversal stack overflow"; return RTG_STATUS_STACK_OVERFLOW; }
        res.extend_rays += rays[0];
        res.shadow_rays += rays[1];
    }
    return RTG_STATUS_OK;
}

}  // namespace rtg
