// Launch interface of the wavefront kernels (rtg_kernels.cu), used by the C-ABI engine.
#pragma once
#include <cuda_runtime.h>

#include "rtg_dev.h"

namespace rtg {

struct JobDev;

// Rounds of a wave: one per vertex up to the depth, plus, when a material is a cut-out, one per
// cut-out a path may pass (at most 64; a pass is no vertex).
inline uint32_t wave_rounds(const SceneDev& S) { return S.max_depth + 1u + (S.any_cutout ? 64u : 0u); }

// The edge mask of an image (pixel_filter.rs:175, the same for any tile cut): one byte per pixel,
// 1 where a neighbour's centre ray sees another part, material or depth. `exact` is scratch of
// w h uint4. Returns the launch status.
cudaError_t launch_edge_mask(const SceneDev& S, const LightsDev* L, uint4* exact, uint8_t* mask, cudaStream_t st, int grid);
// The packed (x | y << 16) edge pixels of the rectangle (x0, y0, w, h) of a mask, in any order;
// their count in *count (device).
// The exact passes (normal, depth, part and material ids) of a rectangle's centre rays, and the
// albedo of a range of its samples added to sums (passes.rs, render.rs:515-640).
cudaError_t launch_exact_passes(const SceneDev& S, const LightsDev* L, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h, float* normal,
                                float* depth, uint32_t* part, uint32_t* material, cudaStream_t st, int grid);
cudaError_t launch_albedo_pass(const SceneDev& S, const LightsDev* L, const uint8_t* edge, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                               uint32_t first, uint32_t count, float* sum, float* weight, float* alpha, cudaStream_t st, int grid);
cudaError_t launch_edge_list(const uint8_t* mask, uint32_t stride, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h, uint32_t* list,
                             uint32_t* count, cudaStream_t st, int grid);

// A segment of a batched wave: samples [first, first + ns) of the full-width rows [y0, y0 + h) of
// one job's image. Its slots start at slot_begin (sample-major, then row-major pixels); its pixels
// start at pix_begin in the wave's accumulation order.
struct SegDev {
    uint32_t job, y0, w, h, first, ns, slot_begin, pix_begin;
};

// A wave of path slots: either the pixels of the rectangle (x0, y0, w, h) for the sample
// indices first .. first + n / (w h) - 1 (slot = s * w * h + row-major pixel), or, when `xys` is
// set, the explicit (x, y, sample index) triples of a device array, or, when `segs` is set, the
// segments of a batched wave (nseg of them, sorted by slot_begin; npix pixels in all), whose jobs
// are `jobs`.
struct WaveDesc {
    uint32_t x0, y0, w, h, first, n;
    const uint32_t* xys;
    const SegDev* segs;
    const JobDev* jobs;
    uint32_t nseg, npix;
    // A list wave when `epix` is set: the k = `ek` samples of each sample index of `ne` listed
    // pixels (packed x | y << 16): slot ((s ne) + e) k + j holds sample index (b + first + s) k + j
    // of pixel e, b = ebase[e] (0 without `ebase`). Edge pixels (render.rs:477, E11) take ek > 1;
    // the pixels of an adaptive pass (adaptive.rs:471, E10) carry their block's first index in b.
    const uint32_t* epix;
    uint32_t ne, ek;
    const uint32_t* ebase;
    // A rectangle wave of a scene with edge samples: the image's edge mask (row stride
    // `edge_stride`); its pixels splat from the edge waves, not from this one.
    const uint8_t* edge;
    uint32_t edge_stride;
    // Guides taken from the wave itself (the film's albedo pass, passes.rs:209): when `alb` is set
    // (one float4 a path slot), the albedo of each camera ray's first hit is read from the first
    // extend, and after the film's accumulate each pixel adds its samples' albedo (an edge pixel
    // the mean of its k) to `guide_sum` (3 a film pixel) with `guide_weight` += 1, in sample order.
    float4* alb;
    float* guide_sum;
    float* guide_weight;
};

// Structure-of-arrays path state of one wave (device pointers).
struct PathBuffers {
    float4* o;       // origin, w: distance since the last scattering vertex (straight events)
    float4* d;       // direction, w: density of the BSDF sample that produced it
    float4* thr;     // throughput, w: alpha
    float4* sum;     // radiance
    float4* sel;     // point of the light selection the MIS weights use
    uint32_t* flags;
    uint32_t* medium;
    uint4* hit;
    uint32_t* queue[2];
    uint32_t* sorted;    // the active queue ordered by material key (shade reads it)
    uint32_t* key;       // per slot: material of the hit (n_materials: floor or miss)
    uint32_t* bins;      // [0, 256) key histogram, [256, 512) scatter cursors
    float4* sh_o;    // shadow rays: origin, w: t_max
    float4* sh_d;
    float4* sh_c;    // contribution, w: slot
    uint32_t* counters;  // [0], [1] queue lengths, [2] shadow queue length, [3] error bits
    unsigned long long* rays;
    // Coherence sort of the rays before each traversal (RaySort); all null: off.
    uint32_t* rbins;   // extension rays: [0, nk) key histogram, [nk, 2 nk) cursors
    uint32_t* sbins;   // shadow rays: the same
    uint32_t* sh_key;  // per shadow ray: its coherence key
};

// How a wave orders its work (the tunable half of the pipeline; none of it changes a film's bits).
// ray_bits > 0: before every traversal after the camera rays, the extension rays are ordered by a
// key of their direction's octant (3 bits) over the Morton code of their origin's cell on a grid of
// 2^ray_bits cells per axis over the scene's box (counting sort: histogram, prefix, scatter);
// shadow_sort: the shadow rays too (by their own origin and direction); material_sort: shade
// reads the paths ordered by the material they hit (otherwise in traversal order).
struct RaySort {
    uint32_t ray_bits = 0, shadow_sort = 0, material_sort = 1;
    float lo[3] = {0, 0, 0}, scale[3] = {0, 0, 0};  // cell = (p - lo) * scale per axis
    // l2_persist: the traversal kernels' launches mark the scene's traversal data (l2_base,
    // l2_bytes: nodes, leaf triangles, top-level leaves) as persisting in L2 for the fraction
    // l2_hit_ratio of it, so that the streamed path state does not evict it.
    uint32_t l2_persist = 0;
    const void* l2_base = nullptr;
    size_t l2_bytes = 0;
    float l2_hit_ratio = 0.0f;
    // tail_paths > 0: from round TAIL_FIRST_ROUND on, a round whose extension queue holds at most
    // tail_paths paths and every later round run in one launch, a path per thread (k_tail).
    uint32_t tail_paths = 0;
};
constexpr uint32_t TAIL_FIRST_ROUND = 2;
constexpr uint32_t RAY_SORT_MAX_BITS = 5;
inline uint32_t ray_sort_keys(uint32_t bits) { return 8u << (3u * bits); }

struct FilmDev {
    uint32_t ox, oy, w, h;
    float* rgb;
    float* weight;
    float* alpha;
    float* lum2;
};

// A job of the batched render queue: its scene constants (camera, image, settings, and its own
// instances, materials and BSDFs; the tree pointers are the shared scene's), lights and film.
struct JobDev {
    SceneDev S;
    const LightsDev* lights;
    FilmDev film;
};

// What the adjoint replay (rtg_adjoint.cuh) reads besides the scene and the wave.
struct AdjointDev {
    // per material m and side s (0 outside, 1 inside), at [2 m + s]: BSDFs at base + h, base - h
    // (every channel), alpha + h, alpha - h
    const Bsdf* albedo_plus;
    const Bsdf* albedo_minus;
    const Bsdf* alpha_plus;
    const Bsdf* alpha_minus;
    float inv_2h_albedo, inv_2h_alpha;
    const float4* dpath;  // d loss / d (one path's radiance): per pixel of the wave's rectangle for
                          // samples before `split`, then per pixel for samples from `split` on
    uint32_t split;
    float* grads;         // per material base R, G, B, alpha (4 n_materials), then per light
    float* residual;      // [0] sum of |radiance left| at the paths' ends, [1] sum of |radiance|
    uint32_t n_materials, n_lights;
    // per path slot
    float4* rem;          // the path's radiance still to come
    uint32_t* pend;       // material of the BSDF sample taken at the last vertex, or ADJ_NONE
    float4* pend_albedo;  // its d f / f over base colour, per channel
    float4* pend_alpha;   // its d f / f over alpha, per channel
    // per shadow ray
    float4* sh_grad;      // the material gradient it adds when unblocked: base R, G, B, alpha
    uint32_t* sh_ids;     // material + 1 (0: none) | (light + 1) << 16 (0: environment)
};
constexpr uint32_t ADJ_NONE = 0xffffffffu;

// CUDA events bracketing every extend launch of a wave (optional).
struct WaveTiming {
    static constexpr int MAX_EVENTS = 512;
    cudaEvent_t ev[MAX_EVENTS];
    int ev_count = 0;
};

void set_sobol(const SobolTable& t, cudaStream_t s);
void launch_wave(const SceneDev& S, const LightsDev* L, const WaveDesc& w, const PathBuffers& P, const FilmDev* film, cudaStream_t st,
                 int grid, WaveTiming* timing, const RaySort& order = RaySort());
// Kernel launches of one launch_wave with a film (camera and accumulate included, guides not).
uint32_t wave_launches(const SceneDev& S, const RaySort& order, const PathBuffers& P, bool batch);
// The adjoint: loss and per-pixel path derivatives of a film against a target (w*h*3 floats on
// the device), then the backward wave: the replay of the wave that rendered the film.
void launch_adjoint_delta(const FilmDev& F, const float* target, float4* dpath, double* loss, const PathBuffers& P, uint32_t count, cudaStream_t st,
                          int grid);
void launch_adjoint_wave(const SceneDev& S, const LightsDev* L, const WaveDesc& w, const PathBuffers& P, const AdjointDev& A, cudaStream_t st,
                         int grid);
// Film::to_srgb8_tonemapped / to_srgb16_tonemapped into `out` (device, w*h*3 bytes or words).
void launch_film_encode(const FilmDev& F, float ev, uint32_t tonemap, uint32_t bits, void* out, cudaStream_t st, int grid);
void launch_trace_batch(const SceneDev& S, const float* rays, uint32_t n, uint32_t mode, uint32_t* out, uint32_t* counters,
                        cudaStream_t st, int grid);

}  // namespace rtg
