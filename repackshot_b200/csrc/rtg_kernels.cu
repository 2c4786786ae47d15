// The wavefront pipeline of the drop-in: camera generation, extend (nearest hit), shade
// (surface, emission, next-event estimation setup, BSDF sampling, roulette), shadow (any hit)
// and accumulate, over persistent grid-stride queues. One wave is a set of path slots; a slot
// is (pixel, sample index) and keeps its own radiance, so the film adds each pixel's samples in
// sample order (integrator/mod.rs:1140-1891, render.rs:388-497, image.rs:82-93).
#include <cuda_runtime.h>

#include "rtg_image.cuh"
#include "rtg_kernels.h"
#include "rtg_shade.cuh"

namespace rtg {

__constant__ SobolTable c_sobol;

// Threads per block of the traversal kernels (the stride of their shared stacks).
constexpr int TRACE_THREADS = 128;
// RTG_REFILL_MIN (build setting): idle lanes a k_extend warp waits for before it takes new rays
// (1: every step with an idle lane; a warp whose lanes are all idle always refills). A refill
// costs the whole warp a ballot, an atomic, a shuffle and two dependent loads, so taking rays for
// eight lanes at a time beats taking them one by one as rays end: on the 1080p product frame the
// extend time fell from 145 to 130 ms (4: 134 ms, 10: 130 ms, 12: 130 ms, 16: 133 ms).
#ifndef RTG_REFILL_MIN
#define RTG_REFILL_MIN 8
#endif
// RTG_SHADOW_REFILL_MIN (build setting): the same for k_shadow (frame 312 ms at 1, 308 at 8, 309
// at 4, 312 at 16).
#ifndef RTG_SHADOW_REFILL_MIN
#define RTG_SHADOW_REFILL_MIN 8
#endif
// RTG_TRACE_MIN_BLOCKS (build setting): blocks per SM the traversal kernels (k_extend, k_shadow)
// are compiled for (0: the compiler's choice of registers, 76). At 8 (64 registers, no spills in
// k_extend, 40 bytes in k_shadow) the 1080p product frame's extend time fell from 163 to 145 ms
// and the frame from 349 to 327 ms: more warps hide the node fetches. 7 and 9 blocks measured
// 337-338 ms, 10 blocks 350 ms.
#ifndef RTG_TRACE_MIN_BLOCKS
#define RTG_TRACE_MIN_BLOCKS 8
#endif
#if RTG_TRACE_MIN_BLOCKS > 0
#define RTG_TRACE_BOUNDS __launch_bounds__(TRACE_THREADS, RTG_TRACE_MIN_BLOCKS)
#else
#define RTG_TRACE_BOUNDS __launch_bounds__(TRACE_THREADS)
#endif
// Blocks of 128 threads per SM that the shade kernels are compiled for (their register cap:
// 65536 / (128 x this)); a build may set it (RTG_SHADE_MIN_BLOCKS) to compare occupancies.
#ifndef RTG_SHADE_MIN_BLOCKS
#define RTG_SHADE_MIN_BLOCKS 8
#endif

// Flags of a path slot.
constexpr uint32_t PF_HAS_PDF = 1, PF_PRIMARY = 2, PF_MEDIUM = 4;
// A panoramic camera's sample that sees nothing (scene/mod.rs:227): its ray has an empty interval
// (no hit, no floor) and its radiance is multiplied by its black weight when it reaches the film.
constexpr uint32_t PF_NOTHING = 8;
// The path's flags also hold the cut-outs it passed (bits 8-14, at most MAX_CUTOUTS) and its vertex
// count (bits 16-26): a cut-out pass is no vertex, so a path's bounce can fall behind the round.
constexpr uint32_t PF_CUT_SHIFT = 8, PF_CUT_MASK = 0x7fu << 8, PF_BOUNCE_SHIFT = 16, PF_BOUNCE_MASK = 0x7ffu << 16;
constexpr uint32_t MAX_CUTOUTS = 64;
// sampler.rs:127-135: the hashed dimension deciding whether vertex `bounce`'s ray passes its
// `crossing`-th cut-out.
RTG_D uint32_t cutout_dim(uint32_t bounce, uint32_t crossing) { return (1u << 20) + bounce * 64u + (crossing < 63u ? crossing : 63u); }

__device__ __forceinline__ void wave_slot(const WaveDesc& w, uint32_t slot, uint32_t& x, uint32_t& y, uint32_t& index) {
    if (w.epix) {
        const uint32_t j = slot % w.ek, r = slot / w.ek, s = r / w.ne, e = r - s * w.ne;
        const uint32_t packed = w.epix[e];
        x = packed & 0xffffu;
        y = packed >> 16;
        index = ((w.ebase ? __ldg(&w.ebase[e]) : 0u) + w.first + s) * w.ek + j;  // render.rs:376 sub_sample (wrapping)
        return;
    }
    if (w.xys) {
        x = w.xys[3 * slot];
        y = w.xys[3 * slot + 1];
        index = w.xys[3 * slot + 2];
        return;
    }
    uint32_t npix = w.w * w.h;
    uint32_t s = slot / npix, rem = slot - s * npix;
    y = w.y0 + rem / w.w;
    x = w.x0 + rem % w.w;
    index = w.first + s;
}

// The segment of a batched wave that holds `slot`: the last with slot_begin <= slot.
__device__ __forceinline__ uint32_t seg_of_slot(const WaveDesc& w, uint32_t slot) {
    uint32_t lo = 0, hi = w.nseg;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&w.segs[mid].slot_begin) <= slot) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Job, pixel and sample index of a slot of a batched wave.
__device__ __forceinline__ void batch_slot(const WaveDesc& w, uint32_t slot, uint32_t& job, uint32_t& x, uint32_t& y, uint32_t& index) {
    const SegDev& g = w.segs[seg_of_slot(w, slot)];
    uint32_t local = slot - g.slot_begin, npix = g.w * g.h;
    uint32_t s = local / npix, rem = local - s * npix;
    job = g.job;
    y = g.y0 + rem / g.w;
    x = rem % g.w;
    index = g.first + s;
}

__device__ __forceinline__ void add_clamped(float4& sum, Rgb c, bool indirect, float clamp) {  // integrator/mod.rs:855
    if (!(finitef(c.r) && finitef(c.g) && finitef(c.b))) return;
    float p = rmax(rmax(c.r, c.g), c.b);
    if (indirect && clamp > 0.0f && p > clamp) c = c * (clamp / p);
    sum.x = sum.x + c.r;
    sum.y = sum.y + c.g;
    sum.z = sum.z + c.b;
}

// ---- camera generation ---------------------------------------------------------------------------
// BATCH: the slots belong to the jobs of a batched wave, each with its own camera.
template <bool BATCH>
__global__ void k_camera(SceneDev S, WaveDesc w, PathBuffers P) {
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < w.n; slot += gridDim.x * blockDim.x) {
        uint32_t x, y, index;
        V3 o, d;
        bool sees;
        if constexpr (BATCH) {
            uint32_t job;
            batch_slot(w, slot, job, x, y, index);
            sees = camera_ray(w.jobs[job].S, c_sobol, x, y, index, o, d);
        } else {
            wave_slot(w, slot, x, y, index);
            sees = camera_ray(S, c_sobol, x, y, index, o, d);
        }
        P.o[slot] = make_float4(o.x, o.y, o.z, 0.0f);  // w: distance since the last scattering vertex
        P.d[slot] = make_float4(d.x, d.y, d.z, 0.0f);  // w: density of the BSDF sample
        P.thr[slot] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);  // w: alpha
        P.sum[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        P.flags[slot] = PF_PRIMARY | (sees ? 0u : PF_NOTHING);
        P.queue[0][slot] = slot;
    }
    if (blockIdx.x == 0) {
        for (uint32_t k = threadIdx.x; k < 512; k += blockDim.x) P.bins[k] = 0;
        if (threadIdx.x == 0) {
            P.counters[0] = w.n;
            P.counters[1] = 0;
            P.counters[2] = 0;
            P.counters[4] = 0;
            P.counters[5] = 0;
        }
    }
}

// Material key of a path's next vertex, for the material-sorted shade.
__device__ __forceinline__ uint32_t material_key(const SceneDev& S, bool got, uint32_t inst) {
    uint32_t k = got ? __ldg(&S.instances[inst].material) : S.n_materials;
    return k < 255u ? k : 255u;
}

// Adds one to bins[key] for every active lane, one atomic per distinct key of the warp.
__device__ __forceinline__ void warp_count(uint32_t* bins, uint32_t key) {
    uint32_t mask = __match_any_sync(__activemask(), key);
    if ((threadIdx.x & 31) == (uint32_t)(__ffs((int)mask) - 1)) atomicAdd(&bins[key], (uint32_t)__popc(mask));
}

// ---- ray order (RaySort): coherence keys, their prefix and the scatter ---------------------------------
// Cell of coordinate v on a grid of n cells from lo with `scale` cells per unit (NaN and below: 0).
__device__ __forceinline__ uint32_t sort_cell(float v, float lo, float scale, uint32_t n) {
    const float f = (v - lo) * scale;
    return f > 0.0f ? (uint32_t)fminf(f, (float)(n - 1u)) : 0u;
}
// The coherence key of a ray: the octant of d (3 bits) over the Morton code of o's cell.
__device__ __forceinline__ uint32_t ray_key(const RaySort& R, V3 o, V3 d) {
    const uint32_t n = 1u << R.ray_bits;
    const uint32_t cx = sort_cell(o.x, R.lo[0], R.scale[0], n), cy = sort_cell(o.y, R.lo[1], R.scale[1], n),
                   cz = sort_cell(o.z, R.lo[2], R.scale[2], n);
    uint32_t m = 0;
#pragma unroll
    for (uint32_t b = 0; b < RAY_SORT_MAX_BITS; ++b)
        m |= (((cx >> b) & 1u) << (3u * b)) | (((cy >> b) & 1u) << (3u * b + 1u)) | (((cz >> b) & 1u) << (3u * b + 2u));
    const uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
    return (oct << (3u * R.ray_bits)) | m;
}

// bins[nk, 2 nk) = exclusive prefix of the histogram bins[0, nk), which is cleared. One block of
// 1024 threads: each warp sums a contiguous chunk, the chunk sums are scanned, then each warp
// scans its chunk row by row (coalesced).
__global__ void __launch_bounds__(1024) k_key_scan(uint32_t* bins, uint32_t nk) {
    __shared__ uint32_t chunk[32];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t per = ((nk + 31u) / 32u + 31u) & ~31u;
    const uint32_t b0 = min(warp * per, nk), b1 = min(b0 + per, nk);
    uint32_t s = 0;
    for (uint32_t e = b0 + lane; e < b1; e += 32u) s += bins[e];
    s = __reduce_add_sync(0xffffffffu, s);
    if (lane == 0) chunk[warp] = s;
    __syncthreads();
    if (warp == 0) {
        const uint32_t v = chunk[lane];
        uint32_t x = v;
#pragma unroll
        for (uint32_t o = 1; o < 32u; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        chunk[lane] = x - v;
    }
    __syncthreads();
    uint32_t off = chunk[warp];
    for (uint32_t r = b0; r < b1; r += 32u) {
        const uint32_t e = r + lane;
        const uint32_t v = e < b1 ? bins[e] : 0u;
        uint32_t x = v;
#pragma unroll
        for (uint32_t o = 1; o < 32u; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (e < b1) {
            bins[nk + e] = off + x - v;
            bins[e] = 0u;
        }
        off += __shfl_sync(0xffffffffu, x, 31);
    }
}

// out = the *count items of `list` (null: 0, 1, 2, ...) ordered by keys[item] (any order within a
// key: every ray's result depends on its own item only).
__global__ void k_key_scatter(const uint32_t* __restrict__ list, const uint32_t* __restrict__ keys, uint32_t* cursors,
                              const uint32_t* count, uint32_t* out) {
    const uint32_t n = *(volatile const uint32_t*)count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t item = list ? list[i] : i;
        out[atomicAdd(&cursors[keys[item]], 1u)] = item;
    }
}

// ---- extend: nearest hit of every active path ------------------------------------------------------------
// Persistent warps over the active queue: a lane whose ray has finished takes the next queue entry
// (one atomic per warp on counters[4]) while the rest of the warp keeps traversing, so no lane idles
// until the slowest ray of its warp is done.
// `order`: the active queue in the order to trace it (P.queue[cur], or its ray-sorted copy).
__global__ void RTG_TRACE_BOUNDS k_extend(SceneDev S, PathBuffers P, int cur, const uint32_t* __restrict__ order) {
    __shared__ uint64_t s_stack[SHORT_STACK * TRACE_THREADS];
    uint64_t deep[STACK_CAP - SHORT_STACK];
    SplitStack stack{s_stack + threadIdx.x, deep, TRACE_THREADS};
    const uint32_t n = *(volatile uint32_t*)&P.counters[cur];
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t err = 0, slot = 0;
    bool busy = false, drained = false;
    Trav T;
    for (;;) {
        if (!drained) {
            const uint32_t idle = __ballot_sync(0xffffffffu, !busy);
            if (idle && (RTG_REFILL_MIN <= 1 || __popc(idle) >= RTG_REFILL_MIN || idle == 0xffffffffu)) {
                const int leader = __ffs((int)idle) - 1;
                uint32_t base = 0;
                if ((int)lane == leader) base = atomicAdd(&P.counters[4], (uint32_t)__popc(idle));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (base + (uint32_t)__popc(idle) >= n) drained = true;
                const uint32_t i = base + (uint32_t)__popc(idle & ((1u << lane) - 1u));
                if (!busy && i < n) {
                    slot = order[i];
                    const float4 o = P.o[slot], d = P.d[slot];
                    const uint32_t pf = P.flags[slot];
                    busy = !(pf & PF_NOTHING) && trav_init(S, T, v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), 1.0e-3f, f_inf(), (pf & PF_PRIMARY) != 0);
                    if (!busy) {
                        P.hit[slot] = make_uint4(0xffffffffu, 0xffffffffu, 0u, 0u);
                        const uint32_t key = material_key(S, false, 0);
                        P.key[slot] = key;
                        warp_count(P.bins, key);
                    }
                }
            }
        }
        if (!__any_sync(0xffffffffu, busy)) {
            if (drained) break;
            continue;
        }
        if (busy) {
            bool got = false;
            if (trav_step<false>(S, T, stack, &err, got)) {
                busy = false;
                P.hit[slot] = got ? make_uint4(T.best_i, T.best_tri, __float_as_uint(T.best_t), 1u)
                                  : make_uint4(0xffffffffu, 0xffffffffu, 0u, 0u);
                const uint32_t key = material_key(S, got, T.best_i);
                P.key[slot] = key;
                warp_count(P.bins, key);
            }
        }
    }
    if (err) atomicOr(&P.counters[3], err);
}

// Exclusive prefix of the key histogram into the scatter cursors; clears the histogram.
__global__ void k_scan(PathBuffers P) {
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int k = 0; k < 256; ++k) {
            uint32_t c = P.bins[k];
            P.bins[256 + k] = acc;
            P.bins[k] = 0;
            acc += c;
        }
    }
}

// The active queue `in` reordered by material key into `out` (the order inside a key does not
// matter: every path's result depends on its own slot only).
__global__ void k_scatter(PathBuffers P, int cur, const uint32_t* __restrict__ in, uint32_t* __restrict__ out) {
    uint32_t n = *(volatile uint32_t*)&P.counters[cur];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t slot = in[i];
        uint32_t key = P.key[slot];
        uint32_t mask = __match_any_sync(__activemask(), key);
        int leader = __ffs((int)mask) - 1;
        uint32_t base = 0;
        if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(&P.bins[256 + key], (uint32_t)__popc(mask));
        base = __shfl_sync(mask, base, leader);
        uint32_t rank = __popc(mask & ((1u << (threadIdx.x & 31)) - 1u));
        out[base + rank] = slot;
    }
}

// ---- shade: one vertex of every active path ----------------------------------------------------------
// One vertex of the path in `slot` with the scene constants S and lights L; xyi(x, y, index) gives
// the path's pixel and sample index (the sampler's key).
// With P.rbins set, each surviving path's next ray gets its coherence key (in P.key) and is counted
// in the histogram; with P.sbins set, each shadow ray likewise (in P.sh_key).
// With `tail` (the tail kernel), the shadow ray goes to *tail instead of the shadow queue and the
// surviving path to no queue. Returns whether the path goes on.
struct TailShadow {
    bool on;
    float4 o, d, c;
};
template <class XYI>
__device__ __forceinline__ bool shade_slot(const SceneDev& S, const LightsDev& L, const PathBuffers& P, const RaySort& R, uint32_t slot, int cur,
                                           XYI xyi, uint32_t& rays_local, uint32_t& shadow_local, TailShadow* tail = nullptr) {
    float4 o4 = P.o[slot], d4 = P.d[slot], thr4 = P.thr[slot], sum = P.sum[slot];
    uint32_t flags = P.flags[slot];
    const uint32_t bounce = (flags & PF_BOUNCE_MASK) >> PF_BOUNCE_SHIFT;
    uint4 hit = P.hit[slot];
    V3 ro = v3(o4.x, o4.y, o4.z), rd = v3(d4.x, d4.y, d4.z);
    float offset = o4.w, pdf = d4.w;
    bool has_pdf = (flags & PF_HAS_PDF) != 0, primary = (flags & PF_PRIMARY) != 0;
    Rgb thr = rgb(thr4.x, thr4.y, thr4.z);
    float alpha = thr4.w;
    rays_local += 1;
    float t_geometry = hit.w ? __uint_as_float(hit.z) : f_inf();
    // floor_t (integrator/mod.rs:493)
    float t_floor = f_inf();
    if ((S.floor_mode == 1) && rd.z != 0.0f && !(flags & PF_NOTHING)) {
        float t = (S.floor_z - ro.z) / rd.z;
        if (t > 1.0e-3f && t < f_inf()) t_floor = t;
    }
    float t_nearest = rmin(t_geometry, t_floor);
    if ((flags & PF_MEDIUM) && finitef(t_nearest)) {
        const DevMaterial& mm = S.materials[P.medium[slot]];
        thr = thr * rgb(fexp(-mm.sigma[0] * t_nearest), fexp(-mm.sigma[1] * t_nearest), fexp(-mm.sigma[2] * t_nearest));
    }
    float4 sel4 = P.sel[slot];
    Sel from;
    from.p = v3(sel4.x, sel4.y, sel4.z);
    from.by_flux = !(L.per_point && L.n_entries > 0);
    from.total = 0.0f;
    if (has_pdf && !from.by_flux) from = select_at(L, from.p);
    Rgb crossed = crossed_from(L, ro, rd, 1.0e-3f, t_nearest, has_pdf, pdf, from, offset);
    add_clamped(sum, thr * crossed, bounce >= 2, S.clamp_indirect);
    bool alive = false;
    do {
        if (t_nearest == f_inf()) {
            if (primary && S.background == 0) {
                Rgb seen = escaped(L, rd, false, 0.0f, from);
                Rgb c = thr * (S.exterior == 1.0f ? seen : seen * S.exterior);
                sum.x = sum.x + c.r; sum.y = sum.y + c.g; sum.z = sum.z + c.b;
            } else if (primary && (S.background == 1 || S.background == 3)) {
                uint32_t x, y, index;
                xyi(x, y, index);
                float su, sv;
                screen_of(S, c_sobol, x, y, index, su, sv);
                Rgb c = thr * backdrop(S, su, sv);
                sum.x = sum.x + c.r; sum.y = sum.y + c.g; sum.z = sum.z + c.b;
            } else if (primary && S.background == 2) {
                alpha = peak(crossed) > 0.0f ? 1.0f : 0.0f;
            } else {
                add_clamped(sum, thr * escaped(L, rd, has_pdf, pdf, from), bounce >= 2, S.clamp_indirect);
            }
            break;
        }
        V3 s_point, s_hit, s_normal, s_geom;
        bool s_inst = false, s_outside = true;
        uint32_t inst = 0;
        const DevInstance* I = nullptr;
        const DevMaterial* mat = nullptr;
        if (t_floor < t_geometry) {
            V3 pp = ro + rd * t_floor;
            V3 point = v3(pp.x, pp.y, S.floor_z);
            V3 nn = v3(0.0f, 0.0f, rd.z < 0.0f ? 1.0f : -1.0f);
            s_point = point; s_hit = point; s_normal = nn; s_geom = nn;
        } else {
            HitInfo h;
            uint4 idx;
            if (!hit_details(S, ro, rd, 1.0e-3f, f_inf(), hit.x, hit.y, __uint_as_float(hit.z), h, I, idx)) break;
            // bevel.rs:232 shading_point without a bevel
            V3 ng = h.geometric, nrm = h.normal;
            if (dot(nrm, ng) < 0.0f) nrm = -nrm;
            if (dot(nrm, rd) >= -1.0e-4f) nrm = ng;
            s_point = terminator_point(S, I, idx, h);
            s_hit = h.point;
            s_normal = nrm;
            s_geom = ng;
            s_inst = true;
            inst = hit.x;
            s_outside = h.outside;
            mat = S.materials + I->material;
            if (mat->kind == MATERIAL_EMISSIVE) {
                // A BSDF-sampled ray that finds a mesh light weighs it against the light's own
                // sample (integrator/mod.rs:1556); other emitters and camera rays weigh 1.
                if (h.front || !(I->flags & 1u)) {
                    const float wgt = has_pdf ? emitter_weight(L, I->emitter, pdf, from, offset + t_geometry, dot(ng, rd)) : 1.0f;
                    add_clamped(sum, thr * rgb(mat->emission[0], mat->emission[1], mat->emission[2]) * wgt, bounce >= 2, S.clamp_indirect);
                }
                break;
            }
            // A cut-out lets the ray through with probability 1 - opacity: no vertex, the same
            // direction, density and selection; the path goes back to the extension queue
            // (integrator/mod.rs:1571).
            const uint32_t cut = (flags & PF_CUT_MASK) >> PF_CUT_SHIFT;
            if (S.any_cutout && mat->opacity < 1.0f && cut < MAX_CUTOUTS) {
                uint32_t x, y, index;
                xyi(x, y, index);
                const float u = sample1(c_sobol, sample_key(S, x, y, index), index, cutout_dim(bounce, cut));
                flags = (flags & ~PF_CUT_MASK) | ((cut + 1u) << PF_CUT_SHIFT);
                if (u >= rmax(mat->opacity, 0.0f)) {
                    const V3 o2 = offset_origin(h.point, -ng);
                    offset += dot(o2 - ro, rd);
                    P.o[slot] = make_float4(o2.x, o2.y, o2.z, offset);
                    P.flags[slot] = flags;
                    alive = true;
                    break;
                }
            }
        }
        if (bounce >= S.max_depth) break;
        const Bsdf& b = S.bsdfs[mat ? 2 * I->material + (s_outside ? 0 : 1) : 2 * S.n_materials];
        // Prepared::frame (integrator/mod.rs:833)
        Frame fr = frame_from_normal(s_normal);
        if (s_inst && I->tangent_on) {
            V3 cands[2] = {cross(ld3(I->tan_axis), s_point - ld3(I->tan_centre)), ld3(I->tan_x)};
            for (int k = 0; k < 2; ++k) {
                V3 t = cands[k] - s_normal * dot(s_normal, cands[k]);
                if (len2(t) > 1.0e-12f) {
                    V3 xx = normalize(t);
                    fr.x = xx; fr.y = cross(s_normal, xx); fr.z = s_normal;
                    break;
                }
            }
        }
        V3 wo = to_local(fr, -rd);
        V3 ng = s_geom;
        V3 origin = offset_origin(s_point, ng);
        uint32_t dims = bounce_dim(bounce);
        uint32_t x, y, index;
        xyi(x, y, index);
        uint64_t key = sample_key(S, x, y, index);
        // Next-event estimation: one light; the shadow ray goes to the shadow queue.
        Sel selection = select_at(L, s_point);
        LightSample ls;
        if (sample_light(L, selection, sample1(c_sobol, key, index, dims + OFF_LIGHT_SELECT), sample1(c_sobol, key, index, dims + OFF_LIGHT),
                         sample1(c_sobol, key, index, dims + OFF_LIGHT + 1), ls)) {
            V3 wi = to_local(fr, ls.wi);
            Rgb f = bsdf_eval(S.energy, b, wo, wi, ls.glossy ? LOBES_ALL : LOBES_DIFFUSE);
            if (peak(f) > 0.0f) {
                V3 from_p = wi.z < 0.0f ? offset_origin(s_hit, -ng) : origin;
                float weight = (ls.delta || !ls.glossy) ? 1.0f : power_heuristic(ls.pdf, bsdf_pdf(S.energy, b, wo, wi));
                Rgb c = thr * f * ls.radiance * (absf(wi.z) * weight / ls.pdf);
                bool finite_c = finitef(c.r) && finitef(c.g) && finitef(c.b);
                // The clamp applies to what arrives: after the shadow walk when it may attenuate.
                const bool walk = ls.shadow && S.any_passable;
                if (finite_c && bounce >= 1 && S.clamp_indirect > 0.0f && !walk) {
                    float p = rmax(rmax(c.r, c.g), c.b);
                    if (p > S.clamp_indirect) c = c * (S.clamp_indirect / p);
                }
                if (!ls.shadow) {
                    if (finite_c) { sum.x = sum.x + c.r; sum.y = sum.y + c.g; sum.z = sum.z + c.b; }
                } else {
                    shadow_local += 1;
                    float tmax = finitef(ls.distance) ? ls.distance * (1.0f - 1.0e-4f) : f_inf();
                    bool floor_blocks = false;
                    if (S.floor_mode == 1 && ls.wi.z != 0.0f) {
                        float t = (S.floor_z - from_p.z) / ls.wi.z;
                        floor_blocks = t > 1.0e-3f && t < tmax;
                    }
                    if (finite_c && !floor_blocks) {
                        const float4 so = make_float4(from_p.x, from_p.y, from_p.z, tmax);
                        const float4 sd = make_float4(ls.wi.x, ls.wi.y, ls.wi.z, bounce >= 1 ? 1.0f : 0.0f);  // w: indirect
                        const float4 sc = make_float4(c.r, c.g, c.b, __uint_as_float(slot));
                        if (tail) {
                            tail->on = true;
                            tail->o = so;
                            tail->d = sd;
                            tail->c = sc;
                        } else {
                            uint32_t k = atomicAdd(&P.counters[2], 1u);
                            P.sh_o[k] = so;
                            P.sh_d[k] = sd;
                            P.sh_c[k] = sc;
                            if (P.sbins) {
                                const uint32_t sk = ray_key(R, from_p, ls.wi);
                                P.sh_key[k] = sk;
                                atomicAdd(&P.sbins[sk], 1u);
                            }
                        }
                    }
                }
            }
        }
        // The next direction.
        BsdfSample bs;
        if (!bsdf_sample(S.energy, b, wo, sample1(c_sobol, key, index, dims + OFF_BSDF), sample1(c_sobol, key, index, dims + OFF_BSDF + 1), bs))
            break;
        bool transmitted = bs.wi.z < 0.0f;
        V3 wi = bs.straight ? rd : normalize(to_world(fr, bs.wi));
        if (transmitted) {
            if (dot(wi, ng) >= 0.0f) break;
        } else if (dot(wi, ng) <= 0.0f) {
            break;
        }
        thr = thr * bs.weight;
        if (bounce >= 2) {
            float survive = rclamp(peak(thr), 0.05f, 1.0f);
            if (sample1(c_sobol, key, index, dims + OFF_ROULETTE) >= survive) break;
            thr = thr / survive;
        }
        float pk = peak(thr);
        if (!(pk > 0.0f && finitef(pk))) break;
        V3 next_origin = transmitted ? offset_origin(s_hit, -ng) : origin;
        if (bs.straight) {
            offset += dot(next_origin - ro, rd);
        } else {
            flags |= PF_HAS_PDF;
            flags &= ~PF_PRIMARY;
            pdf = bs.pdf;
            P.sel[slot] = make_float4(s_point.x, s_point.y, s_point.z, 0.0f);
            offset = 0.0f;
            if (transmitted) {
                if (s_outside && mat && mat->has_medium) {
                    flags |= PF_MEDIUM;
                    P.medium[slot] = I->material;
                } else {
                    flags &= ~PF_MEDIUM;
                }
            }
        }
        P.o[slot] = make_float4(next_origin.x, next_origin.y, next_origin.z, offset);
        P.d[slot] = make_float4(wi.x, wi.y, wi.z, pdf);
        P.flags[slot] = (flags & ~PF_BOUNCE_MASK) | ((bounce + 1u) << PF_BOUNCE_SHIFT);
        alive = true;
    } while (false);
    P.thr[slot] = make_float4(thr.r, thr.g, thr.b, alpha);
    P.sum[slot] = sum;
    if (alive && !tail) {
        uint32_t k = atomicAdd(&P.counters[cur ^ 1], 1u);
        P.queue[cur ^ 1][k] = slot;
        if (P.rbins) {
            const float4 no = P.o[slot], nd = P.d[slot];
            const uint32_t rk = ray_key(R, v3(no.x, no.y, no.z), v3(nd.x, nd.y, nd.z));
            P.key[slot] = rk;
            atomicAdd(&P.rbins[rk], 1u);
        }
    }
    return alive;
}

// BATCH: the slots belong to the jobs of a batched wave, each with its own constants and lights.
// Eight blocks per SM (64 registers, with some spills) beat the 128 registers the compiler would
// use on its own: the kernel waits on scattered hit-detail loads, and more warps hide them (1080p
// frame: 369 -> 383 Mpaths/s; 5, 6 and 7 blocks measured 367, 379 and 372).
// `order`: the active queue in the order to shade it (material-sorted, or as traced).
template <bool BATCH>
__global__ void __launch_bounds__(128, RTG_SHADE_MIN_BLOCKS) k_shade(SceneDev S, const LightsDev* __restrict__ Lg, PathBuffers P, int cur, WaveDesc w,
                                                  const uint32_t* __restrict__ order, RaySort R) {
    uint32_t n = *(volatile uint32_t*)&P.counters[cur];
    uint32_t rays_local = 0, shadow_local = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = order[i];
        if constexpr (BATCH) {
            uint32_t job, x, y, index;
            batch_slot(w, slot, job, x, y, index);
            const JobDev& J = w.jobs[job];
            shade_slot(J.S, *J.lights, P, R, slot, cur, [&](uint32_t& xx, uint32_t& yy, uint32_t& ii) { xx = x; yy = y; ii = index; },
                       rays_local, shadow_local);
        } else {
            shade_slot(S, *Lg, P, R, slot, cur, [&](uint32_t& xx, uint32_t& yy, uint32_t& ii) { wave_slot(w, slot, xx, yy, ii); },
                       rays_local, shadow_local);
        }
    }
    // Ray counts: camera + extension rays in rays[0], shadow rays in rays[1]; one atomic per warp.
    uint32_t total = __reduce_add_sync(0xffffffffu, rays_local);
    uint32_t shadows = __reduce_add_sync(0xffffffffu, shadow_local);
    if ((threadIdx.x & 31) == 0 && total) atomicAdd(P.rays, (unsigned long long)total);
    if ((threadIdx.x & 31) == 0 && shadows) atomicAdd(P.rays + 1, (unsigned long long)shadows);
}

// ---- shadow: any hit of every queued shadow ray; the unblocked add their light ----------------------------
// Persistent warps with lane refill, as k_extend (queue position counter: counters[5]).
__device__ __forceinline__ void shadow_unblocked(const PathBuffers& P, uint32_t i) {
    const float4 c = P.sh_c[i];
    const uint32_t slot = __float_as_uint(c.w);
    float4 s = P.sum[slot];
    s.x = s.x + c.x; s.y = s.y + c.y; s.z = s.z + c.z;
    P.sum[slot] = s;
}

// `perm` (may be null): the shadow queue in the order to trace it.
__global__ void RTG_TRACE_BOUNDS k_shadow(SceneDev S, PathBuffers P, const uint32_t* __restrict__ perm) {
    __shared__ uint64_t s_stack[SHORT_STACK * TRACE_THREADS];
    uint64_t deep[STACK_CAP - SHORT_STACK];
    SplitStack stack{s_stack + threadIdx.x, deep, TRACE_THREADS};
    const uint32_t n = *(volatile uint32_t*)&P.counters[2];
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t err = 0, ray = 0;
    bool busy = false, drained = false;
    Trav T;
    for (;;) {
        if (!drained) {
            const uint32_t idle = __ballot_sync(0xffffffffu, !busy);
            if (idle && (RTG_SHADOW_REFILL_MIN <= 1 || __popc(idle) >= RTG_SHADOW_REFILL_MIN || idle == 0xffffffffu)) {
                const int leader = __ffs((int)idle) - 1;
                uint32_t base = 0;
                if ((int)lane == leader) base = atomicAdd(&P.counters[5], (uint32_t)__popc(idle));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (base + (uint32_t)__popc(idle) >= n) drained = true;
                const uint32_t i = base + (uint32_t)__popc(idle & ((1u << lane) - 1u));
                if (!busy && i < n) {
                    ray = perm ? perm[i] : i;
                    const float4 o = P.sh_o[ray], d = P.sh_d[ray];
                    busy = trav_init(S, T, v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), 1.0e-3f, o.w, false);
                    if (!busy) shadow_unblocked(P, ray);
                }
            }
        }
        if (!__any_sync(0xffffffffu, busy)) {
            if (drained) break;
            continue;
        }
        if (busy) {
            bool blocked = false;
            if (trav_step<true>(S, T, stack, &err, blocked)) {
                busy = false;
                if (!blocked) shadow_unblocked(P, ray);
            }
        }
    }
    if (err) atomicOr(&P.counters[3], err);
}

// ---- the section view: k_extend and k_shadow through the section's queries (geometry/section.rs) -------
// One ray per thread: a query may be several traversals (the kept part, the cap's probe beyond the
// plane, the studio on the removed side), so the lane refill of the plain kernels does not apply.
// Launched instead of them for a scene with a section; they write the same records (a cap is a hit
// with triangle CAP_TRIANGLE).
__global__ void __launch_bounds__(TRACE_THREADS) k_extend_section(SceneDev S, PathBuffers P, int cur, const uint32_t* __restrict__ order) {
    __shared__ uint64_t s_stack[SHORT_STACK * TRACE_THREADS];
    uint64_t deep[STACK_CAP - SHORT_STACK];
    SplitStack stack{s_stack + threadIdx.x, deep, TRACE_THREADS};
    const uint32_t n = *(volatile uint32_t*)&P.counters[cur];
    uint32_t err = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = order[i];
        const float4 o = P.o[slot], d = P.d[slot];
        const uint32_t pf = P.flags[slot];
        TraceResult res;
        const bool got = !(pf & PF_NOTHING) &&
                         trace_q<false>(S, v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), 1.0e-3f, f_inf(), (pf & PF_PRIMARY) != 0, res, &err, stack);
        P.hit[slot] = got ? make_uint4(res.inst, res.tri, __float_as_uint(res.t), 1u) : make_uint4(0xffffffffu, 0xffffffffu, 0u, 0u);
        const uint32_t key = material_key(S, got, got ? res.inst : 0u);
        P.key[slot] = key;
        warp_count(P.bins, key);
    }
    if (err) atomicOr(&P.counters[3], err);
}

__global__ void __launch_bounds__(TRACE_THREADS) k_shadow_section(SceneDev S, PathBuffers P, const uint32_t* __restrict__ perm) {
    __shared__ uint64_t s_stack[SHORT_STACK * TRACE_THREADS];
    uint64_t deep[STACK_CAP - SHORT_STACK];
    SplitStack stack{s_stack + threadIdx.x, deep, TRACE_THREADS};
    const uint32_t n = *(volatile uint32_t*)&P.counters[2];
    uint32_t err = 0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint32_t ray = perm ? perm[j] : j;
        const float4 o = P.sh_o[ray], d = P.sh_d[ray];
        TraceResult unused;
        if (!trace_q<true>(S, v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), 1.0e-3f, o.w, false, unused, &err, stack)) shadow_unblocked(P, ray);
    }
    if (err) atomicOr(&P.counters[3], err);
}

// ---- shadow walk: shadow rays through cut-outs and thin walls (integrator/mod.rs:629-690) ------------
// Nearest hits along the ray: a passable surface multiplies what arrives by its straight
// transmittance (a thin wall's) times its opacity plus 1 - opacity, and the ray goes on from just
// behind it, up to 32 crossings; any other surface blocks it. One thread per ray: only scenes with
// passable instances run it, instead of k_shadow. BATCH: each ray's job gives its materials.
template <bool BATCH>
__global__ void __launch_bounds__(TRACE_THREADS) k_shadow_walk(SceneDev S, PathBuffers P, WaveDesc w, const uint32_t* __restrict__ perm) {
    __shared__ uint64_t s_stack[SHORT_STACK * TRACE_THREADS];
    uint64_t deep[STACK_CAP - SHORT_STACK];
    SplitStack stack{s_stack + threadIdx.x, deep, TRACE_THREADS};
    const uint32_t n = *(volatile uint32_t*)&P.counters[2];
    uint32_t err = 0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint32_t i = perm ? perm[j] : j;
        const float4 o4 = P.sh_o[i], d4 = P.sh_d[i], c4 = P.sh_c[i];
        const uint32_t slot = __float_as_uint(c4.w);
        const SceneDev* Sp = &S;
        if constexpr (BATCH) {
            uint32_t job, x, y, index;
            batch_slot(w, slot, job, x, y, index);
            Sp = &w.jobs[job].S;
        }
        const SceneDev& J = *Sp;
        const V3 d = v3(d4.x, d4.y, d4.z);
        const float t_max = o4.w;
        V3 o = v3(o4.x, o4.y, o4.z);
        float tmax = t_max, travelled = 0.0f;
        Rgb keep = splat(1.0f);
        bool arrives = false;
        for (uint32_t k = 0; k < 32; ++k) {  // MAX_SHADOW_CROSSINGS
            TraceResult res;
            if (!trace_q<false>(J, o, d, 1.0e-3f, tmax, false, res, &err, stack)) { arrives = true; break; }
            if (res.inst >= J.n_instances || !J.instances[res.inst].passable) break;
            HitInfo h;
            uint4 idx;
            const DevInstance* I = nullptr;
            if (!hit_details(J, o, d, 1.0e-3f, f_inf(), res.inst, res.tri, res.t, h, I, idx)) break;
            const uint32_t m = I->material;
            const float opacity = rclamp(J.materials[m].opacity, 0.0f, 1.0f);
            keep = keep * (straight_transmittance(J.bsdfs[2 * m], dot(h.geometric, d)) * opacity + splat(1.0f - opacity));
            if (rmax(rmax(keep.r, keep.g), keep.b) <= 0.0f) break;
            const V3 origin = offset_origin(h.point, -h.geometric);
            travelled += dot(origin - o, d);
            const float next = t_max - travelled;
            if (next != next || next <= 1.0e-3f) { arrives = true; break; }
            o = origin;
            tmax = next;
        }
        if (!(arrives && peak(keep) > 0.0f)) continue;
        Rgb c = rgb(c4.x, c4.y, c4.z) * keep;
        if (d4.w != 0.0f && J.clamp_indirect > 0.0f) {
            const float p = rmax(rmax(c.r, c.g), c.b);
            if (p > J.clamp_indirect) c = c * (J.clamp_indirect / p);
        }
        float4 s4 = P.sum[slot];
        s4.x = s4.x + c.r; s4.y = s4.y + c.g; s4.z = s4.z + c.b;
        P.sum[slot] = s4;
    }
    if (err) atomicOr(&P.counters[3], err);
}

// ---- tail: the last rounds of a wave, a path per thread -----------------------------------------------
// When the round's extension queue holds at most `limit` paths, each thread carries its share of
// them through the wave's remaining `rounds_left` rounds alone: the nearest hit (as k_extend), the
// vertex (shade_slot), the any hit of its shadow ray and its contribution (as k_shadow), the next
// ray; each path's arithmetic in the order the wavefront gives it, so its sum has the same bits.
// A wave whose last rounds hold few paths then pays one launch as long as its slowest path instead
// of a chain of launches, each as long as its slowest ray. k_tail_end then empties the queue, so
// the later rounds' launches find no work. Scenes with passable surfaces (shadow walks) and
// batched waves keep the wavefront.
__global__ void __launch_bounds__(TRACE_THREADS) k_tail(SceneDev S, const LightsDev* __restrict__ Lg, PathBuffers P, int cur, WaveDesc w, uint32_t rounds_left,
                                        uint32_t limit) {
    const uint32_t n = *(volatile uint32_t*)&P.counters[cur];
    if (n == 0 || n > limit) return;
    __shared__ uint64_t s_stack[SHORT_STACK * TRACE_THREADS];
    uint64_t deep[STACK_CAP - SHORT_STACK];
    SplitStack stack{s_stack + threadIdx.x, deep, TRACE_THREADS};
    const uint32_t* __restrict__ queue = P.queue[cur];
    const RaySort R;  // no coherence keys
    uint32_t err = 0, rays_local = 0, shadow_local = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = queue[i];
        for (uint32_t r = 0; r < rounds_left; ++r) {
            const float4 o = P.o[slot], d = P.d[slot];
            const uint32_t pf = P.flags[slot];
            TraceResult res;
            const bool got = !(pf & PF_NOTHING) &&
                             traverse<false>(S, v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), 1.0e-3f, f_inf(), (pf & PF_PRIMARY) != 0, res, &err, stack);
            P.hit[slot] = got ? make_uint4(res.inst, res.tri, __float_as_uint(res.t), 1u) : make_uint4(0xffffffffu, 0xffffffffu, 0u, 0u);
            TailShadow sh;
            sh.on = false;
            const bool alive = shade_slot(S, *Lg, P, R, slot, cur, [&](uint32_t& xx, uint32_t& yy, uint32_t& ii) { wave_slot(w, slot, xx, yy, ii); },
                                          rays_local, shadow_local, &sh);
            if (sh.on) {
                TraceResult unused;
                if (!traverse<true>(S, v3(sh.o.x, sh.o.y, sh.o.z), v3(sh.d.x, sh.d.y, sh.d.z), 1.0e-3f, sh.o.w, false, unused, &err, stack)) {
                    float4 sum = P.sum[slot];  // shadow_unblocked's addition
                    sum.x = sum.x + sh.c.x;
                    sum.y = sum.y + sh.c.y;
                    sum.z = sum.z + sh.c.z;
                    P.sum[slot] = sum;
                }
            }
            if (!alive) break;
        }
    }
    uint32_t total = __reduce_add_sync(0xffffffffu, rays_local);
    uint32_t shadows = __reduce_add_sync(0xffffffffu, shadow_local);
    if ((threadIdx.x & 31) == 0 && total) atomicAdd(P.rays, (unsigned long long)total);
    if ((threadIdx.x & 31) == 0 && shadows) atomicAdd(P.rays + 1, (unsigned long long)shadows);
    if (err) atomicOr(&P.counters[3], err);
}

// After k_tail: a queue it carried to the end is empty for the rest of the wave.
__global__ void k_tail_end(PathBuffers P, int cur, uint32_t limit) {
    const uint32_t n = P.counters[cur];
    if (n > 0 && n <= limit) P.counters[cur] = 0;
}

__global__ void k_next_round(PathBuffers P, int cur) {
    // The queue just consumed becomes the next round's output; the shadow queue empties; the
    // extend and shadow queue positions start again.
    P.counters[cur] = 0;
    P.counters[2] = 0;
    P.counters[4] = 0;
    P.counters[5] = 0;
}

// ---- accumulate: film += each pixel's samples in sample-index order (image.rs:82) -------------------------
// A sample's radiance times its camera weight (render.rs:465): white, or black for a panoramic
// camera's sample that sees nothing.
__device__ __forceinline__ float4 sample_sum(const PathBuffers& P, uint32_t slot) {
    const float4 c = P.sum[slot];
    if (!(P.flags[slot] & PF_NOTHING)) return c;
    return make_float4(c.x * 0.0f, c.y * 0.0f, c.z * 0.0f, c.w);
}
// Film pixel (x, y) += the ns samples in slots slot0, slot0 + stride, ..., in that order
// (Film::splat_alpha, image.rs:82).
__device__ __forceinline__ void accumulate_pixel(const FilmDev& F, uint32_t x, uint32_t y, const PathBuffers& P, uint32_t slot0, uint32_t stride,
                                                 uint32_t ns) {
    if (x < F.ox || y < F.oy || x - F.ox >= F.w || y - F.oy >= F.h) return;
    size_t fi = (size_t)(y - F.oy) * F.w + (x - F.ox);
    float r = F.rgb[3 * fi], g = F.rgb[3 * fi + 1], b = F.rgb[3 * fi + 2];
    float wt = F.weight[fi], al = F.alpha[fi], l2 = F.lum2[fi];
    for (uint32_t s = 0; s < ns; ++s) {
        uint32_t slot = slot0 + s * stride;
        float4 c = sample_sum(P, slot);
        r = r + c.x; g = g + c.y; b = b + c.z;
        wt = wt + 1.0f;
        al = al + P.thr[slot].w;
        float l = luminance(rgb(c.x, c.y, c.z));
        l2 = l2 + l * l;
    }
    F.rgb[3 * fi] = r; F.rgb[3 * fi + 1] = g; F.rgb[3 * fi + 2] = b;
    F.weight[fi] = wt; F.alpha[fi] = al; F.lum2[fi] = l2;
}

__global__ void k_accumulate(WaveDesc w, PathBuffers P, FilmDev F) {
    uint32_t npix = w.w * w.h;
    uint32_t ns = w.n / npix;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        const uint32_t x = w.x0 + p % w.w, y = w.y0 + p / w.w;
        if (w.edge && w.edge[(size_t)y * w.edge_stride + x]) continue;  // splatted by the edge waves
        accumulate_pixel(F, x, y, P, p, npix, ns);
    }
}

// An edge wave: per edge pixel and sample index, the mean of its k samples (summed in order,
// times 1 / k), splatted once (render.rs:477-488), sample indices in order.
__global__ void k_accumulate_edges(WaveDesc w, PathBuffers P, FilmDev F) {
    const uint32_t k = w.ek, ns = w.n / (w.ne * k);
    const float inv = 1.0f / (float)k;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < w.ne; e += gridDim.x * blockDim.x) {
        const uint32_t x = w.epix[e] & 0xffffu, y = w.epix[e] >> 16;
        if (x < F.ox || y < F.oy || x - F.ox >= F.w || y - F.oy >= F.h) continue;
        const size_t fi = (size_t)(y - F.oy) * F.w + (x - F.ox);
        float r = F.rgb[3 * fi], g = F.rgb[3 * fi + 1], b = F.rgb[3 * fi + 2];
        float wt = F.weight[fi], al = F.alpha[fi], l2 = F.lum2[fi];
        for (uint32_t s = 0; s < ns; ++s) {
            float sr = 0.0f, sg = 0.0f, sb = 0.0f, cov = 0.0f;
            for (uint32_t j = 0; j < k; ++j) {
                const uint32_t slot = (s * w.ne + e) * k + j;
                const float4 c = sample_sum(P, slot);
                sr = sr + c.x; sg = sg + c.y; sb = sb + c.z;
                cov = cov + P.thr[slot].w;
            }
            const Rgb m = rgb(sr * inv, sg * inv, sb * inv);
            r = r + m.r; g = g + m.g; b = b + m.b;
            wt = wt + 1.0f;
            al = al + cov * inv;
            const float l = luminance(m);
            l2 = l2 + l * l;
        }
        F.rgb[3 * fi] = r; F.rgb[3 * fi + 1] = g; F.rgb[3 * fi + 2] = b;
        F.weight[fi] = wt; F.alpha[fi] = al; F.lum2[fi] = l2;
    }
}

// ---- edge mask (pixel_filter.rs:149-268) -------------------------------------------------------------
// What the centre ray of a pixel meets first (render.rs:503 centre_ray, integrator/mod.rs:911
// first_hit, passes.rs:168 Exact::of): x = part (instance + 1, 0xffffffff the floor, 0 the
// background), y = material (+ 1, the same codes), z = depth along the view axis (bits).
__global__ void __launch_bounds__(TRACE_THREADS) k_edge_exact(SceneDev S, const LightsDev* __restrict__ Lg, uint4* exact) {
    __shared__ uint64_t s_stack[SHORT_STACK * TRACE_THREADS];
    uint64_t deep[STACK_CAP - SHORT_STACK];
    SplitStack stack{s_stack + threadIdx.x, deep, TRACE_THREADS};
    const LightsDev& L = *Lg;
    const uint32_t n = S.width * S.height;
    uint32_t err = 0;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t x = p % S.width, y = p / S.width;
        V3 o, d;
        const bool sees = camera_ray_at(S, ((float)x + 0.5f) / (float)S.width, ((float)y + 0.5f) / (float)S.height, 0.0f, 0.0f, o, d);
        TraceResult res;
        const bool got = sees && trace_q<false>(S, o, d, 1.0e-3f, f_inf(), true, res, &err, stack);
        const float t_geometry = got ? res.t : f_inf();
        float t_floor = f_inf();
        if (S.floor_mode == 1 && d.z != 0.0f && sees) {
            const float t = (S.floor_z - o.z) / d.z;
            if (t > 1.0e-3f && t < f_inf()) t_floor = t;
        }
        const float t_nearest = rmin(t_geometry, t_floor);
        uint4 e = make_uint4(0u, 0u, __float_as_uint(f_inf()), 0u);
        if (!(t_nearest == f_inf() || camera_sees_panel(L, o, d, t_nearest))) {
            float t = t_floor;
            bool ok = true;
            if (t_floor < t_geometry) {
                e.x = e.y = 0xffffffffu;
            } else {
                HitInfo h;
                uint4 idx;
                const DevInstance* I = nullptr;
                ok = hit_details(S, o, d, 1.0e-3f, f_inf(), res.inst, res.tri, res.t, h, I, idx) && I != nullptr;
                if (ok) {
                    e.x = res.inst + 1u;
                    e.y = I->material < S.n_materials ? I->material + 1u : 0u;
                }
                t = res.t;
            }
            if (ok) {
                const V3 fwd = ld3(S.cam_fwd);
                e.z = __float_as_uint(S.projection ? t * len(d) : t * dot(d, fwd) + dot(o - ld3(S.cam_pos), fwd));
            } else {
                e = make_uint4(0u, 0u, __float_as_uint(f_inf()), 0u);
            }
        }
        exact[p] = e;
    }
    (void)err;
}
// ---- guide passes (passes.rs:141-229, render.rs:515-640) --------------------------------------------
// What a camera ray (o, d) meets first (integrator/mod.rs:911 first_hit): `e` = part, material
// and depth bits as k_edge_exact writes them, the normal facing the ray (the floor's +-z), and the
// albedo (passes.rs:209: the material's base colour, the default material's for an index out of
// range, the floor's colour, black for the background).
// `sees`: false for a panoramic camera's ray that sees nothing (an empty interval: the background).
__device__ void first_hit_passes(const SceneDev& S, const LightsDev& L, V3 o, V3 d, bool sees, SplitStack& stack, uint32_t* err, uint4& e,
                                 V3& normal, Rgb& albedo) {
    TraceResult res;
    const bool got = sees && trace_q<false>(S, o, d, 1.0e-3f, f_inf(), true, res, err, stack);
    const float t_geometry = got ? res.t : f_inf();
    float t_floor = f_inf();
    if (S.floor_mode == 1 && d.z != 0.0f && sees) {
        const float t = (S.floor_z - o.z) / d.z;
        if (t > 1.0e-3f && t < f_inf()) t_floor = t;
    }
    const float t_nearest = rmin(t_geometry, t_floor);
    e = make_uint4(0u, 0u, __float_as_uint(f_inf()), 0u);
    normal = v3(0.0f, 0.0f, 0.0f);
    albedo = rgb(0.0f, 0.0f, 0.0f);
    if (t_nearest == f_inf() || camera_sees_panel(L, o, d, t_nearest)) return;
    float t = t_floor;
    if (t_floor < t_geometry) {
        e.x = e.y = 0xffffffffu;
        normal = v3(0.0f, 0.0f, d.z < 0.0f ? 1.0f : -1.0f);
        albedo = rgb(S.floor_color[0], S.floor_color[1], S.floor_color[2]);
    } else {
        HitInfo h;
        uint4 idx;
        const DevInstance* I = nullptr;
        if (!(hit_details(S, o, d, 1.0e-3f, f_inf(), res.inst, res.tri, res.t, h, I, idx) && I != nullptr)) return;
        e.x = res.inst + 1u;
        const bool known = I->material < S.n_materials;
        e.y = known ? I->material + 1u : 0u;
        normal = h.normal;
        albedo = known ? rgb(S.materials[I->material].base[0], S.materials[I->material].base[1], S.materials[I->material].base[2])
                       : rgb(0.8f, 0.8f, 0.8f);
        t = res.t;
    }
    const V3 fwd = ld3(S.cam_fwd);
    e.z = __float_as_uint(S.projection ? t * len(d) : t * dot(d, fwd) + dot(o - ld3(S.cam_pos), fwd));  // passes.rs:191
}

// passes.rs:221 coverage_of: whether first_hit_passes met a surface of an instance (its part id is
// the instance + 1; the floor's is all ones, the background's and a light panel's 0).
__device__ __forceinline__ bool first_hit_covers(uint4 e) { return e.x != 0u && e.x != 0xffffffffu; }

// The exact passes of the centre rays of a rectangle (render.rs:529), background outside the image.
__global__ void __launch_bounds__(TRACE_THREADS) k_exact_passes(SceneDev S, const LightsDev* __restrict__ Lg, uint32_t x0, uint32_t y0,
                                                                 uint32_t w, uint32_t h, float* normal, float* depth, uint32_t* part,
                                                                 uint32_t* material) {
    __shared__ uint64_t s_stack[SHORT_STACK * TRACE_THREADS];
    uint64_t deep[STACK_CAP - SHORT_STACK];
    SplitStack stack{s_stack + threadIdx.x, deep, TRACE_THREADS};
    uint32_t err = 0;
    const uint32_t n = w * h;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t x = x0 + p % w, y = y0 + p / w;
        uint4 e = make_uint4(0u, 0u, __float_as_uint(f_inf()), 0u);
        V3 nn = v3(0.0f, 0.0f, 0.0f);
        Rgb a;
        if (x < S.width && y < S.height) {
            V3 o, d;
            const bool sees = camera_ray_at(S, ((float)x + 0.5f) / (float)S.width, ((float)y + 0.5f) / (float)S.height, 0.0f, 0.0f, o, d);
            first_hit_passes(S, *Lg, o, d, sees, stack, &err, e, nn, a);
        }
        normal[3 * p] = nn.x;
        normal[3 * p + 1] = nn.y;
        normal[3 * p + 2] = nn.z;
        depth[p] = __uint_as_float(e.z);
        part[p] = e.x;
        material[p] = e.y;
    }
    (void)err;
}

// The albedo of samples [first, first + count) of a rectangle's pixels inside the image, added in
// sample order to `sum` (3 a pixel) with `weight` += 1 each (render.rs:590 render_tile_albedo_traced):
// an edge pixel (`edge`, the image's mask, may be null) adds the mean of its k sub-samples. With
// `alpha` (may be null) the coverage of the same first hits is added likewise (passes.rs:221
// coverage_of: 1 for a surface of an instance, 0 for the floor, a light panel or the background).
__global__ void __launch_bounds__(TRACE_THREADS) k_albedo_pass(SceneDev S, const LightsDev* __restrict__ Lg, const uint8_t* __restrict__ edge,
                                                                uint32_t x0, uint32_t y0, uint32_t w, uint32_t h, uint32_t first,
                                                                uint32_t count, float* sum, float* weight, float* alpha) {
    __shared__ uint64_t s_stack[SHORT_STACK * TRACE_THREADS];
    uint64_t deep[STACK_CAP - SHORT_STACK];
    SplitStack stack{s_stack + threadIdx.x, deep, TRACE_THREADS};
    uint32_t err = 0;
    const uint32_t n = w * h;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t x = x0 + p % w, y = y0 + p / w;
        if (x >= S.width || y >= S.height) continue;
        const uint32_t k = (edge && S.edge_k > 1 && edge[(size_t)y * S.width + x]) ? S.edge_k : 1u;
        float r = sum[3 * p], g = sum[3 * p + 1], b = sum[3 * p + 2], wt = weight[p], cv = alpha ? alpha[p] : 0.0f;
        for (uint32_t s = 0; s < count; ++s) {
            uint4 e;
            V3 nn, o, d;
            Rgb a;
            float c;
            if (k <= 1) {
                const bool sees = camera_ray(S, c_sobol, x, y, first + s, o, d);
                first_hit_passes(S, *Lg, o, d, sees, stack, &err, e, nn, a);
                c = first_hit_covers(e) ? 1.0f : 0.0f;
            } else {
                Rgb acc = rgb(0.0f, 0.0f, 0.0f);
                float covered = 0.0f;
                for (uint32_t j = 0; j < k; ++j) {
                    const bool sees = camera_ray(S, c_sobol, x, y, (first + s) * k + j, o, d);  // render.rs:376 sub_sample
                    first_hit_passes(S, *Lg, o, d, sees, stack, &err, e, nn, a);
                    acc = rgb(acc.r + a.r, acc.g + a.g, acc.b + a.b);
                    covered = covered + (first_hit_covers(e) ? 1.0f : 0.0f);
                }
                const float inv = 1.0f / (float)k;
                a = rgb(acc.r * inv, acc.g * inv, acc.b * inv);
                c = covered * inv;
            }
            r = r + a.r;
            g = g + a.g;
            b = b + a.b;
            wt = wt + 1.0f;
            cv = cv + c;
        }
        sum[3 * p] = r;
        sum[3 * p + 1] = g;
        sum[3 * p + 2] = b;
        weight[p] = wt;
        if (alpha) alpha[p] = cv;
    }
    (void)err;
}

// The albedo of each camera ray's first hit from the wave's first extend (the ray in P.o / P.d,
// the hit in P.hit): first_hit_passes without its traversal, which the extend has done with the
// same ray, class and interval.
__global__ void k_albedo_hits(SceneDev S, const LightsDev* __restrict__ Lg, WaveDesc w, PathBuffers P) {
    const LightsDev& L = *Lg;
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < w.n; slot += gridDim.x * blockDim.x) {
        const float4 of = P.o[slot], df = P.d[slot];
        const V3 o = v3(of.x, of.y, of.z), d = v3(df.x, df.y, df.z);
        const uint4 hit = P.hit[slot];
        const bool got = hit.w != 0u;
        const float t_geometry = got ? __uint_as_float(hit.z) : f_inf();
        float t_floor = f_inf();
        if (S.floor_mode == 1 && d.z != 0.0f && !(P.flags[slot] & PF_NOTHING)) {
            const float t = (S.floor_z - o.z) / d.z;
            if (t > 1.0e-3f && t < f_inf()) t_floor = t;
        }
        const float t_nearest = rmin(t_geometry, t_floor);
        float4 a = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (!(t_nearest == f_inf() || camera_sees_panel(L, o, d, t_nearest))) {
            if (t_floor < t_geometry) {
                a = make_float4(S.floor_color[0], S.floor_color[1], S.floor_color[2], 0.0f);
            } else {
                HitInfo h;
                uint4 idx;
                const DevInstance* I = nullptr;
                if (hit_details(S, o, d, 1.0e-3f, f_inf(), hit.x, hit.y, __uint_as_float(hit.z), h, I, idx) && I != nullptr) {
                    if (I->material < S.n_materials) {
                        const float* b = S.materials[I->material].base;
                        a = make_float4(b[0], b[1], b[2], 0.0f);
                    } else {
                        a = make_float4(0.8f, 0.8f, 0.8f, 0.0f);
                    }
                }
            }
        }
        w.alb[slot] = a;
    }
}

// The wave's albedo into the film's guide sums, each pixel's samples in index order (the edge
// pixels of a list wave the mean of their k sub-samples, render.rs:590).
__global__ void k_accumulate_albedo(WaveDesc w, FilmDev F) {
    const bool list = w.epix != nullptr;
    const uint32_t k = list ? w.ek : 1u;
    const uint32_t units = list ? w.ne : w.w * w.h;
    const uint32_t ns = w.n / (units * k);
    const float inv = 1.0f / (float)k;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < units; e += gridDim.x * blockDim.x) {
        uint32_t x, y;
        if (list) {
            x = w.epix[e] & 0xffffu;
            y = w.epix[e] >> 16;
        } else {
            x = w.x0 + e % w.w;
            y = w.y0 + e / w.w;
            if (w.edge && w.edge[(size_t)y * w.edge_stride + x]) continue;  // from the edge waves
        }
        if (x < F.ox || y < F.oy || x - F.ox >= F.w || y - F.oy >= F.h) continue;
        const size_t fi = (size_t)(y - F.oy) * F.w + (x - F.ox);
        float r = w.guide_sum[3 * fi], g = w.guide_sum[3 * fi + 1], b = w.guide_sum[3 * fi + 2], wt = w.guide_weight[fi];
        for (uint32_t s = 0; s < ns; ++s) {
            float ar, ag, ab;
            if (k > 1) {
                ar = ag = ab = 0.0f;
                for (uint32_t j = 0; j < k; ++j) {
                    const float4 c = w.alb[(s * units + e) * k + j];
                    ar = ar + c.x;
                    ag = ag + c.y;
                    ab = ab + c.z;
                }
                ar = ar * inv;
                ag = ag * inv;
                ab = ab * inv;
            } else {
                const float4 c = w.alb[s * units + e];
                ar = c.x;
                ag = c.y;
                ab = c.z;
            }
            r = r + ar;
            g = g + ag;
            b = b + ab;
            wt = wt + 1.0f;
        }
        w.guide_sum[3 * fi] = r;
        w.guide_sum[3 * fi + 1] = g;
        w.guide_sum[3 * fi + 2] = b;
        w.guide_weight[fi] = wt;
    }
}

// A pixel is an edge when a neighbour inside the image sees another part, another material, or
// a depth more than 2 % away (two background pixels never differ).
__global__ void k_edge_mask(SceneDev S, const uint4* __restrict__ exact, uint8_t* mask) {
    const uint32_t w = S.width, h = S.height, n = w * h;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t x = p % w, y = p / w;
        const uint4 c = exact[p];
        const float cd = __uint_as_float(c.z);
        bool edge = false;
        for (uint32_t ny = y ? y - 1 : 0; ny < min(y + 2, h); ++ny)
            for (uint32_t nx = x ? x - 1 : 0; nx < min(x + 2, w); ++nx) {
                const uint4 o = exact[ny * w + nx];
                const float od = __uint_as_float(o.z);
                edge |= c.x != o.x || c.y != o.y || absf(cd - od) > 0.02f * rmin(cd, od);
            }
        mask[p] = edge ? 1 : 0;
    }
}
__global__ void k_edge_list(const uint8_t* __restrict__ mask, uint32_t stride, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                            uint32_t* list, uint32_t* count) {
    const uint32_t n = w * h;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t x = x0 + p % w, y = y0 + p / w;
        if (mask[(size_t)y * stride + x]) list[atomicAdd(count, 1u)] = x | (y << 16);
    }
}

// A batched wave: every pixel of every segment into its job's film. A job has at most one segment
// per wave, so no pixel is added twice here, and waves run in sample order.
__global__ void k_accumulate_jobs(WaveDesc w, PathBuffers P) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < w.npix; p += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = w.nseg;
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (__ldg(&w.segs[mid].pix_begin) <= p) lo = mid;
            else hi = mid;
        }
        const SegDev& g = w.segs[lo];
        uint32_t local = p - g.pix_begin, npix = g.w * g.h;
        accumulate_pixel(w.jobs[g.job].film, local % g.w, g.y0 + local / g.w, P, g.slot_begin + local, npix, g.ns);
    }
}

// ---- film output (image.rs:186-221): resolve, exposure, then either the tone curve and sRGB at 8 or 16
// bits, or (bits 32) the exposed linear light as floats with no curve and no clamp (to_linear_exposed) ----
__global__ void k_film_encode(FilmDev F, float gain, uint32_t kind, AgxMatrices agx, uint32_t bits, void* out) {
    const uint32_t n = F.w * F.h;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        float w = F.weight[p];
        Rgb px = rgb(0.0f, 0.0f, 0.0f);
        if (w > 0.0f) {
            float inv = 1.0f / w;
            px = rgb(F.rgb[3 * p] * inv, F.rgb[3 * p + 1] * inv, F.rgb[3 * p + 2] * inv);
        }
        if (bits == 32) {
            float* o = static_cast<float*>(out) + 3 * p;
            o[0] = px.r * gain;
            o[1] = px.g * gain;
            o[2] = px.b * gain;
            continue;
        }
        Rgb m = tonemap_apply(kind, px * gain, agx);
        float v[3] = {srgb_encode(m.r), srgb_encode(m.g), srgb_encode(m.b)};
        for (int c = 0; c < 3; ++c) {
            if (bits == 8) static_cast<uint8_t*>(out)[3 * p + c] = (uint8_t)saturate_cast(v[c] * 255.0f + 0.5f, 255.0f);
            else static_cast<uint16_t*>(out)[3 * p + c] = (uint16_t)saturate_cast(v[c] * 65535.0f + 0.5f, 65535.0f);
        }
    }
}

// ---- ray batches for the traversal parity harness ---------------------------------------------------
__global__ void __launch_bounds__(TRACE_THREADS) k_trace_batch(SceneDev S, const float* __restrict__ rays, uint32_t n, uint32_t mode, uint32_t* out,
                                                     uint32_t* counters) {
    __shared__ uint64_t s_stack[SHORT_STACK * TRACE_THREADS];
    uint64_t deep[STACK_CAP - SHORT_STACK];
    SplitStack stack{s_stack + threadIdx.x, deep, TRACE_THREADS};
    uint32_t err = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* r = rays + 8 * i;
        TraceResult res;
        V3 o = v3(r[0], r[1], r[2]), d = v3(r[3], r[4], r[5]);
        if (mode & 2u) {
            out[i] = trace_q<true>(S, o, d, r[6], r[7], (mode & 1u) != 0, res, &err, stack) ? 1u : 0u;
        } else {
            bool got = trace_q<false>(S, o, d, r[6], r[7], (mode & 1u) != 0, res, &err, stack);
            out[3 * i] = got ? res.inst : 0xffffffffu;
            out[3 * i + 1] = got ? res.tri : 0xffffffffu;
            out[3 * i + 2] = got ? __float_as_uint(res.t) : 0u;
        }
    }
    if (err) atomicOr(&counters[3], err);
}

}  // namespace rtg

#include "rtg_adjoint.cuh"

namespace rtg {

// ---- launchers ---------------------------------------------------------------------------------------
void set_sobol(const SobolTable& t, cudaStream_t s) { cudaMemcpyToSymbolAsync(c_sobol, &t, sizeof(t), 0, cudaMemcpyHostToDevice, s); }

// Blocks of the persistent traversal kernels that fit on the device at once (their grid: more
// blocks would only start after the queue has drained).
static int resident_blocks(const void* kernel, int threads) {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess || per_sm < 1)
        return 0;
    return sms * per_sm;
}

// A traversal kernel's launch; with order.l2_persist, with an L2 access-policy window over the
// scene's traversal data (persisting for its hit ratio, the rest streaming).
template <class... KArgs, class... Args>
static void launch_traversal(const RaySort& order, int grid, cudaStream_t st, void (*kernel)(KArgs...), Args... args) {
    if (!(order.l2_persist && order.l2_base && order.l2_bytes)) {
        kernel<<<grid, TRACE_THREADS, 0, st>>>(args...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(TRACE_THREADS);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeAccessPolicyWindow;
    attr[0].val.accessPolicyWindow.base_ptr = const_cast<void*>(order.l2_base);
    attr[0].val.accessPolicyWindow.num_bytes = order.l2_bytes;
    attr[0].val.accessPolicyWindow.hitRatio = order.l2_hit_ratio;
    attr[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    attr[0].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Whether a wave's last rounds run in k_tail: a limit set, no shadow walks, not batched.
// The tail traces with the plain traversal: scenes with passable surfaces or a section keep the wavefront.
static bool tail_on(const SceneDev& S, const RaySort& order, bool batch) {
    return order.tail_paths > 0 && !S.any_passable && !S.section_on && !batch;
}

uint32_t wave_launches(const SceneDev& S, const RaySort& order, const PathBuffers& P, bool batch) {
    const uint32_t rounds = wave_rounds(S);
    const bool rsort = order.ray_bits > 0 && P.rbins, ssort = rsort && order.shadow_sort && P.sbins;
    uint32_t per_round = 5 + (order.material_sort ? 1u : 0u) + (ssort ? 2u : 0u);
    const uint32_t tail = tail_on(S, order, batch) && rounds > TAIL_FIRST_ROUND ? 2u * (rounds - TAIL_FIRST_ROUND) : 0u;
    return 2 + rounds * per_round + (rsort && rounds > 1 ? 2u * (rounds - 1u) : 0u) + tail;
}

void launch_wave(const SceneDev& S, const LightsDev* L, const WaveDesc& w, const PathBuffers& P, const FilmDev* film, cudaStream_t st,
                 int grid, WaveTiming* timing, const RaySort& order) {
    static const int ext_resident = resident_blocks((const void*)k_extend, TRACE_THREADS);
    static const int sh_resident = resident_blocks((const void*)k_shadow, TRACE_THREADS);
    static const int tail_resident = resident_blocks((const void*)k_tail, TRACE_THREADS);
    const int g = grid;
    const int g_ext = ext_resident > 0 && ext_resident < g ? ext_resident : g;
    const int g_sh = sh_resident > 0 && sh_resident < g ? sh_resident : g;
    const bool batch = w.segs != nullptr;
    const bool rsort = order.ray_bits > 0 && order.ray_bits <= RAY_SORT_MAX_BITS && P.rbins;
    const bool ssort = rsort && order.shadow_sort && P.sbins;
    const uint32_t nk = ray_sort_keys(order.ray_bits);
    if (batch) k_camera<true><<<g, 256, 0, st>>>(S, w, P);
    else k_camera<false><<<g, 256, 0, st>>>(S, w, P);
    int cur = 0;
    const uint32_t rounds = wave_rounds(S);
    const bool tail = tail_on(S, order, batch);
    for (uint32_t round = 0; round < rounds; ++round) {
        if (tail && round >= TAIL_FIRST_ROUND) {
            k_tail<<<tail_resident > 0 ? tail_resident : g, TRACE_THREADS, 0, st>>>(S, L, P, cur, w, rounds - round, order.tail_paths);
            k_tail_end<<<1, 1, 0, st>>>(P, cur, order.tail_paths);
        }
        // The camera rays are traced in pixel order; later rounds' rays in coherence order.
        const uint32_t* traced = P.queue[cur];
        if (rsort && round > 0) {
            k_key_scan<<<1, 1024, 0, st>>>(P.rbins, nk);
            k_key_scatter<<<g, 256, 0, st>>>(P.queue[cur], P.key, P.rbins + nk, &P.counters[cur], P.sorted);
            traced = P.sorted;
        }
        if (timing && timing->ev_count + 2 <= WaveTiming::MAX_EVENTS) {
            cudaEventRecord(timing->ev[timing->ev_count++], st);
            launch_traversal(order, g_ext, st, S.section_on ? k_extend_section : k_extend, S, P, cur, traced);
            cudaEventRecord(timing->ev[timing->ev_count++], st);
        } else {
            launch_traversal(order, g_ext, st, S.section_on ? k_extend_section : k_extend, S, P, cur, traced);
        }
        if (round == 0 && w.alb && film && !batch) k_albedo_hits<<<g, 256, 0, st>>>(S, L, w, P);
        k_scan<<<1, 32, 0, st>>>(P);
        // The material-sorted copy goes to whichever list the traversal did not read.
        const uint32_t* shaded = traced;
        if (order.material_sort) {
            uint32_t* sorted = traced == P.sorted ? P.queue[cur] : P.sorted;
            k_scatter<<<g, 256, 0, st>>>(P, cur, traced, sorted);
            shaded = sorted;
        }
        // Keys for the next round's rays (none after the last round) and for this round's shadow rays.
        PathBuffers Q = P;
        Q.rbins = rsort && round + 1 < rounds ? P.rbins : nullptr;
        Q.sbins = ssort ? P.sbins : nullptr;
        if (batch) k_shade<true><<<g, 128, 0, st>>>(S, L, Q, cur, w, shaded, order);
        else k_shade<false><<<g, 128, 0, st>>>(S, L, Q, cur, w, shaded, order);
        // queue[cur] is free once shade has read its list: it holds the shadow rays' order.
        const uint32_t* perm = nullptr;
        if (ssort) {
            k_key_scan<<<1, 1024, 0, st>>>(P.sbins, nk);
            k_key_scatter<<<g, 256, 0, st>>>(nullptr, P.sh_key, P.sbins + nk, &P.counters[2], P.queue[cur]);
            perm = P.queue[cur];
        }
        if (!S.any_passable) launch_traversal(order, g_sh, st, S.section_on ? k_shadow_section : k_shadow, S, P, perm);
        else if (batch) k_shadow_walk<true><<<g, TRACE_THREADS, 0, st>>>(S, P, w, perm);
        else k_shadow_walk<false><<<g, TRACE_THREADS, 0, st>>>(S, P, w, perm);
        k_next_round<<<1, 1, 0, st>>>(P, cur);
        cur ^= 1;
    }
    if (batch) k_accumulate_jobs<<<g, 256, 0, st>>>(w, P);
    else if (film && w.epix) k_accumulate_edges<<<g, 256, 0, st>>>(w, P, *film);
    else if (film) k_accumulate<<<g, 256, 0, st>>>(w, P, *film);
    if (w.alb && film && !batch) k_accumulate_albedo<<<g, 256, 0, st>>>(w, *film);
}

cudaError_t launch_edge_mask(const SceneDev& S, const LightsDev* L, uint4* exact, uint8_t* mask, cudaStream_t st, int grid) {
    k_edge_exact<<<grid, TRACE_THREADS, 0, st>>>(S, L, exact);
    k_edge_mask<<<grid, 256, 0, st>>>(S, exact, mask);
    return cudaGetLastError();
}
cudaError_t launch_exact_passes(const SceneDev& S, const LightsDev* L, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h, float* normal,
                                float* depth, uint32_t* part, uint32_t* material, cudaStream_t st, int grid) {
    k_exact_passes<<<grid, TRACE_THREADS, 0, st>>>(S, L, x0, y0, w, h, normal, depth, part, material);
    return cudaGetLastError();
}
cudaError_t launch_albedo_pass(const SceneDev& S, const LightsDev* L, const uint8_t* edge, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                               uint32_t first, uint32_t count, float* sum, float* weight, float* alpha, cudaStream_t st, int grid) {
    k_albedo_pass<<<grid, TRACE_THREADS, 0, st>>>(S, L, edge, x0, y0, w, h, first, count, sum, weight, alpha);
    return cudaGetLastError();
}
cudaError_t launch_edge_list(const uint8_t* mask, uint32_t stride, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h, uint32_t* list,
                             uint32_t* count, cudaStream_t st, int grid) {
    cudaMemsetAsync(count, 0, 4, st);
    k_edge_list<<<grid, 256, 0, st>>>(mask, stride, x0, y0, w, h, list, count);
    return cudaGetLastError();
}

void launch_adjoint_delta(const FilmDev& F, const float* target, float4* dpath, double* loss, const PathBuffers& P, uint32_t count, cudaStream_t st,
                          int grid) {
    k_adjoint_delta<<<grid, 256, 0, st>>>(F, target, dpath, loss, P, count);
}
void launch_adjoint_wave(const SceneDev& S, const LightsDev* L, const WaveDesc& w, const PathBuffers& P, const AdjointDev& A, cudaStream_t st,
                         int grid) {
    static const int ext_resident = resident_blocks((const void*)k_extend, TRACE_THREADS);
    static const int sh_resident = resident_blocks((const void*)k_shadow_adjoint, TRACE_THREADS);
    const int g = grid;
    const int g_ext = ext_resident > 0 && ext_resident < g ? ext_resident : g;
    const int g_sh = sh_resident > 0 && sh_resident < g ? sh_resident : g;
    k_adjoint_camera<<<g, 256, 0, st>>>(S, w, P, A);
    int cur = 0;
    for (uint32_t bounce = 0; bounce <= S.max_depth; ++bounce) {
        k_extend<<<g_ext, TRACE_THREADS, 0, st>>>(S, P, cur, P.queue[cur]);
        k_scan<<<1, 32, 0, st>>>(P);
        k_scatter<<<g, 256, 0, st>>>(P, cur, P.queue[cur], P.sorted);
        k_shade_adjoint<<<g, 128, 0, st>>>(S, L, P, cur, bounce, w, A);
        k_shadow_adjoint<<<g_sh, TRACE_THREADS, 0, st>>>(S, P, w, A);
        k_next_round<<<1, 1, 0, st>>>(P, cur);
        cur ^= 1;
    }
    k_adjoint_residual<<<g, 256, 0, st>>>(w, P, A);
}
void launch_film_encode(const FilmDev& F, float ev, uint32_t tonemap, uint32_t bits, void* out, cudaStream_t st, int grid) {
    k_film_encode<<<grid, 256, 0, st>>>(F, fexp2(ev), tonemap, agx_matrices(), bits, out);
}
void launch_trace_batch(const SceneDev& S, const float* rays, uint32_t n, uint32_t mode, uint32_t* out, uint32_t* counters,
                        cudaStream_t st, int grid) {
    k_trace_batch<<<grid, TRACE_THREADS, 0, st>>>(S, rays, n, mode, out, counters);
}

}  // namespace rtg
