// The C-ABI drop-in: scene registry, device memory, tile and progressive renders, films, and the
// parity entry points. Mirrors the hand-written ABI of the reference's rt-wasm
// (engine/crates/rt-wasm/src/ffi.rs:28-197, rt-wasm/src/lib.rs:37-164, 562-730).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/repackshot_b200.h"
#include "rtg_adaptive.h"
#include "rtg_denoise.h"
#include "rtg_kernels.h"
#include "rtg_noalloc.h"
#include "rtg_scene.h"
#include "rtg_tables.h"

namespace rtg {
namespace {

#define RTG_CHECK(call)                                                          \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) { cuda_fail(e_, #call); return RTG_STATUS_CUDA_ERROR; } \
    } while (0)

std::mutex g_mu;  // every entry point holds it: calls serialise, as the reference's registry does
std::string g_error;
bool g_device_ready = false;
void* g_energy_dev = nullptr;
EnergyTables g_energy{};
const float* g_filter_table = nullptr;  // the Blackman-Harris inverse CDF on the device
int g_sms = 148;

void cuda_fail(cudaError_t e, const char* what) {
    g_error = std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ") in " + what;
}

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    void release() { if (p) cudaFree(p); p = nullptr; bytes = 0; }
};

// Device buffers released together.
struct BufSet {
    std::vector<DevBuf> bufs;
    LightsDev* lights = nullptr;
    void release() {
        for (auto& b : bufs) b.release();
        bufs.clear();
        if (lights) cudaFree(lights);
        lights = nullptr;
    }
};

struct Scene {
    SceneDev S{};
    LightsDev* d_lights = nullptr;
    BufSet geometry;  // trees, leaf triangles, vertex arrays: kept by updates that keep the meshes
    BufSet shading;   // instances, materials, BSDFs, lights: replaced by every update
    std::vector<HMesh> meshes;  // the host meshes, for updates without MESH sections
    std::vector<HImage> bitmaps;  // the decoded bitmaps, for updates and jobs without BMAP sections
    std::string geom_key;
    // for the adjoint: materials as uploaded, each scene light's power, each area light's scene light
    std::vector<DevMaterial> materials_h;
    std::vector<float> light_power;
    float exposure_ev = 0.0f;  // RNDR's output settings
    uint32_t tonemap = 1, max_samples = 0;
    uint32_t adaptive = 0;          // RNDR.adaptive and RNDR.noise_threshold (E10)
    float noise_threshold = 0.0f;
    std::vector<uint32_t> light_source;  // scene light of each prepared light (areas, suns, spheres)
    DevBuf adjoint_mem;
    // edge samples (E11): the image's edge mask, its centre-ray scratch and an edge-pixel list
    DevBuf edge_mem;
    bool edges_ready = false;
    DevBuf alb_mem;  // one float4 a path slot: the albedo of renders that fill a film's guides
    uint64_t edge_builds = 0;  // masks built so far: what depends on the mask checks it
    cudaStream_t stream = nullptr;
    int device = -1;  // the CUDA device the scene was loaded on
    // path buffers
    PathBuffers P{};
    DevBuf path_mem;
    uint32_t capacity = 0;
    uint32_t max_capacity = 0;  // paths per wave; 0: automatic (wave_limit)
    RaySort order;              // how waves order their rays and paths (rtg_set_tuning)
    size_t hot_bytes = 0;       // the traversal data at the start of the geometry allocation
    float sort_lo[3] = {0, 0, 0}, sort_hi[3] = {0, 0, 0};  // the box the ray sort grids
    // statistics
    uint64_t rays = 0;
    double build_seconds = 0;
    uint64_t nodes = 0, tris = 0, instanced_triangles = 0;
    uint32_t width = 0, height = 0, max_depth = 0;
    // extend-kernel timing
    bool timing = false;
    WaveTiming* wt = nullptr;
    double extend_ms = 0;
    uint64_t extend_launches = 0;
    uint64_t extend_rays = 0, shadow_rays = 0;
    uint64_t launches = 0;        // kernels launched since the last timing reset
    bool own_stream = true;       // false after rtg_set_stream: the caller owns the stream
    ~Scene() {
        geometry.release();
        shading.release();
        path_mem.release();
        adjoint_mem.release();
        edge_mem.release();
        alb_mem.release();
        if (wt) {
            for (int i = 0; i < WaveTiming::MAX_EVENTS; ++i) cudaEventDestroy(wt->ev[i]);
            delete wt;
        }
        if (stream && own_stream) cudaStreamDestroy(stream);
    }
};
struct Film {
    uint32_t scene;
    FilmDev dev{};
    DevBuf mem;
    DevBuf encoded;  // the last 8- or 16-bit image, on its way to the host
    // The denoiser's guide passes (rtg_film_guides): albedo sums (3 a pixel) and their samples,
    // normal (3), depth, part and material ids; and the denoiser's scratch and result.
    DevBuf guides;
    DevBuf denoise;
    bool fuse_guides = false;  // rtg_film_guides_fused: renders add their albedo to `guides`
    ~Film() {
        mem.release();
        encoded.release();
        guides.release();
        denoise.release();
    }
    size_t pixels() const { return (size_t)dev.w * dev.h; }
    float* albedo_sum() const { return (float*)guides.p; }
    float* albedo_weight() const { return albedo_sum() + 3 * pixels(); }
    float* normal() const { return albedo_weight() + pixels(); }
    float* depth() const { return normal() + 3 * pixels(); }
    uint32_t* part() const { return (uint32_t*)(depth() + pixels()); }
    uint32_t* material() const { return part() + pixels(); }
};
// A job of a render queue: one variant of the queue's scene (its own camera, image, materials,
// lights and settings over the scene's geometry), a sample range and the film it renders into.
struct QueueJob {
    BufSet shading;
    SceneDev constants;  // F.scene of the job; geometry pointers are taken from the scene at run time
    SceneDev shade;      // the job's instance, material and BSDF pointers
    std::string geom_key;
    uint32_t film = 0, first = 0, count = 0, width = 0, height = 0;
};
struct Queue {
    uint32_t scene = 0;
    std::vector<std::unique_ptr<QueueJob>> jobs;  // pending until the next run
    DevBuf tables;                                // JobDev and SegDev arrays of a run
    ~Queue() {
        for (auto& j : jobs) j->shading.release();
        tables.release();
    }
};

std::vector<std::unique_ptr<Scene>> g_scenes;
std::vector<std::unique_ptr<Film>> g_films;
std::vector<std::unique_ptr<Queue>> g_queues;

Scene* scene_of(uint32_t h) { return (h == 0 || h > g_scenes.size()) ? nullptr : g_scenes[h - 1].get(); }
Film* film_of(uint32_t h) { return (h == 0 || h > g_films.size()) ? nullptr : g_films[h - 1].get(); }
Queue* queue_of(uint32_t h) { return (h == 0 || h > g_queues.size()) ? nullptr : g_queues[h - 1].get(); }

uint32_t device_init() {
    if (g_device_ready) return RTG_STATUS_OK;
    int dev = 0;
    RTG_CHECK(cudaGetDevice(&dev));
    RTG_CHECK(cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev));
    SobolTable sob;
    build_sobol_table(sob);
    RTG_CHECK(cudaDeviceSynchronize());
    set_sobol(sob, 0);
    RTG_CHECK(cudaGetLastError());
    const EnergyData& E = energy_data();
    size_t n16 = E.albedo.size() + E.schlick.size() + E.clear_in.size() + E.clear_out.size();
    size_t bytes = n16 * 2 + 64 * 4 + 256 * 4;
    RTG_CHECK(cudaMalloc(&g_energy_dev, bytes));
    std::vector<uint8_t> host(bytes);
    uint8_t* p = host.data();
    auto put = [&](const void* src, size_t n) { std::memcpy(p, src, n); p += n; };
    put(E.albedo.data(), E.albedo.size() * 2);
    put(E.schlick.data(), E.schlick.size() * 2);
    put(E.clear_in.data(), E.clear_in.size() * 2);
    put(E.clear_out.data(), E.clear_out.size() * 2);
    put(E.albedo_avg.data(), 32 * 4);
    put(E.schlick_avg.data(), 32 * 4);
    put(blackman_harris_table(), 256 * 4);
    RTG_CHECK(cudaMemcpy(g_energy_dev, host.data(), bytes, cudaMemcpyHostToDevice));
    const uint8_t* d = (const uint8_t*)g_energy_dev;
    g_energy.albedo = (const uint16_t*)d;
    g_energy.schlick = g_energy.albedo + E.albedo.size();
    g_energy.clear_in = g_energy.schlick + E.schlick.size();
    g_energy.clear_out = g_energy.clear_in + E.clear_in.size();
    g_energy.albedo_avg = (const float*)(g_energy.clear_out + E.clear_out.size());
    g_energy.schlick_avg = g_energy.albedo_avg + 32;
    g_filter_table = g_energy.schlick_avg + 32;
    RTG_CHECK(cudaDeviceSynchronize());
    g_device_ready = true;
    return RTG_STATUS_OK;
}

template <class T>
uint32_t upload(BufSet& set, const std::vector<T>& v, const T*& out) {
    DevBuf b;
    b.bytes = v.size() * sizeof(T);
    if (b.bytes == 0) { out = nullptr; return RTG_STATUS_OK; }
    RTG_CHECK(cudaMalloc(&b.p, b.bytes));
    set.bufs.push_back(b);
    RTG_CHECK(cudaMemcpy(b.p, v.data(), b.bytes, cudaMemcpyHostToDevice));
    out = (const T*)b.p;
    return RTG_STATUS_OK;
}

// Uploads the trees, leaf triangles and hit-detail arrays of `F` into `set`, pointers into `S`.
// What traversal reads (nodes, leaf triangles, top-level leaves) lies first, in one allocation,
// so that one L2 access-policy window can cover it (its size in *hot_bytes).
uint32_t upload_geometry(const Flat& F, BufSet& set, SceneDev& S, size_t* hot_bytes = nullptr) {
    std::vector<float4> pos(F.positions.size() / 4), nrm(F.normals.size() / 4);
    std::memcpy(pos.data(), F.positions.data(), F.positions.size() * 4);
    std::memcpy(nrm.data(), F.normals.data(), F.normals.size() * 4);
    std::vector<uint4> ti(F.tri_index.size() / 4);
    std::memcpy(ti.data(), F.tri_index.data(), F.tri_index.size() * 4);
    auto round = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t b_nodes = F.nodes.size() * sizeof(QNode), b_tris = F.tris.size() * sizeof(TriRec), b_blas = F.blas.size() * sizeof(BlasInst);
    const size_t hot = round(b_nodes) + round(b_tris) + round(b_blas);
    if (hot_bytes) *hot_bytes = hot;
    S.nodes = nullptr;
    S.tris = nullptr;
    S.blas = nullptr;
    if (hot) {
        DevBuf b;
        b.bytes = hot;
        RTG_CHECK(cudaMalloc(&b.p, b.bytes));
        set.bufs.push_back(b);
        uint8_t* p = (uint8_t*)b.p;
        if (b_nodes) RTG_CHECK(cudaMemcpy(p, F.nodes.data(), b_nodes, cudaMemcpyHostToDevice));
        if (b_tris) RTG_CHECK(cudaMemcpy(p + round(b_nodes), F.tris.data(), b_tris, cudaMemcpyHostToDevice));
        if (b_blas) RTG_CHECK(cudaMemcpy(p + round(b_nodes) + round(b_tris), F.blas.data(), b_blas, cudaMemcpyHostToDevice));
        if (b_nodes) S.nodes = (const QNode*)p;
        if (b_tris) S.tris = (const TriRec*)(p + round(b_nodes));
        if (b_blas) S.blas = (const BlasInst*)(p + round(b_nodes) + round(b_tris));
    }
    uint32_t st;
    if ((st = upload(set, pos, S.positions)) || (st = upload(set, nrm, S.normals)) || (st = upload(set, ti, S.tri_index)))
        return st;
    return RTG_STATUS_OK;
}

// Uploads instances, materials, BSDFs, lights, the environment map and the background image of
// `F` into `set`, pointers into `S` and the uploaded lights.
uint32_t upload_shading(const Flat& F, BufSet& set, SceneDev& S) {
    uint32_t st;
    if ((st = upload(set, F.instances, S.instances)) || (st = upload(set, F.materials, S.materials)) ||
        (st = upload(set, F.bsdfs, S.bsdfs)))
        return st;
    LightsDev L = F.lights;
    if (!F.ies_data.empty()) {  // the IES lights point into their tables on the device
        const float* dev = nullptr;
        if ((st = upload(set, F.ies_data, dev))) return st;
        for (uint32_t i = 0; i < L.n_lights; ++i)
            if (L.lights[i].ies) L.lights[i].ies = dev + (F.lights.lights[i].ies - F.ies_data.data());
    }
    if (!F.mesh_light_data.empty()) {  // the mesh lights point into their triangles on the device
        const float* dev = nullptr;
        if ((st = upload(set, F.mesh_light_data, dev))) return st;
        for (uint32_t i = 0; i < L.n_lights; ++i)
            if (L.lights[i].kind == LIGHT_MESH)
                L.lights[i].tris = reinterpret_cast<const float4*>(dev + reinterpret_cast<size_t>(F.lights.lights[i].tris));
    }
    if (L.env_is_map && F.env_image) {
        if ((st = upload(set, F.env_image->texels, L.env_map.texels)) || (st = upload(set, F.env_map.weights, L.env_map.weights)) ||
            (st = upload(set, F.env_map.conditional, L.env_map.conditional)) || (st = upload(set, F.env_map.marginal, L.env_map.marginal)))
            return st;
    }
    S.plate = nullptr;
    if (F.plate && (st = upload(set, F.plate->texels, S.plate))) return st;
    S.exempt_boxes = nullptr;
    if (!F.exempt_boxes.empty() && (st = upload(set, F.exempt_boxes, S.exempt_boxes))) return st;
    RTG_CHECK(cudaMalloc(&set.lights, sizeof(LightsDev)));
    RTG_CHECK(cudaMemcpy(set.lights, &L, sizeof(LightsDev), cudaMemcpyHostToDevice));
    return RTG_STATUS_OK;
}

// Keeps what the adjoint needs on the host: the uploaded materials, the lights' powers and which
// scene light each area light came from.
void keep_shading(Scene& sc, const HScene& hs, const Flat& F) {
    sc.materials_h = F.materials;
    sc.exposure_ev = hs.exposure_ev;
    sc.tonemap = hs.tonemap;
    sc.max_samples = hs.max_samples;
    sc.adaptive = hs.adaptive;
    sc.noise_threshold = hs.noise_threshold;
    sc.light_power.clear();
    for (const HLight& l : hs.lights) sc.light_power.push_back(l.power);
    sc.light_source.clear();
    for (uint32_t i = 0; i < F.lights.n_lights; ++i) sc.light_source.push_back(F.lights.lights[i].source);
}

// The scene constants of `F` with the device pointers and tree fields of `geom` and `shade`.
SceneDev compose(const SceneDev& constants, const SceneDev& geom, const SceneDev& shade) {
    SceneDev S = constants;
    S.nodes = geom.nodes; S.tris = geom.tris; S.blas = geom.blas;
    S.positions = geom.positions; S.normals = geom.normals; S.tri_index = geom.tri_index;
    S.tlas_root = geom.tlas_root; S.stack_need = geom.stack_need;
    S.instances = shade.instances; S.materials = shade.materials; S.bsdfs = shade.bsdfs; S.plate = shade.plate;
    S.exempt_boxes = shade.exempt_boxes;
    S.energy = g_energy;
    S.filter_table = g_filter_table;
    return S;
}

// Device bytes of one path slot: o, d, thr, sum, sel, hit, sh_o, sh_d, sh_c (16 each), flags,
// medium, queue[0], queue[1], sorted, key, sh_key (4 each).
constexpr size_t PATH_BYTES = 9 * 16 + 7 * 4;
// The ray sort's two key histograms with their cursors, at the largest key count.
constexpr size_t SORT_BINS_BYTES = 2 * 2 * (size_t)(8u << (3u * RAY_SORT_MAX_BITS)) * 4;
// The default tuning: no ray sort, material-sorted shading. On the 1080p product frame the sort
// made the extend kernel 4% faster and the frame 3-9% slower (its own passes); rtg_autotune
// measures it per scene.
constexpr uint32_t DEFAULT_RAY_BITS = 0, DEFAULT_SHADOW_SORT = 0, DEFAULT_MATERIAL_SORT = 1;
// The default tail limit (RaySort::tail_paths). On the 1080p product scene a limit of 2^14 made a
// 1-spp frame 20% faster, the adaptive frame 6% and the 64-spp frame no slower; 2^18 and more were
// slower everywhere (the tail kernel takes 8-10x the wavefront's time per path).
constexpr uint32_t DEFAULT_TAIL_PATHS = 1u << 14;
constexpr uint64_t AUTO_MIN_PATHS = 1u << 20;
constexpr uint64_t PLAIN_JOB_PATHS = 1u << 24;  // a queue job this large runs as plain waves
constexpr uint64_t MAX_WAVE_PATHS = 0x7fffffffu;

// Paths one wave of a call may hold: the limit set by rtg_set_path_capacity, or by default every
// path the call renders, bounded by half of the device memory that is free (counting the scene's
// own path buffers). Each wave ends with a tail of long paths that leaves the GPU part-idle, so
// the fewer waves a call takes, the faster it runs: a 1080p frame at 64 spp is one wave of
// 132.7 M paths (22 GB).
// The L2 set-aside for persisting accesses this library asked for (0: none), per device.
size_t g_l2_set_aside[64] = {};

// Whether a scene on device `dev` other than `self` has the L2 window on.
bool other_window_on(int dev, const Scene* self) {
    for (const auto& s : g_scenes)
        if (s && s.get() != self && s->device == dev && s->order.l2_persist) return true;
    return false;
}
// Gives the set-aside back when no scene on `dev` has the window on any longer: L2 set aside for
// persisting lines is not all normal accesses' again until the limit returns to 0 (the 1080p frame
// ran 9% slower after the window had been on once).
void release_set_aside(int dev, const Scene* self) {
    if (dev < 0 || dev >= 64 || g_l2_set_aside[dev] == 0 || other_window_on(dev, self)) return;
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != dev) return;
    cudaCtxResetPersistingL2Cache();
    if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0) == cudaSuccess) g_l2_set_aside[dev] = 0;
    cudaGetLastError();
}

// The ray sort's grid over the scene's sort box at the current bits per axis, and the L2 window
// over its traversal data: at most the device's largest window, persisting for the share of it
// the set-aside holds. The set-aside is asked for when a scene turns the window on, and given back
// when the last scene on the device turns it off or is freed; it is a limit of this process's
// CUDA context.
void refresh_order(Scene& sc) {
    int dev = 0, max_window = 0, max_persist = 0;
    size_t aside = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64) {
        cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, dev);
        cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev);
        const size_t want = sc.order.l2_persist ? std::min<size_t>((size_t)std::max(max_persist, 0), sc.hot_bytes) : 0;
        if (want > g_l2_set_aside[dev] && cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) == cudaSuccess)
            g_l2_set_aside[dev] = want;
        cudaGetLastError();
        if (!sc.order.l2_persist) release_set_aside(dev, &sc);
        aside = g_l2_set_aside[dev];
    }
    sc.order.l2_base = sc.S.nodes;
    sc.order.l2_bytes = std::min<size_t>(sc.hot_bytes, (size_t)std::max(max_window, 0));
    sc.order.l2_hit_ratio = sc.order.l2_bytes ? std::min(1.0f, (float)((double)aside / (double)sc.order.l2_bytes)) : 0.0f;
    const float cells = (float)(1u << sc.order.ray_bits);
    for (int k = 0; k < 3; ++k) {
        const float extent = sc.sort_hi[k] - sc.sort_lo[k];
        const bool ok = extent > 0.0f && extent < 3.0e38f;
        sc.order.lo[k] = ok ? sc.sort_lo[k] : 0.0f;
        sc.order.scale[k] = ok ? cells / extent : 0.0f;
    }
}
void set_sort_box(Scene& sc, const Flat& F) {
    for (int k = 0; k < 3; ++k) {
        sc.sort_lo[k] = F.box_lo[k];
        sc.sort_hi[k] = F.box_hi[k];
    }
    refresh_order(sc);
}

uint64_t wave_limit(const Scene& sc, uint64_t call_paths) {
    if (sc.max_capacity) return sc.max_capacity;
    uint64_t by_memory = AUTO_MIN_PATHS;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess)
        by_memory = std::max<uint64_t>(AUTO_MIN_PATHS, (free_b + sc.path_mem.bytes) / 2 / PATH_BYTES);
    return std::max<uint64_t>(1, std::min<uint64_t>(std::min(call_paths, by_memory), MAX_WAVE_PATHS));
}

uint32_t ensure_capacity(Scene& sc, uint32_t paths) {
    if (paths <= sc.capacity) return RTG_STATUS_OK;
    sc.path_mem.release();
    sc.capacity = 0;
    size_t n = paths;
    size_t bytes = n * PATH_BYTES + 17 * 256 + 256 + 512 * 4 + SORT_BINS_BYTES;
    RTG_CHECK(cudaMalloc(&sc.path_mem.p, bytes));
    sc.path_mem.bytes = bytes;
    uint8_t* p = (uint8_t*)sc.path_mem.p;
    auto take = [&](size_t each) { uint8_t* r = p; p += ((n * each + 255) / 256) * 256; return r; };
    // (sizes rounded to 256 bytes; `bytes` above leaves room for the rounding of 14 arrays)
    sc.P.o = (float4*)take(16);
    sc.P.d = (float4*)take(16);
    sc.P.thr = (float4*)take(16);
    sc.P.sum = (float4*)take(16);
    sc.P.sel = (float4*)take(16);
    sc.P.flags = (uint32_t*)take(4);
    sc.P.medium = (uint32_t*)take(4);
    sc.P.hit = (uint4*)take(16);
    sc.P.queue[0] = (uint32_t*)take(4);
    sc.P.queue[1] = (uint32_t*)take(4);
    sc.P.sorted = (uint32_t*)take(4);
    sc.P.key = (uint32_t*)take(4);
    sc.P.bins = (uint32_t*)p;
    p += 512 * 4;
    sc.P.sh_o = (float4*)take(16);
    sc.P.sh_d = (float4*)take(16);
    sc.P.sh_c = (float4*)take(16);
    sc.P.sh_key = (uint32_t*)take(4);
    sc.P.rbins = (uint32_t*)p;
    sc.P.sbins = sc.P.rbins + SORT_BINS_BYTES / 8;
    p += SORT_BINS_BYTES;
    RTG_CHECK(cudaMemsetAsync(sc.P.rbins, 0, SORT_BINS_BYTES, sc.stream));  // histograms start at zero
    sc.P.counters = (uint32_t*)p;
    p += 64;
    sc.P.rays = (unsigned long long*)p;
    p += 64;
    if ((size_t)(p - (uint8_t*)sc.path_mem.p) > bytes) { g_error = "internal: path buffer layout"; return RTG_STATUS_CUDA_ERROR; }
    sc.capacity = paths;
    return RTG_STATUS_OK;
}

int grid_for(uint32_t n, int per_block) {
    long g = ((long)n + per_block - 1) / per_block;
    long cap = (long)g_sms * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// Runs one wave and (when timing) adds the extend-kernel time.
// `S` (default: the scene's) gives the launch its bounce count; batched waves pass the deepest job's.
uint32_t run_wave(Scene& sc, const WaveDesc& w, const FilmDev* film, const SceneDev* S = nullptr, const LightsDev* lights = nullptr) {
    const SceneDev& Sw = S ? *S : sc.S;
    WaveTiming* t = nullptr;
    if (sc.timing) {
        if (!sc.wt) {
            sc.wt = new WaveTiming();
            for (int i = 0; i < WaveTiming::MAX_EVENTS; ++i) RTG_CHECK(cudaEventCreate(&sc.wt->ev[i]));
        }
        sc.wt->ev_count = 0;
        t = sc.wt;
    }
    launch_wave(Sw, lights ? lights : sc.d_lights, w, sc.P, film, sc.stream, grid_for(w.n, 128), t, sc.order);
    RTG_CHECK(cudaGetLastError());
    sc.launches += wave_launches(Sw, sc.order, sc.P, w.segs != nullptr) - ((film || w.segs) ? 0 : 1) + ((w.alb && film && !w.segs) ? 2 : 0);
    if (t) {
        RTG_CHECK(cudaStreamSynchronize(sc.stream));
        for (int i = 0; i + 1 < t->ev_count; i += 2) {
            float ms = 0;
            RTG_CHECK(cudaEventElapsedTime(&ms, t->ev[i], t->ev[i + 1]));
            sc.extend_ms += ms;
            sc.extend_launches += 1;
        }
    }
    return RTG_STATUS_OK;
}

uint32_t finish(Scene& sc, uint64_t* rays_out) {
    uint32_t counters[4];
    unsigned long long rays[2] = {0, 0};
    RTG_CHECK(cudaMemcpyAsync(counters, sc.P.counters, 16, cudaMemcpyDeviceToHost, sc.stream));
    RTG_CHECK(cudaMemcpyAsync(rays, sc.P.rays, 16, cudaMemcpyDeviceToHost, sc.stream));
    RTG_CHECK(cudaStreamSynchronize(sc.stream));
    if (counters[3] & 1u) { g_error = "traversal stack overflow"; return RTG_STATUS_STACK_OVERFLOW; }
    if (rays_out) *rays_out = rays[0] + rays[1];
    sc.rays += rays[0] + rays[1];
    sc.extend_rays += rays[0];
    sc.shadow_rays += rays[1];
    return RTG_STATUS_OK;
}

// The image's edge mask on the device (built once per scene state, pixel_filter.rs:175), with an
// edge-pixel list and its count after it.
uint32_t edge_mask_of(Scene& sc, const uint8_t*& mask, uint32_t*& list, uint32_t*& count) {
    const size_t npix = (size_t)sc.width * sc.height;
    const size_t mask_bytes = (npix + 15) & ~(size_t)15;
    const size_t need = mask_bytes + npix * sizeof(uint4) + npix * 4 + 16;
    if (sc.edge_mem.bytes < need) {
        sc.edge_mem.release();
        RTG_CHECK(cudaMalloc(&sc.edge_mem.p, need));
        sc.edge_mem.bytes = need;
        sc.edges_ready = false;
    }
    uint8_t* base = (uint8_t*)sc.edge_mem.p;
    uint8_t* m = base;
    uint4* exact = (uint4*)(base + mask_bytes);
    list = (uint32_t*)(base + mask_bytes + npix * sizeof(uint4));
    count = list + npix;
    if (!sc.edges_ready) {
        RTG_CHECK(launch_edge_mask(sc.S, sc.d_lights, exact, m, sc.stream, grid_for(npix, 128)));
        sc.launches += 2;
        sc.edges_ready = true;
        sc.edge_builds += 1;
    }
    mask = m;
    return RTG_STATUS_OK;
}

// The edge pixels of the rectangle (x, y, w, h): the image's edge mask, their packed list on the
// device and their count.
uint32_t edge_pixels(Scene& sc, uint32_t x, uint32_t y, uint32_t w, uint32_t h, const uint8_t*& mask, const uint32_t*& list,
                     uint32_t& count) {
    uint32_t *l = nullptr, *c = nullptr;
    const uint32_t st = edge_mask_of(sc, mask, l, c);
    if (st) return st;
    RTG_CHECK(launch_edge_list(mask, sc.width, x, y, w, h, l, c, sc.stream, grid_for((uint64_t)w * h, 256)));
    sc.launches += 1;
    RTG_CHECK(cudaMemcpyAsync(&count, c, 4, cudaMemcpyDeviceToHost, sc.stream));
    RTG_CHECK(cudaStreamSynchronize(sc.stream));
    list = l;
    return RTG_STATUS_OK;
}

// Renders samples [first, first + count) of the image rectangle (x, y, w, h) (clipped to the
// image) into `film`, every pixel's samples added in index order.
uint32_t render_region(Scene& sc, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t first, uint32_t count, const FilmDev& film,
                       uint64_t* rays_out, float* guide_sum = nullptr, float* guide_weight = nullptr) {
    uint64_t x_end = std::min<uint64_t>((uint64_t)x + w, sc.width), y_end = std::min<uint64_t>((uint64_t)y + h, sc.height);
    if (rays_out) *rays_out = 0;
    if (x >= x_end || y >= y_end || count == 0) return RTG_STATUS_OK;
    uint32_t cw = (uint32_t)(x_end - x), ch = (uint32_t)(y_end - y);
    uint64_t npix = (uint64_t)cw * ch;
    // Rows per band so that one band of one sample fits a wave.
    const uint64_t cap = wave_limit(sc, npix * count);
    uint32_t band_rows = ch;
    if (npix > cap) band_rows = std::max<uint32_t>(1, (uint32_t)(cap / cw));
    uint64_t total_rays = 0;
    for (uint32_t by = 0; by < ch; by += band_rows) {
        uint32_t bh = std::min(band_rows, ch - by);
        uint64_t bpix = (uint64_t)cw * bh;
        uint32_t per_wave = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(count, cap / bpix));
        uint32_t need = (uint32_t)(bpix * per_wave);
        // Edge samples (E11): the band's edge pixels splat from edge waves of their own, the
        // mean of k samples per sample index (render.rs:477); the rectangle waves skip them. The
        // edge waves take as many edge pixels (k samples each) and sample indices as fit.
        const uint8_t* mask = nullptr;
        const uint32_t* elist = nullptr;
        uint32_t ne = 0, chunk = 0;
        const uint32_t k = sc.S.edge_k;
        uint32_t st;
        if (k > 1 && (st = edge_pixels(sc, x, y + by, cw, bh, mask, elist, ne))) return st;
        if (ne) {
            chunk = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(ne, cap / k));
            need = std::max<uint32_t>(need, (uint32_t)((uint64_t)chunk * k));
        }
        st = ensure_capacity(sc, need);
        if (st) return st;
        if (guide_sum && sc.alb_mem.bytes < (size_t)sc.capacity * 16) {
            sc.alb_mem.release();
            RTG_CHECK(cudaMalloc(&sc.alb_mem.p, (size_t)sc.capacity * 16));
            sc.alb_mem.bytes = (size_t)sc.capacity * 16;
        }
        auto guides = [&](WaveDesc& wd) {
            if (!guide_sum) return;
            wd.alb = (float4*)sc.alb_mem.p;
            wd.guide_sum = guide_sum;
            wd.guide_weight = guide_weight;
        };
        RTG_CHECK(cudaMemsetAsync(sc.P.counters, 0, 16, sc.stream));
        RTG_CHECK(cudaMemsetAsync(sc.P.rays, 0, 16, sc.stream));
        for (uint32_t s = 0; s < count; s += per_wave) {
            uint32_t ns = std::min(per_wave, count - s);
            WaveDesc wd{x, y + by, cw, bh, first + s, (uint32_t)(bpix * ns), nullptr};
            if (ne) {
                wd.edge = mask;
                wd.edge_stride = sc.width;
            }
            guides(wd);
            st = run_wave(sc, wd, &film);
            if (st) return st;
        }
        for (uint32_t e0 = 0; e0 < ne; e0 += chunk) {
            const uint32_t en = std::min(chunk, ne - e0);
            const uint32_t per_edge_wave = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(count, sc.capacity / ((uint64_t)en * k)));
            for (uint32_t s = 0; s < count; s += per_edge_wave) {
                const uint32_t ns = std::min(per_edge_wave, count - s);
                WaveDesc wd{x, y + by, cw, bh, first + s, (uint32_t)((uint64_t)en * k * ns), nullptr};
                wd.epix = elist + e0;
                wd.ne = en;
                wd.ek = k;
                guides(wd);
                st = run_wave(sc, wd, &film);
                if (st) return st;
            }
        }
        uint64_t r = 0;
        st = finish(sc, &r);
        if (st) return st;
        total_rays += r;
    }
    if (rays_out) *rays_out = total_rays;
    return RTG_STATUS_OK;
}

uint32_t make_film(uint32_t ox, uint32_t oy, uint32_t w, uint32_t h, Film& f) {
    size_t n = (size_t)w * h;
    f.mem.bytes = n * 6 * 4;
    RTG_CHECK(cudaMalloc(&f.mem.p, f.mem.bytes));
    RTG_CHECK(cudaMemset(f.mem.p, 0, f.mem.bytes));
    float* p = (float*)f.mem.p;
    f.dev = FilmDev{ox, oy, w, h, p, p + 3 * n, p + 4 * n, p + 5 * n};
    return RTG_STATUS_OK;
}

// Registers a new zeroed film over (x, y, w, h) of scene `handle`: its handle, or 0.
uint32_t new_film(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h) {
    auto f = std::make_unique<Film>();
    f->scene = handle;
    if (make_film(x, y, w, h, *f) != RTG_STATUS_OK) return 0;
    for (size_t i = 0; i < g_films.size(); ++i)
        if (!g_films[i]) { g_films[i] = std::move(f); return (uint32_t)i + 1; }
    g_films.push_back(std::move(f));
    return (uint32_t)g_films.size();
}

uint32_t render_tile_impl(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t sample, float* out, bool rgba) {
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    uint64_t px = (uint64_t)w * h;
    if (px == 0 || px > RTG_MAX_TILE_PIXELS) return RTG_STATUS_BAD_TILE;
    if (!out) return RTG_STATUS_NULL_POINTER;
    Film f;
    f.scene = handle;
    uint32_t st = make_film(x, y, w, h, f);
    if (st) return st;
    st = render_region(*sc, x, y, w, h, sample, 1, f.dev, nullptr);
    if (st) return st;
    std::vector<float> buf(px * 6);
    RTG_CHECK(cudaMemcpyAsync(buf.data(), f.mem.p, px * 6 * 4, cudaMemcpyDeviceToHost, sc->stream));
    RTG_CHECK(cudaStreamSynchronize(sc->stream));
    const float* rgb = buf.data();
    const float* wt = rgb + 3 * px;
    const float* al = rgb + 4 * px;
    for (uint64_t i = 0; i < px; ++i) {
        float inv = wt[i] > 0.0f ? 1.0f / wt[i] : 0.0f;
        size_t o = rgba ? 4 * i : 3 * i;
        for (int c = 0; c < 3; ++c) out[o + c] = wt[i] > 0.0f ? rgb[3 * i + c] * inv : 0.0f;
        if (rgba) out[o + 3] = wt[i] > 0.0f ? al[i] * inv : 0.0f;
    }
    return RTG_STATUS_OK;
}

// ---- adaptive sampling (E10, adaptive.rs:318-551) --------------------------------------------------
// An adaptive render: the round state on the host (each block's samples when the round began,
// the blocks of the round and its size, the samples of it rendered so far, the photon-map
// iteration, the cap, the noise target, the floor of the mean) and the device buffers of the
// decision and of the pass lists; the film lives on the device and covers the whole image.
struct AdaptiveRun {
    uint32_t scene = 0, film = 0;
    uint32_t width = 0, height = 0, cols = 0, rows = 0;
    std::vector<uint32_t> counts;
    std::vector<uint8_t> active;
    uint32_t round = 0, done = 0, iteration = 0, cap = 0, decisions = 0;
    float target = 0.0f, floor = 0.0f;
    AdDecision last;
    // per block: its plain and its edge pixels, for the edge factor and mask they were found with
    std::vector<uint32_t> pixels;
    uint32_t pixels_k = 0;
    uint64_t pixels_mask = 0;
    DevBuf mem;
    uint32_t* d_counts = nullptr;
    float* d_error = nullptr;
    AdEntry* d_entries = nullptr;
    uint32_t *d_pixels = nullptr, *d_plain = nullptr, *d_plain_base = nullptr, *d_edge = nullptr, *d_edge_base = nullptr;
    size_t blocks() const { return counts.size(); }
    uint32_t left() const { return round - done; }
    uint32_t quota(size_t b) const {  // adaptive.rs:409
        if (!active[b]) return 0;
        if (cap > 0) return std::min(round, cap > counts[b] ? cap - counts[b] : 0u);
        return round;
    }
    uint32_t samples_of(size_t b) const { return counts[b] + std::min(quota(b), done); }
    ~AdaptiveRun() { mem.release(); }
};
std::vector<std::unique_ptr<AdaptiveRun>> g_adaptive;
AdaptiveRun* adaptive_of(uint32_t h) { return (h == 0 || h > g_adaptive.size()) ? nullptr : g_adaptive[h - 1].get(); }

// The end of a round (adaptive.rs:513): its samples counted, the iteration moved past it, and the
// image's decision of the next one: block errors on the device from the film where it lies, the
// choice on the host.
uint32_t adaptive_decide_round(Scene& sc, const Film& f, AdaptiveRun& a) {
    for (size_t b = 0; b < a.blocks(); ++b) a.counts[b] += a.quota(b);
    a.iteration += a.round;
    a.done = 0;
    const size_t nb = a.blocks();
    RTG_CHECK(cudaMemcpyAsync(a.d_counts, a.counts.data(), nb * 4, cudaMemcpyHostToDevice, sc.stream));
    RTG_CHECK(launch_block_error(f.dev.rgb, 3, f.dev.lum2, a.d_counts, a.width, a.height, a.floor, a.d_error, sc.stream,
                                 grid_for((uint32_t)nb, 1)));
    sc.launches += 1;
    std::vector<float> err(nb);
    RTG_CHECK(cudaMemcpyAsync(err.data(), a.d_error, nb * 4, cudaMemcpyDeviceToHost, sc.stream));
    RTG_CHECK(cudaStreamSynchronize(sc.stream));
    a.last = ad_decide_blocks(a.width, a.height, a.counts.data(), err.data(), a.target, a.cap, a.active);
    a.round = a.last.round;
    a.decisions += 1;
    return RTG_STATUS_OK;
}

// Waves over `n` listed pixels (k samples a sample index, first sample index `first` past each
// entry's base), `count` sample indices, each wave at most `cap` paths.
uint32_t list_waves(Scene& sc, const FilmDev& film, const uint32_t* list, const uint32_t* base, uint32_t n, uint32_t k, uint32_t first,
                    uint32_t count, uint64_t cap) {
    if (n == 0 || count == 0) return RTG_STATUS_OK;
    const uint32_t chunk = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(n, cap / k));
    for (uint32_t e0 = 0; e0 < n; e0 += chunk) {
        const uint32_t en = std::min(chunk, n - e0);
        const uint32_t per = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(count, cap / ((uint64_t)en * k)));
        for (uint32_t s = 0; s < count; s += per) {
            const uint32_t ns = std::min(per, count - s);
            WaveDesc wd{0, 0, sc.width, sc.height, first + s, (uint32_t)((uint64_t)en * k * ns), nullptr};
            wd.epix = list + e0;
            wd.ne = en;
            wd.ek = k;
            wd.ebase = base + e0;
            const uint32_t st = run_wave(sc, wd, &film);
            if (st) return st;
        }
    }
    return RTG_STATUS_OK;
}

// A pass of `count` samples of the round (adaptive.rs:471 work): the first round renders the whole
// image as the progressive renderer does (every block active, sample indices from 0, the same
// pixels); a later one renders the pixels of its active blocks from lists, the blocks with the most
// samples to go first, so that sample s of the pass covers a prefix of the lists.
uint32_t adaptive_pass(Scene& sc, const Film& f, AdaptiveRun& a, uint32_t count, uint64_t& rays) {
    rays = 0;
    if (a.decisions == 0) return render_region(sc, 0, 0, a.width, a.height, a.iteration + a.done, count, f.dev, &rays);
    const size_t nb = a.blocks();
    const uint32_t k = sc.S.edge_k > 1 ? sc.S.edge_k : 1;
    const uint8_t* mask = nullptr;
    if (k > 1) {
        uint32_t *l = nullptr, *c = nullptr;
        const uint32_t st = edge_mask_of(sc, mask, l, c);
        if (st) return st;
    }
    // Each block's plain and edge pixels: its size inside the image without edge samples, else
    // counted on the device once per edge mask.
    if (a.pixels.size() != 2 * nb || a.pixels_k != k || (k > 1 && a.pixels_mask != sc.edge_builds)) {
        a.pixels.assign(2 * nb, 0);
        if (k > 1) {
            RTG_CHECK(launch_block_pixels(mask, a.width, a.height, a.d_pixels, sc.stream, grid_for((uint32_t)nb, 128)));
            sc.launches += 1;
            RTG_CHECK(cudaMemcpyAsync(a.pixels.data(), a.d_pixels, nb * 8, cudaMemcpyDeviceToHost, sc.stream));
            RTG_CHECK(cudaStreamSynchronize(sc.stream));
        } else {
            for (size_t b = 0; b < nb; ++b)
                a.pixels[2 * b] = std::min(AD_BLOCK, a.width - (uint32_t)(b % a.cols) * AD_BLOCK) *
                                  std::min(AD_BLOCK, a.height - (uint32_t)(b / a.cols) * AD_BLOCK);
        }
        a.pixels_k = k;
        a.pixels_mask = sc.edge_builds;
    }
    const std::vector<uint32_t>& pixels = a.pixels;
    std::vector<std::pair<uint32_t, uint32_t>> order;  // (quota, block)
    for (size_t b = 0; b < nb; ++b) {
        const uint32_t q = a.quota(b);
        if (q > a.done) order.push_back({q, (uint32_t)b});
    }
    if (order.empty()) return RTG_STATUS_OK;
    std::stable_sort(order.begin(), order.end(), [](const auto& p, const auto& q) { return p.first > q.first; });
    std::vector<AdEntry> entries(order.size());
    std::vector<uint32_t> plain_end(order.size()), edge_end(order.size());
    uint32_t off_p = 0, off_e = 0;
    uint64_t total = 0;
    for (size_t i = 0; i < order.size(); ++i) {
        const uint32_t b = order[i].second;
        entries[i] = AdEntry{b, a.counts[b], off_p, off_e};
        off_p += pixels[2 * b];
        off_e += pixels[2 * b + 1];
        plain_end[i] = off_p;
        edge_end[i] = off_e;
        total += (uint64_t)std::min(order[i].first - a.done, count) * (pixels[2 * b] + (uint64_t)k * pixels[2 * b + 1]);
    }
    RTG_CHECK(cudaMemcpyAsync(a.d_entries, entries.data(), entries.size() * sizeof(AdEntry), cudaMemcpyHostToDevice, sc.stream));
    RTG_CHECK(launch_block_expand(a.d_entries, (uint32_t)entries.size(), mask, a.width, a.height, a.d_plain, a.d_plain_base, a.d_edge,
                                  a.d_edge_base, sc.stream, grid_for((uint32_t)entries.size(), 1)));
    sc.launches += 1;
    const uint64_t cap = std::max<uint64_t>(std::min<uint64_t>(wave_limit(sc, total), total), off_e ? k : 1);
    uint32_t st = ensure_capacity(sc, (uint32_t)cap);
    if (st) return st;
    RTG_CHECK(cudaMemsetAsync(sc.P.counters, 0, 16, sc.stream));
    RTG_CHECK(cudaMemsetAsync(sc.P.rays, 0, 16, sc.stream));
    // Sample s of the pass covers the entries whose quota is above done + s: a prefix.
    size_t n_in = order.size();
    for (uint32_t s = 0; s < count;) {
        while (n_in > 0 && order[n_in - 1].first <= a.done + s) --n_in;
        if (n_in == 0) break;
        const uint32_t s1 = std::min(count, order[n_in - 1].first - a.done);
        st = list_waves(sc, f.dev, a.d_plain, a.d_plain_base, plain_end[n_in - 1], 1, a.done + s, s1 - s, cap);
        if (st) return st;
        st = list_waves(sc, f.dev, a.d_edge, a.d_edge_base, edge_end[n_in - 1], k, a.done + s, s1 - s, cap);
        if (st) return st;
        s = s1;
    }
    return finish(sc, &rays);
}

}  // namespace
}  // namespace rtg

using namespace rtg;

extern "C" {

uint32_t rtg_version(void) { return RTG_ABI_VERSION; }

uint32_t rtg_features(void) { return RTG_FEATURE_SECTION | RTG_FEATURE_IES | RTG_FEATURE_CAMERAS; }

uint32_t rtg_scene_load(const uint8_t* bytes, uint32_t len) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!bytes) { g_error = "null pointer"; return 0; }
    // The scene is parsed, checked and flattened on the host before any device work, so a
    // malformed or unsupported scene is refused the same way with or without a GPU.
    HScene hs;
    std::string err;
    if (!parse_rsb(bytes, len, hs, err)) { g_error = err; return 0; }
    Flat F;
    if (!flatten_scene(hs, F, err)) { g_error = err; return 0; }
    if (device_init() != RTG_STATUS_OK) return 0;
    auto sc = std::make_unique<Scene>();
    if (cudaStreamCreateWithFlags(&sc->stream, cudaStreamNonBlocking) != cudaSuccess) { g_error = "cudaStreamCreate failed"; return 0; }
    if (cudaGetDevice(&sc->device) != cudaSuccess) sc->device = -1;
    SceneDev geom = F.scene, shade = F.scene;
    if (upload_geometry(F, sc->geometry, geom, &sc->hot_bytes) || upload_shading(F, sc->shading, shade)) return 0;
    sc->S = compose(F.scene, geom, shade);
    sc->d_lights = sc->shading.lights;
    sc->geom_key = geometry_key(hs);
    keep_shading(*sc, hs, F);
    sc->meshes = std::move(hs.meshes);
    sc->bitmaps = std::move(hs.bitmaps);
    sc->build_seconds = F.build_seconds;
    sc->nodes = F.nodes.size();
    sc->tris = F.tris.size();
    sc->instanced_triangles = F.instanced_triangles;
    sc->width = F.scene.width;
    sc->height = F.scene.height;
    sc->max_depth = F.scene.max_depth;
    sc->order.ray_bits = DEFAULT_RAY_BITS;
    sc->order.shadow_sort = DEFAULT_SHADOW_SORT;
    sc->order.material_sort = DEFAULT_MATERIAL_SORT;
    sc->order.tail_paths = DEFAULT_TAIL_PATHS;
    set_sort_box(*sc, F);
    g_error.clear();
    for (size_t i = 0; i < g_scenes.size(); ++i)
        if (!g_scenes[i]) { g_scenes[i] = std::move(sc); return (uint32_t)i + 1; }
    g_scenes.push_back(std::move(sc));
    return (uint32_t)g_scenes.size();
}

uint32_t rtg_scene_update(uint32_t handle, const uint8_t* bytes, uint32_t len) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    if (!bytes) { g_error = "rtg_scene_update: null pointer"; return RTG_STATUS_NULL_POINTER; }
    HScene hs;
    std::string err;
    bool kept = false;
    if (!parse_rsb(bytes, len, hs, err, &sc->meshes, &kept, &sc->bitmaps)) { g_error = err; return RTG_STATUS_BAD_SCENE; }
    std::string key = geometry_key(hs);
    const bool same_geometry = kept && key == sc->geom_key;
    Flat F;
    if (!flatten_scene(hs, F, err, !same_geometry)) { g_error = err; return RTG_STATUS_BAD_SCENE; }
    // Everything new is uploaded first; the scene changes only once all of it is on the device.
    RTG_CHECK(cudaStreamSynchronize(sc->stream));
    BufSet geometry, shading;
    SceneDev geom = sc->S, shade = F.scene;
    size_t hot = sc->hot_bytes;
    uint32_t st = same_geometry ? RTG_STATUS_OK : upload_geometry(F, geometry, geom, &hot);
    if (!st) st = upload_shading(F, shading, shade);
    if (st) {
        geometry.release();
        shading.release();
        return st;
    }
    if (same_geometry) {
        geom.tlas_root = sc->S.tlas_root;
        geom.stack_need = sc->S.stack_need;
    } else {
        geom.tlas_root = F.scene.tlas_root;
        geom.stack_need = F.scene.stack_need;
        set_sort_box(*sc, F);
        sc->hot_bytes = hot;
        sc->geometry.release();
        sc->geometry = std::move(geometry);
        sc->nodes = F.nodes.size();
        sc->tris = F.tris.size();
        sc->build_seconds = F.build_seconds;
    }
    sc->shading.release();
    sc->shading = std::move(shading);
    sc->edges_ready = false;
    sc->S = compose(F.scene, geom, shade);
    sc->d_lights = sc->shading.lights;
    refresh_order(*sc);  // the L2 window follows the geometry
    keep_shading(*sc, hs, F);
    if (!kept) sc->meshes = std::move(hs.meshes);
    sc->bitmaps = std::move(hs.bitmaps);
    sc->geom_key = std::move(key);
    sc->instanced_triangles = F.instanced_triangles;
    sc->width = F.scene.width;
    sc->height = F.scene.height;
    sc->max_depth = F.scene.max_depth;
    g_error.clear();
    return RTG_STATUS_OK;
}

uint32_t rtg_scene_error_len(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    return (uint32_t)g_error.size();
}
void rtg_scene_error_copy(uint8_t* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (out) std::memcpy(out, g_error.data(), g_error.size());
}

uint32_t rtg_scene_free(uint32_t handle) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!scene_of(handle)) return RTG_STATUS_BAD_HANDLE;
    Scene* sc = g_scenes[handle - 1].get();
    cudaStreamSynchronize(sc->stream);
    const int dev = sc->device;
    const bool window = sc->order.l2_persist != 0;
    g_scenes[handle - 1].reset();
    if (window) release_set_aside(dev, nullptr);
    return RTG_STATUS_OK;
}

uint32_t rtg_render_tile(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t sample_index, float* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    return render_tile_impl(handle, x, y, w, h, sample_index, out, false);
}
uint32_t rtg_render_tile_rgba(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t sample_index, float* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    return render_tile_impl(handle, x, y, w, h, sample_index, out, true);
}

uint32_t rtg_film_create(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!scene_of(handle)) { g_error = "bad scene handle"; return 0; }
    if ((uint64_t)w * h == 0 || (uint64_t)w * h > (1ull << 28)) { g_error = "bad film size"; return 0; }
    return new_film(handle, x, y, w, h);
}
uint32_t rtg_film_free(uint32_t film) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!film_of(film)) return RTG_STATUS_BAD_FILM;
    cudaDeviceSynchronize();
    g_films[film - 1].reset();
    return RTG_STATUS_OK;
}
uint32_t rtg_film_clear(uint32_t film) {
    std::lock_guard<std::mutex> lk(g_mu);
    Film* f = film_of(film);
    if (!f) return RTG_STATUS_BAD_FILM;
    Scene* sc = scene_of(f->scene);
    RTG_CHECK(cudaMemsetAsync(f->mem.p, 0, f->mem.bytes, sc ? sc->stream : 0));
    if (f->guides.p) RTG_CHECK(cudaMemsetAsync(f->guides.p, 0, f->guides.bytes, sc ? sc->stream : 0));
    if (sc) RTG_CHECK(cudaStreamSynchronize(sc->stream));
    return RTG_STATUS_OK;
}
uint32_t rtg_render_progressive(uint32_t handle, uint32_t film, uint32_t first_sample, uint32_t count, uint64_t* rays) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    Film* f = film_of(film);
    if (!f || f->scene != handle) return RTG_STATUS_BAD_FILM;
    if (f->fuse_guides)
        return render_region(*sc, f->dev.ox, f->dev.oy, f->dev.w, f->dev.h, first_sample, count, f->dev, rays, f->albedo_sum(),
                             f->albedo_weight());
    return render_region(*sc, f->dev.ox, f->dev.oy, f->dev.w, f->dev.h, first_sample, count, f->dev, rays);
}
uint32_t rtg_render_progressive_noalloc(uint32_t handle, uint32_t film, uint32_t first_sample, uint32_t count,
                                        uint64_t* rays) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    Film* f = film_of(film);
    if (!f || f->scene != handle) return RTG_STATUS_BAD_FILM;
    if (rays) *rays = 0;
    if (sc->S.edge_k > 1) {
        g_error = "rtg_render_progressive_noalloc: unsupported: edge samples (their mask needs device memory)";
        return RTG_STATUS_BAD_SCENE;
    }
    NoallocJob job{&sc->S, sc->d_lights, f->dev, sc->width, sc->height, first_sample, count, sc->stream, g_sms};
    if (f->fuse_guides) {
        job.guide_sum = f->albedo_sum();
        job.guide_weight = f->albedo_weight();
    }
    NoallocResult res;
    const char* why = "";
    uint32_t st = noalloc_render(job, res, &why);
    if (st) { g_error = why; return st; }
    sc->launches += res.waves * (2 + 6 * (uint64_t)wave_rounds(sc->S) + (job.guide_sum ? 2 : 0));
    sc->rays += res.extend_rays + res.shadow_rays;
    sc->extend_rays += res.extend_rays;
    sc->shadow_rays += res.shadow_rays;
    if (rays) *rays = res.extend_rays + res.shadow_rays;
    return RTG_STATUS_OK;
}
uint32_t rtg_queue_create(uint32_t scene) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!scene_of(scene)) { g_error = "bad scene handle"; return 0; }
    auto q = std::make_unique<Queue>();
    q->scene = scene;
    for (size_t i = 0; i < g_queues.size(); ++i)
        if (!g_queues[i]) { g_queues[i] = std::move(q); return (uint32_t)i + 1; }
    g_queues.push_back(std::move(q));
    return (uint32_t)g_queues.size();
}

uint32_t rtg_queue_free(uint32_t queue) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!queue_of(queue)) return RTG_STATUS_BAD_HANDLE;
    Scene* sc = scene_of(g_queues[queue - 1]->scene);
    if (sc) cudaStreamSynchronize(sc->stream);
    g_queues[queue - 1].reset();
    return RTG_STATUS_OK;
}

uint32_t rtg_queue_add(uint32_t queue, const uint8_t* bytes, uint32_t len, uint32_t first_sample, uint32_t count, uint32_t* film) {
    std::lock_guard<std::mutex> lk(g_mu);
    Queue* q = queue_of(queue);
    Scene* sc = q ? scene_of(q->scene) : nullptr;
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    if (!bytes || !film) { g_error = "rtg_queue_add: null pointer"; return RTG_STATUS_NULL_POINTER; }
    *film = 0;
    HScene hs;
    std::string err;
    bool kept = false;
    if (!parse_rsb(bytes, len, hs, err, &sc->meshes, &kept, &sc->bitmaps)) { g_error = err; return RTG_STATUS_BAD_SCENE; }
    std::string key = geometry_key(hs);
    if (!kept || key != sc->geom_key) {
        g_error = "a queue job keeps the scene's geometry: no MESH sections, the same instances";
        return RTG_STATUS_BAD_SCENE;
    }
    Flat F;
    if (!flatten_scene(hs, F, err, false)) { g_error = err; return RTG_STATUS_BAD_SCENE; }
    if (F.scene.edge_k > 1) { g_error = "unsupported in the batched queue: edge samples"; return RTG_STATUS_BAD_SCENE; }
    // The queue's traversal reads the shared scene's constants, so a job cannot bring a section.
    if (F.scene.section_on || sc->S.section_on) { g_error = "unsupported in the batched queue: a section view"; return RTG_STATUS_BAD_SCENE; }
    auto job = std::make_unique<QueueJob>();
    job->constants = F.scene;
    job->shade = F.scene;
    uint32_t st = upload_shading(F, job->shading, job->shade);
    if (st) { job->shading.release(); return st; }
    job->geom_key = std::move(key);
    job->first = first_sample;
    job->count = count;
    job->width = F.scene.width;
    job->height = F.scene.height;
    job->film = new_film(q->scene, 0, 0, job->width, job->height);
    if (!job->film) { job->shading.release(); return RTG_STATUS_CUDA_ERROR; }
    *film = job->film;
    q->jobs.push_back(std::move(job));
    g_error.clear();
    return RTG_STATUS_OK;
}

namespace rtg {
namespace {
// Packs the queue's jobs into waves of at most `cap` paths. A job gives each wave one segment at
// most (whole images over a run of samples, or a band of rows of one sample), so a pixel receives
// its samples in index order: wave by wave, and within a wave from one segment only.
void pack_waves(const std::vector<std::unique_ptr<QueueJob>>& jobs, uint64_t cap, std::vector<std::vector<SegDev>>& waves,
                std::vector<uint64_t>& wave_paths, const std::vector<uint8_t>& skip) {
    std::vector<SegDev> cur;
    uint64_t used = 0;
    auto flush = [&]() {
        if (cur.empty()) return;
        waves.push_back(cur);
        wave_paths.push_back(used);
        cur.clear();
        used = 0;
    };
    for (uint32_t j = 0; j < jobs.size(); ++j) {
        if (j < skip.size() && skip[j]) continue;
        const QueueJob& J = *jobs[j];
        const uint64_t W = J.width, H = J.height, npix = W * H;
        uint32_t s = J.first, row = 0;
        const uint32_t s_end = J.first + J.count;
        while (s < s_end) {
            uint64_t space = cap - used;
            SegDev g{};
            g.job = j;
            g.w = (uint32_t)W;
            if (row == 0 && space >= npix) {
                uint64_t ns = std::min<uint64_t>(s_end - s, space / npix);
                g.y0 = 0; g.h = (uint32_t)H; g.first = s; g.ns = (uint32_t)ns;
                s += (uint32_t)ns;
            } else if (space >= W) {
                uint64_t rows = std::min<uint64_t>(H - row, space / W);
                g.y0 = row; g.h = (uint32_t)rows; g.first = s; g.ns = 1;
                row += (uint32_t)rows;
                if (row == H) { row = 0; ++s; }
            } else {
                flush();
                continue;
            }
            g.slot_begin = (uint32_t)used;
            uint64_t seg_pix = (uint64_t)g.w * g.h;
            g.pix_begin = cur.empty() ? 0 : cur.back().pix_begin + cur.back().w * cur.back().h;
            cur.push_back(g);
            used += seg_pix * g.ns;
            if (s < s_end) flush();  // the job goes on: its next segment belongs to the next wave
        }
    }
    flush();
}
}  // namespace
}  // namespace rtg

uint32_t rtg_queue_run(uint32_t queue, uint32_t flags, uint64_t* rays) {
    std::lock_guard<std::mutex> lk(g_mu);
    Queue* q = queue_of(queue);
    Scene* sc = q ? scene_of(q->scene) : nullptr;
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    if (rays) *rays = 0;
    // Jobs and their films as the device reads them; the geometry is the scene's as it is now.
    std::vector<JobDev> jobs_h(q->jobs.size());
    SceneDev Sw = sc->S;
    uint64_t total = 0;
    for (size_t j = 0; j < q->jobs.size(); ++j) {
        QueueJob& J = *q->jobs[j];
        Film* f = film_of(J.film);
        if (!f) { g_error = "a queue job's film was freed"; return RTG_STATUS_BAD_FILM; }
        if (J.geom_key != sc->geom_key) { g_error = "the scene's geometry changed after the job was added"; return RTG_STATUS_BAD_SCENE; }
        jobs_h[j].S = compose(J.constants, sc->S, J.shade);
        jobs_h[j].lights = J.shading.lights;
        jobs_h[j].film = f->dev;
        Sw.max_depth = std::max(Sw.max_depth, J.constants.max_depth);
        Sw.any_cutout |= J.constants.any_cutout;
        Sw.any_passable |= J.constants.any_passable;
        total += (uint64_t)J.width * J.height * J.count;
    }
    if (total == 0) {
        for (auto& j : q->jobs) j->shading.release();
        q->jobs.clear();
        return RTG_STATUS_OK;
    }
    uint64_t cap = wave_limit(*sc, total);
    uint64_t widest = 0;
    for (auto& j : q->jobs) widest = std::max<uint64_t>(widest, j->width);
    cap = std::max(cap, widest);  // a wave holds at least one row of every job
    // A job that fills waves on its own (at least PLAIN_JOB_PATHS paths, a whole sample in one
    // wave) gains nothing from sharing them and would pay the batched kernels' segment lookups and
    // the deepest job's bounce count: it runs as the plain path's waves, with its own scene
    // constants and lights. Its film gets the same bits either way, and its waves are captured
    // into the run's graph like the batched ones.
    const bool graph = (flags & RTG_QUEUE_GRAPH) != 0;
    std::vector<uint8_t> plain(q->jobs.size(), 0);
    uint64_t plain_need = 0;
    for (size_t j = 0; j < q->jobs.size(); ++j) {
        const QueueJob& J = *q->jobs[j];
        const uint64_t npix = (uint64_t)J.width * J.height;
        if (npix * J.count >= PLAIN_JOB_PATHS && npix <= cap) {
            plain[j] = 1;
            plain_need = std::max(plain_need, npix * std::min<uint64_t>(J.count, cap / npix));
        }
    }
    std::vector<std::vector<SegDev>> waves;
    std::vector<uint64_t> wave_paths;
    pack_waves(q->jobs, cap, waves, wave_paths, plain);
    uint64_t max_wave = wave_paths.empty() ? 0 : *std::max_element(wave_paths.begin(), wave_paths.end());
    max_wave = std::max(max_wave, plain_need);
    if (max_wave > MAX_WAVE_PATHS) { g_error = "a queue wave exceeds 2^31 paths"; return RTG_STATUS_BAD_SCENE; }
    uint32_t st = ensure_capacity(*sc, (uint32_t)max_wave);
    if (st) return st;
    // One upload of the job table and every wave's segments.
    size_t nseg = 0;
    for (auto& w : waves) nseg += w.size();
    size_t bytes = jobs_h.size() * sizeof(JobDev) + nseg * sizeof(SegDev);
    if (q->tables.bytes < bytes) {
        q->tables.release();
        RTG_CHECK(cudaMalloc(&q->tables.p, bytes));
        q->tables.bytes = bytes;
    }
    std::vector<uint8_t> host(bytes);
    std::memcpy(host.data(), jobs_h.data(), jobs_h.size() * sizeof(JobDev));
    size_t off = jobs_h.size() * sizeof(JobDev);
    for (auto& w : waves) {
        std::memcpy(host.data() + off, w.data(), w.size() * sizeof(SegDev));
        off += w.size() * sizeof(SegDev);
    }
    RTG_CHECK(cudaMemcpyAsync(q->tables.p, host.data(), bytes, cudaMemcpyHostToDevice, sc->stream));
    const JobDev* jobs_d = (const JobDev*)q->tables.p;
    const SegDev* segs_d = (const SegDev*)((const uint8_t*)q->tables.p + jobs_h.size() * sizeof(JobDev));
    // The waves: enqueued back to back, or captured into one CUDA graph and launched as one.
    const bool timing = sc->timing;
    if (graph) {
        sc->timing = false;
        RTG_CHECK(cudaStreamSynchronize(sc->stream));
        RTG_CHECK(cudaStreamBeginCapture(sc->stream, cudaStreamCaptureModeThreadLocal));
    }
    cudaError_t e = cudaMemsetAsync(sc->P.counters, 0, 16, sc->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(sc->P.rays, 0, 16, sc->stream);
    for (size_t j = 0; j < q->jobs.size() && e == cudaSuccess && st == RTG_STATUS_OK; ++j) {
        if (!plain[j]) continue;
        const QueueJob& J = *q->jobs[j];
        const uint64_t npix = (uint64_t)J.width * J.height;
        const uint32_t per = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(J.count, cap / npix));
        for (uint32_t s = 0; s < J.count && st == RTG_STATUS_OK; s += per) {
            const uint32_t ns = std::min(per, J.count - s);
            WaveDesc wd{0, 0, J.width, J.height, J.first + s, (uint32_t)(npix * ns), nullptr};
            st = run_wave(*sc, wd, &jobs_h[j].film, &jobs_h[j].S, jobs_h[j].lights);
        }
    }
    size_t seg_off = 0;
    for (size_t k = 0; k < waves.size() && e == cudaSuccess && st == RTG_STATUS_OK; ++k) {
        uint32_t npix = waves[k].back().pix_begin + waves[k].back().w * waves[k].back().h;
        WaveDesc wd{0, 0, 0, 0, 0, (uint32_t)wave_paths[k], nullptr, segs_d + seg_off, jobs_d, (uint32_t)waves[k].size(), npix};
        st = run_wave(*sc, wd, nullptr, &Sw);
        seg_off += waves[k].size();
    }
    if (graph) {
        sc->timing = timing;
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(sc->stream, &g);
        if (e == cudaSuccess) e = ce;
        cudaGraphExec_t exec = nullptr;
        if (e == cudaSuccess && st == RTG_STATUS_OK) e = cudaGraphInstantiate(&exec, g, 0);
        if (e == cudaSuccess && st == RTG_STATUS_OK) e = cudaGraphLaunch(exec, sc->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(sc->stream);
        if (exec) cudaGraphExecDestroy(exec);
        if (g) cudaGraphDestroy(g);
    }
    if (e != cudaSuccess) { cuda_fail(e, "rtg_queue_run"); return RTG_STATUS_CUDA_ERROR; }
    if (st) return st;
    uint64_t r = 0;
    st = finish(*sc, &r);
    if (st) return st;
    if (rays) *rays = r;
    for (auto& j : q->jobs) j->shading.release();
    q->jobs.clear();
    return RTG_STATUS_OK;
}

uint32_t rtg_adjoint_params(uint32_t scene, uint32_t* n_materials, uint32_t* n_lights) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(scene);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    if (!n_materials || !n_lights) return RTG_STATUS_NULL_POINTER;
    *n_materials = (uint32_t)sc->materials_h.size();
    *n_lights = (uint32_t)sc->light_power.size();
    return RTG_STATUS_OK;
}

uint32_t rtg_render_adjoint(uint32_t scene, uint32_t film, const float* target, uint32_t first_sample, uint32_t count, uint32_t flags,
                            float* loss, float* grads, uint32_t n_grads, float* residual) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(scene);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    Film* f = film_of(film);
    if (!f || f->scene != scene) return RTG_STATUS_BAD_FILM;
    if (!target || !loss || !grads) { g_error = "rtg_render_adjoint: null pointer"; return RTG_STATUS_NULL_POINTER; }
    if (sc->S.any_passable) {
        g_error = "rtg_render_adjoint: unsupported: cut-outs and thin walls (their shadow rays are not replayed)";
        return RTG_STATUS_BAD_SCENE;
    }
    if (sc->S.edge_k > 1) {
        g_error = "rtg_render_adjoint: unsupported: edge samples (the replay takes one sample per index)";
        return RTG_STATUS_BAD_SCENE;
    }
    if (sc->S.section_on) {
        g_error = "rtg_render_adjoint: unsupported: a section view (the replay traces without it)";
        return RTG_STATUS_BAD_SCENE;
    }
    const FilmDev& F = f->dev;
    const uint32_t nm = (uint32_t)sc->materials_h.size(), na = (uint32_t)sc->light_source.size();
    const uint32_t nl = (uint32_t)sc->light_power.size();
    if (n_grads != 4 * nm + nl) {
        g_error = "rtg_render_adjoint: grads holds 4 per material and 1 per light (" + std::to_string(4 * nm + nl) + " floats)";
        return RTG_STATUS_BAD_ARGUMENT;
    }
    if ((uint64_t)F.ox + F.w > sc->width || (uint64_t)F.oy + F.h > sc->height) {
        g_error = "rtg_render_adjoint: the film must lie inside the image";
        return RTG_STATUS_BAD_FILM;
    }
    if (nm > 64 || count == 0) {
        g_error = nm > 64 ? "rtg_render_adjoint: more than 64 materials" : "rtg_render_adjoint: no samples";
        return RTG_STATUS_BAD_ARGUMENT;
    }
    const uint64_t npix = (uint64_t)F.w * F.h, paths = npix * count;
    if (paths > MAX_WAVE_PATHS) { g_error = "rtg_render_adjoint: more than 2^31 paths in one call"; return RTG_STATUS_BAD_ARGUMENT; }
    // BSDFs of every material and side at base +- h (all channels) and alpha +- h, built as the
    // forward ones are (flatten_scene), for the replay's central differences.
    const float h_albedo = 1.0e-3f, h_alpha = 1.0e-3f;
    const EnergyData& ed = energy_data();
    EnergyTables Eh{ed.albedo.data(), ed.schlick.data(), ed.clear_in.data(), ed.clear_out.data(), ed.albedo_avg.data(), ed.schlick_avg.data()};
    std::vector<Bsdf> tab(4 * 2 * (size_t)nm);
    for (uint32_t m = 0; m < nm; ++m) {
        const DevMaterial& d0 = sc->materials_h[m];
        float alpha = d0.roughness * d0.roughness;
        for (int v = 0; v < 4; ++v) {
            DevMaterial d = d0;
            if (v < 2)
                for (int c = 0; c < 3; ++c) d.base[c] = d0.base[c] + (v == 0 ? h_albedo : -h_albedo);
            else
                d.roughness = sqrt_(rmax(alpha + (v == 2 ? h_alpha : -h_alpha), 0.0f));
            tab[(size_t)v * 2 * nm + 2 * m] = bsdf_surface(Eh, d, true);
            tab[(size_t)v * 2 * nm + 2 * m + 1] = bsdf_surface(Eh, d, false);
        }
    }
    // Work arrays: the BSDF tables, the target, the per-pixel path derivatives, the gradients,
    // the residuals and the loss.
    const uint32_t n_params = 4 * nm + na;
    size_t off_tab = 0, off_target = off_tab + ((tab.size() * sizeof(Bsdf) + 255) / 256) * 256;
    size_t off_dpath = off_target + ((npix * 12 + 255) / 256) * 256;
    size_t off_grads = off_dpath + ((2 * npix * 16 + 255) / 256) * 256;
    size_t off_res = off_grads + ((n_params * 4 + 255) / 256) * 256;
    size_t off_loss = off_res + 256;
    // per path slot: radiance still to come, pending BSDF term (material, two float4); per shadow
    // ray: material gradient, material and light ids
    size_t off_rem = off_loss + 256;
    auto span = [&](size_t each) { return ((paths * each + 255) / 256) * 256; };
    size_t off_pend = off_rem + span(16), off_pa = off_pend + span(4), off_pr = off_pa + span(16);
    size_t off_shg = off_pr + span(16), off_shi = off_shg + span(16);
    size_t bytes = off_shi + span(4);
    if (sc->adjoint_mem.bytes < bytes) {
        sc->adjoint_mem.release();
        RTG_CHECK(cudaMalloc(&sc->adjoint_mem.p, bytes));
        sc->adjoint_mem.bytes = bytes;
    }
    uint8_t* base = (uint8_t*)sc->adjoint_mem.p;
    uint32_t st = ensure_capacity(*sc, (uint32_t)paths);
    if (st) return st;
    cudaStream_t s = sc->stream;
    RTG_CHECK(cudaMemcpyAsync(base + off_tab, tab.data(), tab.size() * sizeof(Bsdf), cudaMemcpyHostToDevice, s));
    RTG_CHECK(cudaMemcpyAsync(base + off_target, target, npix * 12, cudaMemcpyHostToDevice, s));
    RTG_CHECK(cudaMemsetAsync(base + off_grads, 0, off_loss + 8 - off_grads, s));
    // With two halves, the second is drawn with the seed's complement: an independent scramble,
    // so that E[(mean_A - T)(mean_B - T)] is the converged image's loss with no covariance term
    // (two ranges of one Owen-scrambled sequence are stratified together, hence correlated). The
    // launches of this call take the split; the scene's own renders never see it.
    const bool halves = count >= 2 && !(flags & RTG_ADJOINT_CORRELATED);
    struct SplitSeeds {
        SceneDev& S;
        SplitSeeds(SceneDev& s_, bool on, uint32_t split) : S(s_) {
            if (on) { S.split_b = split; S.seed_b = ~S.seed; }
        }
        ~SplitSeeds() { S.split_b = 0xffffffffu; S.seed_b = S.seed; }
    } split_seeds(sc->S, halves, first_sample + count / 2);
    // Forward: every path of the call in one wave, into the cleared film.
    RTG_CHECK(cudaMemsetAsync(f->mem.p, 0, f->mem.bytes, s));
    RTG_CHECK(cudaMemsetAsync(sc->P.counters, 0, 16, s));
    RTG_CHECK(cudaMemsetAsync(sc->P.rays, 0, 16, s));
    WaveDesc wd{F.ox, F.oy, F.w, F.h, first_sample, (uint32_t)paths, nullptr};
    st = run_wave(*sc, wd, &F);
    if (st) return st;
    // Loss and path derivatives, then the replay.
    launch_adjoint_delta(F, (const float*)(base + off_target), (float4*)(base + off_dpath), (double*)(base + off_loss), sc->P,
                         halves ? count : 1, s, grid_for((uint32_t)npix, 256));
    const Bsdf* t0 = (const Bsdf*)(base + off_tab);
    AdjointDev A{t0, t0 + 2 * nm, t0 + 4 * nm, t0 + 6 * nm, 1.0f / (2.0f * h_albedo), 1.0f / (2.0f * h_alpha),
                 (const float4*)(base + off_dpath), halves ? first_sample + count / 2 : first_sample + count,
                 (float*)(base + off_grads), (float*)(base + off_res), nm, na,
                 (float4*)(base + off_rem), (uint32_t*)(base + off_pend), (float4*)(base + off_pa), (float4*)(base + off_pr),
                 (float4*)(base + off_shg), (uint32_t*)(base + off_shi)};
    launch_adjoint_wave(sc->S, sc->d_lights, wd, sc->P, A, s, grid_for((uint32_t)paths, 128));
    RTG_CHECK(cudaGetLastError());
    sc->launches += 3 + 6 * (uint64_t)(sc->S.max_depth + 1);
    uint64_t rays = 0;
    st = finish(*sc, &rays);
    if (st) return st;
    std::vector<float> g(n_params);
    float res[2];
    double lossd = 0.0;
    RTG_CHECK(cudaMemcpy(g.data(), base + off_grads, n_params * 4, cudaMemcpyDeviceToHost));
    RTG_CHECK(cudaMemcpy(res, base + off_res, 8, cudaMemcpyDeviceToHost));
    RTG_CHECK(cudaMemcpy(&lossd, base + off_loss, 8, cudaMemcpyDeviceToHost));
    *loss = (float)lossd;
    for (uint32_t k = 0; k < 4 * nm; ++k) grads[k] = g[k];
    // Every light's radiance is proportional to its power: d/d power = d/d scale / power.
    for (uint32_t j = 0; j < nl; ++j) grads[4 * nm + j] = 0.0f;
    for (uint32_t i = 0; i < na; ++i) {
        uint32_t j = sc->light_source[i];
        if (j >= nl) continue;  // an emissive mesh: its emission is not a parameter
        float p = sc->light_power[j];
        if (p > 0.0f) grads[4 * nm + j] += g[4 * nm + i] / p;
    }
    if (residual) { residual[0] = res[0]; residual[1] = res[1]; }
    return RTG_STATUS_OK;
}

uint32_t rtg_scene_output(uint32_t scene, float* exposure_ev, uint32_t* tonemap, uint32_t* max_samples) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(scene);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    if (exposure_ev) *exposure_ev = sc->exposure_ev;
    if (tonemap) *tonemap = sc->tonemap;
    if (max_samples) *max_samples = sc->max_samples;
    return RTG_STATUS_OK;
}

namespace rtg {
namespace {
uint32_t film_encode(uint32_t film, float ev, uint32_t tonemap, uint32_t bits, void* out) {
    Film* f = film_of(film);
    if (!f) return RTG_STATUS_BAD_FILM;
    if (!out) { g_error = bits == 32 ? "rtg_film_linear: null pointer" : "rtg_film_srgb: null pointer"; return RTG_STATUS_NULL_POINTER; }
    Scene* sc = scene_of(f->scene);
    cudaStream_t s = sc ? sc->stream : 0;
    size_t bytes = (size_t)f->dev.w * f->dev.h * 3 * (bits / 8);
    if (f->encoded.bytes < bytes) {
        f->encoded.release();
        RTG_CHECK(cudaMalloc(&f->encoded.p, bytes));
        f->encoded.bytes = bytes;
    }
    launch_film_encode(f->dev, ev, tonemap, bits, f->encoded.p, s, grid_for(f->dev.w * f->dev.h, 256));
    RTG_CHECK(cudaGetLastError());
    RTG_CHECK(cudaMemcpyAsync(out, f->encoded.p, bytes, cudaMemcpyDeviceToHost, s));
    RTG_CHECK(cudaStreamSynchronize(s));
    return RTG_STATUS_OK;
}
}  // namespace
}  // namespace rtg

uint32_t rtg_film_srgb8(uint32_t film, float ev, uint32_t tonemap, uint8_t* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    return film_encode(film, ev, tonemap, 8, out);
}
uint32_t rtg_film_srgb16(uint32_t film, float ev, uint32_t tonemap, uint16_t* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    return film_encode(film, ev, tonemap, 16, out);
}
uint32_t rtg_film_linear(uint32_t film, float ev, float* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    return film_encode(film, ev, 0, 32, out);
}

uint32_t rtg_encode_planes(const float* rgb, const float* weight, uint32_t width, uint32_t height, float ev, uint32_t tonemap,
                           uint32_t bits, void* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!rgb || !weight || !out) return RTG_STATUS_NULL_POINTER;
    if (width == 0 || height == 0 || width > 16384 || height > 16384) return RTG_STATUS_BAD_TILE;
    if (bits != 8 && bits != 16 && bits != 32) { g_error = "rtg_encode_planes: bits must be 8, 16 or 32"; return RTG_STATUS_BAD_ARGUMENT; }
    uint32_t st = device_init();
    if (st) return st;
    const size_t npix = (size_t)width * height;
    const size_t rgb_bytes = (npix * 12 + 255) & ~(size_t)255, weight_bytes = (npix * 4 + 255) & ~(size_t)255;
    const size_t out_bytes = npix * 3 * (bits / 8);
    DevBuf m;
    struct Release { DevBuf& b; ~Release() { b.release(); } } release{m};
    m.bytes = rgb_bytes + weight_bytes + out_bytes;
    RTG_CHECK(cudaMalloc(&m.p, m.bytes));
    uint8_t* base = (uint8_t*)m.p;
    FilmDev F{0, 0, width, height, (float*)base, (float*)(base + rgb_bytes), nullptr, nullptr};
    void* d_out = base + rgb_bytes + weight_bytes;
    RTG_CHECK(cudaMemcpy(F.rgb, rgb, npix * 12, cudaMemcpyHostToDevice));
    RTG_CHECK(cudaMemcpy(F.weight, weight, npix * 4, cudaMemcpyHostToDevice));
    launch_film_encode(F, ev, tonemap, bits, d_out, 0, grid_for((uint32_t)npix, 256));
    RTG_CHECK(cudaGetLastError());
    RTG_CHECK(cudaMemcpy(out, d_out, out_bytes, cudaMemcpyDeviceToHost));
    return RTG_STATUS_OK;
}

uint32_t rtg_film_read(uint32_t film, float* rgb, float* weight, float* alpha, float* lum2) {
    std::lock_guard<std::mutex> lk(g_mu);
    Film* f = film_of(film);
    if (!f) return RTG_STATUS_BAD_FILM;
    Scene* sc = scene_of(f->scene);
    cudaStream_t s = sc ? sc->stream : 0;
    size_t n = (size_t)f->dev.w * f->dev.h;
    if (rgb) RTG_CHECK(cudaMemcpyAsync(rgb, f->dev.rgb, n * 12, cudaMemcpyDeviceToHost, s));
    if (weight) RTG_CHECK(cudaMemcpyAsync(weight, f->dev.weight, n * 4, cudaMemcpyDeviceToHost, s));
    if (alpha) RTG_CHECK(cudaMemcpyAsync(alpha, f->dev.alpha, n * 4, cudaMemcpyDeviceToHost, s));
    if (lum2) RTG_CHECK(cudaMemcpyAsync(lum2, f->dev.lum2, n * 4, cudaMemcpyDeviceToHost, s));
    RTG_CHECK(cudaStreamSynchronize(s));
    return RTG_STATUS_OK;
}
uint32_t rtg_film_device(uint32_t film, float** rgb, float** weight, float** alpha, float** lum2) {
    std::lock_guard<std::mutex> lk(g_mu);
    Film* f = film_of(film);
    if (!f) return RTG_STATUS_BAD_FILM;
    if (rgb) *rgb = f->dev.rgb;
    if (weight) *weight = f->dev.weight;
    if (alpha) *alpha = f->dev.alpha;
    if (lum2) *lum2 = f->dev.lum2;
    return RTG_STATUS_OK;
}

uint32_t rtg_render_paths(uint32_t handle, const uint32_t* xys, uint32_t n, float* out5) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    if (!xys || !out5) return RTG_STATUS_NULL_POINTER;
    if (n == 0) return RTG_STATUS_OK;
    uint32_t st = ensure_capacity(*sc, n);
    if (st) return st;
    uint32_t* d_xys = nullptr;
    RTG_CHECK(cudaMalloc(&d_xys, (size_t)n * 12));
    std::unique_ptr<uint32_t, void (*)(uint32_t*)> guard(d_xys, [](uint32_t* p) { cudaFree(p); });
    RTG_CHECK(cudaMemcpyAsync(d_xys, xys, (size_t)n * 12, cudaMemcpyHostToDevice, sc->stream));
    RTG_CHECK(cudaMemsetAsync(sc->P.counters, 0, 16, sc->stream));
    RTG_CHECK(cudaMemsetAsync(sc->P.rays, 0, 16, sc->stream));
    WaveDesc wd{0, 0, 1, 1, 0, n, d_xys};
    st = run_wave(*sc, wd, nullptr);
    if (st) return st;
    std::vector<float4> sum(n), thr(n);
    std::vector<uint32_t> flags(n);
    RTG_CHECK(cudaMemcpyAsync(sum.data(), sc->P.sum, (size_t)n * 16, cudaMemcpyDeviceToHost, sc->stream));
    RTG_CHECK(cudaMemcpyAsync(thr.data(), sc->P.thr, (size_t)n * 16, cudaMemcpyDeviceToHost, sc->stream));
    RTG_CHECK(cudaMemcpyAsync(flags.data(), sc->P.flags, (size_t)n * 4, cudaMemcpyDeviceToHost, sc->stream));
    st = finish(*sc, nullptr);
    if (st) return st;
    for (uint32_t i = 0; i < n; ++i) {
        // a panoramic camera's sample that sees nothing weighs black (render.rs:465)
        const float k = (flags[i] & 8u) ? 0.0f : 1.0f;
        out5[5 * i] = k == 1.0f ? sum[i].x : sum[i].x * k;
        out5[5 * i + 1] = k == 1.0f ? sum[i].y : sum[i].y * k;
        out5[5 * i + 2] = k == 1.0f ? sum[i].z : sum[i].z * k;
        out5[5 * i + 3] = thr[i].w;
        out5[5 * i + 4] = 0.0f;
    }
    return RTG_STATUS_OK;
}

uint32_t rtg_mesh_solid(const float* positions, uint32_t n_vertices, const uint32_t* indices, uint32_t n_indices, uint32_t* solid) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!positions || !solid || (n_indices && !indices)) { g_error = "rtg_mesh_solid: null pointer"; return RTG_STATUS_NULL_POINTER; }
    if (n_indices % 3) { g_error = "rtg_mesh_solid: index count is not a multiple of 3"; return RTG_STATUS_BAD_ARGUMENT; }
    HMesh m;
    m.positions.resize(n_vertices);
    V3 lo = v3(f_inf(), f_inf(), f_inf()), hi = v3(-f_inf(), -f_inf(), -f_inf());
    for (uint32_t v = 0; v < n_vertices; ++v) {
        const V3 p = v3(positions[3 * v], positions[3 * v + 1], positions[3 * v + 2]);
        if (!vfinite(p)) { g_error = "rtg_mesh_solid: non-finite vertex position"; return RTG_STATUS_BAD_ARGUMENT; }
        m.positions[v] = p;
        lo = v3(rmin(lo.x, p.x), rmin(lo.y, p.y), rmin(lo.z, p.z));
        hi = v3(rmax(hi.x, p.x), rmax(hi.y, p.y), rmax(hi.z, p.z));
    }
    m.indices.assign(indices, indices + n_indices);
    for (uint32_t i : m.indices)
        if (i >= n_vertices) { g_error = "rtg_mesh_solid: vertex index out of range"; return RTG_STATUS_BAD_ARGUMENT; }
    m.bmin = lo;
    m.bmax = hi;
    m.empty_bounds = m.positions.empty();
    *solid = solid_of(m);
    return RTG_STATUS_OK;
}

uint32_t rtg_trace_rays(uint32_t handle, const float* rays, uint32_t n, uint32_t mode, uint32_t* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    if (!rays || !out) return RTG_STATUS_NULL_POINTER;
    if (n == 0) return RTG_STATUS_OK;
    uint32_t st = ensure_capacity(*sc, 1024);
    if (st) return st;
    size_t words = (mode & 2u) ? n : (size_t)n * 3;
    void* mem = nullptr;
    RTG_CHECK(cudaMalloc(&mem, (size_t)n * 32 + words * 4));
    std::unique_ptr<void, void (*)(void*)> guard(mem, [](void* p) { cudaFree(p); });
    float* d_rays = (float*)mem;
    uint32_t* d_out = (uint32_t*)((uint8_t*)mem + (size_t)n * 32);
    RTG_CHECK(cudaMemcpyAsync(d_rays, rays, (size_t)n * 32, cudaMemcpyHostToDevice, sc->stream));
    RTG_CHECK(cudaMemsetAsync(sc->P.counters, 0, 16, sc->stream));
    launch_trace_batch(sc->S, d_rays, n, mode, d_out, sc->P.counters, sc->stream, grid_for(n, 128));
    RTG_CHECK(cudaGetLastError());
    RTG_CHECK(cudaMemcpyAsync(out, d_out, words * 4, cudaMemcpyDeviceToHost, sc->stream));
    uint32_t counters[4];
    RTG_CHECK(cudaMemcpyAsync(counters, sc->P.counters, 16, cudaMemcpyDeviceToHost, sc->stream));
    RTG_CHECK(cudaStreamSynchronize(sc->stream));
    if (counters[3] & 1u) { g_error = "traversal stack overflow"; return RTG_STATUS_STACK_OVERFLOW; }
    return RTG_STATUS_OK;
}

uint32_t rtg_scene_stats(uint32_t handle, double* out8) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    if (!out8) return RTG_STATUS_NULL_POINTER;
    out8[0] = (double)sc->width;
    out8[1] = (double)sc->height;
    out8[2] = (double)sc->max_depth;
    out8[3] = (double)sc->instanced_triangles;
    out8[4] = (double)sc->nodes;
    out8[5] = (double)sc->tris;
    out8[6] = sc->build_seconds;
    out8[7] = (double)sc->rays;
    return RTG_STATUS_OK;
}

uint32_t rtg_set_path_capacity(uint32_t handle, uint32_t paths) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    if (paths != 0 && paths < 1024) paths = 1024;
    sc->max_capacity = paths;
    return RTG_STATUS_OK;
}

uint32_t rtg_set_tuning(uint32_t handle, const uint32_t* values, uint32_t n) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    if (!values && n) return RTG_STATUS_NULL_POINTER;
    RaySort o = sc->order;
    uint32_t cap = sc->max_capacity;
    if (n > 0) {
        if (values[0] > RAY_SORT_MAX_BITS) { g_error = "rtg_set_tuning: ray-sort bits above 5"; return RTG_STATUS_BAD_SCENE; }
        o.ray_bits = values[0];
    }
    if (n > 1) o.shadow_sort = values[1] != 0;
    if (n > 2) o.material_sort = values[2] != 0;
    if (n > 3) cap = values[3] != 0 && values[3] < 1024 ? 1024 : values[3];
    if (n > 4) o.l2_persist = values[4] != 0;
    if (n > 5) o.tail_paths = values[5];
    // A wave leaves both histograms at zero, but the cursors of fewer bits lie inside the
    // histogram of more: clear them when the key count changes.
    if (o.ray_bits != sc->order.ray_bits && sc->P.rbins) RTG_CHECK(cudaMemsetAsync(sc->P.rbins, 0, SORT_BINS_BYTES, sc->stream));
    sc->order = o;
    sc->max_capacity = cap;
    refresh_order(*sc);
    return RTG_STATUS_OK;
}

// The autotuner: coordinate descent over the tuning, each candidate rendered once to warm up and
// then AUTOTUNE_REPS times, timed with CUDA events on the scene's stream (the median counts); the
// scene keeps the fastest. One timed render of 4 samples of the 1080p frame varied by up to 20%
// between candidates that render identically.
constexpr int AUTOTUNE_REPS = 3;
constexpr double AUTOTUNE_MARGIN = 0.01;
uint32_t rtg_autotune(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t first_sample, uint32_t count, double* report,
                      uint32_t max_report, uint32_t* n_tried) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    if (n_tried) *n_tried = 0;
    const uint64_t x_end = std::min<uint64_t>((uint64_t)x + w, sc->width), y_end = std::min<uint64_t>((uint64_t)y + h, sc->height);
    if (x >= x_end || y >= y_end || count == 0) { g_error = "rtg_autotune: an empty rectangle or no samples"; return RTG_STATUS_BAD_TILE; }
    Film tmp;
    uint32_t st = make_film(x, y, (uint32_t)(x_end - x), (uint32_t)(y_end - y), tmp);
    if (st) return st;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    RTG_CHECK(cudaEventCreate(&e0));
    RTG_CHECK(cudaEventCreate(&e1));
    std::unique_ptr<CUevent_st, cudaError_t (*)(cudaEvent_t)> g0(e0, cudaEventDestroy), g1(e1, cudaEventDestroy);
    const uint64_t paths = (x_end - x) * (y_end - y) * (uint64_t)count;
    const bool timing = sc->timing;
    sc->timing = false;
    struct Cand { uint32_t bits, shadow, msort, cap, l2, tail; };
    std::vector<std::pair<Cand, double>> tried;
    auto measure = [&](const Cand& c, double& ms) -> uint32_t {
        for (const auto& t : tried)
            if (t.first.bits == c.bits && t.first.shadow == c.shadow && t.first.msort == c.msort && t.first.cap == c.cap && t.first.l2 == c.l2 &&
                t.first.tail == c.tail) {
                ms = t.second;
                return 0;
            }
        if (c.bits != sc->order.ray_bits && sc->P.rbins) RTG_CHECK(cudaMemsetAsync(sc->P.rbins, 0, SORT_BINS_BYTES, sc->stream));
        sc->order.ray_bits = c.bits;
        sc->order.shadow_sort = c.shadow;
        sc->order.material_sort = c.msort;
        sc->order.l2_persist = c.l2;
        sc->order.tail_paths = c.tail;
        sc->max_capacity = c.cap;
        refresh_order(*sc);
        uint32_t r = render_region(*sc, tmp.dev.ox, tmp.dev.oy, tmp.dev.w, tmp.dev.h, first_sample, count, tmp.dev, nullptr);  // warm-up
        if (r) return r;
        float t[AUTOTUNE_REPS];
        for (int k = 0; k < AUTOTUNE_REPS; ++k) {
            RTG_CHECK(cudaEventRecord(e0, sc->stream));
            r = render_region(*sc, tmp.dev.ox, tmp.dev.oy, tmp.dev.w, tmp.dev.h, first_sample, count, tmp.dev, nullptr);
            if (r) return r;
            RTG_CHECK(cudaEventRecord(e1, sc->stream));
            RTG_CHECK(cudaEventSynchronize(e1));
            RTG_CHECK(cudaEventElapsedTime(&t[k], e0, e1));
        }
        std::sort(t, t + AUTOTUNE_REPS);
        ms = t[AUTOTUNE_REPS / 2];
        tried.push_back({c, ms});
        return 0;
    };
    Cand best{sc->order.ray_bits, sc->order.shadow_sort, sc->order.material_sort, sc->max_capacity, sc->order.l2_persist, sc->order.tail_paths};
    double best_ms = 1e300;
    // A candidate replaces the best so far only when it is faster by more than AUTOTUNE_MARGIN: a
    // timing's noise must not move the tuning.
    auto consider = [&](const Cand& c) -> uint32_t {
        double ms = 0.0;
        uint32_t r = measure(c, ms);
        if (r) return r;
        if (ms < best_ms * (1.0 - AUTOTUNE_MARGIN)) { best_ms = ms; best = c; }
        return 0;
    };
    // 0. the scene's own tuning, 1. the ray sort's grid (shadow rays sorted with it), 2. shadow
    // rays, 3. material sort, 4. the L2 window over the traversal data, 5. the tail limit, 6. wave
    // size
    const uint32_t tail0 = sc->order.tail_paths;
    st = consider(best);
    for (uint32_t bits : {0u, 3u, 4u, 5u})
        if (!st && (st = consider(Cand{bits, bits > 0 ? 1u : 0u, 1u, 0u, 0u, tail0}))) break;
    if (!st && best.bits > 0) st = consider(Cand{best.bits, 1u - best.shadow, best.msort, best.cap, best.l2, best.tail});
    if (!st) st = consider(Cand{best.bits, best.shadow, 1u - best.msort, best.cap, best.l2, best.tail});
    if (!st) st = consider(Cand{best.bits, best.shadow, best.msort, best.cap, 1u - best.l2, best.tail});
    for (uint32_t tail : {0u, 1u << 16, 1u << 18, 1u << 20}) {
        if (st) break;
        st = consider(Cand{best.bits, best.shadow, best.msort, best.cap, best.l2, tail});
    }
    for (uint64_t div : {2u, 4u}) {
        if (st) break;
        const uint64_t cap = paths / div;
        if (cap >= (1u << 20))
            st = consider(Cand{best.bits, best.shadow, best.msort, (uint32_t)std::min<uint64_t>(cap, MAX_WAVE_PATHS), best.l2, best.tail});
    }
    // keep the fastest
    if (best.bits != sc->order.ray_bits && sc->P.rbins) cudaMemsetAsync(sc->P.rbins, 0, SORT_BINS_BYTES, sc->stream);
    sc->order.ray_bits = best.bits;
    sc->order.shadow_sort = best.shadow;
    sc->order.material_sort = best.msort;
    sc->order.l2_persist = best.l2;
    sc->order.tail_paths = best.tail;
    sc->max_capacity = best.cap;
    refresh_order(*sc);
    sc->timing = timing;
    if (n_tried) *n_tried = (uint32_t)tried.size();
    for (size_t k = 0; report && k < tried.size() && k < max_report; ++k) {
        const Cand& c = tried[k].first;
        double* r = report + 7 * k;
        r[0] = c.bits; r[1] = c.shadow; r[2] = c.msort; r[3] = c.cap; r[4] = c.l2; r[5] = c.tail; r[6] = tried[k].second;
    }
    RTG_CHECK(cudaStreamSynchronize(sc->stream));
    return st;
}

uint32_t rtg_get_tuning(uint32_t handle, uint32_t* values, uint32_t n) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    if (!values && n) return RTG_STATUS_NULL_POINTER;
    const uint32_t v[6] = {sc->order.ray_bits, sc->order.shadow_sort, sc->order.material_sort, sc->max_capacity, sc->order.l2_persist,
                           sc->order.tail_paths};
    for (uint32_t k = 0; k < n && k < 6; ++k) values[k] = v[k];
    return RTG_STATUS_OK;
}

uint32_t rtg_timing(uint32_t handle, uint32_t enable, uint32_t reset, double* out5) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    if (out5) {
        out5[0] = sc->extend_ms;
        out5[1] = (double)sc->extend_launches;
        out5[2] = (double)sc->extend_rays;
        out5[3] = (double)sc->shadow_rays;
        out5[4] = (double)sc->launches;
    }
    if (reset) {
        sc->extend_ms = 0;
        sc->extend_launches = 0;
        sc->extend_rays = 0;
        sc->shadow_rays = 0;
        sc->launches = 0;
    }
    sc->timing = enable != 0;
    return RTG_STATUS_OK;
}

uint32_t rtg_set_stream(uint32_t handle, void* stream) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    RTG_CHECK(cudaStreamSynchronize(sc->stream));
    if (sc->own_stream) RTG_CHECK(cudaStreamDestroy(sc->stream));
    if (stream) {
        sc->stream = (cudaStream_t)stream;
        sc->own_stream = false;
    } else {
        RTG_CHECK(cudaStreamCreateWithFlags(&sc->stream, cudaStreamNonBlocking));
        sc->own_stream = true;
    }
    return RTG_STATUS_OK;
}

uint32_t rtg_synchronize(uint32_t handle) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    RTG_CHECK(cudaStreamSynchronize(sc->stream));
    return RTG_STATUS_OK;
}

// ---- adaptive sampling (E10) -------------------------------------------------------------------------
uint32_t rtg_adaptive_decide(uint32_t width, uint32_t height, float ev, float target, uint32_t cap, const uint8_t* counts,
                             const uint8_t* sums, const uint8_t* lum2, uint8_t* active, uint8_t* decision) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!counts || !sums || !lum2 || !active || !decision) return RTG_STATUS_NULL_POINTER;
    if (width == 0 || height == 0 || width > 16384 || height > 16384) return RTG_STATUS_BAD_TILE;
    uint32_t st = device_init();
    if (st) return st;
    const size_t nb = (size_t)ad_cols(width) * ad_rows(height), npix = (size_t)width * height;
    std::vector<uint32_t> c(nb);
    std::memcpy(c.data(), counts, nb * 4);
    DevBuf m;
    struct Release { DevBuf& b; ~Release() { b.release(); } } release{m};
    const size_t sums_bytes = npix * 16, lum_bytes = (npix * 4 + 255) & ~(size_t)255, nb_bytes = (nb * 4 + 255) & ~(size_t)255;
    m.bytes = sums_bytes + lum_bytes + 2 * nb_bytes;
    RTG_CHECK(cudaMalloc(&m.p, m.bytes));
    uint8_t* base = (uint8_t*)m.p;
    float* d_sums = (float*)base;
    float* d_lum2 = (float*)(base + sums_bytes);
    uint32_t* d_counts = (uint32_t*)(base + sums_bytes + lum_bytes);
    float* d_err = (float*)(base + sums_bytes + lum_bytes + nb_bytes);
    RTG_CHECK(cudaMemcpy(d_sums, sums, sums_bytes, cudaMemcpyHostToDevice));
    RTG_CHECK(cudaMemcpy(d_lum2, lum2, npix * 4, cudaMemcpyHostToDevice));
    RTG_CHECK(cudaMemcpy(d_counts, c.data(), nb * 4, cudaMemcpyHostToDevice));
    RTG_CHECK(launch_block_error(d_sums, 4, d_lum2, d_counts, width, height, ad_floor_for(ev), d_err, 0, grid_for((uint32_t)nb, 1)));
    std::vector<float> err(nb);
    RTG_CHECK(cudaMemcpy(err.data(), d_err, nb * 4, cudaMemcpyDeviceToHost));
    std::vector<uint8_t> act;
    const AdDecision d = ad_decide_blocks(width, height, c.data(), err.data(), target, cap, act);
    std::memcpy(active, act.data(), nb);
    uint32_t words[6] = {d.round, d.active, d.blocks, 0, 0, 0};
    std::memcpy(&words[3], &d.threshold, 4);
    std::memcpy(&words[4], &d.max_error, 4);
    std::memcpy(&words[5], &d.remaining, 4);
    std::memcpy(decision, words, sizeof(words));
    return RTG_STATUS_OK;
}

uint32_t rtg_render_block_rgba(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t sample_index,
                               uint32_t iteration, float* out) {
    (void)iteration;  // the photon map of an iteration: scenes with caustics are refused at load
    if (!out) return RTG_STATUS_NULL_POINTER;
    std::lock_guard<std::mutex> lk(g_mu);
    return render_tile_impl(handle, x, y, w, h, sample_index, out, true);
}

uint32_t rtg_adaptive_create(uint32_t scene, uint32_t film, uint32_t cap) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(scene);
    if (!sc) { g_error = "rtg_adaptive_create: bad scene handle"; return 0; }
    Film* f = film_of(film);
    if (!f || f->scene != scene || f->dev.ox || f->dev.oy || f->dev.w != sc->width || f->dev.h != sc->height) {
        g_error = "rtg_adaptive_create: the film must be one of the scene's and cover its whole image";
        return 0;
    }
    auto a = std::make_unique<AdaptiveRun>();
    a->scene = scene;
    a->film = film;
    a->width = sc->width;
    a->height = sc->height;
    a->cols = ad_cols(sc->width);
    a->rows = ad_rows(sc->height);
    const size_t nb = (size_t)a->cols * a->rows, npix = (size_t)sc->width * sc->height;
    a->counts.assign(nb, 0);
    a->active.assign(nb, 1);
    a->cap = cap;
    a->round = cap > 0 ? std::min(AD_WARMUP, cap) : AD_WARMUP;  // adaptive.rs:349
    a->target = sc->noise_threshold > 0.0f ? sc->noise_threshold : 0.0f;
    a->floor = ad_floor_for(sc->exposure_ev);
    auto round_up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t nb4 = round_up(nb * 4), list = round_up(npix * 4);
    a->mem.bytes = 2 * nb4 + round_up(nb * sizeof(AdEntry)) + round_up(nb * 8) + 4 * list;
    if (cudaMalloc(&a->mem.p, a->mem.bytes) != cudaSuccess) {
        a->mem.p = nullptr;
        g_error = "rtg_adaptive_create: out of device memory";
        return 0;
    }
    uint8_t* p = (uint8_t*)a->mem.p;
    a->d_counts = (uint32_t*)p; p += nb4;
    a->d_error = (float*)p; p += nb4;
    a->d_entries = (AdEntry*)p; p += round_up(nb * sizeof(AdEntry));
    a->d_pixels = (uint32_t*)p; p += round_up(nb * 8);
    a->d_plain = (uint32_t*)p; p += list;
    a->d_plain_base = (uint32_t*)p; p += list;
    a->d_edge = (uint32_t*)p; p += list;
    a->d_edge_base = (uint32_t*)p;
    for (size_t i = 0; i < g_adaptive.size(); ++i)
        if (!g_adaptive[i]) { g_adaptive[i] = std::move(a); return (uint32_t)i + 1; }
    g_adaptive.push_back(std::move(a));
    return (uint32_t)g_adaptive.size();
}

uint32_t rtg_adaptive_run(uint32_t ad, uint32_t pass, uint32_t max_passes, uint32_t* passes_out, uint64_t* rays) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (passes_out) *passes_out = 0;
    if (rays) *rays = 0;
    AdaptiveRun* a = adaptive_of(ad);
    if (!a) return RTG_STATUS_BAD_HANDLE;
    Scene* sc = scene_of(a->scene);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    Film* f = film_of(a->film);
    if (!f) return RTG_STATUS_BAD_FILM;
    if (sc->width != a->width || sc->height != a->height) {
        g_error = "rtg_adaptive_run: the scene's image size changed since rtg_adaptive_create";
        return RTG_STATUS_BAD_SCENE;
    }
    if (pass == 0) pass = UINT32_MAX;  // a whole round a pass: the fewest, largest waves
    uint32_t passes = 0;
    uint64_t total = 0;
    for (;;) {  // adaptive/tests.rs:311
        if (a->left() == 0) {
            if (a->decisions && a->round == 0) break;  // converged
            const uint32_t st = adaptive_decide_round(*sc, *f, *a);
            if (st) return st;
            if (a->round == 0) break;
        }
        if (max_passes && passes >= max_passes) break;
        const uint32_t count = std::min(pass, a->left());
        uint64_t r = 0;
        const uint32_t st = adaptive_pass(*sc, *f, *a, count, r);
        if (st) return st;
        total += r;
        a->done = std::min(a->done + count, a->round);  // adaptive.rs:502
        ++passes;
        if (passes_out) *passes_out = passes;
        if (rays) *rays = total;
    }
    return RTG_STATUS_OK;
}

uint32_t rtg_adaptive_state(uint32_t ad, uint32_t* out16) {
    std::lock_guard<std::mutex> lk(g_mu);
    AdaptiveRun* a = adaptive_of(ad);
    if (!a) return RTG_STATUS_BAD_HANDLE;
    if (!out16) return RTG_STATUS_NULL_POINTER;
    uint32_t lo = UINT32_MAX, hi = 0;
    for (size_t b = 0; b < a->blocks(); ++b) {
        lo = std::min(lo, a->samples_of(b));
        hi = std::max(hi, a->samples_of(b));
    }
    if (lo == UINT32_MAX) lo = hi = 0;
    uint32_t w[16] = {a->round, a->done, a->left(), a->iteration + a->done, (a->decisions && a->round == 0) ? 1u : 0u, a->decisions,
                      lo, hi, a->last.round, a->last.active, a->last.blocks, 0, 0, 0, a->cols, a->rows};
    std::memcpy(&w[11], &a->last.threshold, 4);
    std::memcpy(&w[12], &a->last.max_error, 4);
    std::memcpy(&w[13], &a->last.remaining, 4);
    std::memcpy(out16, w, sizeof(w));
    return RTG_STATUS_OK;
}

uint32_t rtg_adaptive_counts(uint32_t ad, uint32_t* samples, uint8_t* active) {
    std::lock_guard<std::mutex> lk(g_mu);
    AdaptiveRun* a = adaptive_of(ad);
    if (!a) return RTG_STATUS_BAD_HANDLE;
    if (!samples && !active) return RTG_STATUS_NULL_POINTER;
    for (size_t b = 0; b < a->blocks(); ++b) {
        if (samples) samples[b] = a->samples_of(b);
        if (active) active[b] = a->active[b];
    }
    return RTG_STATUS_OK;
}

// ---- guide passes and the denoiser (rt-post/src/denoise.rs) -----------------------------------------
uint32_t rtg_render_tile_passes(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t mask, uint8_t* out) {
    if (!out) return RTG_STATUS_NULL_POINTER;
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    const uint64_t px = (uint64_t)w * h;
    if (px == 0 || px > RTG_MAX_TILE_PIXELS) return RTG_STATUS_BAD_TILE;
    DevBuf m;
    struct Release { DevBuf& b; ~Release() { b.release(); } } release{m};
    m.bytes = px * 24;
    RTG_CHECK(cudaMalloc(&m.p, m.bytes));
    float* normal = (float*)m.p;
    float* depth = normal + 3 * px;
    uint32_t* part = (uint32_t*)(depth + px);
    uint32_t* material = part + px;
    RTG_CHECK(launch_exact_passes(sc->S, sc->d_lights, x, y, w, h, normal, depth, part, material, sc->stream, grid_for((uint32_t)px, 128)));
    sc->launches += 1;
    std::vector<uint32_t> host(px * 6);
    RTG_CHECK(cudaMemcpyAsync(host.data(), m.p, px * 24, cudaMemcpyDeviceToHost, sc->stream));
    RTG_CHECK(cudaStreamSynchronize(sc->stream));
    // The planes of `mask` in the order normal, depth, part id, material id, circle of confusion
    // (passes.rs:475 planes); the albedo and alpha bits and unknown bits are ignored.
    size_t o = 0;
    auto put = [&](const void* src, size_t words) {
        std::memcpy(out + o, src, words * 4);
        o += words * 4;
    };
    if (mask & 2u) put(host.data(), 3 * px);
    if (mask & 4u) put(host.data() + 3 * px, px);
    if (mask & 8u) put(host.data() + 4 * px, px);
    if (mask & 16u) put(host.data() + 5 * px, px);
    if (mask & 32u) {  // passes.rs:130 coc_diameter
        std::vector<float> coc(px, 0.0f);
        const SceneDev& S = sc->S;
        const uint32_t long_side = std::max<uint32_t>(std::max(sc->width, sc->height), 1);
        for (size_t i = 0; i < px; ++i) {
            float depth_v;
            std::memcpy(&depth_v, &host[3 * px + i], 4);
            if (S.lens_radius <= 0.0f || !(depth_v > 0.0f && std::isfinite(depth_v))) continue;
            const float aperture = S.lens_radius * 2.0f;  // focal / fstop, exactly
            const float on_focus_plane = aperture * std::fabs(depth_v - S.focus_dist) / depth_v;
            const float pixel_on_focus_plane = S.sensor_mm / (float)long_side * (S.focus_dist / S.focal_mm);
            coc[i] = on_focus_plane / pixel_on_focus_plane;
        }
        put(coc.data(), px);
    }
    return RTG_STATUS_OK;
}

uint32_t rtg_render_tile_albedo(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t sample_index, float* out) {
    if (!out) return RTG_STATUS_NULL_POINTER;
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    const uint64_t px = (uint64_t)w * h;
    if (px == 0 || px > RTG_MAX_TILE_PIXELS) return RTG_STATUS_BAD_TILE;
    const uint8_t* mask = nullptr;
    if (sc->S.edge_k > 1) {
        uint32_t *l = nullptr, *c = nullptr;
        const uint32_t st = edge_mask_of(*sc, mask, l, c);
        if (st) return st;
    }
    DevBuf m;
    struct Release { DevBuf& b; ~Release() { b.release(); } } release{m};
    m.bytes = px * 16;
    RTG_CHECK(cudaMalloc(&m.p, m.bytes));
    RTG_CHECK(cudaMemsetAsync(m.p, 0, m.bytes, sc->stream));
    float* sum = (float*)m.p;
    RTG_CHECK(launch_albedo_pass(sc->S, sc->d_lights, mask, x, y, w, h, sample_index, 1, sum, sum + 3 * px, nullptr, sc->stream,
                                 grid_for((uint32_t)px, 128)));
    sc->launches += 1;
    RTG_CHECK(cudaMemcpyAsync(out, sum, px * 12, cudaMemcpyDeviceToHost, sc->stream));
    RTG_CHECK(cudaStreamSynchronize(sc->stream));
    return RTG_STATUS_OK;
}

uint32_t rtg_render_tile_alpha(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t sample_index, float* out) {
    if (!out) return RTG_STATUS_NULL_POINTER;
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(handle);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    const uint64_t px = (uint64_t)w * h;
    if (px == 0 || px > RTG_MAX_TILE_PIXELS) return RTG_STATUS_BAD_TILE;
    const uint8_t* mask = nullptr;
    if (sc->S.edge_k > 1) {
        uint32_t *l = nullptr, *c = nullptr;
        const uint32_t st = edge_mask_of(*sc, mask, l, c);
        if (st) return st;
    }
    DevBuf m;
    struct Release { DevBuf& b; ~Release() { b.release(); } } release{m};
    m.bytes = px * 20;
    RTG_CHECK(cudaMalloc(&m.p, m.bytes));
    RTG_CHECK(cudaMemsetAsync(m.p, 0, m.bytes, sc->stream));
    float* sum = (float*)m.p;
    float* alpha = sum + 4 * px;
    RTG_CHECK(launch_albedo_pass(sc->S, sc->d_lights, mask, x, y, w, h, sample_index, 1, sum, sum + 3 * px, alpha, sc->stream,
                                 grid_for((uint32_t)px, 128)));
    sc->launches += 1;
    RTG_CHECK(cudaMemcpyAsync(out, alpha, px * 4, cudaMemcpyDeviceToHost, sc->stream));
    RTG_CHECK(cudaStreamSynchronize(sc->stream));
    return RTG_STATUS_OK;
}

uint32_t rtg_film_guides(uint32_t scene, uint32_t film, uint32_t first_sample, uint32_t count) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(scene);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    Film* f = film_of(film);
    if (!f || f->scene != scene) return RTG_STATUS_BAD_FILM;
    const size_t n = f->pixels();
    if (!f->guides.p) {
        f->guides.bytes = n * 10 * 4;
        RTG_CHECK(cudaMalloc(&f->guides.p, f->guides.bytes));
        RTG_CHECK(cudaMemsetAsync(f->guides.p, 0, f->guides.bytes, sc->stream));
    }
    const uint8_t* mask = nullptr;
    if (sc->S.edge_k > 1) {
        uint32_t *l = nullptr, *c = nullptr;
        const uint32_t st = edge_mask_of(*sc, mask, l, c);
        if (st) return st;
    }
    const FilmDev& d = f->dev;
    RTG_CHECK(launch_exact_passes(sc->S, sc->d_lights, d.ox, d.oy, d.w, d.h, f->normal(), f->depth(), f->part(), f->material(), sc->stream,
                                  grid_for((uint32_t)n, 128)));
    if (count)
        RTG_CHECK(launch_albedo_pass(sc->S, sc->d_lights, mask, d.ox, d.oy, d.w, d.h, first_sample, count, f->albedo_sum(), f->albedo_weight(),
                                     nullptr, sc->stream, grid_for((uint32_t)n, 128)));
    sc->launches += count ? 2 : 1;
    RTG_CHECK(cudaStreamSynchronize(sc->stream));
    return RTG_STATUS_OK;
}

uint32_t rtg_film_guides_fused(uint32_t scene, uint32_t film, uint32_t enable) {
    std::lock_guard<std::mutex> lk(g_mu);
    Scene* sc = scene_of(scene);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    Film* f = film_of(film);
    if (!f || f->scene != scene) return RTG_STATUS_BAD_FILM;
    f->fuse_guides = enable != 0;
    if (!enable) return RTG_STATUS_OK;
    const size_t n = f->pixels();
    if (!f->guides.p) {
        f->guides.bytes = n * 10 * 4;
        RTG_CHECK(cudaMalloc(&f->guides.p, f->guides.bytes));
        RTG_CHECK(cudaMemsetAsync(f->guides.p, 0, f->guides.bytes, sc->stream));
    }
    const FilmDev& d = f->dev;
    RTG_CHECK(launch_exact_passes(sc->S, sc->d_lights, d.ox, d.oy, d.w, d.h, f->normal(), f->depth(), f->part(), f->material(), sc->stream,
                                  grid_for((uint32_t)n, 128)));
    sc->launches += 1;
    RTG_CHECK(cudaStreamSynchronize(sc->stream));
    return RTG_STATUS_OK;
}

namespace {
float strength_of(float s) { return std::isnan(s) ? 1.0f : (s < 0.0f ? 0.0f : (s > 1.0f ? 1.0f : s)); }  // denoise.rs:386
}  // namespace

uint32_t rtg_film_denoise(uint32_t film, uint32_t preset, float strength, uint32_t samples, float* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    Film* f = film_of(film);
    if (!f) return RTG_STATUS_BAD_FILM;
    Scene* sc = scene_of(f->scene);
    if (!sc) return RTG_STATUS_BAD_HANDLE;
    if (preset > 1) return RTG_STATUS_BAD_DENOISE;
    if (!f->guides.p) { g_error = "rtg_film_denoise: the film has no guide passes (rtg_film_guides)"; return RTG_STATUS_BAD_FILM; }
    if (f->dev.ox || f->dev.oy || f->dev.w != sc->width || f->dev.h != sc->height) {
        g_error = "rtg_film_denoise: the film must cover the whole image";
        return RTG_STATUS_BAD_FILM;
    }
    const size_t n = f->pixels();
    const size_t need = dn_scratch_bytes(n) + n * 16 + n * 20;
    if (f->denoise.bytes < need) {
        f->denoise.release();
        RTG_CHECK(cudaMalloc(&f->denoise.p, need));
        f->denoise.bytes = need;
    }
    float* result = (float*)((uint8_t*)f->denoise.p + dn_scratch_bytes(n));
    float* rgba = result + 4 * n;
    float* lum2 = rgba + 4 * n;
    const float s = strength_of(strength);
    const FilmDev& d = f->dev;
    // rt-cli/src/lib.rs:104 denoise_film_at: the sums as sums of `samples` samples and each pixel's
    // variance with its own count (its weight). For a film whose every pixel has `samples` samples
    // this is the plain call bit for bit: the sums keep their bits, and the counts give the same
    // degrees of freedom and the same few-samples test.
    RTG_CHECK(launch_dn_rescale(d.rgb, d.alpha, d.lum2, d.weight, n, samples > 1 ? samples : 1, rgba, lum2, sc->stream, grid_for((uint32_t)n, 256)));
    sc->launches += 1;
    if (s > 0.0f) {
        const DnSrc src{rgba, 4, rgba + 3, 4, lum2, f->albedo_sum(), f->albedo_weight(), f->normal(), f->depth(), f->part(), f->material(),
                        d.weight};
        RTG_CHECK(denoise_band(src, d.w, d.h, samples, dn_preset(preset), f->denoise.p, result, sc->stream, grid_for((uint32_t)n, 256),
                               sc->launches));
    }
    if (out) {
        std::vector<float> noisy;
        if (s < 1.0f) {  // the (rescaled) noisy sums, for strength 0 and the blend (denoise.rs:396)
            noisy.resize(4 * n);
            RTG_CHECK(cudaMemcpyAsync(noisy.data(), rgba, n * 16, cudaMemcpyDeviceToHost, sc->stream));
        }
        if (s > 0.0f) RTG_CHECK(cudaMemcpyAsync(out, result, n * 16, cudaMemcpyDeviceToHost, sc->stream));
        RTG_CHECK(cudaStreamSynchronize(sc->stream));
        if (s <= 0.0f) {
            std::memcpy(out, noisy.data(), n * 16);
        } else if (s < 1.0f) {
            const float k1 = 1.0f - s;
            for (size_t p = 0; p < n; ++p)
                for (int k = 0; k < 3; ++k) out[4 * p + k] = noisy[4 * p + k] * k1 + out[4 * p + k] * s;
        }
    } else {
        RTG_CHECK(cudaStreamSynchronize(sc->stream));
    }
    return RTG_STATUS_OK;
}

uint32_t rtg_denoise_halo(uint32_t preset) { return preset > 1 ? 0u : dn_halo(dn_preset(preset)); }

uint32_t rtg_denoise_with(uint32_t preset, float strength, uint32_t width, uint32_t height, uint32_t origin_y, uint32_t rows, uint32_t samples,
                          uint32_t y0, uint32_t y1, const uint8_t* in, float* out) {
    if (!in || !out) return RTG_STATUS_NULL_POINTER;
    if (preset > 1) return RTG_STATUS_BAD_DENOISE;
    std::lock_guard<std::mutex> lk(g_mu);
    // denoise.rs:274 check and :347 check_rows
    if (width == 0 || (uint64_t)origin_y + rows > height) return RTG_STATUS_BAD_DENOISE;
    const DnPreset pr = dn_preset(preset);
    const uint32_t halo = dn_halo(pr), band_end = origin_y + rows;
    const uint32_t low = y0 > halo ? y0 - halo : 0;
    const uint64_t high = std::min<uint64_t>((uint64_t)y1 + halo, height);
    if (y0 > y1 || y0 < origin_y || y1 > band_end || origin_y > low || band_end < high) return RTG_STATUS_BAD_DENOISE;
    const size_t n = (size_t)width * rows;
    const size_t a = (size_t)(y0 - origin_y) * width * 4, b = (size_t)(y1 - origin_y) * width * 4;
    const float s = strength_of(strength);
    if (s <= 0.0f) {
        std::memcpy(out, in + a * 4, (b - a) * 4);
        return RTG_STATUS_OK;
    }
    uint32_t st = device_init();
    if (st) return st;
    DevBuf m;
    struct Release { DevBuf& bb; ~Release() { bb.release(); } } release{m};
    const size_t in_bytes = n * 14 * 4, scratch = dn_scratch_bytes(n);
    m.bytes = ((in_bytes + 255) & ~(size_t)255) + scratch + n * 16;
    RTG_CHECK(cudaMalloc(&m.p, m.bytes));
    uint8_t* base = (uint8_t*)m.p;
    const float* words = (const float*)base;
    void* scr = base + ((in_bytes + 255) & ~(size_t)255);
    float* result = (float*)((uint8_t*)scr + scratch);
    RTG_CHECK(cudaMemcpy(base, in, in_bytes, cudaMemcpyHostToDevice));
    // rt-wasm/src/lib.rs:448-455: sums (4), lum2, albedo (3), normal (3), depth, part, material
    const DnSrc src{words, 4, words + 3, 4, words + n * 4, words + n * 5, nullptr, words + n * 8, words + n * 11,
                    (const uint32_t*)(words + n * 12), (const uint32_t*)(words + n * 13), nullptr};
    uint64_t launches = 0;
    RTG_CHECK(denoise_band(src, width, rows, samples, pr, scr, result, 0, grid_for((uint32_t)n, 256), launches));
    RTG_CHECK(cudaMemcpy(out, result + a, (b - a) * 4, cudaMemcpyDeviceToHost));
    if (s < 1.0f) {
        std::vector<float> noisy(b - a);
        std::memcpy(noisy.data(), in + a * 4, (b - a) * 4);
        const float k1 = 1.0f - s;
        for (size_t i = 0; i < b - a; ++i)
            if (i % 4 != 3) out[i] = noisy[i] * k1 + out[i] * s;
    }
    return RTG_STATUS_OK;
}

uint32_t rtg_denoise(uint32_t width, uint32_t height, uint32_t origin_y, uint32_t rows, uint32_t samples, uint32_t y0, uint32_t y1,
                     const uint8_t* in, float* out) {
    return rtg_denoise_with(0, 1.0f, width, height, origin_y, rows, samples, y0, y1, in, out);
}

uint32_t rtg_adaptive_free(uint32_t ad) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!adaptive_of(ad)) return RTG_STATUS_BAD_HANDLE;
    Scene* sc = scene_of(g_adaptive[ad - 1]->scene);
    if (sc) cudaStreamSynchronize(sc->stream);
    g_adaptive[ad - 1].reset();
    return RTG_STATUS_OK;
}

}  // extern "C"
