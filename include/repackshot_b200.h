/* repackshot_b200: the C ABI of the B200 path tracer, a drop-in for the progressive
 * sample-and-accumulate render of the Repackshot engine.
 *
 * The reference's engine is Rust; its only C ABI is the hand-written one of the rt-wasm crate
 * (engine/crates/rt-wasm/src/ffi.rs), which every host (the Web Worker pool, the parity tools)
 * binds. The functions below keep its names (rt_ -> rtg_), argument meaning, ownership and
 * status codes; the film and parity entry points have no wasm counterpart and replace the
 * in-process Rust calls cited beside them.
 *
 * Threading: every call holds one library-wide lock, so calls serialise (the reference's
 * registry sits behind a Mutex, rt-wasm/src/lib.rs:10-13). Work runs on a CUDA stream owned by
 * the scene; every call returns after its work is complete unless stated otherwise.
 */
#ifndef REPACKSHOT_B200_H
#define REPACKSHOT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RTG_ABI_VERSION 1u

/* Status codes: 0-5 as rt-wasm/src/lib.rs:37-53; 16 and up are this library's own. */
#define RTG_STATUS_OK 0u
#define RTG_STATUS_BAD_HANDLE 1u
#define RTG_STATUS_BAD_TILE 2u      /* empty tile or more than RTG_MAX_TILE_PIXELS pixels */
#define RTG_STATUS_NULL_POINTER 3u
#define RTG_STATUS_BAD_SCENE 4u
#define RTG_STATUS_BAD_DENOISE 5u   /* the denoiser's preset, sizes, band or halo do not fit */
#define RTG_STATUS_CUDA_ERROR 16u   /* the message is in rtg_scene_error_* */
#define RTG_STATUS_STACK_OVERFLOW 17u
#define RTG_STATUS_BAD_FILM 18u
#define RTG_STATUS_BAD_ARGUMENT 19u  /* a size or count the call cannot take; the message says which */

/* Largest tile rtg_render_tile accepts: 2048 x 2048 (rt-wasm/src/lib.rs:56 MAX_TILE_PIXELS). */
#define RTG_MAX_TILE_PIXELS (1ull << 22)

/* rt_version (ffi.rs): the ABI version. */
uint32_t rtg_version(void);

/* Bits of rtg_features (rt-core/src/lib.rs:76-150 FEATURE_*; the same values). */
#define RTG_FEATURE_SECTION 4u  /* Q1: the section view (SECT), caps of the cut solids */
#define RTG_FEATURE_IES 8u      /* L5: IES lights (LGHT kind 5, IESP sections) */
#define RTG_FEATURE_CAMERAS 16u /* K3: panoramic projections, the exterior factor, instances hidden to the camera */

/* rt_features (ffi.rs:22, lib.rs:159 FEATURES): what this engine reads beyond the RSB every engine
 * reads, as the reference's FEATURE_* bits: RTG_FEATURE_SECTION | RTG_FEATURE_IES | RTG_FEATURE_CAMERAS.
 * The other bits (textures, material programs, pattern nodes, drops, front glass, weather, nested
 * dielectrics) are clear: those sections are refused at load, so a host writes none of them. */
uint32_t rtg_features(void);

/* rt_scene_load (ffi.rs:56-66, lib.rs:145): parses an RSB scene (copied; the caller keeps its
 * bytes), builds its BVHs and uploads it. Returns a handle > 0, or 0 after recording the error
 * (rtg_scene_error_len / _copy). Lights of kinds 0-5 (rect, disk, sun, point, spot, IES) and
 * emissive meshes, HDRI environments and background images (BMAP sections: 8-bit sRGB, linear f32,
 * Radiance files), the classic and the physical sky, panoramic cameras, cut-outs, thin walls and
 * section views (SECT: the model cut by a plane, closed solids capped, the studio exempt) render;
 * features outside the path tracer's core (textures, material programs, lens optics,
 * particles, front glass, weather, nested dielectrics, OpenEXR bitmaps, scattering
 * media, dispersive glass, bevels, caustic photon maps, the shadow catcher) are refused with a
 * message that starts with "unsupported:". */
uint32_t rtg_scene_load(const uint8_t* bytes, uint32_t len);

/* rt_scene_update (ffi.rs:68-88, rt-wasm/src/lib.rs:171-193, Scene::update_from_rsb
 * rt-core/src/scene/rsb.rs:1630): replaces the loaded scene with new RSB bytes (copied). A file
 * without MESH sections keeps the scene's meshes: its INST sections, or the implicit instances of
 * the kept meshes, refer to them; when the instances' meshes, transforms and visibility flags are
 * also unchanged, the device trees are kept and only the camera, image size, materials, lights and
 * settings are uploaded again. A file without BMAP sections keeps the scene's bitmaps, as the
 * reference's update does. Films keep their rectangles. RTG_STATUS_OK, RTG_STATUS_BAD_HANDLE,
 * RTG_STATUS_NULL_POINTER, or RTG_STATUS_BAD_SCENE with the message in rtg_scene_error_*; on any
 * error the scene is unchanged. */
uint32_t rtg_scene_update(uint32_t handle, const uint8_t* bytes, uint32_t len);

/* rt_scene_error_len / rt_scene_error_copy (ffi.rs:90-110): the last error message, UTF-8,
 * without terminator; empty after a successful load. */
uint32_t rtg_scene_error_len(void);
void rtg_scene_error_copy(uint8_t* out);

/* rt_scene_free (ffi.rs:113-116): RTG_STATUS_OK or RTG_STATUS_BAD_HANDLE. */
uint32_t rtg_scene_free(uint32_t handle);

/* rt_render_tile (ffi.rs:118-157, lib.rs:701-710): sample `sample_index` of the pixel rectangle
 * (x, y, w, h) into `out`, w*h*3 floats of linear RGB, row major; one sample, not accumulated;
 * pixels outside the image are zero. */
uint32_t rtg_render_tile(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t sample_index,
                         float* out);

/* rt_render_tile_rgba (ffi.rs:159-197, lib.rs:715): as rtg_render_tile with coverage, w*h*4
 * floats of premultiplied RGBA. */
uint32_t rtg_render_tile_rgba(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t sample_index,
                              float* out);

/* A film on the device: the reference's Film (rt-core/src/image.rs:14-93) over the image
 * rectangle (x, y, w, h): per pixel the sums of RGB, sample count, coverage and squared
 * luminance. Returns a film handle > 0, or 0 (error message as for loads). */
uint32_t rtg_film_create(uint32_t scene, uint32_t x, uint32_t y, uint32_t w, uint32_t h);
uint32_t rtg_film_free(uint32_t film);
uint32_t rtg_film_clear(uint32_t film);

/* render_tile_prepared (rt-core/src/render.rs:272-281) over a range of samples: for every
 * pixel of the film inside the image, film += sample(first_sample) + ... +
 * sample(first_sample + count - 1), added in sample order, as repeated calls of the reference
 * accumulate. `rays` (may be null) receives the camera + extension + shadow rays cast. */
uint32_t rtg_render_progressive(uint32_t scene, uint32_t film, uint32_t first_sample, uint32_t count, uint64_t* rays);

/* No counterpart in the reference. rtg_render_progressive without device allocation, for
 * callers that cannot call cudaMalloc while they render: a host that has handed the device's
 * memory to its own pool allocator, or a render server that must not meet an out-of-memory
 * error in the middle of a frame. (The scene and the film are allocated when they are created,
 * as before; only the per-wave path state differs.)
 *
 * The path state lives in one fixed array of RTG_NOALLOC_SCRATCH_BYTES (12 MiB) in the
 * library's device code. Every GPU that loads the library holds that array until the process
 * exits, whether or not this function is called. A wave holds at most RTG_NOALLOC_MAX_PATHS
 * paths, so the film is rendered in bands of rows and waves of samples that fit; any film of a
 * loadable scene (images are at most 16384 pixels wide) is accepted. A row wider than
 * RTG_NOALLOC_MAX_PATHS pixels would not fit and is refused with RTG_STATUS_BAD_FILM and a
 * message. A scene with edge samples (RNDR edge_supersample above 1) is refused with
 * RTG_STATUS_BAD_SCENE: its edge mask would need device memory.
 *
 * The first call on each device does the set-up: it looks up the array's address on the
 * current device (cudaGetSymbolAddress), which may load the library's device code there. Make
 * that first call before any stream capture. Later calls check the remembered address against
 * the device's mappings (cudaPointerGetAttributes) and look it up again when it is gone, as after
 * a cudaDeviceReset (which also ends every scene and film of that device). Each call zeroes the array's queue counters
 * itself before it renders; nothing else in the array has to start at zero.
 *
 * There is one array per device, shared by every call on that device. Calls through this
 * library serialise on its lock and return after their work is complete, so they do not
 * overlap; work of two calls that ran on the device at the same time would race on the array.
 *
 * Arguments, film result and status codes are those of rtg_render_progressive; the film's bits
 * are the same, and so are its guide sums when the film has fused guides
 * (rtg_film_guides_fused): the first hits' albedo goes through a slice of the same array. Extend-kernel timing (rtg_timing) counts its rays and launches but brackets no
 * launch with events. */
#define RTG_NOALLOC_SCRATCH_BYTES (12ull << 20)
#define RTG_NOALLOC_MAX_PATHS 65536u
uint32_t rtg_render_progressive_noalloc(uint32_t scene, uint32_t film, uint32_t first_sample, uint32_t count,
                                        uint64_t* rays);

/* The batched render queue (no reference counterpart; the reference's product runs its render
 * queue one job after another, src/ui/render-queue.ts, over cameras x studios,
 * src/core/render.ts:71). A queue renders many variants of one loaded scene -- other cameras,
 * image sizes, materials, light rigs, seeds, sample ranges -- over the scene's geometry, packing
 * the paths of all of them into as few waves as device memory allows instead of one call each.
 * Every job's film gets the bits rtg_render_progressive gives after rtg_scene_update with the
 * job's file.
 *
 * rtg_queue_create: a queue over scene `scene`; a handle > 0, or 0 (message as for loads).
 * rtg_queue_add: a job: `bytes` is an RSB file without MESH sections whose instances match the
 * scene's (the form rtg_scene_update takes for a change that keeps the geometry), samples
 * [first_sample, first_sample + count). *film receives a new film over the job's whole image
 * (free it with rtg_film_free). RTG_STATUS_BAD_SCENE (message) when the file is invalid or
 * changes the geometry.
 * rtg_queue_run: renders every job added since the last run, then forgets them (their films stay).
 * flags: RTG_QUEUE_GRAPH captures the run's launches into one CUDA graph and launches that. `rays`
 * (may be null) receives the camera + extension + shadow rays of all jobs.
 * rtg_queue_free: forgets the queue and its pending jobs. */
#define RTG_QUEUE_GRAPH 1u
uint32_t rtg_queue_create(uint32_t scene);
uint32_t rtg_queue_add(uint32_t queue, const uint8_t* bytes, uint32_t len, uint32_t first_sample, uint32_t count, uint32_t* film);
uint32_t rtg_queue_run(uint32_t queue, uint32_t flags, uint64_t* rays);
uint32_t rtg_queue_free(uint32_t queue);

/* The adjoint (no reference counterpart): gradients of an image loss with respect to the scene's
 * parameters, by path replay backpropagation. rtg_adjoint_params gives the parameter counts:
 * every material (4 parameters: base colour R, G, B and GGX alpha = roughness^2) and every scene
 * light (1: its power).
 *
 * rtg_render_adjoint clears `film`, renders samples [first_sample, first_sample + count) into it
 * (the forward pass: with RTG_ADJOINT_CORRELATED the same bits as rtg_render_progressive), and
 * returns
 *   *loss = mean over the film's pixels and channels of (I - target)^2, I = rgb / weight, `target`
 *           w*h*3 floats of linear RGB over the film's rectangle (row major, host memory);
 *   grads[0 .. 4 n_materials): per material d loss / d (base R, base G, base B, alpha);
 *   grads[4 n_materials ..): per light d loss / d power  (n_grads = 4 n_materials + n_lights).
 * The backward pass replays every path from its pixel and sample index (nothing of the paths is
 * stored) and propagates the loss through them; sampling decisions are held fixed (detached).
 * By default the samples are split into two halves, A = [first_sample, first_sample + count/2)
 * and B = the rest, and each half's paths take the loss's derivative from the other half's image.
 * Half B is drawn with the scene's seed complemented (~seed): an independent scramble, since two
 * ranges of one pixel's scrambled sequence are stratified together and so correlated. The
 * gradient is then an unbiased estimate of the gradient of the loss of the noise-free image (a
 * residual and a derivative from the same paths, or from correlated halves, carry a covariance
 * term that shifts the minimum, e.g. towards dimmer lights). With RTG_ADJOINT_CORRELATED every
 * path uses the residual of the whole film, all samples from the scene's seed: the derivative of
 * this very estimate, as a same-seed finite difference measures it.
 * The film must lie inside the image; every path of the call is held in one wave (172 bytes each).
 * `residual` (may be null) receives the sum over replayed paths of |radiance left after the
 * replay| and of |radiance|: the first is 0 up to rounding when the replay retraced the forward
 * paths. A scene with cut-outs or thin walls is refused (RTG_STATUS_BAD_SCENE): the replay does not
 * walk shadow rays through them. */
#define RTG_ADJOINT_CORRELATED 1u
uint32_t rtg_adjoint_params(uint32_t scene, uint32_t* n_materials, uint32_t* n_lights);
uint32_t rtg_render_adjoint(uint32_t scene, uint32_t film, const float* target, uint32_t first_sample, uint32_t count, uint32_t flags,
                            float* loss, float* grads, uint32_t n_grads, float* residual);

/* Copies the film's sums to host memory (any pointer may be null): rgb 3*w*h floats, weight,
 * alpha and lum2 w*h floats each. */
uint32_t rtg_film_read(uint32_t film, float* rgb, float* weight, float* alpha, float* lum2);

/* Film::to_srgb8_tonemapped / to_srgb16_tonemapped (rt-core/src/image.rs:186-214): the film
 * resolved (rgb / weight, black where no sample), `ev` stops of exposure (2^ev), tone curve
 * `tonemap` (the RNDR value: 0 linear, 1 ACES, 2 filmic, 3 AgX, 4 standard; any other ACES;
 * color.rs:95-250), sRGB-encoded and quantised as the reference quantises (v * 255 + 0.5, or
 * * 65535, truncated): `out` w*h*3 bytes or 16-bit words, row major. */
uint32_t rtg_film_srgb8(uint32_t film, float ev, uint32_t tonemap, uint8_t* out);
uint32_t rtg_film_srgb16(uint32_t film, float ev, uint32_t tonemap, uint16_t* out);

/* Film::to_linear_exposed (rt-core/src/image.rs:218-221): the film resolved as above and
 * multiplied by 2^ev, scene-linear light with no tone curve and no clamp: `out` w*h*3 floats, row
 * major. The samples of the reference's 32-bit float TIFF and of its DNG (rt-cli/src/lib.rs:740-760). */
uint32_t rtg_film_linear(uint32_t film, float ev, float* out);

/* The same encodings of film planes given in host memory: `rgb` w*h*3 sums and `weight` w*h
 * sample weights (a Film's rgb and weight, rt-core/src/image.rs), `bits` 8 or 16 (tone curve and
 * sRGB, as rtg_film_srgb8/16) or 32 (linear exposed floats, as rtg_film_linear; `tonemap` unused);
 * `out` w*h*3 bytes, 16-bit words or floats. For images that are no render's film: the
 * denoised film of the command line (rt-cli/src/cli.rs:1886-1900) is encoded through it. */
uint32_t rtg_encode_planes(const float* rgb, const float* weight, uint32_t width, uint32_t height, float ev, uint32_t tonemap,
                           uint32_t bits, void* out);

/* The scene's output settings from its RNDR section: exposure in stops, tone curve, samples per
 * pixel (any pointer may be null). */
uint32_t rtg_scene_output(uint32_t scene, float* exposure_ev, uint32_t* tonemap, uint32_t* max_samples);

/* The film's device arrays (valid until rtg_film_free), for callers that stay on the GPU. */
uint32_t rtg_film_device(uint32_t film, float** rgb, float** weight, float** alpha, float** lum2);

/* radiance_with (rt-core/src/integrator/mod.rs:1107) of explicit paths: for each (x, y,
 * sample index) triple of `xys` (3*n u32), out5[5i..5i+5] = radiance r, g, b, alpha, 0. */
uint32_t rtg_render_paths(uint32_t scene, const uint32_t* xys, uint32_t n, float* out5);

/* Geometry::trace_class / occluded_class (rt-core/src/geometry/mod.rs:566-629) of a ray batch:
 * rays 8*n floats (origin xyz, dir xyz, t_min, t_max). mode bit 0: camera class (instances
 * hidden to the camera are skipped); bit 1: any hit. Nearest: out 3*n u32 = instance, triangle,
 * t bits (instance 0xffffffff: miss). Any: out n u32 = 1 when blocked. */
uint32_t rtg_trace_rays(uint32_t scene, const float* rays, uint32_t n, uint32_t mode, uint32_t* out);

/* What a mesh is as a solid for the caps of a section view (rt-core/src/geometry/solid.rs analyse):
 * `positions` 3*n_vertices floats, `indices` n_indices (a multiple of 3) vertex indices. `solid`
 * gets 0 (open: not capped), 1 (closed, wound counter-clockwise seen from outside) or 2 (closed,
 * wound inward). The host computation a scene load runs for every capped instance's mesh; no GPU. */
uint32_t rtg_mesh_solid(const float* positions, uint32_t n_vertices, const uint32_t* indices, uint32_t n_indices, uint32_t* solid);

/* Facts of a loaded scene: width, height, max depth, instanced triangles, BVH nodes, leaf
 * triangles, BVH build seconds, rays cast so far. */
uint32_t rtg_scene_stats(uint32_t scene, double* out8);

/* Largest number of paths one wave holds (172 bytes of device memory per path, kept until the
 * scene is freed). 0, the default, sizes each wave to every path of the call, bounded by half of
 * the device memory then free: a call then runs as few waves as memory allows, and each wave's
 * tail of long paths is paid once. */
uint32_t rtg_set_path_capacity(uint32_t scene, uint32_t paths);

/* No counterpart in the reference: how the scene's waves order their work. None of it changes a
 * film's bits; it changes how fast the traversal and shading kernels run.
 * values[0]: ray-sort bits per axis, 0-5 (0: off). Before each traversal after the camera rays,
 *   the extension rays are ordered by the octant of their direction over the Morton code of their
 *   origin's cell on a grid of 2^bits cells per axis over the box of the scene's main instances.
 * values[1]: 1 sorts the shadow rays the same way (with ray-sort bits above 0).
 * values[2]: 1 shades the paths ordered by the material they hit; 0 in traversal order.
 * values[3]: paths per wave, as rtg_set_path_capacity (0: automatic).
 * values[4]: 1 marks the scene's traversal data (tree nodes, leaf triangles) as persisting in L2
 *   for the traversal kernels (an access-policy window on their launches; the process's CUDA
 *   context sets L2 aside for it the first time), so the streamed path state does not evict it.
 * values[5]: the tail limit (0: off). From a wave's third round on, a round whose extension queue
 *   holds at most this many paths runs them, and every later round of the wave, in one launch:
 *   each thread carries its paths to the end alone (nearest hit, vertex, shadow ray, next ray).
 *   Scenes with cut-outs or thin walls and batched queue waves keep the wavefront.
 * rtg_set_tuning sets the first n values (n <= 6; later ones keep theirs); RTG_STATUS_BAD_SCENE for
 * ray-sort bits above 5. rtg_get_tuning writes the first n (n <= 6). A loaded scene starts at
 * 0, 0, 1, 0, 0, 16384. */
uint32_t rtg_set_tuning(uint32_t scene, const uint32_t* values, uint32_t n);
uint32_t rtg_get_tuning(uint32_t scene, uint32_t* values, uint32_t n);

/* No counterpart in the reference: the autotuner. Chooses the scene's tuning (the six values of
 * rtg_set_tuning) by rendering samples [first_sample, first_sample + count) of the rectangle
 * (x, y, w, h) of the image (clipped to it; into a film of its own) under candidate settings, by
 * coordinate descent from the scene's own tuning: the ray sort's bits 0, 3, 4 and 5 (shadow rays
 * sorted along), then shadow rays sorted or not, shading material-sorted or not, the L2 window on
 * or off, the tail limit 0, 2^16, 2^18 or 2^20, then waves of the whole call, a half or a quarter
 * of its paths (at least 2^20). Each candidate renders once to warm up, then three times timed
 * with CUDA events on the scene's stream; its median counts, and a candidate replaces the fastest
 * so far only when it is more than 1% faster. The scene keeps the fastest.
 * `report` (may be null) receives 7 doubles per candidate tried, at most max_report of them: its
 * six values and its milliseconds; *n_tried (may be null) the number tried. Films are not touched; a render of the
 * candidate is what a call with those samples would cost, so pick a count that is representative
 * of the calls to come. RTG_STATUS_BAD_TILE for an empty rectangle or no samples. */
uint32_t rtg_autotune(uint32_t scene, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t first_sample, uint32_t count,
                      double* report, uint32_t max_report, uint32_t* n_tried);

/* Extend-kernel timing: when enabled, every extend launch is bracketed by CUDA events on the
 * scene's stream. out5 = total extend milliseconds, extend launches, camera + extension rays,
 * shadow rays, kernels launched, accumulated since the last reset (read before this call's
 * reset). */
uint32_t rtg_timing(uint32_t scene, uint32_t enable, uint32_t reset, double* out5);

/* Runs the scene's work on `stream` (a cudaStream_t the caller owns and keeps alive until the
 * scene is freed or another stream is set); null restores a stream of the scene's own. */
uint32_t rtg_set_stream(uint32_t scene, void* stream);

uint32_t rtg_synchronize(uint32_t scene);

/* ---- Adaptive sampling (E10, rt-core/src/adaptive.rs) ------------------------------------------
 * The image is sampled in rounds: every pixel gets 16 samples first, then each round goes to the
 * 8 x 8 blocks whose smoothed relative error of the mean is at or above the median of those still
 * above the noise target (RNDR.noise_threshold) and under the cap; the round's size grows when few
 * blocks are active. A block that stops keeps its samples: every pixel stays the plain mean of its
 * own samples 0..n, the pixel a progressive render of n samples gives it.
 *
 * rt_adaptive_decide (rt-wasm/src/ffi.rs:237-289): the decision of a width x height image from
 * its blocks' samples (`counts`, u32 each, ceil(width/8) x ceil(height/8) of them, row by row), its
 * RGBA sums (`sums`, 4 f32 a pixel), its squared-luminance sums (`lum2`, f32), the exposure `ev`,
 * the noise `target` and the sample `cap` (0: none). Writes one byte a block to `active` (1: in the
 * next round) and six u32 words to `decision`: the round's samples (0: converged), the active
 * blocks, the blocks, then the bits of the threshold, the largest block error and the pixel-samples
 * still needed. Pointers need no alignment. RTG_STATUS_NULL_POINTER for a null pointer,
 * RTG_STATUS_BAD_TILE for an empty image (or a side above 16384). The per-pixel errors are found
 * on the GPU, the per-block choice on the host, with the reference's bits. */
uint32_t rtg_adaptive_decide(uint32_t width, uint32_t height, float ev, float target, uint32_t cap, const uint8_t* counts,
                             const uint8_t* sums, const uint8_t* lum2, uint8_t* active, uint8_t* decision);

/* rt_render_block_rgba (rt-wasm/src/ffi.rs:196-235): sample `sample_index` of the pixel rectangle
 * (x, y, w, h), a block of a round, as rtg_render_tile_rgba gives it (w*h*4 floats, RGBA; edge
 * pixels take their edge samples). `iteration` names the photon map of the reference's caustics;
 * scenes with caustics are refused at load, so it is unused. Status as rtg_render_tile_rgba. */
uint32_t rtg_render_block_rgba(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t sample_index,
                               uint32_t iteration, float* out);

/* An adaptive render of `scene` into `film` (one of the scene's films covering its whole image,
 * normally cleared) with at most `cap` samples a pixel (0: none), the noise target and exposure of
 * the scene's RNDR section (adaptive.rs:349 Adaptive::new). Returns its handle, or 0 (the reason
 * in rtg_scene_error_*). */
uint32_t rtg_adaptive_create(uint32_t scene, uint32_t film, uint32_t cap);
/* Runs the host loop of an adaptive render (adaptive/tests.rs:311): at the end of a round decides
 * the next (block errors on the GPU from the film where it lies); renders passes of at most `pass`
 * samples of the round (0: the whole round, the fewest and largest waves), the first round over
 * the whole image, later ones over the pixels
 * of the active blocks only; stops when converged or after `max_passes` passes (0: no limit).
 * `passes` and `rays` (may be null) get the passes rendered and the rays cast. The film is the
 * same for any `pass` and any split into calls. */
uint32_t rtg_adaptive_run(uint32_t ad, uint32_t pass, uint32_t max_passes, uint32_t* passes, uint64_t* rays);
/* out16: the round's samples, the samples of it rendered, those left, the photon-map iteration of
 * the next sample, converged (0/1), decisions taken, the fewest and the most samples of a pixel,
 * the last decision's six words (as rtg_adaptive_decide's), the columns and rows of blocks. */
uint32_t rtg_adaptive_state(uint32_t ad, uint32_t* out16);
/* Each block's samples now (u32, row by row) and whether it is in the round (one byte each);
 * either pointer may be null, not both. */
uint32_t rtg_adaptive_counts(uint32_t ad, uint32_t* samples, uint8_t* active);
uint32_t rtg_adaptive_free(uint32_t ad);

/* ---- Guide passes and the denoiser (rt-post/src/denoise.rs, rt-core/src/passes.rs) ----------------
 * rt_render_tile_passes (rt-wasm/src/ffi.rs:303-343, lib.rs:484): the exact passes of `mask`
 * (normal 2, depth 4, part id 8, material id 16, circle of confusion 32; the albedo bit 1, the
 * alpha bit 64 and unknown bits are ignored) of the rectangle (x, y, w, h), from one ray through
 * each pixel's centre: the planes one after another in that order, w*h*3 words for the normal and
 * w*h for the others (f32; u32 for the ids), rows from the top. Status as rtg_render_tile. */
uint32_t rtg_render_tile_passes(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t mask, uint8_t* out);
/* rt_render_tile_albedo (ffi.rs:345-384, lib.rs:510): the albedo of sample `sample_index` of the
 * rectangle's pixels, w*h*3 floats: the base colour of what that sample's camera ray met first
 * (0 for the background and outside the image; an edge pixel's mean over its sub-samples). */
uint32_t rtg_render_tile_albedo(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t sample_index, float* out);
/* rt_render_tile_alpha (ffi.rs:379-418, lib.rs:537): the coverage (the alpha pass) of sample
 * `sample_index` of the rectangle's pixels, w*h floats: 1 where that sample's camera ray met a
 * surface of an instance first, 0 where it met the floor, a light panel or nothing (0 outside the
 * image; an edge pixel's mean over its sub-samples). Status as rtg_render_tile. */
uint32_t rtg_render_tile_alpha(uint32_t handle, uint32_t x, uint32_t y, uint32_t w, uint32_t h, uint32_t sample_index, float* out);
/* rt_denoise / rt_denoise_with (ffi.rs:599-683, lib.rs:420-475): the denoiser on a band of `rows`
 * image rows from `origin_y` of a width x height image of `samples` samples a pixel. `in` holds
 * width*rows*14 little-endian words: the planes sums (RGBA), lum2, albedo (3), normal (3), depth,
 * part id and material id, one after another. Writes the denoised RGBA sums of image rows y0 .. y1
 * (width*(y1-y0)*4 floats) to `out`. `preset` 0 is the full filter, 1 the viewport's; `strength`
 * (0..1, NaN: 1) blends noisy x (1 - s) + denoised x s per colour channel, and at 0 no filter runs.
 * RTG_STATUS_NULL_POINTER, or RTG_STATUS_BAD_DENOISE when the preset, the sizes, the band or its
 * halo do not fit. The filter runs on the GPU with the reference's bits. */
uint32_t rtg_denoise(uint32_t width, uint32_t height, uint32_t origin_y, uint32_t rows, uint32_t samples, uint32_t y0, uint32_t y1,
                     const uint8_t* in, float* out);
uint32_t rtg_denoise_with(uint32_t preset, float strength, uint32_t width, uint32_t height, uint32_t origin_y, uint32_t rows, uint32_t samples,
                          uint32_t y0, uint32_t y1, const uint8_t* in, float* out);
/* rt_denoise_halo (ffi.rs:685-691): rows a band of `preset` holds above and below the rows it
 * computes (72 for the full filter, 24 for the viewport's), 0 for an unknown preset. */
uint32_t rtg_denoise_halo(uint32_t preset);
/* No counterpart in the reference (its hosts render the passes tile by tile and hand the planes
 * to rt_denoise): the guide passes of a film on the device. Writes the exact passes of the film's
 * pixels and adds the albedo of samples [first_sample, first_sample + count) to the film's albedo
 * sums (rtg_film_clear clears them with the film). */
uint32_t rtg_film_guides(uint32_t scene, uint32_t film, uint32_t first_sample, uint32_t count);
/* No counterpart in the reference. With `enable`, writes the film's exact passes now and makes
 * every later rtg_render_progressive on the film add each sample's albedo to the film's albedo
 * sums as well, read from the first hit its camera ray already traced: the guides of
 * rtg_film_guides, bit for bit, without tracing the camera rays a second time. 0 stops it.
 * Only rtg_render_progressive fills the guides this way; the allocation-free render, the queue
 * and the adaptive passes do not, so call rtg_film_guides for films rendered through them. */
uint32_t rtg_film_guides_fused(uint32_t scene, uint32_t film, uint32_t enable);
/* The denoiser on a film that covers the whole image, with its guide passes, as rtg_denoise_with
 * on the film's planes: the film stays on the device, and `out` (may be null: the result stays on
 * the device) gets width*height*4 floats of RGBA sums of `samples` samples. A film whose pixels
 * have their own counts (an adaptive render) is denoised as the reference's CLI does it
 * (rt-cli/src/lib.rs:104): its sums rescaled to `samples` samples (adaptive.rs:260) and each
 * pixel's variance divided by its own count; a film whose every pixel has `samples` samples gives
 * the plain result bit for bit. */
uint32_t rtg_film_denoise(uint32_t film, uint32_t preset, float strength, uint32_t samples, float* out);

#ifdef __cplusplus
}
#endif

#endif /* REPACKSHOT_B200_H */
