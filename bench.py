#!/usr/bin/env python
"""Benchmark of the drop-in path tracer on the 1080p product scene.

Workload (one step): a 1920x1080 frame at 64 samples per pixel, path depth 12, of the seeded
product scene (a displaced (2,3) torus knot of 1,048,576 triangles in 16 materials: GGX
conductors, rough dielectrics, Lambert; three rect softboxes and a gradient dome), rendered by
``Film.render`` (rtg_render_progressive) into a device film. ``value`` is Mpaths/s over all
ranks, device-timed with CUDA events on the stream the kernels run on; ``e2e`` is the same
render through the C ABI with the film read back to pinned host memory every step.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Multi-GPU: one process per GPU under torch.distributed.run; each rank renders its own sample
range of the frame (replicas, no data-path collective; "weak" scaling).

``--impl reference`` times the reference's CPU path tracer instead (the C++ restatement in
oracle/, bit-exact with the reference's pinned hashes) on the host's cores, on bounded samples
of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mpaths/s at equal rel-MSE: plain vs batched queue; adjoint ms/iter vs forward"
WIDTH, HEIGHT, SPP, DEPTH = 1920, 1080, 64, 12
WORKLOAD = ("1080p product scene: 1920x1080, 64 spp, max depth 12, seeded displaced (2,3) torus knot "
            "(1024x512 segments, 1,048,576 triangles) in 16 materials (6 GGX conductors, 4 rough dielectrics, "
            "6 Lambert) on a floor quad, 3 rect softboxes (radiance 5-20) and a gradient dome")
DATA = "synthetic (seeded procedural scene; no dataset)"
FALLBACK_HBM_GBS = 6650.0
BYTES_RAY_IO = 32 + 12  # ray in, hit out
# DRAM bytes (read + write) per extend ray, from one ncu capture of k_extend on this scene (round 0
# of a 4 Mi-path wave: 341 MB for 4,147,200 rays). Scaled to a launch by the rays it traces.
DRAM_BYTES_PER_EXTEND_RAY = 82.0


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


def product_rsb():
    from repackshot_b200 import scenes
    return scenes.to_rsb(scenes.product_scene(width=WIDTH, height=HEIGHT, spp=SPP, depth=DEPTH))


def sample_bands(n_bands: int, rows: int = 8):
    """Row bands spread evenly over the image (the CPU samples and the traversal statistics)."""
    step = HEIGHT // n_bands
    return [(i * step + (step - rows) // 2, rows) for i in range(n_bands)]


def oracle_sample(orc_scene, bands, first, count, threads, images=None):
    """Renders the bands with the oracle; returns (seconds, paths, stats summed). With `images`
    (a list), each band's resolved pixels are appended to it."""
    import oracle
    t0 = time.perf_counter()
    stats = np.zeros(11, np.int64)
    paths = 0
    for y, rows in bands:
        rgb, wt, _, _, st = orc_scene.render_film(first, count, x=0, y=y, w=WIDTH, h=rows, tile=32, threads=threads)
        if images is not None:
            images.append(oracle.resolve(rgb, wt))
        stats += np.array(st, np.int64)
        paths += WIDTH * rows * count
    return time.perf_counter() - t0, paths, stats


def rel_mse(a, b, eps=1.0e-2) -> float:
    """Mean over pixels and channels of (a - b)^2 / (b^2 + eps): the image error at equal spp
    (the reference defines none; the epsilon is this benchmark's)."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.mean((a - b) ** 2 / (b * b + eps)))


def traversal_bytes(stats, merged=True) -> float:
    """Algorithmic bytes per nearest-hit ray: ray in + hit out + the reference BVH8 layout's
    256-byte wide nodes and 160-byte triangle packets it visits (engine/crates/rt-core/src/
    geometry/bvh.rs:96-102, triangle.rs:163-171). `merged`: visits in one reference-layout BVH8
    over all the scene's triangles (the tree this path traverses); otherwise in the reference's
    own two-level tree of per-material instances."""
    nq = max(stats[1], 1)
    nodes, packets = (stats[7], stats[8]) if merged else (stats[2], stats[3])
    return BYTES_RAY_IO + (256.0 * nodes + 160.0 * packets) / nq


class Clocks:
    """nvidia-smi samples every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.file.seek(0)
        rows = [r.split(", ") for r in self.file.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "gloo" if args.impl == "reference" else "nccl"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def run_reference(args, world, rank):
    """The reference arm: the CPU path tracer on the host's cores over the whole frame, a bounded
    number of samples per step (each step the next sample indices of the 64)."""
    import oracle
    threads = os.cpu_count() or 1
    rsb = product_rsb()
    o = oracle.OracleScene(rsb)
    # Calibrate on a band at 1 spp, then size a step to about 2.5 s of whole-frame work.
    o.render_tile(WIDTH // 2, HEIGHT // 2, 8, 8, 0)  # first use generates the energy tables
    dt, paths, _ = oracle_sample(o, sample_bands(4), 0, 1, threads)
    rate = paths / max(dt, 1e-6)
    spp_step = int(max(1, min(SPP, rate * 2.5 / (WIDTH * HEIGHT))))
    times, total_paths = [], 0
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        o.render_film((i * spp_step) % SPP, spp_step, tile=32, threads=threads)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
            total_paths += WIDTH * HEIGHT * spp_step
    value = total_paths / sum(times) / 1e6
    sample = f"the whole 1920x1080 frame at {spp_step} spp per step (sample indices cycling through the frame's 64)"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": DATA,
        "config": {"workload": WORKLOAD, "width": WIDTH, "height": HEIGHT, "spp": SPP, "max_depth": DEPTH,
                   "sample_per_step": sample},
        "cpu_baseline": {"value": value, "unit": "Mpaths/s", "cores": threads, "kind": "port",
                         "sample": sample + " (C++ restatement of the reference, bit-exact with its pinned hashes)"},
        "e2e": {"value": value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def adaptive_comparison(rtg, scene, dist, world, target, uniform_ms):
    """The frame rendered adaptively (E10): the product scene with a noise target and its 64 spp as
    the cap, updated into the loaded scene (same geometry), to convergence, a pass a round.
    Wall time around the synchronous run, max over ranks; its pixel-samples against the uniform
    frame's, and its throughput against the uniform frame's time."""
    from repackshot_b200 import scenes, shards
    s = scenes.product_scene(width=WIDTH, height=HEIGHT, spp=SPP, depth=DEPTH)
    s.adaptive, s.noise_threshold = 1, target
    scene.update(scenes.to_rsb(s, meshes=False))
    film = scene.film()
    warm = rtg.Adaptive(scene, film, 2)  # warm-up: the kernels of a pass and of a decision
    warm.run(2)
    warm.close()
    film.clear()
    ad = rtg.Adaptive(scene, film, SPP)
    scene.synchronize()
    t0 = time.perf_counter()
    passes, rays = ad.run(0)
    scene.synchronize()
    dt = shards.max_over_ranks(time.perf_counter() - t0, dist)
    st = ad.state()
    samples, _ = ad.counts()
    per_pixel = np.repeat(np.repeat(samples, 8, 0), 8, 1)[:HEIGHT, :WIDTH]
    paths = int(per_pixel.astype(np.int64).sum())
    ad.close()
    return {"noise_target": target, "cap": SPP, "passes": passes, "decisions": st["decisions"], "converged": bool(st["converged"]),
            "samples_lo_hi": [st["lo"], st["hi"]], "paths_per_gpu": paths, "pixel_samples_vs_uniform": paths / (WIDTH * HEIGHT * SPP),
            "ms": dt * 1e3, "mpaths_s": world * paths / dt / 1e6, "uniform_frame_ms": uniform_ms,
            "last_max_error": float(np.frombuffer(np.uint32(st["last"][4]).tobytes(), np.float32)[0]),
            "path": "rtg_adaptive_create + rtg_adaptive_run (first round: the progressive renderer over the image; later "
                    "rounds: list waves over the active 8x8 blocks; block errors on the device, the choice on the host)"}


def denoise_comparison(rtg, film, samples, stream, dist, clocks_note=None):
    """The 1080p frame's guide passes and the denoiser (rt-post/src/denoise.rs, the full filter)
    on the device: rtg_film_guides over the frame's samples, then rtg_film_denoise with the result
    kept on the device; device time by CUDA events on the scene's stream, max over ranks; the
    oracle's filter timed on a bounded band of rows beside it."""
    import torch
    from repackshot_b200 import shards
    film.guides(0, samples)  # warm-up
    film.denoise(samples, out=False)
    times = {}
    for name, fn in (("guides_ms", lambda: film.guides(0, samples)), ("denoise_ms", lambda: film.denoise(samples, out=False)),
                     ("denoise_viewport_ms", lambda: film.denoise(samples, preset=1, out=False))):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        times[name] = shards.max_over_ranks(a.elapsed_time(b) / 1e3, dist) * 1e3
    # the guides read from the render's own first hits instead (rtg_film_guides_fused)
    film.clear()
    film.fuse_guides(True)
    film.render(0, 1)  # warm-up of the fused kernels
    film.clear()
    film.fuse_guides(True)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    film.render(0, samples)
    b.record(stream)
    torch.cuda.synchronize()
    times["render_with_fused_guides_ms"] = shards.max_over_ranks(a.elapsed_time(b) / 1e3, dist) * 1e3
    film.fuse_guides(False)
    out = film.denoise(samples)
    n = WIDTH * HEIGHT
    # algorithmic bytes of the filter: per level the 25 taps' guides, light, variance and
    # luminance stay in L1/L2; DRAM sees each plane once per kernel
    return {**times, "pixels": n, "mpixels_s": n / (times["denoise_ms"] / 1e3) / 1e6,
            "image_mean": float(out[..., :3].mean()),
            "path": "rtg_film_guides (centre-ray exact passes + per-sample albedo, traced on the device) and rtg_film_denoise "
                    "(a-trous, 5 levels, bit-exact with the oracle; result left on the device); render_with_fused_guides_ms: the "
                    "frame's render with rtg_film_guides_fused (the albedo from its own first hits), against the plain frame"}


def stress_comparison(rtg, spp, dist, world, stream):
    """The large stress workload at `spp` samples: 10 M triangles (1000 rigid instances of a
    10,000-triangle displaced sphere), 3840 x 2160, depth 16, 16 materials: one rig rendered plainly,
    its 8 rig variants as one batched queue, then the adjoint (35+ parameters) on a 1024 x 1024
    crop. Device time by CUDA events (plain), wall time around synchronous calls (queue, adjoint),
    max over ranks."""
    import torch
    from repackshot_b200 import scenes, shards
    W4, H4, D4 = 3840, 2160, 16
    t0 = time.perf_counter()
    base = scenes.cfg4_scene(width=W4, height=H4, spp=spp, depth=D4)
    s = rtg.Scene(scenes.to_rsb(base))
    load_s = time.perf_counter() - t0
    s.set_stream(stream.cuda_stream)
    f = s.film()
    f.render(1_000_000, 1)  # warm-up
    f.clear()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    f.render(0, spp)
    b.record(stream)
    torch.cuda.synchronize()
    plain_s = shards.max_over_ranks(a.elapsed_time(b) / 1e3, dist)
    paths = W4 * H4 * spp
    rigs = [scenes.to_rsb(scenes.cfg4_scene(width=W4, height=H4, spp=spp, depth=D4, rig=scenes.light_rig(r), seed=1 + r), meshes=False)
            for r in range(8)]
    # the 8 rigs back to back through the plain path (rtg_scene_update + rtg_render_progressive),
    # then as one batched queue (a captured graph): wall time around synchronous calls for both,
    # alternated twice and the faster of each kept (a few seconds each at full power: the two
    # should see the same clocks)
    plain_times, queue_times = [], []
    for _ in range(2):
        s.synchronize()
        t0 = time.perf_counter()
        keep = []
        for r in rigs:
            s.update(r)
            fr = s.film()
            fr.render(0, spp)
            keep.append(fr)
        s.synchronize()
        plain_times.append(shards.max_over_ranks(time.perf_counter() - t0, dist))
        del keep
        q = rtg.Queue(s)
        s.synchronize()
        t0 = time.perf_counter()
        films = [q.add(r, 0, spp, W4, H4) for r in rigs]
        q.run(graph=True)
        queue_times.append(shards.max_over_ranks(time.perf_counter() - t0, dist))
        del films
        q.close()
    plain8_s, queue_s = min(plain_times), min(queue_times)
    s.update(scenes.to_rsb(base, meshes=False))
    crop = ((W4 - 1024) // 2, (H4 - 1024) // 2, 1024, 1024)
    target = np.full((1024, 1024, 3), 0.5, np.float32)
    fc = s.film(*crop)
    s.adjoint(fc, target, 0, 2, correlated=False)  # warm-up
    s.synchronize()
    t0 = time.perf_counter()
    loss, grads, _ = s.adjoint(fc, target, 0, spp, correlated=False)
    adjoint_s = shards.max_over_ranks(time.perf_counter() - t0, dist)
    nm, nl = s.adjoint_params()
    return {"workload": "10,000,002 triangles (1000 rigid instances, PCG32 seed 11, of a 10,000-triangle displaced sphere, "
                        "two-level) + floor, 3840x2160, depth 16, 16 materials", "spp": spp, "scene_load_s": load_s,
            "plain_mpaths_s": world * paths / plain_s / 1e6, "plain_ms": plain_s * 1e3,
            "plain_8_rigs_back_to_back_mpaths_s": world * 8 * paths / plain8_s / 1e6, "plain_8_rigs_s": plain8_s,
            "queue_8_rigs_mpaths_s": world * 8 * paths / queue_s / 1e6, "queue_8_rigs_s": queue_s,
            "plain_8_rigs_times_s": plain_times, "queue_8_rigs_times_s": queue_times,
            "adjoint_crop_1024_ms": adjoint_s * 1e3, "adjoint_params": 4 * nm + nl, "adjoint_loss": float(loss)}


def steady_rates(scene, jobs, rsbs, min_paths=64_000_000):
    """Paths per second of each of the 8 cameras' path mixes at steady state: the first job with
    that camera rendered with enough samples for one wave of at least `min_paths` paths, so that
    its tail of long paths costs a few percent (device time around a synchronous call)."""
    import math
    rates = {}
    for cam in range(8):
        j = next(k for k in range(len(jobs)) if k % 8 == cam)
        scene.update(rsbs[j])
        npix = jobs[j].width * jobs[j].height
        spp = max(1, math.ceil(min_paths / npix))
        f = scene.film()
        f.render(10_000, 1)  # warm-up
        scene.synchronize()
        t0 = time.perf_counter()
        f.render(0, spp)
        scene.synchronize()
        rates[cam] = npix * spp / (time.perf_counter() - t0)
    return rates


def batched_comparison(rtg, scene, spp_scale, dist, world, steady_mpaths_s):
    """The metric's plain-vs-batched half: the 64 camera x light-rig jobs of uneven resolution and
    spp on this scene's geometry, rendered back to back through the plain path (rtg_scene_update +
    rtg_render_progressive per job) and as one batched queue (rtg_queue_*, run as one captured CUDA
    graph), both with the autotuned tuning. Wall time around synchronous calls, max over ranks;
    each rank renders the whole job set (replicas). The ideal time, which no schedule of these
    paths beats, is every job's paths at the steady rate of its camera's path mix (steady_rates);
    `steady_mpaths_s` is the 1080p product frame's rate, for comparison."""
    from repackshot_b200 import scenes, shards
    jobs = scenes.product_jobs(spp_scale=spp_scale)
    rsbs = [scenes.to_rsb(j, meshes=False) for j in jobs]
    paths = sum(j.width * j.height * j.max_samples for j in jobs)
    # warm-up of both paths on four small jobs
    q = rtg.Queue(scene)
    keep = [q.add(rsbs[k], 0, 1, jobs[k].width, jobs[k].height) for k in range(4)]
    q.run()
    for k in range(4):
        scene.update(rsbs[k])
        keep.append(scene.film())
        keep[-1].render(0, 1)
    del keep
    scene.synchronize()
    t0 = time.perf_counter()
    films = []
    for j, b in zip(jobs, rsbs):
        scene.update(b)
        f = scene.film()
        f.render(0, j.max_samples)
        films.append(f)
    scene.synchronize()
    t_plain = shards.max_over_ranks(time.perf_counter() - t0, dist)
    plain_img = films[-1].resolve()
    del films
    q = rtg.Queue(scene)
    t0 = time.perf_counter()
    films = [q.add(b, 0, j.max_samples, j.width, j.height) for j, b in zip(jobs, rsbs)]
    q.run(graph=True)
    t_batched = shards.max_over_ranks(time.perf_counter() - t0, dist)
    same = bool(np.array_equal(films[-1].resolve(), plain_img))
    del films
    rates = steady_rates(scene, jobs, rsbs)
    ideal_s = shards.max_over_ranks(sum(j.width * j.height * j.max_samples / rates[k % 8] for k, j in enumerate(jobs)), dist)
    return {"jobs": len(jobs), "paths_per_gpu": paths, "spp_scale": spp_scale,
            "ideal_s": ideal_s, "ideal_note": "every job's paths at the steady rate of its camera's path mix (one wave of at "
                                              "least 64 M paths per camera): no schedule of these paths beats it",
            "steady_mpaths_s_per_camera": [rates[c] / 1e6 for c in range(8)], "frame_mpaths_s": steady_mpaths_s,
            "batched_over_ideal": ideal_s / t_batched, "plain_over_ideal": ideal_s / t_plain,
            "workload": "64 jobs on the product geometry: 8 orbit cameras (0-315 deg, 35-135 mm) x 8 light rigs (1-4 "
                        "softboxes, radiance 1-20); per job a resolution from {256^2, 512^2, 1280x720, 1920x1080, "
                        "2048x1152} and spp from {4, 16, 64, 256} x spp_scale, drawn from PCG32 seeded with the job id",
            "plain_back_to_back_mpaths_s": world * paths / t_plain / 1e6, "batched_mpaths_s": world * paths / t_batched / 1e6,
            "batched_over_plain": t_plain / t_batched, "plain_s": t_plain, "batched_s": t_batched,
            "last_job_bits_equal": same}


def adjoint_comparison(rtg, dist, world, iterations):
    """The metric's adjoint half on the differentiable workload (the small scene's icosphere in 16
    materials, 512 x 512, 32 spp, depth 6, three lights; the target rendered at 512 spp with every
    parameter perturbed by U(0.8, 1.2), PCG32 seed 3): the forward render's time, one adjoint
    iteration's (rtg_scene_update + rtg_render_adjoint + the Adam step), and a fit of `iterations`
    steps. Wall time around synchronous calls, max over ranks."""
    from repackshot_b200 import fit, scenes, shards
    W = H = 512
    SPP, DEPTH = 32, 6
    base = scenes.adjoint_scene(W, H, SPP, DEPTH)
    tgt = scenes.adjoint_scene(W, H, SPP, DEPTH, perturb_seed=3)
    ts = rtg.Scene(scenes.to_rsb(tgt))
    tf = ts.film()
    tf.render(100_000, 512)
    rgb, wt, _, _ = tf.read()
    target = (rgb / wt[..., None]).astype(np.float32)
    s = rtg.Scene(scenes.to_rsb(base))
    f = s.film()
    f.render(0, SPP)
    fwd = []
    for i in range(5):
        f.clear()
        s.synchronize()
        t0 = time.perf_counter()
        f.render(i * SPP, SPP)
        s.synchronize()
        fwd.append(time.perf_counter() - t0)
    F = fit.Fit(s, base, target, SPP, lr=0.02, decay=0.985)
    F.step()  # warm-up (allocations)
    t0 = time.perf_counter()
    for _ in range(iterations):
        F.step()
    s.synchronize()
    t_fit = shards.max_over_ranks(time.perf_counter() - t0, dist)
    t_fwd = shards.max_over_ranks(statistics.median(fwd), dist)
    want = np.array([l.power for l in tgt.lights])
    want_c = np.array([m.base_color for m in tgt.materials[:16]])
    want_a = np.array([m.roughness ** 2 for m in tgt.materials[:16]])
    cols, alphas, powers = F.params()
    return {"workload": "differentiable render: small-scene icosphere split into 16 instances with the product "
                        "material table (16 base colours, 16 GGX alphas in 0.05-0.8), 3 rect lights, 512x512, 32 spp, "
                        "depth 6; target at parameters perturbed by U(0.8, 1.2) (PCG32 seed 3), 512 spp",
            "forward_ms": t_fwd * 1e3, "adjoint_ms_per_iter": t_fit / iterations * 1e3,
            "adjoint_over_forward": (t_fit / iterations) / t_fwd, "iterations": iterations,
            "loss_first": F.state.losses[0], "loss_last": F.state.losses[-1],
            "light_power_error_first": float(np.abs(np.array([l.power for l in base.lights]) - want).sum()),
            "light_power_error_last": float(np.abs(powers - want).sum()),
            "colour_error_first": float(np.abs(np.array([m.base_color for m in base.materials[:16]]) - want_c).mean()),
            "colour_error_last": float(np.abs(cols - want_c).mean()),
            "alpha_error_first": float(np.abs(np.array([m.roughness ** 2 for m in base.materials[:16]]) - want_a).mean()),
            "alpha_error_last": float(np.abs(alphas - want_a).mean()),
            "errors": "light power: sum over the 3 lights of |power - target power| (W); colour and alpha: mean over the "
                      "16 materials (and channels) of |value - target value|",
            "iteration": "rtg_scene_update (parameters) + rtg_render_adjoint (forward wave, loss, backward wave) + Adam step"}


def run_ours(args, world, rank, local, dist):
    import torch

    import repackshot_b200 as rtg
    from repackshot_b200 import shards
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    hbm_peak, peak_src = peaks()
    t0 = time.perf_counter()
    rsb = product_rsb()
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    scene = rtg.Scene(rsb)
    load_s = time.perf_counter() - t0
    if args.capacity:
        scene.set_path_capacity(args.capacity)
    stream = torch.cuda.current_stream(dev)
    scene.set_stream(stream.cuda_stream)
    film = scene.film()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    base, _ = shards.sample_range(rank, world, SPP)  # each rank its own sample range: a replica frame per rank

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # The autotuner picks the wave tuning on the frame itself (its 64 samples, at sample indices
    # outside the timed ones), before the warm-up: a few samples make a smaller wave, and what
    # pays there need not pay on the frame (the ray sort timed 8% faster at 4 spp and rendered the
    # 64-spp frame 4% slower).
    t0 = time.perf_counter()
    tuned = scene.autotune(base + 90_000, SPP) if args.autotune else {"chosen": scene.tuning(), "tried": []}
    tune_s = time.perf_counter() - t0
    for i in range(args.warmup):
        film.clear()
        film.render(base + 10_000 * (i + 1), SPP)
    barrier()
    scene.timing(True, reset=True)
    clocks = Clocks(local) if rank == 0 else None
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    rays = 0
    barrier()
    for i in range(args.steps):
        flush.zero_()  # evict the previous step from the 126 MB L2
        film.clear()
        ev[i][0].record(stream)
        rays += film.render(base, SPP)
        ev[i][1].record(stream)
    barrier()
    clk = clocks.stop() if clocks else None
    ext_ms, ext_launches, ext_rays, shadow_rays, launches = scene.timing(False)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = shards.max_over_ranks(sum(step_ms), dist)
    paths_step = WIDTH * HEIGHT * SPP
    value = world * args.steps * paths_step / (total_ms / 1e3) / 1e6

    # e2e: the same render through the C ABI with the film copied to pinned host memory.
    n = WIDTH * HEIGHT
    host = tuple(torch.empty(k, dtype=torch.float32, pin_memory=True).numpy() for k in (3 * n, n, n, n))
    e2e_steps = max(2, min(args.steps, 3))
    barrier()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        film.clear()
        film.render(base, SPP)
        film.read(host)
    torch.cuda.synchronize(dev)
    e2e_local = shards.max_over_ranks(time.perf_counter() - t0, dist)
    e2e_value = world * e2e_steps * paths_step / e2e_local / 1e6
    img = film.resolve()
    denoised = denoise_comparison(rtg, film, SPP, stream, dist) if args.denoise else None
    stress = stress_comparison(rtg, args.stress_spp, dist, world, stream) if args.stress_spp > 0 else None
    adaptive = adaptive_comparison(rtg, scene, dist, world, args.adaptive_target, total_ms / args.steps) if args.adaptive_target > 0 else None
    # The metric's other halves (0 leaves a section out, e.g. for a profiler's launch list).
    batched = (batched_comparison(rtg, scene, args.batched_spp_scale, dist, world, value / world)
               if args.batched_spp_scale > 0 else None)
    adjoint = adjoint_comparison(rtg, dist, world, args.fit_iterations) if args.fit_iterations > 0 else None

    if rank != 0:
        return
    # Roofline of the extend kernel: algorithmic bytes from the reference BVH8 visit counts of
    # this workload's own paths (oracle, bounded sample of row bands at 1 spp).
    import oracle
    threads = os.cpu_count() or 1
    o = oracle.OracleScene(rsb)
    o.enable_merged_stats()
    o.render_tile(WIDTH // 2, HEIGHT // 2, 8, 8, 0)  # first use generates the energy tables
    bands = sample_bands(16)
    st_dt, st_paths, stats = oracle_sample(o, bands, 0, 1, threads)
    b_ray = traversal_bytes(stats, merged=True)
    b_ray_two_level = traversal_bytes(stats, merged=False)
    achieved = ext_rays * b_ray / (ext_ms / 1e3) / 1e9 if ext_ms > 0 else 0.0
    o = oracle.OracleScene(rsb)  # without the statistics tree, for the timed CPU baseline
    # CPU baseline: the oracle (C++ restatement of the reference) on this host over the 16 bands
    # at the frame's own samples (10-30 s of work); the same rows of the device frame against
    # them give the image error at equal spp.
    cpu_images = []
    cpu_dt, cpu_paths, _ = oracle_sample(o, bands, base, SPP, threads, images=cpu_images)
    cpu_value = cpu_paths / cpu_dt / 1e6
    gpu_rows = np.concatenate([img[y:y + rows] for y, rows in bands])
    cpu_rows = np.concatenate(cpu_images)
    rel_mse_cpu = rel_mse(gpu_rows, cpu_rows)
    bit_equal_cpu = float(np.mean(gpu_rows.astype(np.float32).view(np.uint32) == cpu_rows.astype(np.float32).view(np.uint32)))
    line = {
        "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": DATA,
        "config": {"workload": WORKLOAD, "width": WIDTH, "height": HEIGHT, "spp": SPP, "max_depth": DEPTH,
                   "triangles": scene.triangles, "paths_per_step_per_gpu": paths_step,
                   "l2": "flushed between steps (512 MiB write); the per-step working set (172 B of path state per path, "
                         "23 GB for the frame) exceeds L2",
                   "parallelism": f"replicas x{world}: each rank renders its own sample range of the frame",
                   "scene_gen_s": round(gen_s, 3), "scene_load_s": round(load_s, 3), "bvh_build_s": round(scene.build_seconds, 3),
                   "tuning": tuned["chosen"]},
        "autotune": {"seconds": round(tune_s, 3), "workload": "the frame at its 64 spp per candidate (a warm-up and three timed renders, the median counts)",
                     "tried": tuned["tried"]},
        "mrays_per_s": world * rays / (total_ms / 1e3) / 1e6 if rank == 0 else None,
        "roofline": {"kernel": "k_extend (nearest-hit traversal)", "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                     "unit": "GB/s", "frac": achieved / hbm_peak, "peak_source": peak_src,
                     "traffic": DRAM_BYTES_PER_EXTEND_RAY * ext_rays / max(ext_launches, 1),
                     "traffic_note": "dram read + write bytes per extend launch: the ncu figure per ray (a 4 Mi-path "
                                     "wave) times this run's mean rays per launch; the BVH is L2-resident",
                     "bytes_per_ray": b_ray, "bytes_per_ray_reference_two_level": b_ray_two_level,
                     "frac_reference_two_level": ext_rays * b_ray_two_level / (ext_ms / 1e3) / 1e9 / hbm_peak if ext_ms > 0 else None,
                     "extend_ms_per_launch": ext_ms / max(ext_launches, 1),
                     "extend_launches": ext_launches, "extend_rays": ext_rays,
                     "mrays_per_s_in_extend": ext_rays / (ext_ms / 1e3) / 1e6 if ext_ms > 0 else None,
                     "note": "achieved = extend rays x algorithmic bytes per ray / extend kernel time (CUDA events around every "
                             "launch). Bytes per ray: 44 B ray I/O + 256 B per wide node + 160 B per 4-triangle packet of the "
                             "reference BVH8 layout, visits counted by the oracle on this workload's own paths in one reference-"
                             "layout BVH8 over all triangles; the reference's own two-level tree of 16 interleaved per-material "
                             "instances visits ~10x more (bytes_per_ray_reference_two_level)."},
        "cpu_baseline": {"value": cpu_value, "unit": "Mpaths/s", "cores": threads, "kind": "port",
                         "sample": f"{len(bands)} bands of 8 rows x 1920 px spread over the frame at the frame's {SPP} spp "
                                   "(C++ restatement of the reference, bit-exact with its pinned hashes)"},
        "rel_mse_vs_cpu": rel_mse_cpu,
        "rel_mse_note": f"the device frame's {len(bands)} bands against the CPU path's render of the same pixels and "
                        f"samples (64 spp): mean of (a - b)^2 / (b^2 + 1e-2); {bit_equal_cpu * 100:.4f}% of the values "
                        "bit-equal",
        "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 24 * n,
                "path": "rtg_film_clear + rtg_render_progressive + rtg_film_read into pinned host buffers (C ABI); the scene "
                        "is resident after rtg_scene_load (scene_load_s in config)"},
        "gpu_launches": launches,
        "clocks": clk,
        "image_mean": float(img.mean()),
        "batched": batched,
        "adjoint": adjoint,
        "adaptive": adaptive,
        "denoise": denoised,
        "stress": stress,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--capacity", type=int, default=0, help="paths per wave (default: the library's automatic size)")
    ap.add_argument("--fit-iterations", type=int, default=200, help="adjoint fit iterations of the differentiable workload")
    ap.add_argument("--batched-spp-scale", type=float, default=1.0,
                    help="spp of the batched-queue comparison's 64 jobs, as a fraction of theirs (1: the full 6.5 G paths)")
    ap.add_argument("--stress-spp", type=int, default=8,
                    help="spp of the 10 M-triangle 4K stress section (plain, 8-rig queue, adjoint on a crop; 0 leaves it out)")
    ap.add_argument("--autotune", type=int, default=1, help="choose the wave tuning with rtg_autotune before the warm-up (0: the default)")
    ap.add_argument("--denoise", type=int, default=1, help="time the guide passes and the denoiser on the frame (0 leaves it out)")
    ap.add_argument("--adaptive-target", type=float, default=0.02,
                    help="noise target of the adaptive-sampling comparison (0 leaves it out)")
    args = ap.parse_args()
    if args.impl == "reference":
        # The CPU reference runs on rank 0 alone; the other ranks have no work.
        if int(os.environ.get("RANK", "0")) == 0:
            run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), 0)
        return
    world, rank, local, dist = dist_setup(args)
    try:
        run_ours(args, world, rank, local, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
