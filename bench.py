"""Benchmark: Mrays/s of the plain wavefront path tracer at 1080p.

One step renders one frame of the 1080p workload (the seeded sphere field:
4096 instanced, Perlin-displaced icospheres, 1.07M unique and 13.7M
instanced triangles, 64 emissive triangles and a 2048x1024 importance-
sampled sky) at 16 samples per pixel, max depth 8, NEE + MIS, through the
CUDA backend's C ABI. A frame's rays are its camera, extension and shadow
rays; value = rays over device time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N > 1 every rank renders its own frames (independent sample indices)
on its own GPU and rank 0 prints the job's total: replicas, no collective
on the data path (weak scaling). `--impl reference` times the CPU oracle
(the scalar restatement of the reference's path tracer) on the host cores
on a bounded band of the same frame.

The line's last key, `time_to_relmse`, summarises the metric's other half
(rank 0, `--convergence 0` skips it): device seconds until the running
image's relMSE falls to 1e-3 for plain PT, the learned radiance cache,
ReSTIR DI in three modes and the cache with each, on the many-light and the
single-light box room at 1080p (`time_to_relmse_detail` holds the
checkpoints). Its `converged` object compares the box-room workload and a
band of the benchmarked frame with the CPU oracle's converged images. Its `batch` object
(`--batch 0` skips it) times the 64-scene batch workload rendered as one
wavefront against the same scenes one at a time.
"""

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from hydra_lotus_b200 import abi, scenes  # noqa: E402

WIDTH, HEIGHT, SPP, DEPTH = 1920, 1080, 16, 8
METRIC = "Mrays/s at 1080p (plain wavefront PT)"
WORKLOAD = ("sphere-field seed 0: 4096 instanced Perlin-displaced icospheres (subdiv 3/4, "
            "1.07M unique / 13.7M instanced triangles) on a 100x100 grid, 64 emissive "
            "triangles + 2048x1024 importance-sampled sky; 1920x1080, 16 spp, max depth 8, "
            "wavefront PT, NEE+MIS, FP32 transport, FP64 accumulation")
# Algorithmic bytes per extension ray outside the BVH walk: the queue
# entry (4), origin, direction and radiance sections (48), the hit section
# (16) and the hit-queue entry (4).
EXTEND_STATE_BYTES = 72
# A 4-wide node visit reads its six box bounds and four child references
# (112 of its 128 bytes); a triangle test its three corners (48 of 64); an
# instance entry its 64-byte traversal record.
NODE_BYTES, TRIANGLE_BYTES, INSTANCE_BYTES = 112, 48, 64
# DRAM bytes (read + write) per extension ray of k_wf_extend, from an Nsight
# Compute capture of one launch (the sphere field at 960x540, one wave of
# eight samples, bounce 1: 2,832,833 rays in key order, 499.4 MB read +
# 63.3 MB written, caches flushed before the launch). Scaled by rays to the
# bench's launches.
EXTEND_DRAM_BYTES_PER_RAY = 198.6
# B200's nominal HBM3e bandwidth (GB/s), for the fraction against it.
NOMINAL_HBM_GBS = 8000.0


def settings(sample_index):
    return abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT,
                                light_sampling=abi.LIGHT_SAMPLING_MIS,
                                max_bounces=DEPTH, sample_index=sample_index)


def launches_per_sample(max_bounces, rounds):
    # camera; shade and shadow per round, extend per round after the first
    # with the queue reordering's scan and scatter before it; the tail
    # kernel when the rounds stop short of max_bounces + 1; resolve, finish,
    # advance
    return 1 + 2 * rounds + 3 * (rounds - 1) + (1 if rounds <= max_bounces else 0) + 3


def wave_count(spp, wave=8):
    """Wavefronts a call adding `spp` samples runs: waves of `wave`, halved
    while fewer samples remain."""
    count = 0
    while spp > 0:
        while wave > spp:
            wave //= 2
        spp -= wave
        count += 1
    return count


def measured_peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,"
              "clocks.mem,clocks.max.mem,utilization.gpu")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mem, util, mx, mem_mx, reasons = [], [], [], None, None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for name, v in zip(names, r[5:9]):
                    if v.strip() == "Active":
                        reasons.add(name)
                mem.append(float(r[9]))
                mem_mx = float(r[10])
                util.append(float(r[11]))
            except (ValueError, IndexError):
                continue
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
               "samples": len(sm)}
        if mem:
            out.update({"mem_mhz": statistics.median(mem), "mem_max_mhz": mem_mx,
                        "gpu_util_pct": statistics.median(util) if util else None})
        return out


def cpu_baseline(scene, seconds, rows=64):
    """The oracle (the scalar CPU restatement of the reference's path
    tracer) on a band of the frame, one sample per pass, until `seconds`."""
    from oracle import oracle
    o = oracle.OracleScene(scene)
    threads = os.cpu_count() or 1
    y0 = (HEIGHT - rows) // 2
    frame = scene.frame(settings(0), data_window=(0, y0, WIDTH, rows))
    rays = 0
    passes = 0
    t0 = time.perf_counter()
    while True:
        _, r = o.sample(frame, passes, threads=threads)
        rays += int(r.sum())
        passes += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": rays / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "port",
            "sample": f"rows {y0}-{y0 + rows - 1} of the 1920x1080 frame, {passes} passes of 1 spp "
                      f"({rays} rays in {dt:.1f} s), OpenMP over {threads} threads"}


def rank_sample_base(rank):
    """First sample index of a rank's frames: ranks render independent
    samples of the same workload (replicas, no data-path collective)."""
    return 1000003 * rank


def reduce_over_ranks(rays, e2e_rays, ms, e2e_ms, world, device):
    """The job's totals: rays summed over ranks, device times as the
    slowest rank's (the rank that finishes last bounds the job)."""
    import torch
    stats = torch.tensor([rays, e2e_rays, ms, e2e_ms], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        sums = stats[:2].clone()
        dist.all_reduce(sums)
        maxes = stats[2:].clone()
        dist.all_reduce(maxes, op=dist.ReduceOp.MAX)
        stats = torch.cat([sums, maxes])
    return stats.tolist()


def run_reference(args, rank):
    """--impl reference: the CPU oracle on the host cores."""
    if rank != 0:
        return
    scene = scenes.sphere_field(seed=0)
    for _ in range(args.warmup):
        cpu_baseline(scene, 0.0, rows=32)
    results = []
    total_rays, total_s = 0, 0.0
    for k in range(args.steps):
        b = cpu_baseline(scene, 2.0, rows=64)
        results.append(b)
    # Aggregate: mean throughput over steps.
    value = statistics.mean(b["value"] for b in results)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
        "config": {"workload": WORKLOAD, "sample": "a 64-row band of the frame per pass"},
        "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s",
                         "cores": results[0]["cores"], "kind": "port",
                         "sample": results[0]["sample"]},
        "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _time_to_relmse(renderer_module, scene, label, budgets, depth=6, rows=64, spp=16384, target=1e-3):
    from hydra_lotus_b200 import convergence
    band_list = convergence.bands(scene.height, rows)
    out = {"scene": label, "target": target, "epsilon": 1e-2, "unit": "s (device time)"}
    with renderer_module.CudaOffscreenRenderer(0) as r:
        renderer_module.check(r.update_scene(scene), "update_scene")
        ref, noise, ref_s = convergence.reference(r, scene, depth, spp, band_list)
        out["reference"] = {"method": "plain wavefront PT, FP64 accumulation (paths bit-identical to the CPU oracle)",
                            "spp": spp, "bands": [list(b) for b in band_list],
                            "relmse_noise_subtracted": float(f"{noise:.3g}"), "device_s": round(ref_s, 3)}
        for method, budget in budgets.items():
            t, pts = convergence.time_to_relmse(r, scene, method, ref, noise, depth, band_list, target=target,
                                                max_seconds=budget)
            entry = {"seconds": None if t is None else round(t, 4),
                     "checkpoints": [[round(a, 4), float(f"{b:.4g}")] for a, b in pts]}
            if t is None and pts:
                entry["extrapolated_seconds"] = round(pts[-1][0] * pts[-1][1] / target, 2)
            out[method] = entry
    return out


def _seconds(entry):
    return entry["seconds"] if entry["seconds"] is not None else entry.get("extrapolated_seconds")


def time_to_relmse_report(renderer_module):
    """The metric's first half: device seconds to relMSE 1e-3 (epsilon 1e-2)
    at 1080p, depth 6, static camera, for plain wavefront PT, the learned
    radiance cache (paths ending into it at their second vertex, and at
    their third: `cache_v3`), ReSTIR DI in three modes (temporal + spatial
    reuse, initial candidates only, spatial reuse only; the spatial pass
    draws 5 neighbours from a 30-pixel disk) and the cache with ReSTIR: on the box
    room with 10,000 emissive floor triangles (power log-normal, sigma 2;
    `many_lights`) and on the config-1 box room with its one ceiling light
    (`single_light`). The reference is plain PT at 16,384 spp with FP64
    accumulation over three 64-row bands (top, middle, bottom), its own
    noise subtracted. A method that does not reach the target within its
    budget reports null with an extrapolation from its last checkpoint
    (relMSE falling as 1/time)."""
    many = _time_to_relmse(
        renderer_module, scenes.box_room_wide(seed=0, emitters=10000),
        "box room + 10,000 emissive floor triangles (power log-normal sigma 2), 1920x1080, depth 6, static camera",
        {"plain": 40.0, "cache": 12.0, "cache_v3": 12.0, "restir": 4.0, "restir_initial": 4.0,
         "restir_spatial": 4.0, "cache+restir": 12.0, "cache+restir_initial": 12.0,
         "cache_v3+restir_initial": 12.0})
    single = _time_to_relmse(
        renderer_module, scenes.box_room_wide(seed=0),
        "config-1 box room (one ceiling quad light), 1920x1080, depth 6, static camera",
        {"plain": 10.0, "cache": 6.0, "cache_v3": 6.0, "restir": 3.0, "restir_initial": 3.0,
         "restir_spatial": 3.0, "cache+restir": 6.0, "cache+restir_initial": 6.0,
         "cache_v3+restir_initial": 6.0})
    return {"many_lights": many, "single_light": single}


def time_to_relmse_summary(report):
    """The compact summary (seconds per method and speed-ups over plain PT)
    that closes the bench line."""
    out = {"target_relmse": 1e-3, "epsilon": 1e-2, "unit": "s (device time, 1080p, static camera)",
           "reference": "plain PT, 16,384 spp, FP64, three 64-row bands; its noise subtracted"}
    for name, rep in report.items():
        methods = [m for m in rep if isinstance(rep[m], dict) and "checkpoints" in rep[m]]
        secs = {m: _seconds(rep[m]) for m in methods}
        plain = secs.get("plain")
        modes = [m for m in methods if m.startswith("cache") and "restir" in m]
        best = min(modes, key=lambda m: secs[m] if secs[m] else float("inf"))
        entry = {"noise": rep["reference"]["relmse_noise_subtracted"],
                 "seconds": {m: (round(v, 3) if v else None) for m, v in secs.items()},
                 "reached": {m: rep[m]["seconds"] is not None for m in methods},
                 "best_cache_restir_mode": best}
        if plain:
            entry["speedup_vs_plain"] = {m: round(plain / v, 2) for m, v in secs.items() if v and m != "plain"}
        out[name] = entry
    return out


def converged_report(renderer_module):
    """Converged images against the CPU oracle's (committed fixtures: FP64
    accumulations of 16,384 samples per pixel for the box room, 4,096 for a
    16-row band of the sphere field, per-pixel variances from batches): the
    box-room workload exactly as specified (256x256, 64 spp, depth 6, NEE +
    MIS) and the benchmarked frame's band at depth 8 and 1024 spp, through
    the wavefront integrator. Per image: device ms, relMSE (epsilon 1e-2)
    beside the relMSE its noise explains (the oracle's variance over the
    image's and the oracle's samples), and the reference's DES-Q5 per-pixel
    z statistics. The sphere field's caustic paths are heavy-tailed, so its
    band is held to the band-wide z per channel (the oracle's own 1024-spp
    band fails the per-tile test against its 4096-spp one)."""
    from hydra_lotus_b200 import metrics
    out = {}
    cases = [("box_room_256_64spp_depth6", "box_room_256_oracle.npz", lambda: scenes.box_room(seed=0, size=256),
              64, 6, None),
             ("sphere_field_band_1024spp_depth8", "sphere_field_band_oracle.npz",
              lambda: scenes.sphere_field(seed=0), 1024, 8, "band")]
    with renderer_module.CudaOffscreenRenderer(0) as r:
        for name, fixture, make, spp, depth, band in cases:
            path = os.path.join(HERE, "tests", "golden", fixture)
            if not os.path.exists(path):
                out[name] = {"error": f"missing fixture {fixture}"}
                continue
            g = np.load(path)
            scene = make()
            renderer_module.check(r.update_scene(scene), "update_scene")
            st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                                      max_bounces=depth, sample_index=0)
            kw = {}
            y0, rows = 0, scene.height
            if band:
                y0, rows = (int(v) for v in g["band"])
                kw["data_window"] = (0, y0, scene.width, rows)
            res, color = r.render_scene(scene.frame(st, spp, **kw))
            renderer_module.check(res, name)
            img = color[y0:y0 + rows]
            ref_spp = int(g["samples"])
            c = metrics.compare(img, spp, g["mean"], g["variance"], ref_spp)
            v = g["variance"].astype(np.float64) * (1.0 / spp + 1.0 / ref_spp)
            m = g["mean"].astype(np.float64)
            expected = float(np.mean(v / (m * m + metrics.RELMSE_EPSILON)))
            rays = res.camera_rays + res.extension_rays + res.shadow_rays
            out[name] = {"gpu_ms": round(res.gpu_ms, 3), "mrays_per_s": round(rays / res.gpu_ms / 1e3, 1),
                         "oracle_spp": ref_spp, "relmse": float(f"{metrics.relmse(img, m):.4g}"),
                         "relmse_expected_from_noise": float(f"{expected:.4g}"),
                         "des_q5_pass": c.ok,
                         "image_z_pass": all(abs(z) <= metrics.MATCH_Z for z in c.image_z),
                         "image_z": [round(z, 3) for z in c.image_z],
                         "max_tile_z": round(c.max_tile_z, 3), "mean_tile_z2": round(c.mean_tile_z2, 3)}
    return out


def scene_update_report(renderer_module, repeats=3):
    """Scene uploads and edits on the shape of the reference's `geometry-v1`
    workload (one indexed 512 x 512-quad grid: 524,288 triangles, 263,169
    vertices), as the reference's performance baseline times them: the
    initial upload and build, a compatible point edit of every position
    (y += 0.01 x, lotus_cuda_update_geometry) and a transform edit (x +=
    0.01, lotus_cuda_update_instances). Per kind, the median over `repeats`
    of the device time of the update's uploads and builds (build_gpu_ms;
    the initial one also spans its host staging) and of the call's host
    wall time."""
    grid = scenes.grid_mesh(quads=512)
    out = {"workload": "one indexed 512x512-quad grid, 524,288 triangles, 263,169 vertices (geometry-v1's shape)",
           "unit": "ms"}

    def med(v):
        return round(statistics.median(v), 4)

    with renderer_module.CudaOffscreenRenderer(0) as r:
        full, full_wall = [], []
        for _ in range(repeats):
            t0 = time.perf_counter()
            res = renderer_module.check(r.update_scene(grid), "update_scene")
            full_wall.append((time.perf_counter() - t0) * 1e3)
            full.append(res.build_gpu_ms)
        p0 = grid.geometries[0][0].copy()
        edit, edit_wall, move, move_wall = [], [], [], []
        for k in range(repeats):
            q = p0.copy()
            q[:, 1] += 0.01 * (k + 1) * p0[:, 0]
            grid.set_positions(0, q)
            t0 = time.perf_counter()
            res = renderer_module.check(r.update_geometry(grid, 0), "update_geometry")
            edit_wall.append((time.perf_counter() - t0) * 1e3)
            edit.append(res.build_gpu_ms)
            m = np.array(grid.instances[0][0], dtype=np.float32)
            m[12] += 0.01
            grid.set_instance(0, m)
            t0 = time.perf_counter()
            res = renderer_module.check(r.update_instances(grid), "update_instances")
            move_wall.append((time.perf_counter() - t0) * 1e3)
            move.append(res.build_gpu_ms)
    out["initial_build"] = {"gpu_ms": med(full), "wall_ms": med(full_wall)}
    out["point_edit"] = {"gpu_ms": med(edit), "wall_ms": med(edit_wall)}
    out["transform_edit"] = {"gpu_ms": med(move), "wall_ms": med(move_wall)}
    out["reference_published"] = {
        "hardware": "RTX A5000 (Vulkan, driver-built acceleration structures)",
        "initial_build": {"gpu_upload_ms": 0.36, "gpu_blas_build_ms": 1.628, "gpu_tlas_build_ms": 0.033,
                          "wall_ms": 8.241},
        "point_edit": {"gpu_upload_ms": 0.359, "gpu_blas_refit_ms": 0.455, "gpu_tlas_refit_ms": 0.010,
                       "wall_ms": 2.645},
        "transform_edit": {"gpu_upload_ms": 0.001, "gpu_tlas_refit_ms": 0.010, "wall_ms": 0.183}}
    return out


def temporal_report(renderer_module, frames=120, checked=(0, 30, 60, 90, 119), ref_spp=4096, rows=64):
    """The temporal configurations at 1920x1080, 1 spp per frame, over the
    120-frame orbit of the box room with 10,000 emissive floor triangles,
    depth 6: config 3 (ReSTIR DI with temporal reuse, M cap 20, one spatial
    pass of 5 neighbours drawn from a 30 px disk; SVGF with FP16 moments
    and 5 a-trous iterations) and config 5 (the learned radiance cache plus
    the same ReSTIR DI, no a-trous iterations). Frames per second from the
    median device time of frames 8.. (the histories full). Frames 0, 30,
    60, 90 and 119 of config 3 are each checked against an FP64 plain-PT
    reference of that frame's camera at 4,096 spp over three 64-row bands
    (top, middle, bottom): the relMSE (epsilon 1e-2) of the filtered
    composite and of the frame's own 1-spp batch."""
    from hydra_lotus_b200 import convergence, metrics
    width, height = 1920, 1080
    scene = scenes.restir_room(seed=0, size=height, emitters=10000, aspect=width / height)
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT,
                              light_sampling=abi.LIGHT_SAMPLING_RESTIR_INITIAL, max_bounces=6, sample_index=0,
                              restir_candidates=8, restir_temporal=1, restir_max_history_candidates=20,
                              restir_spatial=1, restir_spatial_radius=30, restir_spatial_neighbours=5)
    band_list = convergence.bands(height, rows)
    out = {"resolution": [width, height], "depth": 6, "spp_per_frame": 1, "orbit_frames": frames}
    for name, cache, filt in (("restir+svgf", False, 5), ("cache+restir", True, 0)):
        ms = []
        checks = []
        previous = None
        with renderer_module.CudaOffscreenRenderer(0) as r:
            renderer_module.check(r.update_scene(scene), "update_scene")
            if cache:
                r.configure_cache(enable=True, seed=1)
            for k in range(frames):
                view, w2c = scenes.orbit_camera(k, frames=120, aspect=width / height)
                check = not cache and k in checked
                frame = abi.make_frame(w2c, width, height, st, 1, read_back=check)
                d = abi.temporal_desc(frame, view, previous[0] if previous else None,
                                      previous[1] if previous else None, history_available=k > 0,
                                      accumulate_radiance=True, max_history_samples=5, filter_iterations=filt,
                                      moment_precision=abi.MOMENTS_FP16)
                res, img = r.render_temporal(d)
                renderer_module.check(res, name)
                previous = (view, w2c)
                ms.append(res.gpu_ms)
                if check:
                    batch = r.read_product(abi.PRODUCT_BATCH, height, width)
                    checks.append((k, img.copy(), batch.copy(), w2c))
        if checks:
            entries = []
            with renderer_module.CudaOffscreenRenderer(0) as ref_r:
                renderer_module.check(ref_r.update_scene(scene), "update_scene")
                camera = scene.world_to_clip
                for k, img, batch, w2c in checks:
                    scene.world_to_clip = w2c
                    ref, noise, _ = convergence.reference(ref_r, scene, 6, ref_spp, band_list)
                    entries.append({"frame": k,
                                    "relmse_composite": float(f"{metrics.relmse(convergence.band_pixels(img, band_list), ref):.4g}"),
                                    "relmse_batch_1spp": float(f"{metrics.relmse(convergence.band_pixels(batch, band_list), ref):.4g}"),
                                    "reference_noise": float(f"{noise:.3g}")})
                scene.world_to_clip = camera
            out[name + "_checked_frames"] = {"reference": f"plain PT, {ref_spp} spp, FP64, three {rows}-row bands",
                                            "frames": entries}
        med = statistics.median(ms[8:])
        out[name] = {"ms_per_frame": round(med, 3), "frames_per_s": round(1e3 / med, 1)}
    return out


# Tensor-core work the radiance cache's kernels issue per record: the
# forward pass is five 64x64 layers and one 64x16 (three outputs padded to
# 16) = 21,504 multiply-adds; training adds the input gradients and the
# weight gradients of every layer, twice that again.
CACHE_INFER_FLOPS = 2 * 21504
CACHE_TRAIN_FLOPS = 3 * 2 * 21504


def cache_kernels_report(renderer_module, samples=16, warmup=8):
    """The radiance cache's kernels on the config-5 scene's 1080p frame
    (scenes.box_room_wide, wavefront PT, depth 8, paths ending into the
    cache at their second vertex, one path in 32 training): per sample, the
    device time of inference (its spatial query sort included) and of
    training (targets, the training pass, Adam), the records each handled,
    and the tensor-core work they issued per second as a fraction of the
    measured sustained BF16 GEMM rate."""
    peaks_path = os.path.join(HERE, "MEASURED_PEAKS.json")
    peak, kind = 1400.0, "fallback"
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            peak, kind = float(json.load(f)["bf16_tflops_sustained"]), "measured sustained"
    scene = scenes.box_room_wide(seed=0, width=WIDTH, height=HEIGHT)
    infer, train, queries, records = [], [], [], []
    with renderer_module.CudaOffscreenRenderer(0) as r:
        renderer_module.check(r.update_scene(scene), "update_scene")
        r.configure_cache(enable=True, seed=1)
        for k in range(warmup + samples):
            st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                                      max_bounces=DEPTH, sample_index=k)
            res, _ = r.render_scene(scene.frame(st, 1, read_back=False, flags=abi.FRAME_TIMINGS))
            renderer_module.check(res, "cache frame")
            if k >= warmup:
                infer.append(res.cache_infer_gpu_ms)
                train.append(res.cache_train_gpu_ms)
                queries.append(res.cache_queries)
                records.append(res.cache_training_records)
    i_ms, t_ms = statistics.median(infer), statistics.median(train)
    q, n = statistics.median(queries), statistics.median(records)
    i_tf = q * CACHE_INFER_FLOPS / (i_ms * 1e-3) / 1e12
    t_tf = n * CACHE_TRAIN_FLOPS / (t_ms * 1e-3) / 1e12
    return {"workload": f"box room, {WIDTH}x{HEIGHT}, 1 spp per sample, depth {DEPTH}, cache at the second vertex",
            "infer_ms_per_sample": round(i_ms, 4), "queries_per_sample": int(q),
            "train_ms_per_sample": round(t_ms, 4), "training_records_per_sample": int(n),
            "infer_tflops": round(i_tf, 1), "infer_frac": round(i_tf / peak, 4),
            "train_tflops": round(t_tf, 1), "train_frac": round(t_tf / peak, 4),
            "peak_tflops": peak, "peak_kind": kind,
            "flops_per_record": {"infer": CACHE_INFER_FLOPS, "train": CACHE_TRAIN_FLOPS}}


def analytic_lights_report(renderer_module, frames=64, warmup=8):
    """Analytic lights on the shape of the reference's many-lights-v1
    workload (scenes.light_grid: the box room under a grid of sphere
    lights), wavefront PT with NEE + MIS, 64 bounces, one sample per frame:
    the median device milliseconds per frame at 128^2 and 512^2 pixels for
    1 and 256 lights, beside the reference's published figures for its
    light-crossing hierarchy (RTX A5000)."""
    out = {"workload": "box room + side x side sphere lights (r 0.025) at y 0.85 (many-lights-v1's grid), "
                       "wavefront, NEE+MIS, 64 bounces, 1 spp per frame", "unit": "ms per frame (device)"}
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=64, sample_index=0)
    with renderer_module.CudaOffscreenRenderer(0) as r:
        for side in (1, 16):
            for size in (128, 512):
                scene = scenes.light_grid(side=side, size=size)
                renderer_module.check(r.update_scene(scene), "update_scene")
                ms = []
                for k in range(warmup + frames):
                    st.sample_index = k
                    res, _ = r.render_scene(scene.frame(st, 1, read_back=False))
                    renderer_module.check(res, "light grid frame")
                    if k >= warmup:
                        ms.append(res.gpu_ms)
                out[f"{side * side}_lights_{size}px"] = round(statistics.median(ms), 4)
    out["reference_published"] = {
        "hardware": "RTX A5000 (Vulkan ray query), light-crossing hierarchy, wavefront",
        "1_lights_128px": 0.227, "256_lights_128px": 0.384, "1_lights_512px": 0.829, "256_lights_512px": 1.077}
    return out


def gltf_cost_report(renderer_module, size=1024, frames=64, warmup=8):
    """What the glTF PBR closure costs beside UsdPreviewSurface's on one
    scene: the reference's cornell-v1 and cornell-gltf-v1 benchmark
    workloads (the Cornell box, then with every material glTF PBR) at
    size^2, one sample per frame, 64 bounces, BSDF sampling (the reference
    benchmark's defaults): the median device milliseconds per frame under
    each integrator, beside the reference's published figures."""
    out = {"workload": f"cornell-v1 and cornell-gltf-v1, {size}x{size}, 1 spp per frame, 64 bounces, "
                       "BSDF sampling", "unit": "ms per frame (device)"}
    with renderer_module.CudaOffscreenRenderer(0) as r:
        for name, integrator in (("reference", abi.INTEGRATOR_REFERENCE), ("wavefront", abi.INTEGRATOR_WAVEFRONT)):
            st = abi.default_settings(integrator=integrator, light_sampling=abi.LIGHT_SAMPLING_BSDF,
                                      max_bounces=64, sample_index=0)
            for workload, scene in (("cornell-v1", scenes.cornell_reference(size=size)),
                                    ("cornell-gltf-v1", scenes.cornell_gltf(size=size))):
                renderer_module.check(r.update_scene(scene), "update_scene")
                ms = []
                for k in range(warmup + frames):
                    st.sample_index = k
                    res, _ = r.render_scene(scene.frame(st, 1, read_back=False))
                    renderer_module.check(res, workload)
                    if k >= warmup:
                        ms.append(res.gpu_ms)
                out[f"{name}_{workload}"] = round(statistics.median(ms), 4)
            out[f"{name}_ratio"] = round(out[f"{name}_cornell-gltf-v1"] / out[f"{name}_cornell-v1"], 3)
    out["reference_published"] = {
        "hardware": "the reference's development workstation (Vulkan ray query, unlocked clocks), 1024^2",
        "reference_cornell-v1": 1.62, "reference_cornell-gltf-v1": 3.85,
        "wavefront_cornell-v1": 2.21, "wavefront_cornell-gltf-v1": 3.63}
    return out


def batch_report(renderer_module, spp=8, depth=8):
    """Config 4: the 64-scene batch workload (scenes.batch_workload: traced
    triangles log-uniform in [1e4, 2e6], 256^2 .. 1024^2 targets), 8 spp,
    depth 8, rendered as one wavefront per sample under a CUDA graph with
    the tuner's launch shape, against the same scenes rendered one after
    another by one renderer: with its samples in waves of eight (the
    renderer's default: each scene's samples share a wavefront) and with one
    sample per wavefront (no batching of scenes or samples). Device time
    only (CUDA events)."""
    from hydra_lotus_b200 import autotune
    work = scenes.batch_workload(64, seed=0)

    def st(k, first=0):
        return abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                                    max_bounces=depth, sample_index=first + 1000 * k)

    out = {"scenes": len(work), "pixels": sum(s.width * s.height for s in work),
           "traced_triangles": sum(s.traced_triangle_count for s in work), "spp": spp, "depth": depth}
    with renderer_module.CudaBatch(0) as batch:
        res = batch.set_scenes(work)
        if any(r.status != abi.PASS for r in res):
            return {"error": [r.detail.decode() for r in res if r.status != abi.PASS][0]}
        frames = [s.frame(st(k), frame_count=spp, read_back=False) for k, s in enumerate(work)]
        best, times = autotune.tune_batch(batch, frames)
        out["tuned"] = {"knobs": dict(zip(autotune.KNOBS, best)),
                        "candidates_ms_per_sample": {autotune.shape_name(s): round(t, 3) for s, t in times.items()}}
        frames = [s.frame(st(k, 7), frame_count=spp, read_back=False) for k, s in enumerate(work)]
        _, _, total = batch.render(frames)
        renderer_module.check(total, "batch")
        rays = total.camera_rays + total.extension_rays + total.shadow_rays
        out["batched"] = {"ms": round(total.gpu_ms, 2), "mrays_per_s": round(rays / total.gpu_ms / 1e3, 1),
                          "scene_samples_per_s": round(len(work) * spp / (total.gpu_ms * 1e-3), 1)}
    for name, wave in (("sequential", 0), ("sequential_one_sample_per_wavefront", 1)):
        seq_ms, seq_rays = 0.0, 0
        with renderer_module.CudaOffscreenRenderer(0, trace_refill_below=best[0], trace_blocks_per_sm=best[1],
                                                   samples_per_wave=wave) as r:
            for k, s in enumerate(work):
                renderer_module.check(r.update_scene(s), "update_scene")
                f = s.frame(st(k, 7), frame_count=spp, read_back=False)
                res, _ = r.render_scene(f)
                renderer_module.check(res, name)
                seq_ms += res.gpu_ms
                seq_rays += res.camera_rays + res.extension_rays + res.shadow_rays
        out[name] = {"ms": round(seq_ms, 2), "mrays_per_s": round(seq_rays / seq_ms / 1e3, 1)}
    out["speedup_batched_vs_sequential"] = round(out["sequential"]["ms"] / out["batched"]["ms"], 3)
    out["speedup_batched_vs_one_sample_per_wavefront"] = round(
        out["sequential_one_sample_per_wavefront"]["ms"] / out["batched"]["ms"], 3)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--batch", type=int, default=1,
                    help="1: also measure the 64-scene batch (config 4), batched vs one scene at a time")
    ap.add_argument("--temporal", type=int, default=1,
                    help="1: also measure frames/s of ReSTIR+SVGF (config 3) and cache+ReSTIR (config 5) at 1080p")
    ap.add_argument("--updates", type=int, default=1,
                    help="1: also time scene uploads and edits on the geometry-v1-shaped grid")
    ap.add_argument("--lights", type=int, default=1,
                    help="1: also time the many-lights-v1-shaped analytic light grid (1 and 256 sphere lights)")
    ap.add_argument("--convergence", type=int, default=1,
                    help="1: also measure time to relMSE 1e-3 (plain PT, cache, ReSTIR, cache+ReSTIR)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank)

    import torch
    import torch.distributed as dist

    from hydra_lotus_b200 import renderer

    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    scene = scenes.sphere_field(seed=0)
    r = renderer.CudaOffscreenRenderer(local_rank)
    sres = renderer.check(r.update_scene(scene), "update_scene")
    stream = torch.cuda.ExternalStream(r.stream)

    base = rank_sample_base(rank)
    step_index = [0]

    def frame(read_back=False, flags=0):
        f = scene.frame(settings(base + SPP * step_index[0]), frame_count=SPP,
                        read_back=read_back, flags=flags)
        step_index[0] += 1
        return f

    for _ in range(args.warmup):
        renderer.check(r.render_scene(frame())[0], "warmup")

    # Timed region: K frames, device time by CUDA events on the renderer's
    # stream, bracketed by a barrier and synchronize.
    barrier()
    torch.cuda.synchronize()
    rays = 0
    with ClockSampler(local_rank) as clocks:
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        step_ms = []
        for _ in range(args.steps):
            res, _ = r.render_scene(frame())
            renderer.check(res, "render")
            rays += res.camera_rays + res.extension_rays + res.shadow_rays
            step_ms.append(res.gpu_ms)
        stop.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = start.elapsed_time(stop)
    clock = clocks.summary()

    # End to end through the C ABI: per step the frame description goes to
    # the device and the RGBA32F image comes back into pinned host memory.
    pinned = torch.empty((HEIGHT, WIDTH, 4), dtype=torch.float32, pin_memory=True)
    color = np.frombuffer((C.c_float * (HEIGHT * WIDTH * 4)).from_address(pinned.data_ptr()),
                          dtype=np.float32).reshape(HEIGHT, WIDTH, 4)
    barrier()
    torch.cuda.synchronize()
    e2e_rays = 0
    e_start = torch.cuda.Event(enable_timing=True)
    e_stop = torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(args.steps):
        res, _ = r.render_scene(frame(read_back=True), color=color)
        renderer.check(res, "render e2e")
        e2e_rays += res.camera_rays + res.extension_rays + res.shadow_rays
    e_stop.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = e_start.elapsed_time(e_stop)

    # Kernel timings (one instrumented frame) and BVH visits (another).
    timed, _ = r.render_scene(frame(flags=abi.FRAME_TIMINGS))
    renderer.check(timed, "timed frame")
    counted, _ = r.render_scene(frame(flags=abi.FRAME_COUNT_VISITS))
    renderer.check(counted, "counted frame")

    total_rays, total_e2e_rays, max_ms, max_e2e_ms = reduce_over_ranks(rays, e2e_rays, ms, e2e_ms, world, "cuda")

    if rank == 0:
        peak, peak_kind = measured_peaks()
        # Extension kernel roofline: algorithmic bytes of the last sample's
        # extension rays over the extension kernels' device time.
        n_ext = max(counted.visit_rays[1], 1)
        per_ray = (EXTEND_STATE_BYTES + NODE_BYTES * counted.node_visits[1] / n_ext +
                   TRIANGLE_BYTES * counted.triangle_visits[1] / n_ext +
                   INSTANCE_BYTES * counted.instance_visits[1] / n_ext)
        # The rays the extension kernel traced: those of the rounds' bounces
        # (the tail kernel traces the rest).
        ext_rays_timed = sum(timed.wavefront_path_counts[b]
                             for b in range(1, min(timed.wavefront_rounds, timed.wavefront_path_count_size)))
        ext_bytes = ext_rays_timed * per_ray
        achieved = ext_bytes / (timed.extend_gpu_ms * 1e-3) / 1e9 if timed.extend_gpu_ms else 0.0
        launches = timed.extend_launches or DEPTH
        cpu = cpu_baseline(scene, args.cpu_seconds)
        line = {
            "metric": METRIC,
            "value": round(total_rays / (max_ms * 1e-3) / 1e6, 2),
            "unit": "Mrays/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(max_ms / args.steps, 3),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded procedural scene; no dataset)",
            "config": {"workload": WORKLOAD, "rays_per_step": int(total_rays / args.steps / world),
                       "l2": "inputs larger than L2: path state 166 MB + BVH/triangles/normals "
                             f"{sres.device_bytes / 1e6:.0f} MB per frame pass",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": round(total_e2e_rays / (max_e2e_ms * 1e-3) / 1e6, 2),
                    "unit": "Mrays/s", "h2d_bytes_per_step": 160,
                    "d2h_bytes_per_step": WIDTH * HEIGHT * 16 + 64},
            # Per step: SPP samples in waves of eight (each wave's launches
            # as one sample's, its frame constants in place of the advance),
            # chained 16 samples at a time, each chain advancing the frame
            # constants once.
            "gpu_launches": (launches_per_sample(DEPTH, timed.wavefront_rounds) * wave_count(SPP) +
                             (SPP + 15) // 16) * args.steps,
            "roofline": {
                "kernel": "k_wf_extend",
                "bound": "hbm",
                "achieved": round(achieved, 1),
                "peak": peak,
                "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                # The same bytes over the extension kernels' time plus the
                # queue reordering that prepares their queues.
                "frac_with_reordering": round(ext_bytes / ((timed.extend_gpu_ms + timed.sort_gpu_ms) * 1e-3) / 1e9
                                              / peak, 4) if timed.extend_gpu_ms else 0.0,
                "peak_kind": peak_kind,
                "frac_of_nominal": round(achieved / NOMINAL_HBM_GBS, 4),
                "traffic": round(EXTEND_DRAM_BYTES_PER_RAY * ext_rays_timed / launches),
                "traffic_basis": "ncu dram__bytes_read.sum + dram__bytes_write.sum per extension ray "
                                 "(one 960x540 launch of an 8-sample wave), times this wave's rays per extend "
                                 "launch",
                "bytes_per_ray": round(per_ray, 1),
                "nodes_per_ray": round(counted.node_visits[1] / n_ext, 2),
                "triangles_per_ray": round(counted.triangle_visits[1] / n_ext, 2),
                "instances_per_ray": round(counted.instance_visits[1] / n_ext, 2),
                # The instrumented frame's last wave (its samples together).
                "last_wave_samples": timed.last_wave_samples,
                "extend_ms_last_wave": round(timed.extend_gpu_ms, 4),
                "extend_launches_last_wave": launches,
                "kernel_ms_last_wave": {
                    "camera": round(timed.camera_gpu_ms, 4), "extend": round(timed.extend_gpu_ms, 4),
                    "shade": round(timed.shade_gpu_ms, 4), "shadow": round(timed.shadow_gpu_ms, 4),
                    "tail": round(timed.tail_gpu_ms, 4), "resolve": round(timed.resolve_gpu_ms, 4),
                    "reorder": round(timed.sort_gpu_ms, 4)},
                "wavefront_rounds": timed.wavefront_rounds,
            },
            "cpu_baseline": cpu,
            "clocks": clock,
            # The renderer's own per-step device times (its events around each
            # frame's samples): a spread far above the median means the GPU
            # was shared or throttled during the timed region.
            "step_gpu_ms": {"min": round(min(step_ms), 2), "median": round(statistics.median(step_ms), 2),
                            "max": round(max(step_ms), 2)},
        }
        line["converged"] = converged_report(renderer)
        convergence_report = time_to_relmse_report(renderer) if args.convergence else None
        if convergence_report:
            line["time_to_relmse_detail"] = convergence_report
        if args.batch:
            line["batch"] = batch_report(renderer)
        if args.updates:
            line["scene_updates"] = scene_update_report(renderer)
        if args.temporal:
            line["temporal"] = temporal_report(renderer)
            line["cache_kernels"] = cache_kernels_report(renderer)
        if args.lights:
            line["analytic_lights"] = analytic_lights_report(renderer)
            line["gltf_cost"] = gltf_cost_report(renderer)
        # Last, so that a reader of the line's tail sees it.
        if convergence_report:
            line["time_to_relmse"] = time_to_relmse_summary(convergence_report)
        print(json.dumps(line), flush=True)
    r.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
