"""Time to a relMSE target: the cumulative device time a method spends
rendering a static view progressively until its running image's relMSE
against a converged reference falls to the target.

relMSE is the mean over pixels and RGB of (x - r)^2 / (r^2 + 1e-2)
(metrics.relmse). The reference is plain wavefront PT with FP64
accumulation, rendered over a band of rows (the target's data window) in
two independent halves, so that its own noise can be estimated,
(mean over pixels of ((a - b) / 2)^2 / (r^2 + 1e-2)), and taken off the
measured error: with independent noise, E[relMSE(x, r)] is x's error plus
r's.

Methods:
  plain        RenderScene, wavefront PT, NEE + MIS.
  cache        the same with the learned radiance cache: paths end into the
               cache at their second vertex; the cache starts untrained and
               trains for `warmup` samples (timed, not averaged) before the
               progressive average starts.
  restir       RenderTemporalScene, one sample per frame with ReSTIR DI
               (initial, temporal, spatial) for the primary vertex's direct
               light, frames averaged by the temporal accumulation.
  cache+restir both.
"""

import numpy as np

from . import abi, metrics

EPSILON = metrics.RELMSE_EPSILON


def _settings(sample_index, depth, restir=False):
    s = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                             max_bounces=depth, sample_index=sample_index)
    if restir:
        s.light_sampling = abi.LIGHT_SAMPLING_RESTIR_INITIAL
        s.restir_candidates = 8
        s.restir_temporal = 1
        s.restir_max_history_candidates = 20
        s.restir_spatial = 1
        s.restir_spatial_radius = 30
    return s


def band_rows(height, rows):
    y0 = max(0, height // 2 - rows // 2)
    return y0, min(rows, height - y0)


def reference(r, scene, depth, spp, rows, chunk=256, seed=1 << 26):
    """Plain PT over a band of rows at `spp` samples, in two halves:
    (mean band image, its estimated relMSE noise, device seconds)."""
    from .renderer import check
    y0, h = band_rows(scene.height, rows)
    halves = []
    seconds = 0.0
    for k in range(2):
        done = 0
        img = None
        while done < spp // 2:
            n = min(chunk, spp // 2 - done)
            f = scene.frame(_settings(seed + k * (1 << 24), depth), frame_count=n, read_back=True,
                            data_window=(0, y0, scene.width, h))
            res, img = r.render_scene(f)
            check(res, "reference")
            seconds += res.gpu_ms * 1e-3
            done += n
        halves.append(img[y0:y0 + h, :, :3].astype(np.float64))
    ref = 0.5 * (halves[0] + halves[1])
    noise = float(np.mean(((halves[0] - halves[1]) * 0.5) ** 2 / (ref * ref + EPSILON)))
    return ref, noise, seconds


def _crossing(points, target):
    """Interpolates (log t, log e) between the last point above the target
    and the first at or below it."""
    for (t0, e0), (t1, e1) in zip(points, points[1:]):
        if e0 > target >= e1:
            if e1 <= 0.0 or t0 <= 0.0:
                return t1
            a = (np.log(target) - np.log(e0)) / (np.log(e1) - np.log(e0))
            return float(np.exp(np.log(t0) + a * (np.log(t1) - np.log(t0))))
    if points and points[0][1] <= target:
        return points[0][0]
    return None


def time_to_relmse(r, scene, method, ref, noise, depth, rows, target=1e-3, max_seconds=30.0,
                   warmup=32, seed=12345):
    """Cumulative device seconds until relMSE <= target (None if the budget
    runs out), with the measured (seconds, relMSE) checkpoints."""
    from .renderer import check
    y0, h = band_rows(scene.height, rows)
    cache = method.startswith("cache")
    restir = method.endswith("restir")
    if cache:
        r.configure_cache(enable=True, seed=1)
    seconds = 0.0
    points = []

    def error(img):
        return max(metrics.relmse(img[y0:y0 + h], ref) - noise, 1e-12)

    if not restir:
        if cache and warmup:
            res, _ = r.render_scene(scene.frame(_settings(seed + 999_999, depth), frame_count=warmup,
                                                read_back=False))
            check(res, "cache warm-up")
            seconds += res.gpu_ms * 1e-3
        spp, step = 0, 1
        while seconds < max_seconds:
            res, img = r.render_scene(scene.frame(_settings(seed, depth), frame_count=step, read_back=True))
            check(res, method)
            seconds += res.gpu_ms * 1e-3
            spp += step
            points.append((seconds, error(img)))
            if points[-1][1] <= target:
                break
            step = spp  # doubling
    else:
        view = scene.view
        frame_index = 0
        if cache and warmup:
            res, _ = r.render_scene(scene.frame(_settings(seed + 999_999, depth), frame_count=warmup,
                                                read_back=False))
            check(res, "cache warm-up")
            seconds += res.gpu_ms * 1e-3
        next_check = 1
        while seconds < max_seconds:
            # One sample index for the whole stream: the renderer advances its
            # own sample offset per frame, and a changed setting would reset
            # the temporal history.
            f = scene.frame(_settings(seed, depth, restir=True), frame_count=1, read_back=True)
            d = abi.temporal_desc(f, view, view, scene.world_to_clip, history_available=frame_index > 0,
                                  accumulate_radiance=True, max_history_samples=65536, filter_iterations=0)
            res, img = r.render_temporal(d)
            check(res, method)
            seconds += res.gpu_ms * 1e-3
            frame_index += 1
            if frame_index == next_check:
                points.append((seconds, error(img)))
                if points[-1][1] <= target:
                    break
                next_check *= 2
    if cache:
        r.configure_cache(enable=False, seed=1)
    return _crossing(points, target), points
