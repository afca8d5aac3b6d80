"""Time to a relMSE target: the cumulative device time a method spends
rendering a static view progressively until its running image's relMSE
against a converged reference falls to the target.

relMSE is the mean over pixels and RGB of (x - r)^2 / (r^2 + 1e-2)
(metrics.relmse), taken over bands of rows through the top, middle and
bottom of the frame. The reference is plain wavefront PT with FP64
accumulation over the same bands (the target's data window), 16,384
samples per pixel, whose every path is bit-identical to the CPU oracle's
(tests/test_gpu_integrators.py). It is rendered in two independent halves
so that its own noise can be estimated (mean over pixels of
((a - b) / 2)^2 / (r^2 + 1e-2)) and taken off the measured error: with
independent noise, E[relMSE(x, r)] is x's error plus r's. Reports state the
noise beside the numbers.

Methods:
  plain            RenderScene, wavefront PT, NEE + MIS.
  cache            the same with the learned radiance cache: paths end into
                   the cache at their second vertex; the cache starts
                   untrained and trains for `warmup` samples (timed, not
                   averaged) before the progressive average starts.
  restir           RenderTemporalScene, one sample per frame with ReSTIR DI
                   for the primary vertex's direct light (initial
                   candidates, temporal reuse, one spatial pass of five
                   neighbours drawn from a 30-pixel disk), frames averaged
                   by the temporal accumulation.
  restir_initial   the same without reuse: each frame's reservoirs are its
                   own initial candidates.
  restir_spatial   the initial candidates and one spatial pass, no temporal
                   reuse.
  cache+<restir*>  the cache with one of the ReSTIR modes.
  cache_v3...      the same with the paths ending into the cache at their
                   third vertex (lotus_cache_desc::terminate_bounce 2)
                   instead of the second.
"""

import numpy as np

from . import abi, metrics

EPSILON = metrics.RELMSE_EPSILON

# ReSTIR modes: (temporal reuse, spatial reuse).
RESTIR_MODES = {
    "restir": (1, 1),
    "restir_initial": (0, 0),
    "restir_spatial": (0, 1),
}


def _settings(sample_index, depth, restir=None):
    s = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                             max_bounces=depth, sample_index=sample_index)
    if restir:
        temporal, spatial = RESTIR_MODES[restir]
        s.light_sampling = abi.LIGHT_SAMPLING_RESTIR_INITIAL
        s.restir_candidates = 8
        s.restir_temporal = temporal
        s.restir_max_history_candidates = 20
        s.restir_spatial = spatial
        s.restir_spatial_radius = 30
        s.restir_spatial_neighbours = 5
    return s


def bands(height, rows, count=3):
    """`count` bands of `rows` rows, evenly spread from the top of the frame
    to its bottom (top, middle and bottom for 3), as (first row, rows)."""
    rows = min(rows, height // count)
    if count == 1:
        return [(max(0, height // 2 - rows // 2), rows)]
    step = (height - rows) / (count - 1)
    return [(int(round(k * step)), rows) for k in range(count)]


def band_pixels(img, band_list):
    return np.concatenate([img[y0:y0 + h, :, :3] for y0, h in band_list], axis=0)


def reference(r, scene, depth, spp, band_list, chunk=256, seed=1 << 26):
    """Plain PT over `band_list` at `spp` samples, in two halves: (the bands'
    mean image stacked, its estimated relMSE noise, device seconds)."""
    from .renderer import check
    halves = [[], []]
    seconds = 0.0
    for y0, h in band_list:
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
            halves[k].append(img[y0:y0 + h, :, :3].astype(np.float64))
    a = np.concatenate(halves[0], axis=0)
    b = np.concatenate(halves[1], axis=0)
    ref = 0.5 * (a + b)
    noise = float(np.mean(((a - b) * 0.5) ** 2 / (ref * ref + EPSILON)))
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


def time_to_relmse(r, scene, method, ref, noise, depth, band_list, target=1e-3, max_seconds=30.0,
                   warmup=32, seed=12345):
    """Cumulative device seconds until relMSE <= target over the bands
    (None if the budget runs out), with the measured (seconds, relMSE)
    checkpoints, the reference's noise taken off."""
    from .renderer import check
    cache = method.startswith("cache")
    restir = method.split("+")[-1] if "restir" in method else None
    if cache:
        r.configure_cache(enable=True, seed=1, terminate_bounce=2 if method.startswith("cache_v3") else 1)
    seconds = 0.0
    points = []

    def error(img):
        return max(metrics.relmse(band_pixels(img, band_list), ref) - noise, 1e-12)

    if cache and warmup:
        res, _ = r.render_scene(scene.frame(_settings(seed + 999_999, depth), frame_count=warmup,
                                            read_back=False))
        check(res, "cache warm-up")
        seconds += res.gpu_ms * 1e-3
    if not restir:
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
        next_check = 1
        while seconds < max_seconds:
            # One sample index for the whole stream: the renderer advances its
            # own sample offset per frame, and a changed setting would reset
            # the temporal history.
            f = scene.frame(_settings(seed, depth, restir=restir), frame_count=1, read_back=True)
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
