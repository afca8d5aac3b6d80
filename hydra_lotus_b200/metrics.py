"""Image metrics: the reference's DES-Q5 statistical match and relMSE.

``compare`` restates ``Compare`` (adapters/common/reference.cpp:285-379 in
hydra-lotus): an image of N samples per pixel matches a reference of M
samples when, in each channel, the mean difference over the whole image and
over every tile is within ``MATCH_Z`` standard errors, a pixel's difference
having variance s2 (1/N + 1/M) with s2 the reference's per-sample variance.
A tile is 8x8 pixels, doubled until it holds at least 1024 samples.
"""

import math

import numpy as np

MATCH_Z = 5.0  # kMatchZ (reference.hpp:80)


class Comparison:
    def __init__(self):
        self.samples = 0
        self.tile = 0
        self.image_z = [0.0, 0.0, 0.0]
        self.max_tile_z = 0.0
        self.mean_tile_z2 = 0.0
        self.failure = ""

    @property
    def ok(self):
        return not self.failure

    def __repr__(self):
        return (f"Comparison(samples={self.samples}, tile={self.tile}, "
                f"image_z={[round(z, 3) for z in self.image_z]}, "
                f"max_tile_z={self.max_tile_z:.3f}, mean_tile_z2={self.mean_tile_z2:.3f}, "
                f"failure={self.failure!r})")


def _z(diff, var, mag, pixels):
    floor = 1e-6 + 1e-5 * mag / pixels
    return diff / pixels / math.sqrt(var / (pixels * pixels) + floor * floor)


def compare(image, samples, ref_mean, ref_variance, ref_samples):
    """DES-Q5: `image` (H, W, >=3) with `samples` spp against a reference
    mean and per-sample variance (H, W, 3) of `ref_samples` spp."""
    r = Comparison()
    r.samples = samples
    mean = np.asarray(ref_mean, dtype=np.float64)
    var = np.asarray(ref_variance, dtype=np.float64)
    img = np.asarray(image, dtype=np.float32)[..., :3].astype(np.float64)
    h, w = mean.shape[:2]
    if samples == 0 or ref_samples == 0 or var.shape != mean.shape:
        r.failure = "the reference is incomplete"
        return r
    if img.shape != mean.shape:
        r.failure = f"the image is {img.shape[1]}x{img.shape[0]} instead of {w}x{h}"
        return r
    if not np.all(np.isfinite(img)):
        bad = int(np.argmax(~np.isfinite(img).reshape(-1)) // 3)
        r.failure = f"a non-finite value at pixel {bad}"
        return r
    weight = 1.0 / samples + 1.0 / ref_samples
    diff = img - mean
    vw = var * weight
    mag = np.abs(mean)
    for c in range(3):
        z = _z(diff[..., c].sum(), vw[..., c].sum(), mag[..., c].sum(), float(h * w))
        r.image_z[c] = z
        if not (abs(z) <= MATCH_Z) and not r.failure:
            r.failure = f"{samples} spp: the image, channel {c}: {z:.3f} standard errors"
    r.tile = 8
    while r.tile * r.tile * samples < 1024 and r.tile < max(w, h):
        r.tile *= 2
    z2 = 0.0
    tests = 0
    for y0 in range(0, h, r.tile):
        for x0 in range(0, w, r.tile):
            sl = (slice(y0, min(h, y0 + r.tile)), slice(x0, min(w, x0 + r.tile)))
            n = float((sl[0].stop - y0) * (sl[1].stop - x0))
            for c in range(3):
                z = _z(diff[sl][..., c].sum(), vw[sl][..., c].sum(), mag[sl][..., c].sum(), n)
                z2 += z * z
                tests += 1
                r.max_tile_z = max(r.max_tile_z, abs(z))
                if not (abs(z) <= MATCH_Z) and not r.failure:
                    r.failure = (f"{samples} spp: the tile at {x0},{y0}, channel {c}: "
                                 f"{z:.3f} standard errors")
    r.mean_tile_z2 = z2 / tests
    return r


RELMSE_EPSILON = 1e-2


def relmse(image, reference, epsilon=RELMSE_EPSILON):
    """Mean over pixels and RGB of (x - r)^2 / (r^2 + epsilon)."""
    x = np.asarray(image, dtype=np.float64)[..., :3]
    r = np.asarray(reference, dtype=np.float64)[..., :3]
    return float(np.mean((x - r) ** 2 / (r * r + epsilon)))
