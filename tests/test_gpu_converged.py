"""Converged images against the oracle's (tests/golden/make_oracle_images.py:
the CPU oracle's FP64 accumulation of 16,384 samples per pixel for the box
room, 4,096 for a band of the 1080p sphere field, with per-pixel variances
from batches).

The box-room image must pass the reference's DES-Q5 per-pixel statistics
(metrics.compare: the whole image and every tile within 5 standard errors)
and its relMSE (epsilon 1e-2) must be the one its noise explains: at most
RELMSE_SLACK times the expected relMSE of an unbiased estimator with the
oracle's per-sample variance, the mean over pixels of var (1/N + 1/M) /
(r^2 + epsilon). The sphere-field band is held to the band-wide z per
channel (see its test).
"""

import os

import numpy as np
import pytest

from hydra_lotus_b200 import abi, metrics, scenes

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RELMSE_SLACK = 1.25


def load(name):
    g = np.load(os.path.join(ROOT, "tests", "golden", name))
    return {k: g[k] for k in g.files}


def expected_relmse(variance, reference, samples, ref_samples):
    v = variance.astype(np.float64) * (1.0 / samples + 1.0 / ref_samples)
    r = reference.astype(np.float64)
    return float(np.mean(v / (r * r + metrics.RELMSE_EPSILON)))


@pytest.mark.parametrize("integrator", [abi.INTEGRATOR_WAVEFRONT, abi.INTEGRATOR_REFERENCE])
def test_box_room_converges_to_oracle(cuda, integrator):
    """The small box-room workload exactly as specified: 256x256, 64 spp,
    max depth 6, NEE + MIS."""
    g = load("box_room_256_oracle.npz")
    scene = scenes.box_room(seed=0, size=256)
    st = abi.default_settings(integrator=integrator, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=6, sample_index=0)
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        res, color = r.render_scene(scene.frame(st, 64))
        cuda.check(res, "render_scene")
    assert res.samples_per_pixel == 64
    c = metrics.compare(color, 64, g["mean"], g["variance"], int(g["samples"]))
    err = metrics.relmse(color, g["mean"])
    bound = RELMSE_SLACK * expected_relmse(g["variance"], g["mean"], 64, int(g["samples"]))
    print(c, err, bound)
    assert c.ok, c
    assert err <= bound, (err, bound)


@pytest.mark.parametrize("integrator", [abi.INTEGRATOR_WAVEFRONT, abi.INTEGRATOR_REFERENCE])
def test_sphere_field_band_converges_to_oracle(cuda, integrator):
    """A 16-row band through the middle of the benchmarked 1080p frame at
    depth 8, 1024 spp. The sphere field's dielectrics and sun give caustic
    paths whose radiance is heavy-tailed: the CPU oracle's own 1024-spp
    image fails the per-tile z-test against its 4096-spp image (largest
    tile |z| about 21), so only the band-wide z per channel (within 5
    standard errors) is asserted here; the per-path agreement of this frame
    with the oracle is bit-exact (test_gpu_integrators.py)."""
    g = load("sphere_field_band_oracle.npz")
    y0, rows = (int(v) for v in g["band"])
    scene = scenes.sphere_field(seed=0)
    st = abi.default_settings(integrator=integrator, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=8, sample_index=0)
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        res, color = r.render_scene(scene.frame(st, 1024, data_window=(0, y0, scene.width, rows)))
        cuda.check(res, "render_scene")
    band = color[y0:y0 + rows]
    c = metrics.compare(band, 1024, g["mean"], g["variance"], int(g["samples"]))
    print(c, metrics.relmse(band, g["mean"]))
    assert all(abs(z) <= metrics.MATCH_Z for z in c.image_z), c
