"""CPU: the oracle's analytic lights (Lotus::Light; gpu_scene.cpp:272-610,
scene.slang:680-1178, transport.slang:139-247) against facts that do not
depend on it: the light table's weights (an analytic light's estimated power
over 2 pi), the closed-form direct light of a sphere and a disk over a
Lambert plane, and the agreement of BSDF sampling (which finds the lights
only by crossing them) with next event estimation plus MIS."""

import math

import numpy as np
import pytest

from hydra_lotus_b200 import abi, scenes

ANALYTIC = 0x80000000


def as_float(u):
    return np.asarray(u, dtype=np.uint32).view(np.float32)


def test_light_table_weights(oracle_lib):
    """Entries: the two ceiling triangles, then one per analytic light in the
    scene's order; each analytic entry's probability is proportional to its
    mean radiance times its area over 2 (a distant light's projected solid
    angle times the scene radius squared)."""
    scene = scenes.lit_room(parallel=True)
    rec, _ = oracle_lib.OracleScene(scene).light_table()
    assert rec.shape[0] == 2 + len(scene.lights)
    instance = rec[:, 3]
    assert np.all(instance[:2] < ANALYTIC)
    np.testing.assert_array_equal(instance[2:], ANALYTIC | np.arange(len(scene.lights), dtype=np.uint32))
    pdf = as_float(rec[:, 0]).astype(np.float64)
    assert abs(pdf.sum() - 1.0) < 1e-6

    def power(light):
        mean = sum(light.radiance) / 3.0
        if light.shape == abi.LIGHT_SPHERE:
            m = np.asarray(light.world_from_light).reshape(4, 4, order="F")[:3, :3]
            r = light.radius * abs(np.linalg.det(m)) ** (1.0 / 3.0)
            return mean * 4.0 * math.pi * r * r / 2.0
        if light.shape == abi.LIGHT_RECT:
            return mean * light.width * light.height / 2.0
        if light.shape == abi.LIGHT_DISK:
            area = math.pi * light.radius ** 2
            return (mean / area if light.normalize else mean) * area / 2.0
        return None

    bounded = [(k, power(l)) for k, l in enumerate(scene.lights) if power(l) is not None]
    k0, p0 = bounded[0]
    for k, p in bounded[1:]:
        assert pdf[2 + k] / pdf[2 + k0] == pytest.approx(p / p0, rel=1e-5)


def direct_mean(oracle_lib, scene, light_sampling, samples, first=0):
    st = abi.default_settings(integrator=abi.INTEGRATOR_REFERENCE, light_sampling=light_sampling,
                              max_bounces=1, sample_index=first)
    o = oracle_lib.OracleScene(scene)
    frame = scene.frame(st)
    batches = []
    for b in range(8):
        sums, _ = o.accumulate(frame, first + b * samples // 8, samples // 8)
        batches.append(sums[..., :3] / np.maximum(sums[..., 3:4], 1.0))
    return np.stack(batches)


@pytest.mark.parametrize("shape", [abi.LIGHT_SPHERE, abi.LIGHT_DISK])
def test_direct_light_closed_form(oracle_lib, shape):
    """Next event estimation with MIS converges to the closed form at the
    plane's centre: albedo L r^2 / h^2 under a sphere, albedo L r^2 /
    (r^2 + h^2) under a downward disk (h = 1, r = 0.25, L = 2, albedo 0.5)."""
    scene = scenes.lit_plane(shape, size=33)
    r2, h2 = 0.25 ** 2, 1.0
    want = 0.5 * 2.0 * (r2 / h2 if shape == abi.LIGHT_SPHERE else r2 / (r2 + h2))
    means = direct_mean(oracle_lib, scene, abi.LIGHT_SAMPLING_MIS, 4096)
    # A pixel spans 0.032 of the plane: the irradiance's mean over it is
    # within 3e-4 of the value at its centre.
    centre = means[:, 16, 16, :]
    got = centre.mean(axis=0)
    err = centre.std(axis=0, ddof=1) / math.sqrt(centre.shape[0])
    print(got, err, want)
    assert np.all(np.abs(got - want) <= 4.0 * err + 2e-3 * want)


@pytest.mark.parametrize("make", [lambda: scenes.lit_room(size=24, parallel=False),
                                  lambda: scenes.many_lights(size=24, count=24)])
def test_bsdf_sampling_agrees_with_mis(oracle_lib, make):
    """With one bounce, BSDF sampling finds the analytic lights only by
    crossing them, MIS also by sampling them: both estimate the same direct
    light. Compared over the image's mean, within four standard errors."""
    scene = make()
    mis = direct_mean(oracle_lib, scene, abi.LIGHT_SAMPLING_MIS, 256).mean(axis=(1, 2, 3))
    bsdf = direct_mean(oracle_lib, scene, abi.LIGHT_SAMPLING_BSDF, 2048, first=1 << 16).mean(axis=(1, 2, 3))
    err = math.hypot(mis.std(ddof=1) / math.sqrt(mis.size), bsdf.std(ddof=1) / math.sqrt(bsdf.size))
    print(mis.mean(), bsdf.mean(), err)
    assert abs(mis.mean() - bsdf.mean()) <= 4.0 * err + 1e-3 * mis.mean()


def test_invalid_light_rejected(oracle_lib):
    scene = scenes.lit_plane(abi.LIGHT_SPHERE, size=8)
    scene.lights[0].shape = 9
    scene._desc = None
    with pytest.raises(RuntimeError):
        oracle_lib.OracleScene(scene)
