"""GPU: analytic lights (Lotus::Light: sphere, rect, disk, distant and
parallel lights) through the C ABI. Per-path parity with the oracle's
restatement for both integrators under BSDF and MIS light sampling, the
light table entry for entry, the closed-form direct light of a sphere and a
disk over a Lambert plane, and batches that give each scene its own image."""

import math

import numpy as np
import pytest

from hydra_lotus_b200 import abi, scenes

from parity import PathParity

pytestmark = pytest.mark.gpu

INTEGRATORS = [abi.INTEGRATOR_REFERENCE, abi.INTEGRATOR_WAVEFRONT]
SAMPLING = [abi.LIGHT_SAMPLING_BSDF, abi.LIGHT_SAMPLING_MIS]


@pytest.fixture(scope="module")
def renderer(cuda):
    r = cuda.CudaOffscreenRenderer(0)
    yield r
    r.close()


def lit_room_sky():
    return scenes.lit_room(seed=1, size=96, environment=True)


SCENES = {
    "lit_room": lambda: scenes.lit_room(seed=0, size=96),
    "lit_room_sky": lit_room_sky,
    "many_lights": lambda: scenes.many_lights(seed=2, size=96, count=48),
}


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("integrator", INTEGRATORS)
@pytest.mark.parametrize("light_sampling", SAMPLING)
def test_paths_match_oracle(cuda, renderer, oracle_lib, name, integrator, light_sampling):
    scene = SCENES[name]()
    st = abi.default_settings(integrator=integrator, light_sampling=light_sampling, max_bounces=6,
                              sample_index=13)
    cuda.check(renderer.update_scene(scene), "update_scene")
    res, color = renderer.render_scene(scene.frame(st, 1))
    cuda.check(res, "render_scene")
    want, rays = oracle_lib.OracleScene(scene).sample(scene.frame(st), 13)
    p = PathParity(color, want)
    print(name, p, res.shadow_rays, rays)
    p.assert_ok()
    assert p.exact > 0.9, p
    assert res.camera_rays == rays[0]
    if integrator == abi.INTEGRATOR_REFERENCE:
        assert res.shadow_rays == rays[2]


@pytest.mark.parametrize("name", list(SCENES))
def test_light_table_matches_oracle(cuda, renderer, oracle_lib, name):
    scene = SCENES[name]()
    cuda.check(renderer.update_scene(scene), "update_scene")
    got_rec, got_off = renderer.light_table()
    want_rec, want_off = oracle_lib.OracleScene(scene).light_table()
    np.testing.assert_array_equal(got_rec, want_rec)
    np.testing.assert_array_equal(got_off, want_off)
    assert (got_rec[:, 3] & 0x80000000).any()


@pytest.mark.parametrize("shape", [abi.LIGHT_SPHERE, abi.LIGHT_DISK])
@pytest.mark.parametrize("light_sampling", SAMPLING)
def test_direct_light_closed_form(cuda, renderer, shape, light_sampling):
    """The plane's centre under a sphere (albedo L r^2 / h^2) and a
    downward disk (albedo L r^2 / (r^2 + h^2)), one bounce, 4096 samples
    (BSDF sampling, which finds the light only by crossing it: 32768)."""
    scene = scenes.lit_plane(shape, size=33)
    r2 = 0.25 ** 2
    want = 0.5 * 2.0 * (r2 if shape == abi.LIGHT_SPHERE else r2 / (r2 + 1.0))
    n = 4096 if light_sampling == abi.LIGHT_SAMPLING_MIS else 32768
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=light_sampling, max_bounces=1,
                              sample_index=0)
    cuda.check(renderer.update_scene(scene), "update_scene")
    res, color = renderer.render_scene(scene.frame(st, n))
    cuda.check(res, "render_scene")
    got = color[15:18, 15:18, :3].mean(axis=(0, 1))
    # BSDF sampling's estimate at a pixel is a Bernoulli trial of the light's
    # projected solid angle (p about r^2 / h^2): relative standard error
    # sqrt((1 - p) / (p n)) over the 9 pixels.
    p = r2
    tol = 4.0 * math.sqrt((1.0 - p) / (p * n * 9)) if light_sampling == abi.LIGHT_SAMPLING_BSDF else 0.01
    print(got, want, tol)
    np.testing.assert_allclose(got, want, rtol=tol + 0.003)


def test_batch_with_analytic_lights_matches_single_renders(cuda):
    scs = [scenes.many_lights(seed=4, size=48, count=24), scenes.lit_room(seed=3, size=40),
           scenes.box_room(seed=1, size=32)]

    def settings(k, sample_index):
        return abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT,
                                    light_sampling=abi.LIGHT_SAMPLING_BSDF if k == 1 else abi.LIGHT_SAMPLING_MIS,
                                    max_bounces=5, sample_index=sample_index)

    with cuda.CudaBatch(0) as batch:
        res = batch.set_scenes(scs)
        assert all(r.status == abi.PASS for r in res), [r.detail for r in res]
        frames = [s.frame(settings(k, 40 + k), frame_count=3) for k, s in enumerate(scs)]
        results, colors, total = batch.render(frames)
        cuda.check(total, "batch render")
    with cuda.CudaOffscreenRenderer(0) as r:
        for k, s in enumerate(scs):
            cuda.check(r.update_scene(s), "update_scene")
            res, want = r.render_scene(s.frame(settings(k, 40 + k), frame_count=3))
            cuda.check(res, "render_scene")
            assert np.array_equal(colors[k], want), f"scene {k}: {np.count_nonzero(colors[k] != want)} values differ"


def test_invalid_lights_fail_without_poisoning(cuda, renderer):
    scene = scenes.lit_plane(abi.LIGHT_SPHERE, size=16)
    scene.lights[0].shape = 7
    scene._desc = None
    res = renderer.update_scene(scene)
    assert res.status == abi.FAIL and b"analytic light" in res.detail
    scene.lights[0].shape = abi.LIGHT_SPHERE
    scene.lights[0].radiance[0] = float("nan")
    scene._desc = None
    assert renderer.update_scene(scene).status == abi.FAIL
    cuda.check(renderer.update_scene(scenes.lit_plane(abi.LIGHT_DISK, size=16)), "update after rejects")


def test_spatial_overflow_fails_the_frame_and_latches(cuda):
    """The reference's SpatialOverflow case (validation/restir-gpu-test.cpp,
    SpatialOverflow): a white Lambert plane under a parallel light of
    radiance 2.4e38, one candidate, spatial reuse. Every initial reservoir is
    finite; merging neighbours overflows float, so the frame Fails with the
    spatial pass's detail, and the failure latches."""
    s = scenes.Scene("spatial-overflow")
    white = s.add_material(scenes.preview_material((1.0, 1.0, 1.0), roughness=1.0, ior=1.0))
    s.add_instance(s.add_geometry(*scenes.quad([[-9, 0, 9], [9, 0, 9], [9, 0, -9], [-9, 0, -9]])), white)
    s.add_light(abi.LIGHT_DISTANT, scenes.affine(linear=scenes.towards((0.2, 1.0, 0.1))),
                radiance=(2.4e38, 2.4e38, 2.4e38), angle=0.0)
    view = scenes.look_at((0.0, 3.0, 1e-3), (0.0, 0.0, 0.0), up=(0.0, 0.0, -1.0))
    w2c = scenes.multiply(scenes.perspective(40.0, 1.0, 0.1, 100.0), view)
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_RESTIR_INITIAL,
                              max_bounces=1, sample_index=0, restir_candidates=1, restir_temporal=1,
                              restir_spatial=1, restir_spatial_radius=2)
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(s), "update_scene")
        d = abi.temporal_desc(abi.make_frame(w2c, 8, 8, st, 1), view)
        res, _ = r.render_temporal(d)
        assert res.status == abi.FAIL and b"spatial reservoir arithmetic" in res.detail, res.detail
        res, _ = r.render_temporal(d)
        assert res.status == abi.FAIL
        st.restir_spatial = 0
        res, _ = r.render_temporal(abi.temporal_desc(abi.make_frame(w2c, 8, 8, st, 1), view))
        assert res.status == abi.FAIL
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(s), "update_scene")
        st.restir_spatial = 0
        res, _ = r.render_temporal(abi.temporal_desc(abi.make_frame(w2c, 8, 8, st, 1), view))
        cuda.check(res, "the same frame without spatial reuse")
