"""GPU parity of the integrators against the oracle, through the C ABI."""

import numpy as np
import pytest

from hydra_lotus_b200 import abi, metrics, scenes

from parity import PathParity

pytestmark = pytest.mark.gpu

INTEGRATORS = [abi.INTEGRATOR_REFERENCE, abi.INTEGRATOR_WAVEFRONT]


def small_sphere_field():
    return scenes.sphere_field(seed=3, width=160, height=96, prototypes=8, grid=12,
                               spacing=2.0, spheres=60, emitters=8, sky_size=(256, 128))


@pytest.fixture(scope="module")
def renderer(cuda):
    r = cuda.CudaOffscreenRenderer(0)
    yield r
    r.close()


def render(cuda, renderer, scene, settings, frame_count=1, **kw):
    cuda.check(renderer.update_scene(scene), "update_scene")
    res, color = renderer.render_scene(scene.frame(settings, frame_count, **kw))
    cuda.check(res, "render_scene")
    return res, color


@pytest.mark.parametrize("integrator", INTEGRATORS)
@pytest.mark.parametrize("light_sampling", [abi.LIGHT_SAMPLING_BSDF, abi.LIGHT_SAMPLING_MIS])
def test_box_room_paths_match_oracle(cuda, renderer, oracle_lib, integrator, light_sampling):
    scene = scenes.box_room(seed=0, size=128)
    st = abi.default_settings(integrator=integrator, light_sampling=light_sampling,
                              max_bounces=6, sample_index=7)
    res, color = render(cuda, renderer, scene, st)
    want, rays = oracle_lib.OracleScene(scene).sample(scene.frame(st), 7)
    p = PathParity(color, want)
    print(p)
    p.assert_ok()
    assert p.exact > 0.9, p
    assert res.camera_rays == rays[0]


@pytest.mark.parametrize("integrator", INTEGRATORS)
def test_sphere_field_paths_match_oracle(cuda, renderer, oracle_lib, integrator):
    scene = small_sphere_field()
    st = abi.default_settings(integrator=integrator, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=8, sample_index=3)
    res, color = render(cuda, renderer, scene, st)
    want, rays = oracle_lib.OracleScene(scene).sample(scene.frame(st), 3)
    p = PathParity(color, want)
    print(p, res.camera_rays, res.extension_rays, res.shadow_rays, rays)
    p.assert_ok()


@pytest.mark.parametrize("integrator", INTEGRATORS)
def test_large_mesh_paths_match_oracle(cuda, renderer, oracle_lib, integrator):
    """A mesh above the per-CTA SAH builder's limit builds as an LBVH."""
    scene = scenes.big_mesh()
    st = abi.default_settings(integrator=integrator, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=6, sample_index=5)
    res, color = render(cuda, renderer, scene, st)
    want, _ = oracle_lib.OracleScene(scene).sample(scene.frame(st), 5)
    p = PathParity(color, want)
    print(p)
    p.assert_ok()


def test_light_table_matches_oracle(cuda, renderer, oracle_lib):
    for scene in (scenes.box_room(), scenes.cornell_reference(), small_sphere_field()):
        cuda.check(renderer.update_scene(scene), "update_scene")
        got_rec, got_off = renderer.light_table()
        want_rec, want_off = oracle_lib.OracleScene(scene).light_table()
        np.testing.assert_array_equal(got_rec, want_rec)
        np.testing.assert_array_equal(got_off, want_off)


def test_wavefront_equals_reference_integrator(cuda, renderer):
    scene = scenes.box_room(seed=0, size=128)
    out = []
    for integrator in INTEGRATORS:
        st = abi.default_settings(integrator=integrator, light_sampling=abi.LIGHT_SAMPLING_MIS,
                                  max_bounces=6, sample_index=11)
        _, color = render(cuda, renderer, scene, st, frame_count=4)
        out.append(color)
    p = PathParity(out[1], out[0])
    print(p)
    assert p.within >= 0.999, p


@pytest.mark.parametrize("integrator", INTEGRATORS)
@pytest.mark.parametrize("light_sampling", [abi.LIGHT_SAMPLING_BSDF, abi.LIGHT_SAMPLING_MIS])
def test_cornell_matches_reference_golden(cuda, renderer, golden, integrator, light_sampling):
    """DES-Q5 against the reference's committed 1024-spp Cornell images,
    from sample index 2^20 as renderer.path.reference renders it."""
    scene = scenes.cornell_reference()
    st = abi.default_settings(integrator=integrator, light_sampling=light_sampling,
                              max_bounces=64, sample_index=1 << 20)
    res, color = render(cuda, renderer, scene, st, frame_count=1024)
    assert res.samples_per_pixel == 1024
    c = metrics.compare(color, 1024, golden["mean"], golden["variance"], golden["samples"])
    print(c)
    assert c.ok, c


def test_cornell_negative_control_rejected(cuda, renderer, golden):
    scene = scenes.cornell_reference(red_scale=1.1)
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT,
                              light_sampling=abi.LIGHT_SAMPLING_BSDF, max_bounces=64,
                              sample_index=1 << 20)
    _, color = render(cuda, renderer, scene, st, frame_count=1024)
    c = metrics.compare(color, 1024, golden["mean"], golden["variance"], golden["samples"])
    assert not c.ok, c


@pytest.mark.parametrize("name", ["box_room", "lit_room"])
@pytest.mark.parametrize("light_sampling", [abi.LIGHT_SAMPLING_BSDF, abi.LIGHT_SAMPLING_MIS])
def test_tail_kernel_paths_match_oracle(cuda, renderer, oracle_lib, name, light_sampling):
    """Above LOTUS_WAVEFRONT_ROUNDS - 1 bounces the wavefront integrator's
    tail kernel follows the paths still queued after its rounds: each path
    is the oracle's, and the per-bounce queue counts equal those of a
    sample run in rounds throughout (counting visits keeps every bounce in
    rounds)."""
    scene = scenes.box_room(seed=2, size=96) if name == "box_room" else scenes.lit_room(seed=2, size=96)
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=light_sampling, max_bounces=64,
                              sample_index=21)
    res, color = render(cuda, renderer, scene, st)
    assert res.wavefront_rounds == abi.WAVEFRONT_ROUNDS
    want, rays = oracle_lib.OracleScene(scene).sample(scene.frame(st), 21)
    p = PathParity(color, want)
    print(name, p, res.wavefront_path_count_size, rays, res.extension_rays, res.shadow_rays)
    p.assert_ok()
    assert p.exact > 0.9, p
    assert res.wavefront_path_count_size > abi.WAVEFRONT_ROUNDS
    counted, color2 = render(cuda, renderer, scene, st, flags=abi.FRAME_COUNT_VISITS)
    assert counted.wavefront_rounds == 65
    assert np.array_equal(color, color2)
    assert list(res.wavefront_path_counts[:64]) == list(counted.wavefront_path_counts[:64])
    assert (res.extension_rays, res.shadow_rays) == (counted.extension_rays, counted.shadow_rays)


@pytest.mark.parametrize("frames", [2, 7, 16, 35])
def test_sample_chains_equal_one_sample_at_a_time(cuda, renderer, frames):
    """A call that adds several samples runs them two in flight, in chains of
    up to 16 (each resolving after the one before): its image is bit for bit
    the one `frames` calls of one sample give, the FP64 accumulation adding
    the samples in the same order."""
    scene = scenes.lit_room(seed=5, size=64)
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=12, sample_index=300)
    res, chained = render(cuda, renderer, scene, st, frame_count=frames)
    assert res.samples_per_pixel == frames
    cuda.check(renderer.update_scene(scene), "update_scene")
    for k in range(frames):
        res, single = renderer.render_scene(scene.frame(st, 1))
        cuda.check(res, "one sample")
    assert res.samples_per_pixel == frames
    assert np.array_equal(chained, single), f"{np.count_nonzero(chained != single)} values differ"


def test_reference_integrator_on_queues_matches_oracle(cuda, renderer, oracle_lib):
    """A reference-integrator frame of at least the extension kernel's
    resident threads (here 512^2 paths) runs on the wavefront's queues:
    path for path the oracle's, with the reference integrator's evidence
    (no wavefront path counts or rounds)."""
    scene = scenes.box_room(seed=0, size=512)
    st = abi.default_settings(integrator=abi.INTEGRATOR_REFERENCE, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=12, sample_index=5)
    res, color = render(cuda, renderer, scene, st)
    assert res.wavefront_rounds == 0 and res.wavefront_path_count_size == 0
    want, rays = oracle_lib.OracleScene(scene).sample(scene.frame(st), 5)
    p = PathParity(color, want)
    print(p)
    p.assert_ok()
    assert p.exact > 0.9, p
    assert res.camera_rays == rays[0]


def test_reference_integrator_queued_accumulation_equals_per_thread_loop(cuda, renderer):
    """Eight samples in one call at 192^2 (a wave of eight holds 294,912
    paths: the queues) equal eight one-sample calls (36,864 paths each: the
    per-thread loop, k_reference_pt) bit for bit: the two schedules compute
    each path and add the samples to the FP64 accumulation identically."""
    scene = scenes.lit_room(seed=2, size=192)
    st = abi.default_settings(integrator=abi.INTEGRATOR_REFERENCE, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=12, sample_index=40)
    res, queued = render(cuda, renderer, scene, st, frame_count=8)
    assert res.samples_per_pixel == 8
    cuda.check(renderer.update_scene(scene), "update_scene")
    for k in range(8):
        res, single = renderer.render_scene(scene.frame(st, 1))
        cuda.check(res, "one sample")
    assert res.samples_per_pixel == 8
    assert np.array_equal(queued, single), f"{np.count_nonzero(queued != single)} values differ"


MATERIAL_MODES = [(abi.INTEGRATOR_REFERENCE, abi.LIGHT_SAMPLING_BSDF),
                  (abi.INTEGRATOR_REFERENCE, abi.LIGHT_SAMPLING_MIS),
                  (abi.INTEGRATOR_WAVEFRONT, abi.LIGHT_SAMPLING_MIS),
                  (abi.INTEGRATOR_WAVEFRONT, abi.LIGHT_SAMPLING_BSDF)]


@pytest.mark.parametrize("integrator,light_sampling", MATERIAL_MODES)
def test_material_basics_matches_reference_golden(cuda, renderer, golden_materials, integrator,
                                                  light_sampling):
    """DES-Q5 against the reference's committed 4096-spp material-basics-v1
    images (GGX conductors, rough and smooth coats, metallic mixes, ior
    2.5, the specular workflow, a constant dome and a rect light), at the
    reference's levels 16 and 256 spp in one accumulation (kMaterialLevels,
    adapters/headless/main.cpp) and then at 1024 spp."""
    scene = scenes.material_basics()
    st = abi.default_settings(integrator=integrator, light_sampling=light_sampling,
                              max_bounces=64, sample_index=1 << 20)
    g = golden_materials
    cuda.check(renderer.update_scene(scene), "update_scene")
    rendered = 0
    for level in (16, 256, 1024):
        res, color = renderer.render_scene(scene.frame(st, level - rendered))
        cuda.check(res, "render_scene")
        rendered = level
        assert res.samples_per_pixel == level
        c = metrics.compare(color, level, g["mean"], g["variance"], g["samples"])
        print(level, c)
        assert c.ok, c


def test_material_basics_negative_control_rejected(cuda, renderer, golden_materials):
    """The half-rough copper 10% darker (DarkerMetal) must not match."""
    scene = scenes.material_basics(metal50_scale=0.9)
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=64, sample_index=1 << 20)
    _, color = render(cuda, renderer, scene, st, frame_count=256)
    g = golden_materials
    c = metrics.compare(color, 256, g["mean"], g["variance"], g["samples"])
    assert not c.ok, c


@pytest.mark.parametrize("integrator", INTEGRATORS)
@pytest.mark.parametrize("light_sampling", [abi.LIGHT_SAMPLING_BSDF, abi.LIGHT_SAMPLING_MIS])
def test_material_basics_paths_match_oracle(cuda, renderer, oracle_lib, integrator, light_sampling):
    """Every path of the material fixture (corner normals, every
    UsdPreviewSurface lobe, the dome and the rect light) against the
    oracle's, whose image the previous tests pin to the reference's."""
    scene = scenes.material_basics()
    st = abi.default_settings(integrator=integrator, light_sampling=light_sampling,
                              max_bounces=64, sample_index=9)
    res, color = render(cuda, renderer, scene, st)
    want, rays = oracle_lib.OracleScene(scene).sample(scene.frame(st), 9)
    p = PathParity(color, want)
    print(p)
    p.assert_ok()
    assert p.exact > 0.9, p
    assert res.camera_rays == rays[0]


@pytest.fixture(scope="module")
def bench_frame_scene():
    return scenes.sphere_field(seed=0)


@pytest.mark.parametrize("integrator", INTEGRATORS)
@pytest.mark.parametrize("band", [300, 536, 1064])
def test_bench_frame_band_paths_match_oracle(cuda, renderer, oracle_lib, bench_frame_scene,
                                             integrator, band):
    """The benchmarked frame itself (the seeded 1080p sphere field: 13.7M
    instanced triangles, the 2048x1024 sky), 16 rows at the horizon (the
    rows above it see only sky), the middle and the bottom, one sample at
    depth 8: each path against the oracle's."""
    scene = bench_frame_scene
    st = abi.default_settings(integrator=integrator, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=8, sample_index=40)
    window = (0, band, scene.width, 16)
    cuda.check(renderer.update_scene(scene), "update_scene")
    res, color = renderer.render_scene(scene.frame(st, 1, data_window=window))
    cuda.check(res, "render_scene")
    want, rays = oracle_lib.OracleScene(scene).sample(scene.frame(st, data_window=window), 40)
    p = PathParity(color[band:band + 16], want[band:band + 16])
    print(p, res.camera_rays, res.extension_rays, res.shadow_rays, rays)
    p.assert_ok()
    assert res.camera_rays == rays[0] == scene.width * 16
