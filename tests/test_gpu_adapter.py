"""GPU: a reference host's calls through the C++ adapter
(CudaOffscreenRenderer, the reference's Lotus::OffscreenRenderer over the C
ABI) render exactly what the C ABI renders for the same scene and frame:
the adapter's SceneUpdate -> scene description and PathTracingSettings ->
frame mapping loses nothing. The harness (tests/adapter_harness.cpp) builds
the reference's own scene types from the same data."""

import os

import numpy as np
import pytest

from hydra_lotus_b200 import abi, scenes

import adapter_scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def harness():
    if not os.path.exists(adapter_scene.HARNESS):
        pytest.skip("the adapter's driver builds only where the reference's headers are present")
    return adapter_scene.HARNESS


def small_sphere_field():
    return scenes.sphere_field(seed=3, width=96, height=64, prototypes=6, grid=10, spacing=2.0,
                               spheres=40, emitters=6, sky_size=(128, 64))


ADAPTER_SCENES = {
    "box_room": lambda: scenes.box_room(seed=0, size=64),
    "sphere_field": small_sphere_field,
    # Lotus::Light of every shape, mapped by the adapter to lotus_light.
    "lit_room": lambda: scenes.lit_room(seed=2, size=64, environment=True),
    # Textures, texture inputs on every PreviewSurface slot, coordinate sets
    # and fallbacks, normal maps, mapped by the adapter from the
    # reference's Texture / TextureInput / MeshGeometry::texcoords.
    "material_textures": lambda: scenes.material_textures(size=64),
    # glTF PBR materials with every extension and their lookups.
    "material_gltf": lambda: scenes.material_gltf(size=64),
    "material_gltf_extensions": lambda: scenes.material_gltf_extensions(size=64),
    "material_normals": lambda: scenes.material_normals(size=64),
    "texture_cutouts": lambda: scenes.texture_cutouts(size=64),
}


@pytest.mark.parametrize("integrator", [abi.INTEGRATOR_REFERENCE, abi.INTEGRATOR_WAVEFRONT])
@pytest.mark.parametrize("scene_name", list(ADAPTER_SCENES))
def test_adapter_renders_what_the_c_abi_renders(cuda, harness, tmp_path, integrator, scene_name):
    scene = ADAPTER_SCENES[scene_name]()
    st = abi.default_settings(integrator=integrator, light_sampling=abi.LIGHT_SAMPLING_MIS, max_bounces=6,
                              sample_index=11)
    code, evidence, color = adapter_scene.run(str(tmp_path), scene, st, 4)
    assert code == 0, evidence
    assert evidence["capability"] is True
    assert evidence["update"] == "pass" and evidence["render"] == "pass", evidence
    assert evidence["instances"] == len(scene.instances)
    assert evidence["spp"] == 4
    assert evidence["pixel_format"] == "rgba32-sfloat" and evidence["row_pitch"] == scene.width * 16
    assert evidence["bootstrap"] == "skip" and evidence["present"] == "skip"
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        res, want = r.render_scene(scene.frame(st, frame_count=4))
        cuda.check(res, "render_scene")
    assert color is not None
    assert np.array_equal(color, want), f"{np.count_nonzero(color != want)} values differ"


def test_adapter_incremental_updates_render_what_full_updates_render(cuda, harness, tmp_path):
    """An instance-only SceneUpdate and a same-topology geometry replacement
    go through lotus_cuda_update_instances / lotus_cuda_update_geometry and
    give the images a full update of the edited scene gives; ReadBackScene
    then returns the edited instances and the points each one names."""
    scene = scenes.box_room(seed=0, size=48)
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=5, sample_index=3)
    code, evidence, colors = adapter_scene.run(str(tmp_path), scene, st, 4, edit_dx=0.05)
    assert code == 0, evidence
    assert evidence[-1]["instance_edit"] == "pass" and evidence[-1]["point_edit"] == "pass", evidence
    assert evidence[-1]["readback"] == "pass" and evidence[-1]["materials"] == len(scene.materials), evidence
    moved = scenes.box_room(seed=0, size=48)
    m = np.array(moved.instances[0][0], dtype=np.float32)
    m[12] += np.float32(0.05)
    moved.set_instance(0, m)
    edited = scenes.box_room(seed=0, size=48)
    edited.set_instance(0, m)
    p, t, n = edited.geometries[0]
    q = p.copy()
    q[:, 1] += np.float32(0.01) * p[:, 0]
    edited.set_positions(0, q)
    for want_scene, got in ((moved, colors[1]), (edited, colors[2])):
        with cuda.CudaOffscreenRenderer(0) as r:
            cuda.check(r.update_scene(want_scene), "update_scene")
            res, want = r.render_scene(want_scene.frame(st, frame_count=4))
            cuda.check(res, "render_scene")
        assert got is not None
        assert np.array_equal(got, want), f"{np.count_nonzero(got != want)} values differ"


def test_adapter_temporal_products_equal_the_c_abi(cuda, harness, tmp_path):
    """RenderTemporalScene through the adapter returns the reference's
    TemporalProducts and RestirProducts (surface, validity, radiance, batch,
    initial / temporal / spatial reservoirs, spatial sources) and colour,
    byte for byte what the C ABI's products are for the same two frames."""
    scene = scenes.restir_room(seed=0, size=48, emitters=200)
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=4, sample_index=5)
    code, evidence, frames = adapter_scene.run_temporal(str(tmp_path), scene, st)
    assert code == 0, evidence
    assert [e["history"] for e in evidence] == [False, True], evidence
    assert all(e["temporal"] and e["restir"] for e in evidence), evidence
    assert evidence[1]["previous_pixels"] == scene.width * scene.height
    rst = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT,
                               light_sampling=abi.LIGHT_SAMPLING_RESTIR_INITIAL, max_bounces=4, sample_index=5,
                               restir_temporal=1, restir_spatial=1, restir_spatial_radius=2)
    identity = [1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0]
    names = {"surface": abi.PRODUCT_SURFACE, "validity": abi.PRODUCT_VALIDITY, "radiance": abi.PRODUCT_RADIANCE,
             "batch": abi.PRODUCT_BATCH, "restir_initial": abi.PRODUCT_RESTIR_INITIAL,
             "restir_temporal": abi.PRODUCT_RESTIR_TEMPORAL, "restir_spatial": abi.PRODUCT_RESTIR_SPATIAL,
             "restir_sources": abi.PRODUCT_RESTIR_SOURCES}
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        for k in range(2):
            frame = abi.make_frame(scene.world_to_clip, scene.width, scene.height, rst, 1)
            d = abi.temporal_desc(frame, identity, identity, scene.world_to_clip, history_available=k > 0,
                                  accumulate_radiance=True, max_history_samples=5, filter_iterations=2)
            res, color = r.render_temporal(d)
            cuda.check(res, f"render_temporal {k}")
            got = frames[k]
            assert got["color"] == color.tobytes(), f"frame {k}: colour differs"
            for name, product in names.items():
                want = r.read_product(product, scene.height, scene.width).tobytes()
                assert got[name] == want, f"frame {k}: {name} differs"
