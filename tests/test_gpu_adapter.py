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


@pytest.mark.parametrize("integrator", [abi.INTEGRATOR_REFERENCE, abi.INTEGRATOR_WAVEFRONT])
@pytest.mark.parametrize("scene_name", ["box_room", "sphere_field"])
def test_adapter_renders_what_the_c_abi_renders(cuda, harness, tmp_path, integrator, scene_name):
    scene = scenes.box_room(seed=0, size=64) if scene_name == "box_room" else small_sphere_field()
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
    give the images a full update of the edited scene gives."""
    scene = scenes.box_room(seed=0, size=48)
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=5, sample_index=3)
    code, evidence, colors = adapter_scene.run(str(tmp_path), scene, st, 4, edit_dx=0.05)
    assert code == 0, evidence
    assert evidence[-1]["instance_edit"] == "pass" and evidence[-1]["point_edit"] == "pass", evidence
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
