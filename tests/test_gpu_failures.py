"""Device-side bounds that run out are reported, not silent.

A BVH walk ends early when it has used its step budget or when a child does
not fit on its traversal stack; either leaves the frame's hits incomplete.
The kernels count such walks in a failure word that the renderer reads back
with the frame's ray totals: the frame Fails with a detail naming the cause
and the renderer is poisoned, as for any device failure. The tests lower the
step budget (lotus_cuda_options::traversal_step_limit) so that it runs out;
the kernels return normally, so nothing waits or faults.
"""

import pytest

from hydra_lotus_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def small_sphere_field():
    return scenes.sphere_field(seed=3, width=160, height=96, prototypes=8, grid=12,
                               spacing=2.0, spheres=60, emitters=8, sky_size=(256, 128))


@pytest.mark.parametrize("integrator", [abi.INTEGRATOR_REFERENCE, abi.INTEGRATOR_WAVEFRONT])
def test_step_budget_running_out_fails_the_frame(cuda, integrator):
    scene = small_sphere_field()
    st = abi.default_settings(integrator=integrator, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=8, sample_index=3)
    with cuda.CudaOffscreenRenderer(0, traversal_step_limit=16) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        res, _ = r.render_scene(scene.frame(st, 2))
        assert res.status == abi.FAIL
        detail = res.detail.decode()
        assert "ran out of its 16 steps" in detail, detail
        assert "BVH walk" in detail, detail
        # The renderer is poisoned.
        again, _ = r.render_scene(scene.frame(st, 1))
        assert again.status == abi.FAIL
        assert "failed earlier" in again.detail.decode()


def test_default_step_budget_passes(cuda):
    scene = small_sphere_field()
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=8, sample_index=3)
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        cuda.check(r.render_scene(scene.frame(st, 2))[0], "render_scene")


def test_step_budget_running_out_fails_a_temporal_frame(cuda):
    scene = scenes.restir_room(seed=0, size=48, emitters=64)
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT,
                              light_sampling=abi.LIGHT_SAMPLING_RESTIR_INITIAL, max_bounces=4,
                              sample_index=0, restir_candidates=4)
    with cuda.CudaOffscreenRenderer(0, traversal_step_limit=4) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        view, w2c = scenes.orbit_camera(0)
        frame = abi.make_frame(w2c, scene.width, scene.height, st, 1)
        d = abi.temporal_desc(frame, view, None, None, history_available=False,
                              accumulate_radiance=True, max_history_samples=5, filter_iterations=1)
        res, _ = r.render_temporal(d)
        assert res.status == abi.FAIL
        assert "steps" in res.detail.decode(), res.detail.decode()


def test_step_budget_running_out_fails_a_batch(cuda):
    work = [scenes.box_room(seed=k, size=48) for k in range(3)]
    with cuda.CudaBatch(0) as batch:
        res = batch.set_scenes(work)
        assert all(x.status == abi.PASS for x in res)
        st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                                  max_bounces=4, sample_index=0)
        _, _, total = batch.render([s.frame(st, 1, read_back=False) for s in work])
        cuda.check(total, "batch with the default budget")
