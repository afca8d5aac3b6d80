"""GPU: a batch of scenes rendered as one wavefront gives every scene the
image lotus_cuda_render gives it alone, bit for bit, over two calls that
continue the accumulation, whatever the tuner's launch shape (refill,
blocks per SM, rounds before the tail, camera order)."""

import numpy as np
import pytest

from hydra_lotus_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def batch_scenes():
    a = scenes.box_room(seed=0, size=64)
    b = scenes.sphere_field(seed=3, width=96, height=64, prototypes=6, grid=10, spacing=2.0, spheres=40,
                            emitters=6, sky_size=(128, 64))
    c = scenes.box_room(seed=5, size=48)
    c.width, c.height = 40, 56
    return [a, b, c]


def settings(k, sample_index):
    return abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT,
                                light_sampling=abi.LIGHT_SAMPLING_MIS if k != 2 else abi.LIGHT_SAMPLING_BSDF,
                                max_bounces=6 if k != 1 else 8, sample_index=sample_index)


TUNINGS = [
    (0, 0, 0, 0),
    (24, 4, 5, abi.CAMERA_TILE_8X4),
    (0, 0, 9, abi.CAMERA_TILE_4X8),
    (16, 0, 3, abi.CAMERA_TILE_16X2),  # 16x2 does not divide 40: rows
]


@pytest.mark.parametrize("tuning", TUNINGS, ids=lambda t: "/".join(map(str, t)))
def test_batch_matches_single_renders(cuda, tuning):
    scs = batch_scenes()
    with cuda.CudaBatch(0) as batch:
        batch.set_tuning(*tuning)
        res = batch.set_scenes(scs)
        assert all(r.status == abi.PASS for r in res), [r.detail for r in res]
        frames = [s.frame(settings(k, 100 + k), frame_count=2) for k, s in enumerate(scs)]
        results, colors, total = batch.render(frames)
        cuda.check(total, "batch render")
        results, colors, total = batch.render(frames)
        cuda.check(total, "batch render")
        assert all(r.samples_per_pixel == 4 for r in results)
        assert total.camera_rays == 2 * sum(s.width * s.height for s in scs)
    with cuda.CudaOffscreenRenderer(0) as r:
        for k, s in enumerate(scs):
            cuda.check(r.update_scene(s), "update_scene")
            res, want = r.render_scene(s.frame(settings(k, 100 + k), frame_count=4))
            cuda.check(res, "render_scene")
            assert np.array_equal(colors[k], want), f"scene {k}: {np.count_nonzero(colors[k] != want)} values differ"


def test_batch_rejects_mismatched_frames(cuda):
    scs = batch_scenes()[:2]
    with cuda.CudaBatch(0) as batch:
        batch.set_scenes(scs)
        frames = [scs[0].frame(settings(0, 0), frame_count=1), scs[1].frame(settings(1, 0), frame_count=2)]
        _, _, total = batch.render(frames)
        assert total.status == abi.FAIL
        frames = [s.frame(abi.default_settings(integrator=abi.INTEGRATOR_REFERENCE), frame_count=1) for s in scs]
        _, _, total = batch.render(frames)
        assert total.status == abi.FAIL
        # The batch stays usable after rejected frames.
        frames = [s.frame(settings(k, 0), frame_count=1) for k, s in enumerate(scs)]
        _, _, total = batch.render(frames)
        cuda.check(total, "batch render")
