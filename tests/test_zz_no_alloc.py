"""The allocation-free render entry point (lotus_cuda_render_static).

Hosts that cannot call cudaMalloc when they want a frame (a delegate inside
another framework's frame loop that owns every allocation, or a real-time
caller that must not block in the allocator) render through this entry
point, whose scratch is a fixed device array inside the library. This file
checks, through the C ABI, that it produces what the allocating entry point
lotus_cuda_render produces for the same frame, on two calls in a row (the
second reuses the scratch the first left behind), and that it rejects
targets larger than its scratch. It is collected last so that a run that
stops at the first failure has run every other test before it.
"""

import numpy as np
import pytest

from hydra_lotus_b200 import abi, scenes

from parity import PathParity

pytestmark = pytest.mark.gpu


CASES = {
    # The box room at 6 bounces: the wavefront's rounds only.
    "box_room": (lambda: scenes.box_room(seed=0, size=128), 6, None),
    # Analytic lights at 12 bounces: the paths still queued after the
    # rounds go to the tail kernel.
    "lit_room": (lambda: scenes.lit_room(seed=1, size=96), 12, None),
    # A data window smaller than the target: the pixels outside it keep
    # the clear colour.
    "data_window": (lambda: scenes.box_room(seed=3, size=128), 6, (16, 24, 80, 64)),
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("integrator", [abi.INTEGRATOR_WAVEFRONT, abi.INTEGRATOR_REFERENCE])
def test_static_entry_matches_allocating_entry(cuda, integrator, case):
    import torch

    make, bounces, window = CASES[case]
    scene = make()
    st = abi.default_settings(integrator=integrator, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=bounces, sample_index=21)
    kw = {"data_window": window, "clear_color": (0.25, 0.5, 0.75, 1.0)} if window else {}
    frame = scene.frame(st, frame_count=4, **kw)
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        res, want = r.render_scene(frame)
        cuda.check(res, "render_scene")
        out = torch.full((scene.height, scene.width, 4), float("nan"), dtype=torch.float32,
                         device="cuda")
        for call in range(2):
            got_res = r.render_static(frame, out.data_ptr())
            cuda.check(got_res, f"render_static call {call}")
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            p = PathParity(got, want)
            print(call, p)
            assert p.finite
            assert p.within == 1.0, p
            assert np.array_equal(got, want), f"{np.count_nonzero(got != want)} values differ"
            assert got_res.samples_per_pixel == 4
            assert (got_res.camera_rays, got_res.extension_rays, got_res.shadow_rays) == \
                (res.camera_rays, res.extension_rays, res.shadow_rays)
            out.fill_(float("nan"))


def test_static_entry_rejects_oversized_target(cuda):
    import torch

    scene = scenes.box_room(seed=0, size=257)
    scene.height = 256
    frame = scene.frame(abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, max_bounces=4))
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        out = torch.zeros((256, 257, 4), dtype=torch.float32, device="cuda")
        res = r.render_static(frame, out.data_ptr())
        assert res.status == abi.FAIL
        assert str(abi.STATIC_MAX_PIXELS) in res.detail.decode()
        # A failed call leaves the renderer usable.
        ok, _ = r.render_scene(frame)
        cuda.check(ok, "render_scene after a rejected static call")


def test_static_entry_caps_samples_and_refuses_the_cache(cuda):
    import torch

    scene = scenes.box_room(seed=0, size=64)
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=6, sample_index=5)
    st.max_samples = 3
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        res, want = r.render_scene(scene.frame(st, frame_count=8))
        cuda.check(res, "render_scene")
        assert res.samples_per_pixel == 3
        out = torch.zeros((64, 64, 4), dtype=torch.float32, device="cuda")
        got_res = r.render_static(scene.frame(st, frame_count=8), out.data_ptr())
        cuda.check(got_res, "render_static")
        assert got_res.samples_per_pixel == 3
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), want)
        r.configure_cache(enable=True, seed=1)
        refused = r.render_static(scene.frame(st, frame_count=1), out.data_ptr())
        assert refused.status == abi.FAIL
        assert "radiance cache" in refused.detail.decode()
