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


@pytest.mark.parametrize("integrator", [abi.INTEGRATOR_WAVEFRONT, abi.INTEGRATOR_REFERENCE])
def test_static_entry_matches_allocating_entry(cuda, integrator):
    import torch

    scene = scenes.box_room(seed=0, size=128)
    st = abi.default_settings(integrator=integrator, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=6, sample_index=21)
    frame = scene.frame(st, frame_count=4)
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
