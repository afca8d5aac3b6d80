"""GPU: the diagnostic outputs of RenderScene (SceneOutput Barycentrics,
ShadingNormal, Albedo, RoughnessMetallic; path_trace.slang's surface pass)
through the C ABI. Each pixel centre's closest hit, traced with the fixed
coverage sequence, is the hit the oracle's WriteTemporalSurface finds for
the same pixel: the hit mask equals the oracle's, the albedo and shading
normal equal its packed ones within their packing, roughness and metallic
are the hit material's, barycentric weights sum to one; a diagnostic call
leaves the radiance accumulation as it was."""

import numpy as np
import pytest

from hydra_lotus_b200 import abi, scenes
from oracle import oracle

pytestmark = pytest.mark.gpu

IDENTITY = [1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0]
CLEAR = (0.25, 0.5, 0.75, 0.0)


def small_sphere_field():
    s = scenes.sphere_field(seed=3, width=80, height=56, prototypes=6, grid=10, spacing=2.0,
                            spheres=40, emitters=6, sky_size=(128, 64))
    extent = 10 * 2.0
    s.view = scenes.look_at((0.24 * extent, 0.11 * extent, 0.24 * extent), (0.0, 0.0, 0.0))
    return s


def room():
    return scenes.box_room_wide(seed=0, width=64, height=48)


def unpack_albedo(a):
    return np.stack([(a & 0xFF), (a >> 8) & 0xFF, (a >> 16) & 0xFF], -1).astype(np.float32) / 255.0


def unpack_normal(v):
    ex = np.maximum(((v & 0xFFFF).astype(np.uint16).view(np.int16)).astype(np.float32) / 32767.0, -1.0)
    ey = np.maximum(((v >> 16).astype(np.uint16).view(np.int16)).astype(np.float32) / 32767.0, -1.0)
    n = np.stack([ex, ey, 1.0 - np.abs(ex) - np.abs(ey)], -1)
    fold = np.maximum(-n[..., 2], 0.0)
    n[..., 0] += np.where(n[..., 0] >= 0.0, -fold, fold)
    n[..., 1] += np.where(n[..., 1] >= 0.0, -fold, fold)
    return n / np.linalg.norm(n, axis=-1, keepdims=True)


def diagnostic(r, scene, output):
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=4, sample_index=0, output=output)
    res, img = r.render_scene(scene.frame(st, frame_count=1, clear_color=CLEAR))
    assert res.status == abi.PASS, res.detail
    assert res.samples_per_pixel == 0
    return img


@pytest.mark.parametrize("make", [room, small_sphere_field])
def test_diagnostics_match_the_oracle_surface(cuda, make):
    scene = make()
    frame = scene.frame(abi.default_settings(), frame_count=1)
    want = oracle.OracleTemporalScene(scene).temporal_surface(frame, oracle.oracle_temporal(
        abi.temporal_desc(frame, scene.view)))
    hit = (want["flags"] & 1) != 0
    assert hit.any()
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        bary = diagnostic(r, scene, abi.OUTPUT_BARYCENTRICS)
        normal = diagnostic(r, scene, abi.OUTPUT_SHADING_NORMAL)
        albedo = diagnostic(r, scene, abi.OUTPUT_ALBEDO)
        rm = diagnostic(r, scene, abi.OUTPUT_ROUGHNESS_METALLIC)
    clear = np.array(CLEAR, dtype=np.float32)
    for img in (bary, normal, albedo, rm):
        assert np.array_equal(np.all(img == clear, axis=-1), ~hit)
        assert np.all(img[hit][:, 3] == 1.0)
    w = bary[hit][:, :3]
    assert np.all(w >= -1e-6) and np.all(np.abs(w.sum(-1) - 1.0) <= 1e-5)
    np.testing.assert_allclose(albedo[hit][:, :3], unpack_albedo(want["albedo"][hit]), atol=0.5 / 255 + 1e-6)
    n = normal[hit][:, :3]
    np.testing.assert_allclose(np.linalg.norm(n, axis=-1), 1.0, atol=1e-5)
    np.testing.assert_allclose(n, unpack_normal(want["shading_normal"][hit]), atol=2e-4)
    mats = scene.materials
    slots = want["material_id"][hit].astype(np.int64)
    np.testing.assert_array_equal(rm[hit][:, 0], np.array([mats[k].roughness for k in slots], dtype=np.float32))
    np.testing.assert_array_equal(rm[hit][:, 1], np.array([mats[k].metallic for k in slots], dtype=np.float32))


def test_diagnostic_leaves_the_accumulation(cuda):
    scene = scenes.box_room(seed=0, size=32)
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=4, sample_index=9)
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        cuda.check(r.render_scene(scene.frame(st, frame_count=2))[0], "radiance")
        diagnostic(r, scene, abi.OUTPUT_ALBEDO)
        res, split = r.render_scene(scene.frame(st, frame_count=2))
        cuda.check(res, "radiance")
        assert res.samples_per_pixel == 4
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        res, whole = r.render_scene(scene.frame(st, frame_count=4))
        cuda.check(res, "radiance")
    assert np.array_equal(split, whole)


def test_diagnostics_outside_render_scene_fail(cuda):
    scene = scenes.box_room(seed=0, size=16)
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT,
                                  light_sampling=abi.LIGHT_SAMPLING_RESTIR_INITIAL, output=abi.OUTPUT_ALBEDO)
        res, _ = r.render_temporal(abi.temporal_desc(scene.frame(st, frame_count=1), IDENTITY))
        assert res.status == abi.FAIL
        st.output = 7
        assert r.render_scene(scene.frame(st, frame_count=1))[0].status == abi.FAIL
        cuda.check(r.render_scene(scene.frame(abi.default_settings(), frame_count=1))[0], "render after rejects")


def depth_plane_scene(size=48, half=10.0):
    """One quad at z = -2 facing the camera at z = +3 (the Cornell camera's
    view): every pixel centre hits it at view depth 5 when it spans the
    view (`half` large), a central square of pixels when it is small."""
    s = scenes.Scene("depth-plane")
    q = s.add_geometry(*scenes.quad([[-half, -half, -2.0], [half, -half, -2.0], [half, half, -2.0],
                                     [-half, half, -2.0]]))
    s.add_instance(q, s.add_material(scenes.preview_material((0.5, 0.5, 0.5))))
    s.world_to_clip = scenes.cornell_camera()
    s.width = s.height = size
    return s


def plane_depth(world_to_clip):
    """The Vulkan window depth of a point at view depth 5 on the axis: the
    OpenGL clip z and w of the Cornell projection, z mapped to (z + w) / 2."""
    m = np.asarray(world_to_clip, dtype=np.float64)
    p = np.array([0.0, 0.0, -2.0, 1.0])
    clip = np.array([sum(m[c * 4 + r] * p[c] for c in range(4)) for r in range(4)])
    return 0.5 * (clip[2] + clip[3]) / clip[3]


def test_depth_product_of_a_plane(cuda):
    scene = depth_plane_scene()
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, max_bounces=2)
    want = plane_depth(scene.world_to_clip)
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        res, _ = r.render_scene(scene.frame(st, 2, flags=abi.FRAME_DEPTH))
        cuda.check(res, "render_scene")
        depth = r.read_depth(scene.height, scene.width)
    print(want, depth.min(), depth.max())
    assert 0.0 < want < 1.0
    np.testing.assert_allclose(depth, want, rtol=1e-5)


def test_depth_product_clears_and_keeps(cuda):
    """Pixels whose centre misses keep the clear depth; with DEPTH_KEEP they
    keep the preceding frame's; a frame without DEPTH has no depth product;
    the hit pixels are the diagnostic pass's."""
    scene = depth_plane_scene(half=0.5)
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, max_bounces=2)
    want = plane_depth(scene.world_to_clip)
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        cuda.check(r.render_scene(scene.frame(st, 1, flags=abi.FRAME_DEPTH, clear_depth=0.75))[0], "first")
        first = r.read_depth(scene.height, scene.width)
        hit = first != np.float32(0.75)
        assert 0 < hit.sum() < hit.size
        np.testing.assert_allclose(first[hit], want, rtol=1e-5)
        cuda.check(r.render_scene(scene.frame(st, 1, flags=abi.FRAME_DEPTH | abi.FRAME_DEPTH_KEEP,
                                              clear_depth=0.25))[0], "keep")
        kept = r.read_depth(scene.height, scene.width)
        assert np.array_equal(kept, first)
        cuda.check(r.render_scene(scene.frame(st, 1, flags=abi.FRAME_DEPTH, clear_depth=0.25))[0], "clear")
        cleared = r.read_depth(scene.height, scene.width)
        assert np.array_equal(cleared[~hit], np.full((~hit).sum(), 0.25, np.float32))
        dst = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, output=abi.OUTPUT_BARYCENTRICS)
        res, bary = r.render_scene(scene.frame(dst, 1, clear_color=CLEAR))
        cuda.check(res, "barycentrics")
        assert np.array_equal(bary[..., 3] == 1.0, hit)
        cuda.check(r.render_scene(scene.frame(st, 1))[0], "no depth")
        with pytest.raises(cuda.RendererError):
            r.read_depth(scene.height, scene.width)
