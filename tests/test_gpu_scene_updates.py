"""GPU: incremental scene updates through the C ABI. An instance-only
update (lotus_cuda_update_instances) and a point edit of one geometry
(lotus_cuda_update_geometry) give the images a full UpdateScene of the
edited scene gives, bit for bit, for the binned-SAH and LBVH builders and
with the light table changing; invalid edits Fail without poisoning the
renderer (the reference's UpdateScene conventions, vulkan_backend.hpp:
812-815)."""

import numpy as np
import pytest

from hydra_lotus_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def render(r, scene, spp=4):
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=5, sample_index=7)
    res, img = r.render_scene(scene.frame(st, frame_count=spp))
    return res, img


def fresh_image(cuda, scene):
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        res, img = render(r, scene)
        cuda.check(res, "render")
        return img


def same(a, b):
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


def moved_room():
    s = scenes.box_room(seed=0, size=64)
    for i, (m, g, mat) in enumerate(list(s.instances)):
        m2 = np.array(m, dtype=np.float32).copy()
        if i >= 5:  # the light and the boxes move; the walls stay
            m2[12] += 0.03 * (i - 4)
            m2[14] -= 0.02
        s.set_instance(i, m2, material=mat if i != 6 else 0)
    return s


def test_instance_update_matches_full_update(cuda):
    before = scenes.box_room(seed=0, size=64)
    after = moved_room()
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(before), "update_scene")
        cuda.check(render(r, before)[0], "render")
        res = r.update_instances(after)
        cuda.check(res, "update_instances")
        assert res.instance_count == len(after.instances) and res.build_gpu_ms > 0.0
        out, img = render(r, after)
        cuda.check(out, "render")
        # The accumulation restarted: the frame holds only the new samples.
        assert out.samples_per_pixel == 4
    assert same(img, fresh_image(cuda, after))


def displaced(scene, geometry, amount):
    p, t, n = scene.geometries[geometry]
    q = p.copy()
    q[:, 1] += amount * p[:, 0]
    normals = scenes.corner_normals(q, t) if n is not None else None
    scene.set_positions(geometry, q, normals)
    return scene


@pytest.mark.parametrize("make,geometry", [
    (lambda: scenes.big_mesh(seed=1, size=64, subdivisions=5), 0),   # 20,480 triangles: binned SAH
    (lambda: scenes.grid_mesh(quads=200, size=64), 0),              # 80,000 triangles: LBVH
])
def test_point_edit_matches_full_update(cuda, make, geometry):
    before = make()
    after = displaced(make(), geometry, 0.05)
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(before), "update_scene")
        cuda.check(render(r, before)[0], "render")
        res = r.update_geometry(after, geometry)
        cuda.check(res, "update_geometry")
        out, img = render(r, after)
        cuda.check(out, "render")
    assert same(img, fresh_image(cuda, after))


def test_invalid_edits_fail_without_poisoning(cuda):
    scene = scenes.box_room(seed=0, size=32)
    with cuda.CudaOffscreenRenderer(0) as r:
        assert r.update_instances(scene).status == abi.FAIL  # nothing resident yet
        cuda.check(r.update_scene(scene), "update_scene")
        bad = scenes.box_room(seed=0, size=32)
        m, g, mat = bad.instances[0]
        bad.instances[0] = (m, len(bad.geometries) + 3, mat)
        bad._desc = None
        assert r.update_instances(bad).status == abi.FAIL
        p, t, n = scene.geometries[0]
        short = scenes.box_room(seed=0, size=32)
        short.geometries[0] = (p[:-1].copy(), t, n)
        short._desc = None
        assert r.update_geometry(short, 0).status == abi.FAIL
        extra = scenes.box_room(seed=0, size=32)
        extra.add_geometry(*scenes.quad([[0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1]]))
        assert r.update_geometry(extra, len(extra.geometries) - 1).status == abi.FAIL
        cuda.check(render(r, scene)[0], "render after rejected edits")


def test_scene_readback_equals_the_scene(cuda):
    """ReadBackScene (lotus_cuda_read_scene): the device's geometry arrays,
    instance records and material table decode to the scene that was
    uploaded, after an instance edit too."""
    from hydra_lotus_b200 import abi
    scene = scenes.material_basics(size=32)
    scene.environment_constant = (0.5, 0.25, 0.125)
    with cuda.CudaOffscreenRenderer(0) as r:
        cuda.check(r.update_scene(scene), "update_scene")
        for g, (p, t, n) in enumerate(scene.geometries):
            assert np.array_equal(r.read_scene(abi.SCENE_POSITIONS, g), p)
            assert np.array_equal(r.read_scene(abi.SCENE_TRIANGLES, g), t)
            normals = r.read_scene(abi.SCENE_NORMALS, g)
            assert (n is None and normals.size == 0) or np.array_equal(normals, n)
        insts = r.read_scene(abi.SCENE_INSTANCES)
        assert len(insts) == len(scene.instances)
        for got, (m, g, mat) in zip(insts, scene.instances):
            assert np.array_equal(np.array(got.world_from_object[:], np.float32), m)
            assert (got.geometry, got.material) == (g, mat)
        mats = r.read_scene(abi.SCENE_MATERIALS)
        assert len(mats) == len(scene.materials)
        for got, want in zip(mats, scene.materials):
            assert bytes(got) == bytes(want)
        assert np.array_equal(r.read_scene(abi.SCENE_ENVIRONMENT), np.array([0.5, 0.25, 0.125], np.float32))
        m = np.array(scene.instances[3][0], dtype=np.float32)
        m[12] += 0.25
        scene.set_instance(3, m, material=1)
        cuda.check(r.update_instances(scene), "update_instances")
        got = r.read_scene(abi.SCENE_INSTANCES)[3]
        assert np.array_equal(np.array(got.world_from_object[:], np.float32), m)
        assert got.material == 1
