"""CPU: the oracle's glTF PBR closure in the reference's white furnace
(renderer.path.gltf_furnace, GltfFurnaceFailure, adapters/headless/
main.cpp:1632-1770): a white glTF PBR plane under a white constant
environment, seen orthographically at view cosines 1, 0.5 and 0.125, under
BSDF sampling and NEE/MIS, 32 spp: each image's mean (over pixels whose
samples all hit) is the closure's directional albedo, which must be 1
within five standard errors and the albedo tables' bound of 8e-3 — for
dielectrics and metals at two roughnesses, a clearcoat, a rough half-weight
clearcoat, a white sheen, full and half thin transmission, and every
extension together."""

import numpy as np
import pytest

from hydra_lotus_b200 import abi, scenes

SAMPLES = 32
# lotus-bsdf-test's bound on the furnace of a compensated lobe under two
# layers (the reference's kTableError).
TABLE_ERROR = 8.0e-3


def furnace_check(image):
    """The reference's acceptance: |mean - 1| <= 5 SE + 8e-3 per channel."""
    hit = image[..., 3] == 1.0
    assert hit.sum() >= 2, "no pixel's samples all hit"
    v = image[hit][:, :3].astype(np.float64)
    assert np.all(np.isfinite(v)), "non-finite radiance in the furnace"
    mean = v.mean(axis=0)
    se = v.std(axis=0, ddof=1) / np.sqrt(v.shape[0])
    tol = 5.0 * se + TABLE_ERROR
    return mean, tol, bool(np.all(np.abs(mean - 1.0) <= tol))


@pytest.mark.parametrize("light_sampling", [abi.LIGHT_SAMPLING_BSDF, abi.LIGHT_SAMPLING_MIS])
@pytest.mark.parametrize("cos_view", [1.0, 0.5, 0.125])
@pytest.mark.parametrize("plane", sorted(scenes.GLTF_FURNACE_PLANES))
def test_oracle_gltf_furnace(oracle_lib, plane, cos_view, light_sampling):
    scene = scenes.gltf_furnace(plane, cos_view, size=48)
    st = abi.default_settings(integrator=abi.INTEGRATOR_REFERENCE, light_sampling=light_sampling,
                              max_bounces=64, sample_index=0)
    sums, _ = oracle_lib.OracleScene(scene).accumulate(scene.frame(st, SAMPLES), 0, SAMPLES)
    image = (sums / SAMPLES).astype(np.float32)
    mean, tol, ok = furnace_check(image)
    assert ok, (plane, cos_view, mean, tol)
