"""CPU: the oracle against the reference's own golden Cornell images
(validation/reference/cornell-box-{mean,variance}.pfm, 1024 spp, written by
the reference's GPU renderer; fixtures in tests/golden) with the
reference's DES-Q5 comparison, and the red-wall negative control."""

import numpy as np
import pytest

from hydra_lotus_b200 import abi, metrics, scenes

SPP = 256


def oracle_image(oracle_lib, scene, light_sampling):
    st = abi.default_settings(integrator=abi.INTEGRATOR_REFERENCE, light_sampling=light_sampling,
                              max_bounces=64, sample_index=1 << 20)
    frame = scene.frame(st, SPP)
    sums, _ = oracle_lib.OracleScene(scene).accumulate(frame, 1 << 20, SPP)
    return (sums / SPP).astype(np.float32)


@pytest.mark.parametrize("light_sampling", [abi.LIGHT_SAMPLING_BSDF, abi.LIGHT_SAMPLING_MIS])
def test_oracle_matches_reference_golden(oracle_lib, golden, light_sampling):
    img = oracle_image(oracle_lib, scenes.cornell_reference(), light_sampling)
    c = metrics.compare(img, SPP, golden["mean"], golden["variance"], golden["samples"])
    assert c.ok, c


def test_oracle_negative_control_rejected(oracle_lib, golden):
    img = oracle_image(oracle_lib, scenes.cornell_reference(red_scale=1.1), abi.LIGHT_SAMPLING_BSDF)
    c = metrics.compare(img, SPP, golden["mean"], golden["variance"], golden["samples"])
    assert not c.ok, c
