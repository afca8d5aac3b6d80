"""CPU: the C++ Lotus::OffscreenRenderer adapter (hydra_lotus_b200/host)
compiles against the reference's headers and links with nothing but the
CUDA library; without a GPU, creating it reports Skip, as the reference's
CreateOffscreenRenderer does without a capable device."""

import os

import pytest

from hydra_lotus_b200 import abi, build, renderer, scenes

import adapter_scene


def harness():
    path = build.build_host()
    if path is None:
        pytest.skip("the adapter builds only where the reference's headers are present")
    return path


def test_adapter_builds_and_links_against_the_c_abi_only():
    path = harness()
    assert os.path.exists(path)


def test_adapter_without_gpu_reports_skip(tmp_path):
    harness()
    status, _ = renderer.capability(0)
    if status == abi.PASS:
        pytest.skip("a usable GPU is present")
    scene = scenes.box_room(seed=0, size=16)
    st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT, max_bounces=2)
    code, evidence, _ = adapter_scene.run(str(tmp_path), scene, st, 1)
    assert code == 77, evidence
    assert evidence.get("create") == "skip"
