import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and the CUDA library")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import build, oracle
    build.build()
    return oracle


@pytest.fixture(scope="session")
def cuda():
    """The CUDA library on an sm_100 device. GPU tests fail loudly (never
    fall back) when the library is missing or the device is not usable."""
    from hydra_lotus_b200 import abi, renderer
    status, detail = renderer.capability(0)
    assert status == abi.PASS, f"no usable sm_100 device: {detail}"
    return renderer


def load_golden(name):
    import numpy as np
    g = np.load(os.path.join(ROOT, "tests", "golden", name))
    return {"mean": g["mean"], "variance": g["variance"], "samples": int(g["samples"])}


@pytest.fixture(scope="session")
def golden():
    """The reference's Cornell box golden images (1024 spp)."""
    return load_golden("cornell_box.npz")


@pytest.fixture(scope="session")
def golden_materials():
    """The reference's material-basics-v1 golden images (4096 spp)."""
    return load_golden("material_basics_v1.npz")


@pytest.fixture(scope="session")
def golden_alpha():
    """The reference's material-alpha-v1 golden images (4096 spp)."""
    return load_golden("material_alpha_v1.npz")


@pytest.fixture(scope="session")
def golden_normals():
    """The reference's material-normals-v1 golden images (4096 spp)."""
    return load_golden("material_normals_v1.npz")


@pytest.fixture(scope="session")
def golden_fixtures():
    """The reference's material-transmission-v1, material-transforms-v1,
    material-emission-v1, material-gltf-v1, material-gltf-extensions-v1,
    material-primvars-v1, material-subsets-v1, material-mtlx-v1 and
    material-graphs-v1 golden images (4096 spp), by fixture name."""
    return {name: load_golden(f"material_{name}_v1.npz")
            for name in ("transmission", "transforms", "emission", "gltf", "gltf_extensions", "primvars",
                         "subsets", "mtlx", "graphs")}


@pytest.fixture(scope="session")
def golden_textures():
    """The reference's material-textures-v1 golden images (4096 spp)."""
    return load_golden("material_textures_v1.npz")
