"""CPU: the CUDA library loads without a GPU, exports every entry point
include/lotus_cuda.h declares, and its structs match the Python mirrors.
No compute call is made."""

import os
import re

from hydra_lotus_b200 import abi, renderer

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "lotus_cuda.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lotus_cuda_\w+)\s*\(", text)))


def test_library_exports_every_declared_function():
    names = declared_functions()
    assert len(names) >= 20
    lib = renderer.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_struct_sizes():
    lib = renderer.lib()
    assert lib.lotus_cuda_abi_version() == abi.ABI_VERSION == 10
    sizes = abi.check_struct_sizes(lib)
    assert len(sizes) == len(abi.STRUCTS)


def test_capability_without_gpu_is_skip_or_pass():
    status, detail = renderer.capability(0)
    assert status in (abi.PASS, abi.SKIP), detail
