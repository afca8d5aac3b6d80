"""The reference's own CPU code for the temporal and reservoir paths,
built from its sources into oracle/_ref: its unit tests pass, and the
bridge the GPU tests use reproduces its known answers."""

import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from oracle import build_ref, ref

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref is not built")


@pytest.mark.parametrize("name", build_ref.TESTS)
def test_reference_unit_tests_pass(name):
    exe = os.path.join(build_ref.OUT, name)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "PASS" in out.stdout or "passed" in out.stdout


def reservoir(sample=0xFFFFFFFF, weight_sum=0.0, target=0.0, count=0):
    return np.array([(sample, weight_sum, target, count)],
                    dtype=[("s", "<u4"), ("w", "<f4"), ("t", "<f4"), ("m", "<u4")])


def test_bridge_stream_and_merge():
    L = ref.lib()
    sel = C.c_int()
    r = reservoir()
    assert L.ref_stream_candidate(r.ctypes.data, 3, 2.0, 0.5, 0.9, C.byref(sel)) == 0
    # The first positive weight is selected with probability one.
    assert sel.value == 1 and r["s"][0] == 3 and r["w"][0] == pytest.approx(4.0) and r["m"][0] == 1
    assert L.ref_stream_candidate(r.ctypes.data, 5, 0.0, 0.5, 0.0, C.byref(sel)) == 0
    assert sel.value == 0 and r["m"][0] == 2
    # Invalid input is rejected without changing the reservoir.
    before = r.copy()
    assert L.ref_stream_candidate(r.ctypes.data, 5, -1.0, 0.5, 0.5, C.byref(sel)) == 1
    assert np.array_equal(r, before)
    status = C.c_int()
    assert L.ref_normalization(r.ctypes.data, C.byref(status)) == pytest.approx(4.0 / 2 / 2.0)
    d = reservoir()
    src = reservoir(7, 4.0, 2.0, 10)
    assert L.ref_merge_reevaluated(d.ctypes.data, src.ctypes.data, 0.2, 3.0, 4, 0.5, C.byref(sel)) == 0
    assert sel.value == 1 and d["m"][0] == 4 and d["w"][0] == pytest.approx(3.0 * 0.2 * 4)
