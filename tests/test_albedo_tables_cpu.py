"""The composed closure's directional albedo tables (csrc/albedo_tables.inc,
written by csrc/albedo_tables_gen.cpp) against the reference's own tables
(backend/vulkan/bsdf-albedo-tables.inc of hydra-lotus, sampled into
tests/golden/albedo_tables_reference.npz), and against a fresh cubature of
the lobes at the nodes and at cell centres."""

import os
import subprocess

import numpy as np
import pytest

from hydra_lotus_b200 import build

HERE = os.path.dirname(os.path.abspath(__file__))
INC = os.path.join(os.path.dirname(HERE), "hydra_lotus_b200", "csrc", "albedo_tables.inc")

# albedo.slang's layout: E1 and Eschlick 32x32, the dielectric's three
# sheets of 16 indices x 48 x 32, the sheen 32x32.
PARTS = {"E1": (0, 1024), "Eschlick": (1024, 2048), "entering": (2048, 2048 + 24576),
         "leaving": (2048 + 24576, 2048 + 2 * 24576), "thin": (2048 + 2 * 24576, 2048 + 3 * 24576),
         "sheen": (2048 + 3 * 24576, 76800)}


def read_inc(path):
    values = []
    with open(path) as f:
        for line in f:
            if not line.startswith("//"):
                values += [float(v) for v in line.strip().split(",") if v.strip()]
    return np.array(values, dtype=np.float64)


def test_layout_size():
    assert read_inc(INC).size == 76800


def test_tables_match_reference_tables():
    ours = read_inc(INC)
    ref = np.load(os.path.join(HERE, "golden", "albedo_tables_reference.npz"))
    assert int(ref["size"]) == ours.size
    index = ref["index"].astype(np.int64)
    diff = np.abs(ours[index] - ref["value"]) / np.maximum(1.0, np.abs(ref["value"]))
    for name, (lo, hi) in PARTS.items():
        part = diff[(index >= lo) & (index < hi)]
        # Both are quadratures of the same lobes to about 1e-5. The largest
        # differences (up to 1.7e-3) sit at normal incidence for small
        # alpha, where GGX's tail beyond 45 degrees (alpha^2 / (1 +
        # alpha^2) of the visible normals) reflects below the horizon: this
        # table keeps that loss, evaluated in double precision.
        assert part.max() < 2.5e-3, (name, part.max())
        assert part.mean() < 5e-5, (name, part.mean())
        assert np.percentile(part, 99) < 1e-3, (name, np.percentile(part, 99))


def test_fresh_cubature_reproduces_nodes():
    tool = build.build_table_tool()
    out = subprocess.run([tool, "--check", INC, "1499"], check=True, capture_output=True,
                         text=True, timeout=600).stdout
    rows = [line.split() for line in out.strip().splitlines()]
    assert len(rows) == 6, out
    for row in rows:
        node_error = float(row[row.index("node") + 2])
        centre_error = float(row[row.index("centre") + 2])
        assert node_error < 1e-6, out
        # The splines' error between nodes, bounded by the grid's spacing.
        assert centre_error < 1e-2, out


@pytest.mark.parametrize("fn", ["E1", "sheen"])
def test_tables_are_finite_and_bounded(fn):
    data = read_inc(INC)
    lo, hi = PARTS[fn]
    part = data[lo:hi]
    assert np.all(np.isfinite(part))
    assert part.min() >= 0.0
    # E1 is at most 1; the sheen's fitted lobe reflects more than it
    # receives toward grazing directions at small roughness.
    assert part.max() <= (1.0 + 1e-6 if fn == "E1" else 8.0)
