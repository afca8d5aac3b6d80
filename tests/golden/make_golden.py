"""Writes the golden fixtures under tests/golden/ from the reference tree.

The reference tree is found at $LOTUS_REFERENCE, else at ../reference beside
this checkout. The fixtures it writes are committed, so tests never read the
reference at run time. Each is the reference's own golden image pair
(validation/reference/<stem>-{mean,variance}.pfm of hydra-lotus v0.9.0),
written by its GPU renderer with BSDF sampling, 64 bounces, from sample
index 0 (docs/reference/SCENE.md, "Deterministic mode"), stored as float32
arrays with rows from the top (the PFMs hold rows from the bottom,
little-endian; ReadPfm, adapters/common/reference.cpp:100-131):

- cornell_box.npz: the Cornell box fixture (adapters/common/reference.cpp:
  221-279) at 128x128, 1024 samples per pixel.
- material_basics_v1.npz: the material-basics-v1 fixture
  (adapters/common/material_fixtures.cpp:161-211: a 4x4 grid of
  UsdPreviewSurface balls under a constant dome and a rect light) at
  128x128, 4096 samples per pixel (kMaterialReferenceSamples,
  adapters/headless/main.cpp).
- material_textures_v1.npz: the material-textures-v1 fixture
  (adapters/common/material_fixtures.cpp:390-500: 25 texture-mapped cards
  under the same studio) at 160x160, 4096 samples per pixel.
- material_alpha_v1.npz: the material-alpha-v1 fixture
  (adapters/common/material_fixtures.cpp:1056-1200: constant and texture
  coverage on 24 cards and a coarse sphere) at 160x160, 4096 samples per
  pixel.
- material_normals_v1.npz: the material-normals-v1 fixture
  (adapters/common/material_fixtures.cpp:692-828: corner normals of every
  kind and tangent-space normal maps on coarse spheres and cards) at
  160x160, 4096 samples per pixel.
- material_transmission_v1.npz and material_transforms_v1.npz: the
  material-transmission-v1 and material-transforms-v1 fixtures
  (adapters/common/material_fixtures.cpp:1588-1671, 1749-1825: solid and
  thin-walled transmission; st transforms on every textured input) at
  160x160, 4096 samples per pixel.
- material_emission_v1.npz: the material-emission-v1 fixture
  (adapters/common/material_fixtures.cpp:875-1009: constant emitters and
  emission maps, float images included) at 160x160, 4096 samples per
  pixel.
- material_primvars_v1.npz: the material-primvars-v1 fixture
  (adapters/common/material_fixtures.cpp:1941-2031: colour sets read as a
  UsdPreviewSurface base colour, displayColor and displayOpacity) at
  160x160, 4096 samples per pixel.
- material_subsets_v1.npz: the material-subsets-v1 fixture
  (adapters/common/material_fixtures.cpp:1840-1939: GeomSubset bindings as
  extraction splits them) at 160x160, 4096 samples per pixel.
- material_mtlx_v1.npz: the material-mtlx-v1 fixture
  (adapters/common/material_fixtures.cpp:1247-1382: Standard Surface
  networks as translated) at 160x160, 4096 samples per pixel.
- material_graphs_v1.npz: the material-graphs-v1 fixture
  (adapters/common/material_fixtures.cpp:1440-1564: MaterialX node graphs
  as translated) at 160x160, 4096 samples per pixel.
- material_gltf_v1.npz and material_gltf_extensions_v1.npz: the
  material-gltf-v1 and material-gltf-extensions-v1 fixtures
  (adapters/common/material_fixtures.cpp:2035-2300: MaterialX's glTF PBR
  surface, its core and its extensions) at 160x160, 4096 samples per
  pixel.

It also writes albedo_tables_reference.npz: every 7th value of the
reference's directional albedo tables (backend/vulkan/
bsdf-albedo-tables.inc, 76800 floats in albedo.slang's layout) with its
index, which the library's own tables are compared with.

Arguments name the fixtures to write (file names); none writes all.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE = os.environ.get("LOTUS_REFERENCE",
                           os.path.join(HERE, "..", "..", "..", "reference"))

FIXTURES = [("cornell-box", "cornell_box.npz", 1024),
            ("material-basics-v1", "material_basics_v1.npz", 4096),
            ("material-textures-v1", "material_textures_v1.npz", 4096),
            ("material-alpha-v1", "material_alpha_v1.npz", 4096),
            ("material-normals-v1", "material_normals_v1.npz", 4096),
            ("material-transmission-v1", "material_transmission_v1.npz", 4096),
            ("material-transforms-v1", "material_transforms_v1.npz", 4096),
            ("material-emission-v1", "material_emission_v1.npz", 4096),
            ("material-gltf-v1", "material_gltf_v1.npz", 4096),
            ("material-gltf-extensions-v1", "material_gltf_extensions_v1.npz", 4096),
            ("material-primvars-v1", "material_primvars_v1.npz", 4096),
            ("material-subsets-v1", "material_subsets_v1.npz", 4096),
            ("material-mtlx-v1", "material_mtlx_v1.npz", 4096),
            ("material-graphs-v1", "material_graphs_v1.npz", 4096)]
TABLES = "albedo_tables_reference.npz"
TABLE_STRIDE = 7


def read_table_inc(path):
    values = []
    with open(path) as f:
        for line in f:
            if line.startswith("//"):
                continue
            values += [float(v) for v in line.strip().split(",") if v.strip()]
    return np.array(values, dtype=np.float32)


def read_pfm(path):
    with open(path, "rb") as f:
        data = f.read()
    parts = data.split(b"\n", 3)
    magic, dims, scale = parts[0].strip(), parts[1].split(), float(parts[2])
    if magic != b"PF" or scale >= 0:
        raise ValueError(f"{path}: not a little-endian RGB PFM")
    w, h = int(dims[0]), int(dims[1])
    body = np.frombuffer(parts[3][:w * h * 12], dtype="<f4").reshape(h, w, 3)
    return np.ascontiguousarray(body[::-1]).astype(np.float32)


def main():
    ref = os.path.join(REFERENCE, "validation", "reference")
    if not os.path.isdir(ref):
        print(f"no reference tree at {REFERENCE}; set LOTUS_REFERENCE", file=sys.stderr)
        return 1
    wanted = set(sys.argv[1:])
    for stem, name, samples in FIXTURES:
        if wanted and name not in wanted:
            continue
        mean = read_pfm(os.path.join(ref, f"{stem}-mean.pfm"))
        variance = read_pfm(os.path.join(ref, f"{stem}-variance.pfm"))
        out = os.path.join(HERE, name)
        np.savez_compressed(out, mean=mean, variance=variance, samples=np.uint32(samples))
        print("wrote", out, mean.shape)
    if not wanted or TABLES in wanted:
        table = read_table_inc(os.path.join(REFERENCE, "backend", "vulkan", "bsdf-albedo-tables.inc"))
        index = np.arange(0, table.size, TABLE_STRIDE, dtype=np.uint32)
        out = os.path.join(HERE, TABLES)
        np.savez_compressed(out, index=index, value=table[index], size=np.uint32(table.size))
        print("wrote", out, index.size)
    return 0


if __name__ == "__main__":
    sys.exit(main())
