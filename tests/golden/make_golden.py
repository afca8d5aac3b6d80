"""Writes the golden fixtures under tests/golden/ from the reference tree.

Run in a checkout that has the reference at REFERENCE (default
/root/reference); the fixtures it writes are committed, so tests never
read the reference at run time.

- cornell_box.npz: validation/reference/cornell-box-mean.pfm and
  cornell-box-variance.pfm of hydra-lotus v0.9.0: the Cornell box fixture
  (adapters/common/reference.cpp:221-279) at 128x128, 1024 samples per
  pixel from sample index 0, BSDF sampling, 64 bounces, as the reference's
  GPU renderer wrote them (docs/reference/SCENE.md, "Deterministic mode").
  Stored as float32 arrays with rows from the top (the PFMs hold rows from
  the bottom, little-endian; ReadPfm, reference.cpp:100-131).
"""

import os
import sys

import numpy as np

REFERENCE = os.environ.get("LOTUS_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))


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
    mean = read_pfm(os.path.join(ref, "cornell-box-mean.pfm"))
    variance = read_pfm(os.path.join(ref, "cornell-box-variance.pfm"))
    out = os.path.join(HERE, "cornell_box.npz")
    np.savez_compressed(out, mean=mean, variance=variance, samples=np.uint32(1024))
    print("wrote", out, mean.shape)


if __name__ == "__main__":
    sys.exit(main())
