"""Writes converged oracle images (test fixtures) under tests/golden/.

Each is the CPU oracle's (oracle/lotus_oracle.cpp, the scalar restatement of
the reference's path tracer, itself pinned to the reference's golden images)
FP64 accumulation of many samples per pixel from sample index 2^24, with the
per-sample variance estimated from batches of 256 samples as the
reference's WriteReferenceFiles does (adapters/headless/main.cpp):
per-batch means, their variance, times the batch size.

- box_room_256_oracle.npz: the seeded box room (scenes.box_room(seed=0)) at
  256x256, NEE + MIS, max depth 6, 16,384 samples per pixel from 64
  batches: the converged image of the small box-room workload.
- sphere_field_band_oracle.npz: the benchmarked 1080p sphere field
  (scenes.sphere_field(seed=0)), rows 536..551 (a 16-row band through the
  middle of the frame), NEE + MIS, max depth 8, 4,096 samples per pixel
  from 16 batches.

The CPU oracle runs on all host cores (OpenMP); each fixture takes a few
minutes. Run: python tests/golden/make_oracle_images.py [box_room|band]
"""

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hydra_lotus_b200 import abi, scenes  # noqa: E402
from oracle import oracle  # noqa: E402

FIRST_SAMPLE = 1 << 24
BATCH = 256
BAND = (536, 16)


def converge(scene, settings, batches, window=None):
    o = oracle.OracleScene(scene)
    kw = {"data_window": window} if window else {}
    frame = scene.frame(settings, BATCH, **kw)
    h, w = scene.height, scene.width
    total = np.zeros((h, w, 3))
    squares = np.zeros((h, w, 3))
    for b in range(batches):
        t = time.time()
        sums, _ = o.accumulate(frame, FIRST_SAMPLE + b * BATCH, BATCH)
        mean = sums[..., :3] / BATCH
        total += mean
        squares += mean * mean
        print(f"batch {b + 1}/{batches} {time.time() - t:.1f} s", flush=True)
    mean = total / batches
    batch_var = np.maximum(0.0, (squares - batches * mean * mean) / (batches - 1))
    return mean.astype(np.float32), (batch_var * BATCH).astype(np.float32)


def box_room():
    scene = scenes.box_room(seed=0, size=256)
    st = abi.default_settings(integrator=abi.INTEGRATOR_REFERENCE, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=6, sample_index=FIRST_SAMPLE)
    mean, variance = converge(scene, st, 64)
    out = os.path.join(HERE, "box_room_256_oracle.npz")
    np.savez_compressed(out, mean=mean, variance=variance, samples=np.uint32(64 * BATCH))
    print("wrote", out)


def band():
    scene = scenes.sphere_field(seed=0)
    st = abi.default_settings(integrator=abi.INTEGRATOR_REFERENCE, light_sampling=abi.LIGHT_SAMPLING_MIS,
                              max_bounces=8, sample_index=FIRST_SAMPLE)
    y0, rows = BAND
    mean, variance = converge(scene, st, 16, window=(0, y0, scene.width, rows))
    out = os.path.join(HERE, "sphere_field_band_oracle.npz")
    np.savez_compressed(out, mean=mean[y0:y0 + rows], variance=variance[y0:y0 + rows],
                        samples=np.uint32(16 * BATCH), band=np.array(BAND, dtype=np.uint32))
    print("wrote", out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["box_room", "band"]
    for name in which:
        {"box_room": box_room, "band": band}[name]()
