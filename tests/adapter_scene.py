"""Writes a scene and a frame in the adapter harness's input format
(tests/adapter_harness.cpp) and runs the harness."""

import json
import os
import struct
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "hydra_lotus_b200", "_lib", "adapter_harness")


def write(path, scene, settings, frame_count):
    out = [b"LTSC", struct.pack("<I", 1)]
    out.append(struct.pack("<3I", len(scene.geometries), len(scene.instances), len(scene.materials)))
    out.append(struct.pack("<3f", *scene.environment_constant))
    if scene.environment is not None:
        texels, scale, rows = scene.environment
        out.append(struct.pack("<3I", 1, texels.shape[1], texels.shape[0]))
        out.append(struct.pack("<3f", *scale))
        out.append(np.asarray(rows, dtype=np.float32).reshape(9).tobytes())
        out.append(np.ascontiguousarray(texels, dtype=np.float32).tobytes())
    else:
        out.append(struct.pack("<I", 0))
    for p, t, n in scene.geometries:
        out.append(struct.pack("<3I", p.shape[0], t.shape[0], 0 if n is None else 1))
        out.append(np.ascontiguousarray(p, dtype=np.float32).tobytes())
        out.append(np.ascontiguousarray(t, dtype=np.uint32).tobytes())
        if n is not None:
            out.append(np.ascontiguousarray(n, dtype=np.float32).tobytes())
    for m, g, mat in scene.instances:
        out.append(np.asarray(m, dtype=np.float32).reshape(16).tobytes())
        out.append(struct.pack("<2I", g, mat))
    for mat in scene.materials:
        out.append(bytes(mat))
    out.append(np.asarray(scene.world_to_clip, dtype=np.float32).reshape(16).tobytes())
    out.append(struct.pack("<7I", scene.width, scene.height, settings.integrator, settings.light_sampling,
                           settings.max_bounces, settings.sample_index, frame_count))
    with open(path, "wb") as f:
        f.write(b"".join(out))


def run(tmpdir, scene, settings, frame_count):
    """(exit code, evidence dict, colour (H, W, 4) or None)."""
    inp = os.path.join(tmpdir, "scene.bin")
    outp = os.path.join(tmpdir, "color.bin")
    write(inp, scene, settings, frame_count)
    p = subprocess.run([HARNESS, inp, outp], capture_output=True, text=True, timeout=600)
    evidence = json.loads(p.stdout.strip().splitlines()[-1]) if p.stdout.strip() else {}
    color = None
    if os.path.exists(outp) and os.path.getsize(outp) == scene.width * scene.height * 16:
        color = np.fromfile(outp, dtype=np.float32).reshape(scene.height, scene.width, 4)
    return p.returncode, evidence, color
