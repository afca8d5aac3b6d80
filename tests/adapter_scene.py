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
    out = [b"LTSC", struct.pack("<I", 3)]
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
    for g, (p, t, n) in enumerate(scene.geometries):
        out.append(struct.pack("<3I", p.shape[0], t.shape[0], 0 if n is None else 1))
        out.append(np.ascontiguousarray(p, dtype=np.float32).tobytes())
        out.append(np.ascontiguousarray(t, dtype=np.uint32).tobytes())
        if n is not None:
            out.append(np.ascontiguousarray(n, dtype=np.float32).tobytes())
        sets = scene.texcoords.get(g)
        out.append(struct.pack("<I", 0 if sets is None else sets.shape[0]))
        if sets is not None:
            out.append(np.ascontiguousarray(sets, dtype=np.float32).tobytes())
    for i, (m, g, mat) in enumerate(scene.instances):
        out.append(np.asarray(m, dtype=np.float32).reshape(16).tobytes())
        out.append(struct.pack("<3I", g, mat, scene.instance_texcoords.get(i, 0)))
    for mat in scene.materials:
        out.append(bytes(mat))
    out.append(struct.pack("<I", len(scene.textures)))
    for texels, fmt in scene.textures:
        out.append(struct.pack("<3I", texels.shape[1], texels.shape[0], fmt))
        out.append(np.ascontiguousarray(texels).tobytes())
    out.append(struct.pack("<I", len(scene.texture_inputs)))
    for t in scene.texture_inputs:
        out.append(bytes(t))
    out.append(struct.pack("<I", len(scene.lights)))
    for light in scene.lights:
        out.append(bytes(light))
    out.append(np.asarray(scene.world_to_clip, dtype=np.float32).reshape(16).tobytes())
    out.append(struct.pack("<7I", scene.width, scene.height, settings.integrator, settings.light_sampling,
                           settings.max_bounces, settings.sample_index, frame_count))
    with open(path, "wb") as f:
        f.write(b"".join(out))


def _image(path, scene):
    if os.path.exists(path) and os.path.getsize(path) == scene.width * scene.height * 16:
        return np.fromfile(path, dtype=np.float32).reshape(scene.height, scene.width, 4)
    return None


def run(tmpdir, scene, settings, frame_count, edit_dx=None):
    """(exit code, evidence dict, colour (H, W, 4) or None). With edit_dx,
    the driver then moves instance 0 by edit_dx in x (an instance-only
    plan) and edits geometry 0 (y += 0.01 x, a same-topology replacement),
    rendering after each: returns (code, [evidence dicts], [3 colours])."""
    inp = os.path.join(tmpdir, "scene.bin")
    outs = [os.path.join(tmpdir, f"color{k}.bin") for k in range(3)]
    write(inp, scene, settings, frame_count)
    args = [HARNESS, inp, outs[0]]
    if edit_dx is not None:
        args += [repr(float(edit_dx)), outs[1], outs[2]]
    p = subprocess.run(args, capture_output=True, text=True, timeout=600)
    lines = [json.loads(line) for line in p.stdout.strip().splitlines() if line.startswith("{")]
    if edit_dx is None:
        return p.returncode, (lines[-1] if lines else {}), _image(outs[0], scene)
    return p.returncode, lines, [_image(o, scene) for o in outs]


TEMPORAL_PRODUCTS = ["color", "surface", "validity", "radiance", "batch", "restir_initial", "restir_temporal",
                     "restir_spatial", "restir_sources"]


def run_temporal(tmpdir, scene, settings):
    """The driver's temporal mode: two still-camera temporal frames through
    RenderTemporalScene. Returns (exit code, [evidence per frame],
    [{product name: raw bytes} per frame])."""
    inp = os.path.join(tmpdir, "scene.bin")
    prefix = os.path.join(tmpdir, "t")
    write(inp, scene, settings, 1)
    p = subprocess.run([HARNESS, inp, os.path.join(tmpdir, "unused.bin"), "--temporal", prefix],
                       capture_output=True, text=True, timeout=600)
    lines = [json.loads(line) for line in p.stdout.strip().splitlines() if line.startswith("{")]
    frames = []
    for k in range(2):
        frames.append({name: open(f"{prefix}{k}_{name}.bin", "rb").read()
                       for name in TEMPORAL_PRODUCTS if os.path.exists(f"{prefix}{k}_{name}.bin")})
    return p.returncode, lines, frames
