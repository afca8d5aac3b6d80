"""Renders frames of a named workload through the C ABI, for profilers.

    python -m hydra_lotus_b200.profile_frame --workload sphere-field \
        --width 960 --height 540 --spp 1 --frames 2

Prints the rays, device time and paths per bounce (the extension
kernel's rays at bounces 1 and up) of each frame. Used as the command under
Nsight Compute: the workload's sizes are arguments so that a capture can
run on a small case of the same kernels.
"""

import argparse
import json

from . import abi, renderer, scenes


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="sphere-field",
                    choices=["sphere-field", "box-room", "cornell", "cornell-gltf"],
                    help="cornell and cornell-gltf: the reference's cornell-v1 and cornell-gltf-v1 workloads "
                         "(square, --height pixels a side)")
    ap.add_argument("--light-sampling", default="mis", choices=["mis", "bsdf"])
    ap.add_argument("--width", type=int, default=960)
    ap.add_argument("--height", type=int, default=540)
    ap.add_argument("--spp", type=int, default=1)
    ap.add_argument("--frames", type=int, default=2)
    ap.add_argument("--depth", type=int, default=8)
    ap.add_argument("--integrator", default="wavefront", choices=["wavefront", "reference"])
    ap.add_argument("--rounds", type=int, default=0,
                    help="wavefront rounds before the tail kernel (0: chosen from the first sample)")
    ap.add_argument("--cache", action="store_true", help="paths end into the learned radiance cache")
    ap.add_argument("--temporal", action="store_true",
                    help="temporal frames of the many-light room: ReSTIR DI (temporal + spatial) and SVGF")
    ap.add_argument("--filter", type=int, default=5, help="a-trous iterations of the temporal frames")
    ap.add_argument("--updates", action="store_true",
                    help="scene upload and edits on the 512x512-quad grid (the geometry-v1 shape): one full "
                         "update, one point edit, one transform edit")
    ap.add_argument("--batch", type=int, default=0,
                    help="render the first N scenes of the 64-scene batch workload as one wavefront")
    args = ap.parse_args()
    if args.temporal:
        scene = scenes.restir_room(seed=0, size=args.height, emitters=10000, aspect=args.width / args.height)
        st = abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT,
                                  light_sampling=abi.LIGHT_SAMPLING_RESTIR_INITIAL, max_bounces=args.depth,
                                  sample_index=0, restir_candidates=8, restir_temporal=1,
                                  restir_max_history_candidates=20, restir_spatial=1, restir_spatial_radius=30,
                                  restir_spatial_neighbours=5)
        previous = None
        with renderer.CudaOffscreenRenderer(0) as r:
            renderer.check(r.update_scene(scene), "update_scene")
            if args.cache:
                r.configure_cache(enable=True, seed=1)
            for k in range(args.frames):
                view, w2c = scenes.orbit_camera(k, frames=120, aspect=args.width / args.height)
                frame = abi.make_frame(w2c, args.width, args.height, st, 1, read_back=False)
                d = abi.temporal_desc(frame, view, previous[0] if previous else None,
                                      previous[1] if previous else None, history_available=k > 0,
                                      accumulate_radiance=True, max_history_samples=5,
                                      filter_iterations=args.filter)
                res, _ = r.render_temporal(d)
                renderer.check(res, "render_temporal")
                previous = (view, w2c)
                rays = res.camera_rays + res.extension_rays + res.shadow_rays
                print(json.dumps({"frame": k, "rays": rays, "gpu_ms": round(res.gpu_ms, 3)}))
        return
    if args.updates:
        grid = scenes.grid_mesh(quads=512)
        with renderer.CudaOffscreenRenderer(0) as r:
            res = renderer.check(r.update_scene(grid), "update_scene")
            print(json.dumps({"update": "initial", "gpu_ms": round(res.build_gpu_ms, 3)}))
            p = grid.geometries[0][0]
            q = p.copy()
            q[:, 1] += 0.01 * p[:, 0]
            grid.set_positions(0, q)
            res = renderer.check(r.update_geometry(grid, 0), "update_geometry")
            print(json.dumps({"update": "point edit", "gpu_ms": round(res.build_gpu_ms, 3)}))
            m = grid.instances[0][0].copy()
            m[12] += 0.01
            grid.set_instance(0, m)
            res = renderer.check(r.update_instances(grid), "update_instances")
            print(json.dumps({"update": "transform edit", "gpu_ms": round(res.build_gpu_ms, 3)}))
        return
    if args.batch:
        work = scenes.batch_workload(64, seed=0)[:args.batch]
        with renderer.CudaBatch(0) as b:
            for r in b.set_scenes(work):
                renderer.check(r, "batch scene")
            for k in range(args.frames):
                frames = [s.frame(abi.default_settings(integrator=abi.INTEGRATOR_WAVEFRONT,
                                                       light_sampling=abi.LIGHT_SAMPLING_MIS, max_bounces=args.depth,
                                                       sample_index=1000 * i + k * args.spp),
                                  frame_count=args.spp, read_back=False) for i, s in enumerate(work)]
                _, _, total = b.render(frames)
                renderer.check(total, "batch render")
                rays = total.camera_rays + total.extension_rays + total.shadow_rays
                print(json.dumps({"frame": k, "rays": rays, "gpu_ms": round(total.gpu_ms, 3),
                                  "mrays_per_s": round(rays / total.gpu_ms / 1e3, 1)}))
        return
    if args.workload == "sphere-field":
        scene = scenes.sphere_field(seed=0, width=args.width, height=args.height)
    elif args.workload == "cornell":
        scene = scenes.cornell_reference(size=args.height)
    elif args.workload == "cornell-gltf":
        scene = scenes.cornell_gltf(size=args.height)
    else:
        scene = scenes.box_room_wide(seed=0, width=args.width, height=args.height)
    light_sampling = abi.LIGHT_SAMPLING_MIS if args.light_sampling == "mis" else abi.LIGHT_SAMPLING_BSDF
    integrator = abi.INTEGRATOR_WAVEFRONT if args.integrator == "wavefront" else abi.INTEGRATOR_REFERENCE
    with renderer.CudaOffscreenRenderer(0, wavefront_rounds=args.rounds) as r:
        renderer.check(r.update_scene(scene), "update_scene")
        if args.cache:
            r.configure_cache(enable=True, seed=1)
        for k in range(args.frames):
            st = abi.default_settings(integrator=integrator, light_sampling=light_sampling,
                                      max_bounces=args.depth, sample_index=k * args.spp)
            res, _ = r.render_scene(scene.frame(st, frame_count=args.spp, read_back=False))
            renderer.check(res, "render")
            rays = res.camera_rays + res.extension_rays + res.shadow_rays
            counts = [res.wavefront_path_counts[b] for b in range(res.wavefront_path_count_size)]
            print(json.dumps({"frame": k, "rays": rays, "gpu_ms": round(res.gpu_ms, 3),
                              "wavefront_rounds": res.wavefront_rounds,
                              "mrays_per_s": round(rays / res.gpu_ms / 1e3, 1),
                              "paths_per_bounce": counts}))


if __name__ == "__main__":
    main()
