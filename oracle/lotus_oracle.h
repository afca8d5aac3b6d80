/* SPDX-License-Identifier: Apache-2.0
 *
 * TEST INFRASTRUCTURE ONLY. The oracle is a scalar CPU restatement of the
 * reference's integrator (its Slang path tracer and host-side table
 * builders). Only tests, the smoke check and the CPU-baseline leg of the
 * benchmark may load it, as the checker; the product never calls it.
 *
 * It takes the same plain-data scene and frame descriptions as the CUDA
 * library (include/lotus_cuda.h) and returns per-sample radiance or FP64
 * accumulated sums.
 */
#ifndef LOTUS_ORACLE_H
#define LOTUS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/lotus_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_scene oracle_scene;

oracle_scene* oracle_scene_create(const lotus_scene_desc* scene, char* error,
    size_t error_size);
void oracle_scene_destroy(oracle_scene* scene);

/* One sample per pixel of the frame's data window with random sequence
 * `sample_index`, as the reference's radiance pass draws it
 * (path_trace.slang:353-367): rgba[pixel] = (radiance, 1) for a camera ray
 * that hits and (0, 0, 0, 0) for one that misses. Pixels outside the data
 * window are left untouched. rays[0..2] receive the camera, extension and
 * shadow rays traced. `threads` <= 0 uses every core. */
int32_t oracle_sample(const oracle_scene* scene, const lotus_frame_desc* frame,
    uint32_t sample_index, float* rgba, uint64_t* rays, int32_t threads);

/* Adds samples first_sample .. first_sample + count - 1 of every pixel to
 * FP64 sums (4 doubles per pixel: radiance and hit count). */
int32_t oracle_accumulate(const oracle_scene* scene,
    const lotus_frame_desc* frame, uint32_t first_sample, uint32_t count,
    double* sums, uint64_t* rays, int32_t threads);

/* The light table BuildLightTable makes (gpu_scene.cpp:515-610): 4 words
 * per entry {pdf, threshold, alias, instance}, then one first entry per
 * instance. Returns the entry count. */
int64_t oracle_light_table(const oracle_scene* scene, uint32_t* records,
    uint64_t record_capacity, uint32_t* offsets, uint64_t offset_capacity);

/* Traversal statistics on the oracle's own BVH over the camera rays of
 * `frame`: mean nodes and triangles visited per ray. */
int32_t oracle_traversal_stats(const oracle_scene* scene,
    const lotus_frame_desc* frame, uint32_t max_rays, double* nodes_per_ray,
    double* triangles_per_ray);

#ifdef __cplusplus
}
#endif

#endif /* LOTUS_ORACLE_H */
