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

/* The temporal passes' constants (the kernels' TemporalConst). */
typedef struct oracle_temporal {
  float current_view[16];
  float previous_view[16];
  float previous_world_to_clip[16];  /* Vulkan clip */
  float previous_display[4];
  uint32_t previous_data[4];
  uint32_t restir_candidates;
  uint32_t restir_history;
  uint32_t restir_max_history;
  uint32_t restir_radius;
  uint32_t restir_neighbours;  /* 0: four axis neighbours; 1..8: disk neighbours */
  uint32_t restir_proposal;
  uint32_t max_bounces;
} oracle_temporal;

/* WriteTemporalSurface (temporal.slang:557-627) for every pixel: 64-byte
 * TemporalPixel records. `ids` may be NULL (index ids, static, flags 6). */
int32_t oracle_temporal_surface(const oracle_scene* scene, const lotus_frame_desc* frame,
    const oracle_temporal* temporal, const lotus_temporal_instance* ids, void* out);

/* The ReSTIR DI passes (restir.slang:163-491) over the same records as the
 * kernels: RestirPixel (48 B), RestirReuse (64 B), RestirSurface (160 B). */
int32_t oracle_restir_initial(const oracle_scene* scene, const lotus_frame_desc* frame,
    const oracle_temporal* temporal, uint32_t sample_index, void* out);
int32_t oracle_restir_temporal(const oracle_scene* scene, const lotus_frame_desc* frame,
    const oracle_temporal* temporal, const lotus_temporal_instance* ids, uint32_t sample_index,
    const void* initial, const void* validity, const void* surface, const void* previous,
    const void* previous_surfaces, void* out, void* out_surfaces);
int32_t oracle_restir_spatial(const oracle_scene* scene, const lotus_frame_desc* frame,
    const oracle_temporal* temporal, uint32_t sample_index, const void* temporal_records,
    const void* surfaces, void* out, uint32_t* sources);

/* oracle_sample with RestirInitial light sampling: the depth-0 direct light
 * is InitialDirectLight over `final_records` (RestirPixel records `stride`
 * bytes apart). */
int32_t oracle_sample_restir(const oracle_scene* scene, const lotus_frame_desc* frame,
    uint32_t sample_index, const void* final_records, uint32_t stride, float* rgba, uint64_t* rays,
    int32_t threads);

#ifdef __cplusplus
}
#endif

#endif /* LOTUS_ORACLE_H */
