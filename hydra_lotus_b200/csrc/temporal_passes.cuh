// SPDX-License-Identifier: Apache-2.0
// Launchers of the temporal passes (temporal.cu).
#pragma once

#include "integrator.cuh"
#include "temporal.cuh"

namespace lotus {

void launch_temporal_surface(const SceneView& S, const FrameConst* fc, const TemporalConst* tc,
    const TemporalInstance* ids, TemporalPixel* out, uint32_t pixels, cudaStream_t s);

void launch_reproject(const TemporalConst* tc, const TemporalPixel* current, const TemporalPixel* previous,
    ValidityPixel* out, uint32_t pixels, cudaStream_t s);

// The ReSTIR passes queue their selected samples' shadow rays in `vq`
// (passes 0, 1 and 2); launch_visibility after each completes its records.
// The initial pass also keeps each pixel's camera-ray hit and random state
// in primary_hit / primary_rng for the passes after it.
void launch_restir_initial(const SceneView& S, const FrameConst* fc, const TemporalConst* tc,
    RestirPixel* out, uint4* primary_hit, uint32_t* primary_rng, const VisibilityQueue& vq, uint32_t pixels,
    cudaStream_t s);

void launch_restir_temporal(const SceneView& S, const FrameConst* fc, const TemporalConst* tc,
    const uint4* primary_hit, const TemporalInstance* ids, const RestirPixel* initial,
    const ValidityPixel* validity, const TemporalPixel* surface, const RestirReuse* previous,
    const RestirSurface* previous_surfaces, RestirReuse* out, RestirSurface* out_surfaces,
    const VisibilityQueue& vq, uint32_t pixels, cudaStream_t s);

void launch_restir_spatial(const SceneView& S, const FrameConst* fc, const TemporalConst* tc,
    const RestirReuse* temporal, const RestirSurface* surfaces, RestirReuse* out, uint4* sources,
    const VisibilityQueue& vq, uint32_t pixels, cudaStream_t s);

// Accumulation, variance, the a-trous iterations and the composite into
// `color` (or the accumulated colour without iterations).
void launch_svgf(const TemporalConst* tc, const TemporalConst& host_tc, const float4* batch,
    const TemporalPixel* surface, const ValidityPixel* validity, const RadiancePixel* old,
    RadiancePixel* radiance, float4* filter, float4* color, uint32_t pixels, cudaStream_t s);

}  // namespace lotus
