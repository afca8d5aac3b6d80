// SPDX-License-Identifier: Apache-2.0
//
// TEST INFRASTRUCTURE ONLY. A C interface over the reference's own CPU code
// for the temporal and reservoir paths (hydra-lotus
// backend/vulkan/temporal.cpp and reservoir.cpp, compiled from their sources
// by oracle/build_ref.py into oracle/_ref/). The tests feed it buffers the
// CUDA kernels produced and compare: it is the checker, never the product.
#include <cstdint>
#include <cstring>
#include <span>
#include <stdexcept>

#include "lotus/temporal.hpp"
#include "reservoir.hpp"

using Lotus::TemporalPixel;
using Lotus::TemporalRadiancePixel;
using Lotus::TemporalValidityPixel;
using Lotus::vulkan_internal::Reservoir;

extern "C" {

// EstimateTemporalVariance (temporal.hpp:264-268) at one pixel.
float ref_estimate_variance(const void* surface, const void* radiance, uint32_t x, uint32_t y,
    uint32_t width, uint32_t height, uint32_t batch_samples, uint32_t max_history_samples) {
  const size_t n = size_t{width} * height;
  return Lotus::EstimateTemporalVariance(
      std::span<const TemporalPixel>(static_cast<const TemporalPixel*>(surface), n),
      std::span<const TemporalRadiancePixel>(static_cast<const TemporalRadiancePixel*>(radiance), n), x, y,
      width, height, batch_samples, max_history_samples);
}

// FilterTemporalRadiance (temporal.hpp:332-336): the composite after
// `iterations` a-trous iterations; 0 on success.
int ref_filter(const void* surface, const void* radiance, uint32_t width, uint32_t height,
    uint32_t batch_samples, uint32_t max_history_samples, uint32_t iterations, float* out) {
  const size_t n = size_t{width} * height;
  const auto result = Lotus::FilterTemporalRadiance(
      std::span<const TemporalPixel>(static_cast<const TemporalPixel*>(surface), n),
      std::span<const TemporalRadiancePixel>(static_cast<const TemporalRadiancePixel*>(radiance), n), width,
      height, batch_samples, max_history_samples, iterations);
  if (result.size() != n) return 1;
  std::memcpy(out, result.data(), n * sizeof(float) * 4);
  return 0;
}

// ReprojectTemporalHistory (temporal.hpp:341-345) at one pixel.
void ref_reproject(const void* current, uint32_t x, uint32_t y, uint32_t width, uint32_t height,
    const void* previous, uint64_t previous_count, const float* validation, void* out) {
  Lotus::TemporalValidationSettings settings;
  settings.absolute_depth_tolerance = validation[0];
  settings.relative_depth_tolerance = validation[1];
  settings.minimum_normal_cosine = validation[2];
  settings.max_motion_pixels = validation[3];
  const TemporalValidityPixel v = Lotus::ReprojectTemporalHistory(*static_cast<const TemporalPixel*>(current),
      x, y, width, height,
      std::span<const TemporalPixel>(static_cast<const TemporalPixel*>(previous), previous_count), settings);
  std::memcpy(out, &v, sizeof(v));
}

// Reservoir arithmetic (reservoir.hpp): 0 success, 1 invalid argument,
// 2 overflow. The reservoir is updated only on success.
int ref_stream_candidate(void* reservoir, uint32_t sample, float target, float proposal, float random,
    int* selected) {
  try {
    *selected = Lotus::vulkan_internal::StreamReservoirCandidate(*static_cast<Reservoir*>(reservoir), sample,
        target, proposal, random) ? 1 : 0;
    return 0;
  } catch (const std::invalid_argument&) {
    return 1;
  } catch (const std::overflow_error&) {
    return 2;
  }
}

int ref_merge_reevaluated(void* destination, const void* source, double normalization, float target,
    uint32_t cap, float random, int* selected) {
  try {
    *selected = Lotus::vulkan_internal::MergeReevaluatedReservoir(*static_cast<Reservoir*>(destination),
        *static_cast<const Reservoir*>(source), normalization, target, cap, random) ? 1 : 0;
    return 0;
  } catch (const std::invalid_argument&) {
    return 1;
  } catch (const std::overflow_error&) {
    return 2;
  }
}

double ref_normalization(const void* reservoir, int* status) {
  try {
    *status = 0;
    return Lotus::vulkan_internal::ReservoirNormalization(*static_cast<const Reservoir*>(reservoir));
  } catch (const std::exception&) {
    *status = 1;
    return 0.0;
  }
}

double ref_reuse_normalization(const void* reservoir, uint32_t supporting, int* status) {
  try {
    *status = 0;
    return Lotus::vulkan_internal::ReservoirReuseNormalization(*static_cast<const Reservoir*>(reservoir),
        supporting);
  } catch (const std::exception&) {
    *status = 1;
    return 0.0;
  }
}

}  // extern "C"
