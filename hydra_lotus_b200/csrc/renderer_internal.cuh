// SPDX-License-Identifier: Apache-2.0
// Internal access to a renderer for the library's other entry points.
#pragma once

#include <string>

#include "../../include/lotus_cuda.h"
#include "integrator.cuh"

namespace lotus {

struct RendererAccess {
  int device = 0;
  cudaStream_t stream = nullptr;
  const SceneView* view = nullptr;
  TraceTuning tuning;
  uint32_t step_limit = 0;     // the BVH walks' step budget
  bool cache_enabled = false;  // the radiance cache is configured on
};

// The renderer's device, stream and resident scene; false (with the
// reason) when it has failed earlier or holds no scene.
bool renderer_access(lotus_cuda_renderer* r, RendererAccess& out, std::string& detail);

// Latches a device failure: every later call on the renderer Fails with it.
void renderer_poison(lotus_cuda_renderer* r, const std::string& detail);

// The detail for a frame whose BVH walks failed (the two words of
// SceneView::walk_failure, read back after the frame), or "" when none did.
std::string walk_failure_detail(const uint32_t words[2], uint32_t step_limit);

// Validates a frame's target, settings and camera as RenderScene does and
// fills its constants and data window. sample_index, accumulated and
// add_sample are left for the caller.
bool make_frame_constants(const lotus_frame_desc& d, FrameConst& fc, uint32_t rect[4],
    std::string& detail);

}  // namespace lotus
