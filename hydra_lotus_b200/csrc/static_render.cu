// SPDX-License-Identifier: Apache-2.0
// lotus_cuda_render_static: a render entry point that allocates nothing.
//
// Some hosts cannot allocate device memory at the moment they want a frame:
// a render delegate that runs inside another framework's frame loop where
// that framework owns every allocation (and a cudaMalloc would synchronize
// the device or break its memory budget), or a caller on a real-time path
// that must not block in the allocator. For them this entry point renders a
// small frame with scratch memory that already exists: one file-scope
// __device__ array, which every GPU that loads the library holds until the
// process exits. The caller passes the inputs (the renderer, whose scene is
// resident, and the frame description) and the output (device memory for
// the colour). Nothing here calls cudaMalloc, cudaFree or an allocating
// library routine.
//
// Limits and sharing:
//   - frames of at most LOTUS_STATIC_MAX_PIXELS (65,536) pixels;
//   - every call shares the one scratch array and leaves its contents
//     behind; each call starts its own accumulation from zero, so nothing
//     carries over, but two calls whose GPU work overlaps (other streams,
//     other threads) race on the scratch and corrupt each other;
//   - the scratch's device address is looked up (cudaGetSymbolAddress) on
//     the first call on each device, with that device current; make that
//     first call before any stream capture. A cudaDeviceReset invalidates
//     it together with every renderer on that device;
//   - a renderer whose radiance cache is configured on Fails: this entry
//     point never uses the cache, so its image would not be RenderScene's;
//   - a launch or device error Fails the call and poisons the renderer, as
//     lotus_cuda_render does; so does a BVH walk that ran out of steps or
//     stack.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/lotus_cuda.h"
#include "integrator.cuh"
#include "renderer_internal.cuh"

namespace lotus {
namespace {

constexpr size_t kMaxPixels = LOTUS_STATIC_MAX_PIXELS;
constexpr size_t kAlign = 256;

constexpr size_t align_up(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }

// The scratch layout.
constexpr size_t kFrameOffset = 0;
constexpr size_t kTotalsOffset = kFrameOffset + align_up(sizeof(FrameConst));
constexpr size_t kCountsOffset = kTotalsOffset + align_up(sizeof(RayTotals));
constexpr size_t kCountsBytes = align_up(sizeof(uint32_t) * kQueueCounterWords * (LOTUS_MAX_BOUNCES + 2));
constexpr size_t kAccumOffset = kCountsOffset + kCountsBytes;
constexpr size_t kPathOffset = kAccumOffset + align_up(sizeof(double4) * kMaxPixels);
constexpr size_t kPathSectionBytes = align_up(16 * kMaxPixels);
constexpr size_t kQueueOffset = kPathOffset + 5 * kPathSectionBytes;
constexpr size_t kQueueBytes = align_up(sizeof(uint32_t) * kMaxPixels);
constexpr size_t kShadowOffset = kQueueOffset + 3 * kQueueBytes;
constexpr size_t kScratchBytes = kShadowOffset + 4 * kPathSectionBytes;

// About 12 MB per device.
__device__ __align__(256) unsigned char g_static_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
unsigned char* g_scratch_address[kMaxDevices] = {};

// The scratch's device address on `device` (which must be current).
cudaError_t scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_address[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_address[device] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_address[device];
  return cudaSuccess;
}

void set_detail(lotus_frame_result& res, const std::string& s) {
  std::snprintf(res.detail, sizeof(res.detail), "%s", s.c_str());
}

}  // namespace
}  // namespace lotus

extern "C" int32_t lotus_cuda_render_static(lotus_cuda_renderer* renderer,
    const lotus_frame_desc* frame, float* color_device, lotus_frame_result* result) {
  using namespace lotus;
  lotus_frame_result local{};
  lotus_frame_result& res = result ? *result : local;
  std::memset(&res, 0, sizeof(res));
  auto fail = [&](const std::string& d) {
    set_detail(res, d);
    return res.status = LOTUS_FAIL;
  };
  if (!renderer || !frame || !color_device) return fail("no renderer, frame or output");
  auto poison = [&](const std::string& d) {
    renderer_poison(renderer, d);
    return fail(d);
  };
  RendererAccess access;
  std::string detail;
  if (!renderer_access(renderer, access, detail)) return fail(detail);
  const lotus_target& t = frame->target;
  if ((uint64_t)t.width * t.height > kMaxPixels)
    return fail("the allocation-free entry point renders at most " + std::to_string(kMaxPixels) +
                " pixels; the target has " + std::to_string((uint64_t)t.width * t.height));
  if (frame->frame_count == 0) return fail("frame_count must be at least 1");
  if (access.cache_enabled)
    return fail("the allocation-free entry point does not use the radiance cache; configure it off first");
  const uint32_t max_samples = frame->settings.max_samples;
  const uint32_t samples = max_samples ? std::min(frame->frame_count, max_samples) : frame->frame_count;
  FrameConst fc{};
  uint32_t rect[4];
  if (!make_frame_constants(*frame, fc, rect, detail)) return fail(detail);
  fc.sample_index = frame->settings.sample_index;
  fc.accumulated = 0;
  fc.add_sample = 1;
  if (cudaSetDevice(access.device) != cudaSuccess) return fail("cudaSetDevice failed");
  unsigned char* base = nullptr;
  cudaError_t e = scratch_address(access.device, &base);
  if (e != cudaSuccess) return fail(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  FrameConst* d_frame = reinterpret_cast<FrameConst*>(base + kFrameOffset);
  RayTotals* d_totals = reinterpret_cast<RayTotals*>(base + kTotalsOffset);
  double4* accum = reinterpret_cast<double4*>(base + kAccumOffset);
  PathState P;
  P.origin = reinterpret_cast<float4*>(base + kPathOffset);
  P.direction = reinterpret_cast<float4*>(base + kPathOffset + kPathSectionBytes);
  P.throughput = reinterpret_cast<float4*>(base + kPathOffset + 2 * kPathSectionBytes);
  P.radiance = reinterpret_cast<float4*>(base + kPathOffset + 3 * kPathSectionBytes);
  P.hit = reinterpret_cast<uint4*>(base + kPathOffset + 4 * kPathSectionBytes);
  Queues Q;
  Q.ray[0] = reinterpret_cast<uint32_t*>(base + kQueueOffset);
  Q.ray[1] = reinterpret_cast<uint32_t*>(base + kQueueOffset + kQueueBytes);
  Q.hit = reinterpret_cast<uint32_t*>(base + kQueueOffset + 2 * kQueueBytes);
  Q.shadow.ray_o = reinterpret_cast<float4*>(base + kShadowOffset);
  Q.shadow.ray_d = reinterpret_cast<float4*>(base + kShadowOffset + kPathSectionBytes);
  Q.shadow.fl = reinterpret_cast<float4*>(base + kShadowOffset + 2 * kPathSectionBytes);
  Q.shadow.thr = reinterpret_cast<float4*>(base + kShadowOffset + 3 * kPathSectionBytes);
  Q.counts = reinterpret_cast<uint32_t*>(base + kCountsOffset);
  Q.capacity = t.width * t.height;
  cudaStream_t s = access.stream;
  const float4 clear = make_float4(t.clear_color[0], t.clear_color[1], t.clear_color[2], t.clear_color[3]);
  if ((e = cudaMemcpyAsync(d_frame, &fc, sizeof(fc), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(d_totals, 0, sizeof(RayTotals), s)) != cudaSuccess ||
      (e = cudaMemsetAsync(access.view->walk_failure, 0, 2 * sizeof(uint32_t), s)) != cudaSuccess)
    return poison(std::string("scratch set-up: ") + cudaGetErrorString(e));
  float4* color = reinterpret_cast<float4*>(color_device);
  if (rect[2] < t.width || rect[3] < t.height || rect[2] == 0)
    launch_clear_color(color, t.width * t.height, clear, s);
  const bool wavefront = frame->settings.integrator == LOTUS_INTEGRATOR_WAVEFRONT;
  for (uint32_t k = 0; k < samples; ++k) {
    if (wavefront)
      launch_wavefront_sample(*access.view, d_frame, rect, t.width, t.height,
          frame->settings.max_bounces, P, Q, accum, color, d_totals, s, nullptr, access.tuning);
    else
      launch_reference_pt(*access.view, d_frame, rect, accum, color, d_totals, s);
    launch_advance(d_frame, s);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return poison(std::string("launch: ") + cudaGetErrorString(e));
  RayTotals totals{};
  uint32_t walks[2] = {0, 0};
  if ((e = cudaMemcpyAsync(&totals, d_totals, sizeof(totals), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(walks, access.view->walk_failure, sizeof(walks), cudaMemcpyDeviceToHost, s)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return poison(std::string("render: ") + cudaGetErrorString(e));
  if (walks[0]) return poison(walk_failure_detail(walks, access.step_limit));
  res.status = LOTUS_PASS;
  res.frames_rendered = samples;
  res.samples_per_pixel = samples;
  res.camera_rays = totals.camera;
  res.extension_rays = totals.extension;
  res.shadow_rays = totals.shadow;
  return LOTUS_PASS;
}
