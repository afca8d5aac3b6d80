// SPDX-License-Identifier: Apache-2.0
// Batched rendering: up to LOTUS_BATCH_MAX_SCENES independent scenes, each
// with its own target, rendered as one wavefront. Every sample runs one
// camera launch over all scenes' pixels, then per bounce one persistent
// extension launch, one shading launch and one persistent shadow launch
// over all scenes' queued paths, then one resolve: small scenes fill the
// GPU together instead of one after another. A sample is captured as one
// CUDA graph and replayed per sample. Each scene's resident data (BVHs,
// materials, lights, environment) is built by the same code as
// lotus_cuda_update_scene, into a renderer the batch owns.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lotus_cuda.h"
#include "integrator.cuh"
#include "renderer_internal.cuh"

struct lotus_cuda_batch {
  int device = 0;
  lotus::TraceTuning tuning;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  std::string failure;
  std::vector<lotus_cuda_renderer*> scenes;
  // The combined wavefront state, sized to the scenes' pixels.
  uint32_t capacity = 0;
  void* buffers[19] = {};
  lotus::PathState P{};
  lotus::Queues Q{};
  double4* accum = nullptr;
  float4* color = nullptr;
  lotus::RayTotals* totals = nullptr;
  lotus::SceneView* views = nullptr;
  lotus::FrameConst* frames = nullptr;
  uint32_t* slot_base = nullptr;
  // Per scene: the last frame description and samples accumulated.
  std::vector<lotus_frame_desc> last;
  std::vector<uint32_t> accumulated;
  std::vector<uint64_t> completion;
  // A second path state and queue set and per-scene frame constants, for
  // the second of two samples in flight (its rounds beside the first's
  // tail, on a second stream; it resolves after the first).
  void* buffers2[16] = {};
  uint32_t capacity2 = 0;
  lotus::PathState P2{};
  lotus::Queues Q2{};
  lotus::FrameConst* frames2 = nullptr;
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_first = nullptr, ev_join = nullptr;
  cudaGraphExec_t graph_pair = nullptr;
  std::vector<uint32_t> pair_layout;
  uint32_t pair_bounces = 0, pair_rounds = 0;
  // The captured sample.
  cudaGraphExec_t graph = nullptr;
  std::vector<uint32_t> graph_layout;
  uint32_t graph_bounces = 0;
  uint32_t graph_rounds = 0;
  // The wavefront rounds before the tail, chosen from the first sample of a
  // layout (choose_wavefront_rounds over every scene's pixels).
  std::vector<uint32_t> rounds_layout;
  uint32_t rounds_bounces = 0;
  uint32_t auto_rounds = 0;
};

namespace lotus {
namespace {

constexpr uint32_t kMaxScenes = LOTUS_BATCH_MAX_SCENES;
// The camera order a batch uses unless tuned otherwise (the tuner's choice
// on the 64-scene workload: 8x4 tiles, 2% faster per sample than rows).
constexpr uint32_t kDefaultBatchCameraTile = LOTUS_CAMERA_TILE_8X4;

void set_detail(char* dst, size_t n, const std::string& s) {
  if (dst && n) std::snprintf(dst, n, "%s", s.c_str());
}

void release_buffers(lotus_cuda_batch& b) {
  for (void*& p : b.buffers) {
    if (p) cudaFree(p);
    p = nullptr;
  }
  for (void*& p : b.buffers2) {
    if (p) cudaFree(p);
    p = nullptr;
  }
  b.capacity = 0;
  b.capacity2 = 0;
  if (b.graph_pair) {
    cudaGraphExecDestroy(b.graph_pair);
    b.graph_pair = nullptr;
  }
}

// The second sample's path state, queues and frame constants.
cudaError_t ensure_pair_buffers(lotus_cuda_batch& b) {
  if (b.capacity2 >= b.capacity && b.buffers2[0]) return cudaSuccess;
  const size_t n = std::max<uint32_t>(b.capacity, 1);
  const size_t sizes[16] = {16 * n, 16 * n, 16 * n, 16 * n, 16 * n, 4 * n, 4 * n, 4 * n, 16 * n, 16 * n, 16 * n,
      16 * n + sizeof(uint32_t) * kQueueCounterWords * (LOTUS_MAX_BOUNCES + 2), sizeof(FrameConst) * kMaxScenes,
      4 * n, 4 * n, sizeof(uint32_t) * kSortBinWords};  // queue keys, sorted queue, key histogram
  for (int i = 0; i < 16; ++i) {
    if (b.buffers2[i]) cudaFree(b.buffers2[i]);
    b.buffers2[i] = nullptr;
    const cudaError_t e = cudaMalloc(&b.buffers2[i], sizes[i]);
    if (e != cudaSuccess) return e;
  }
  auto f4 = [&](int i) { return static_cast<float4*>(b.buffers2[i]); };
  b.P2 = PathState{f4(0), f4(1), f4(2), f4(3), static_cast<uint4*>(b.buffers2[4])};
  b.Q2 = b.Q;
  b.Q2.ray[0] = static_cast<uint32_t*>(b.buffers2[5]);
  b.Q2.ray[1] = static_cast<uint32_t*>(b.buffers2[6]);
  b.Q2.hit = static_cast<uint32_t*>(b.buffers2[7]);
  b.Q2.shadow = ShadowQueue{f4(8), f4(9), f4(10), f4(11)};
  b.Q2.counts = reinterpret_cast<uint32_t*>(static_cast<char*>(b.buffers2[11]) + 16 * n);
  b.frames2 = static_cast<FrameConst*>(b.buffers2[12]);
  b.Q2.keys = static_cast<uint32_t*>(b.buffers2[13]);
  b.Q2.sorted = static_cast<uint32_t*>(b.buffers2[14]);
  b.Q2.bins = static_cast<uint32_t*>(b.buffers2[15]);
  b.capacity2 = (uint32_t)n;
  if (b.graph_pair) {
    cudaGraphExecDestroy(b.graph_pair);
    b.graph_pair = nullptr;
  }
  return cudaSuccess;
}

// The combined state for `pixels` path slots and `scenes` scenes.
cudaError_t ensure_buffers(lotus_cuda_batch& b, uint32_t pixels, uint32_t scenes) {
  if (b.capacity >= pixels && b.buffers[0]) return cudaSuccess;
  release_buffers(b);
  const size_t n = std::max<uint32_t>(pixels, 1);
  const size_t sizes[19] = {16 * n, 16 * n, 16 * n, 16 * n, 16 * n,   // path state
      4 * n, 4 * n, 4 * n,                                           // ray x2, hit queues
      16 * n, 16 * n, 16 * n, 16 * n,                                // shadow queue
      sizeof(uint32_t) * kQueueCounterWords * (LOTUS_MAX_BOUNCES + 2),
      sizeof(double4) * n + sizeof(float4) * n,                      // accumulation, colour
      sizeof(RayTotals) + sizeof(SceneView) * kMaxScenes + sizeof(FrameConst) * kMaxScenes,
      sizeof(uint32_t) * (kMaxScenes + 1),
      4 * n, 4 * n, sizeof(uint32_t) * kSortBinWords};               // queue keys, sorted queue, key histogram
  for (int i = 0; i < 19; ++i) {
    const cudaError_t e = cudaMalloc(&b.buffers[i], sizes[i]);
    if (e != cudaSuccess) {
      release_buffers(b);
      return e;
    }
  }
  auto f4 = [&](int i) { return static_cast<float4*>(b.buffers[i]); };
  b.P = PathState{f4(0), f4(1), f4(2), f4(3), static_cast<uint4*>(b.buffers[4])};
  b.Q.ray[0] = static_cast<uint32_t*>(b.buffers[5]);
  b.Q.ray[1] = static_cast<uint32_t*>(b.buffers[6]);
  b.Q.hit = static_cast<uint32_t*>(b.buffers[7]);
  b.Q.shadow = ShadowQueue{f4(8), f4(9), f4(10), f4(11)};
  b.Q.counts = static_cast<uint32_t*>(b.buffers[12]);
  b.accum = static_cast<double4*>(b.buffers[13]);
  b.color = reinterpret_cast<float4*>(static_cast<char*>(b.buffers[13]) + sizeof(double4) * n);
  char* misc = static_cast<char*>(b.buffers[14]);
  b.totals = reinterpret_cast<RayTotals*>(misc);
  b.views = reinterpret_cast<SceneView*>(misc + sizeof(RayTotals));
  b.frames = reinterpret_cast<FrameConst*>(misc + sizeof(RayTotals) + sizeof(SceneView) * kMaxScenes);
  b.slot_base = static_cast<uint32_t*>(b.buffers[15]);
  b.Q.keys = static_cast<uint32_t*>(b.buffers[16]);
  b.Q.sorted = static_cast<uint32_t*>(b.buffers[17]);
  b.Q.bins = static_cast<uint32_t*>(b.buffers[18]);
  b.capacity = (uint32_t)n;
  (void)scenes;
  if (b.graph) {
    cudaGraphExecDestroy(b.graph);
    b.graph = nullptr;
  }
  return cudaSuccess;
}

void destroy_scenes(lotus_cuda_batch& b) {
  for (lotus_cuda_renderer* r : b.scenes) lotus_cuda_destroy(r);
  b.scenes.clear();
  b.last.clear();
  b.accumulated.clear();
  b.completion.clear();
}

}  // namespace
}  // namespace lotus

using namespace lotus;

extern "C" int32_t lotus_cuda_batch_create(const lotus_cuda_options* options, lotus_cuda_batch** out, char* error,
    size_t error_size) {
  if (!out) return LOTUS_FAIL;
  *out = nullptr;
  const int device = options ? options->device : 0;
  const int32_t cap = lotus_cuda_capability(device, error, error_size);
  if (cap != LOTUS_PASS) return cap;
  auto* b = new (std::nothrow) lotus_cuda_batch();
  if (!b) {
    set_detail(error, error_size, "out of host memory");
    return LOTUS_FAIL;
  }
  b->device = device;
  if (options) {
    b->tuning.refill_below = options->trace_refill_below;
    b->tuning.blocks_per_sm = options->trace_blocks_per_sm;
    b->tuning.rounds = options->wavefront_rounds;
  }
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->stream2, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev_first, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&b->ev_start) != cudaSuccess || cudaEventCreate(&b->ev_stop) != cudaSuccess) {
    set_detail(error, error_size, "stream or event creation failed");
    lotus_cuda_batch_destroy(b);
    return LOTUS_FAIL;
  }
  *out = b;
  return LOTUS_PASS;
}

extern "C" void lotus_cuda_batch_destroy(lotus_cuda_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  release_buffers(*b);
  destroy_scenes(*b);
  if (b->ev_start) cudaEventDestroy(b->ev_start);
  if (b->ev_stop) cudaEventDestroy(b->ev_stop);
  for (cudaEvent_t e : {b->ev_fork, b->ev_first, b->ev_join})
    if (e) cudaEventDestroy(e);
  if (b->stream2) cudaStreamDestroy(b->stream2);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

extern "C" int32_t lotus_cuda_batch_set_tuning(lotus_cuda_batch* b, uint32_t refill_below, uint32_t blocks_per_sm,
    uint32_t wavefront_rounds, uint32_t camera_tile) {
  if (!b || refill_below > 32 || blocks_per_sm > 64 || wavefront_rounds > LOTUS_MAX_BOUNCES + 1 ||
      camera_tile > LOTUS_CAMERA_TILE_16X2)
    return LOTUS_FAIL;
  b->tuning.refill_below = refill_below;
  b->tuning.blocks_per_sm = blocks_per_sm;
  b->tuning.rounds = wavefront_rounds;
  b->tuning.camera_tile = camera_tile;
  cudaSetDevice(b->device);
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  if (b->graph_pair) {
    cudaGraphExecDestroy(b->graph_pair);
    b->graph_pair = nullptr;
  }
  return LOTUS_PASS;
}

extern "C" int32_t lotus_cuda_batch_set_scenes(lotus_cuda_batch* b, const lotus_scene_desc* scenes, uint32_t count,
    lotus_scene_result* results) {
  if (!b || (!scenes && count)) return LOTUS_FAIL;
  auto fail_all = [&](const std::string& why) {
    for (uint32_t k = 0; results && k < count; ++k) {
      results[k].status = LOTUS_FAIL;
      set_detail(results[k].detail, sizeof(results[k].detail), why);
    }
    return LOTUS_FAIL;
  };
  if (!b->failure.empty()) return fail_all("the batch failed earlier: " + b->failure);
  if (count > kMaxScenes)
    return fail_all("a batch holds at most " + std::to_string(kMaxScenes) + " scenes");
  cudaSetDevice(b->device);
  destroy_scenes(*b);
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  if (b->graph_pair) {
    cudaGraphExecDestroy(b->graph_pair);
    b->graph_pair = nullptr;
  }
  int32_t status = LOTUS_PASS;
  for (uint32_t k = 0; k < count; ++k) {
    lotus_cuda_options o{};
    o.device = b->device;
    o.trace_refill_below = b->tuning.refill_below;
    o.trace_blocks_per_sm = b->tuning.blocks_per_sm;
    o.wavefront_rounds = b->tuning.rounds;
    lotus_cuda_renderer* r = nullptr;
    char err[256] = {};
    int32_t s = lotus_cuda_create(&o, &r, err, sizeof(err));
    lotus_scene_result local{};
    lotus_scene_result& res = results ? results[k] : local;
    if (s == LOTUS_PASS) s = lotus_cuda_update_scene(r, &scenes[k], &res);
    else set_detail(res.detail, sizeof(res.detail), err);
    res.status = s;
    if (s != LOTUS_PASS) status = LOTUS_FAIL;
    b->scenes.push_back(r);
  }
  b->last.assign(count, lotus_frame_desc{});
  b->accumulated.assign(count, 0);
  b->completion.assign(count, 0);
  if (status != LOTUS_PASS) destroy_scenes(*b);
  return status;
}

extern "C" int32_t lotus_cuda_batch_render(lotus_cuda_batch* b, const lotus_frame_desc* frames, uint32_t count,
    lotus_frame_result* results, float* const* colors, lotus_frame_result* total) {
  lotus_frame_result local_total{};
  lotus_frame_result& tot = total ? *total : local_total;
  std::memset(&tot, 0, sizeof(tot));
  auto fail = [&](const std::string& why, bool poison = false) {
    set_detail(tot.detail, sizeof(tot.detail), why);
    for (uint32_t k = 0; results && k < count; ++k) {
      results[k].status = LOTUS_FAIL;
      set_detail(results[k].detail, sizeof(results[k].detail), why);
    }
    if (poison) b->failure = why;
    return tot.status = LOTUS_FAIL;
  };
  if (!b || !frames) return LOTUS_FAIL;
  if (!b->failure.empty()) return fail("the batch failed earlier: " + b->failure);
  if (count != b->scenes.size() || count == 0)
    return fail("one frame per scene of the batch is needed (" + std::to_string(b->scenes.size()) + ")");
  const uint32_t frame_count = frames[0].frame_count;
  if (frame_count == 0) return fail("frame_count must be at least 1");
  std::vector<FrameConst> fcs(count);
  std::vector<uint32_t> base(count + 1, 0);
  std::vector<uint32_t> layout;
  uint32_t max_bounces = 0;
  std::string detail;
  for (uint32_t k = 0; k < count; ++k) {
    const lotus_frame_desc& d = frames[k];
    if (d.frame_count != frame_count) return fail("every frame of a batch has the same frame_count");
    if (d.settings.integrator != LOTUS_INTEGRATOR_WAVEFRONT ||
        d.settings.light_sampling > LOTUS_LIGHT_SAMPLING_MIS)
      return fail("a batch renders with the wavefront integrator and Bsdf or Mis light sampling");
    if (d.settings.max_samples != 0) return fail("a batch takes no max_samples");
    uint32_t rect[4];
    if (!make_frame_constants(d, fcs[k], rect, detail)) return fail("scene " + std::to_string(k) + ": " + detail);
    // Accumulation continues while a scene's frame description is unchanged.
    lotus_frame_desc key = d;
    key.frame_count = 0;
    key.target.read_back = 0;
    key.flags = 0;
    if (std::memcmp(&key, &b->last[k], sizeof(key)) != 0) {
      b->last[k] = key;
      b->accumulated[k] = 0;
    }
    fcs[k].sample_index = d.settings.sample_index + b->accumulated[k];
    fcs[k].accumulated = b->accumulated[k];
    fcs[k].add_sample = 1u;
    const uint64_t pixels = (uint64_t)d.target.width * d.target.height;
    if ((uint64_t)base[k] + pixels > 0xFFFFFFF0ull) return fail("the batch's targets exceed 2^32 pixels");
    base[k + 1] = base[k] + (uint32_t)pixels;
    max_bounces = std::max(max_bounces, d.settings.max_bounces);
    layout.push_back(d.target.width);
    layout.push_back(d.target.height);
    layout.insert(layout.end(), rect, rect + 4);
  }
  cudaSetDevice(b->device);
  cudaStream_t s = b->stream;
  cudaError_t e = ensure_buffers(*b, base[count], count);
  if (e != cudaSuccess) return fail(std::string("batch buffers: ") + cudaGetErrorString(e), true);
  std::vector<SceneView> views(count);
  bool analytic = false, full_shading = false;
  // Every scene's walks report to the first scene's walk-failure words.
  uint32_t* walk_failure = nullptr;
  uint32_t step_limit = 0;
  for (uint32_t k = 0; k < count; ++k) {
    RendererAccess a;
    if (!renderer_access(b->scenes[k], a, detail)) return fail("scene " + std::to_string(k) + ": " + detail);
    views[k] = *a.view;
    if (!walk_failure) {
      walk_failure = a.view->walk_failure;
      step_limit = a.step_limit;
    }
    views[k].walk_failure = walk_failure;
    analytic = analytic || a.view->analytic_count != 0;
    full_shading = full_shading || a.view->full_shading != 0;
  }
  SceneTable B;
  B.views = b->views;
  B.frames = b->frames;
  B.slot_base = b->slot_base;
  B.count = count;
  B.total_slots = base[count];
  B.analytic = analytic;
  B.full_shading = full_shading;
  {
    // Warp tiles where every scene's size is a multiple of the tile.
    const uint32_t tile = b->tuning.camera_tile ? b->tuning.camera_tile : kDefaultBatchCameraTile;
    const uint32_t k = tile >= LOTUS_CAMERA_TILE_4X8 && tile <= LOTUS_CAMERA_TILE_16X2 ? tile : 0u;
    bool fits = k != 0;
    for (uint32_t j = 0; fits && j < count; ++j)
      fits = frames[j].target.width % (1u << k) == 0 && frames[j].target.height % (32u >> k) == 0;
    B.camera_tile = fits ? k : 0u;
  }
  Queues Q = b->Q;
  Q.capacity = base[count];
  // Clear colours first: pixels outside a data window keep them.
  for (uint32_t k = 0; k < count; ++k) {
    const lotus_target& t = frames[k].target;
    launch_clear_color(b->color + base[k], t.width * t.height,
        make_float4(t.clear_color[0], t.clear_color[1], t.clear_color[2], t.clear_color[3]), s);
  }
  if ((e = cudaMemcpyAsync(b->views, views.data(), sizeof(SceneView) * count, cudaMemcpyHostToDevice, s)) !=
          cudaSuccess ||
      (e = cudaMemcpyAsync(b->frames, fcs.data(), sizeof(FrameConst) * count, cudaMemcpyHostToDevice, s)) !=
          cudaSuccess ||
      (e = cudaMemcpyAsync(b->slot_base, base.data(), sizeof(uint32_t) * (count + 1), cudaMemcpyHostToDevice, s)) !=
          cudaSuccess ||
      (e = cudaMemsetAsync(b->totals, 0, sizeof(RayTotals), s)) != cudaSuccess ||
      (e = cudaMemsetAsync(walk_failure, 0, 2 * sizeof(uint32_t), s)) != cudaSuccess)
    return fail(std::string("batch upload: ") + cudaGetErrorString(e), true);
  // One graph per layout and round count: the sample over every scene.
  TraceTuning tuning = b->tuning;
  const bool rounds_known = b->rounds_layout == layout && b->rounds_bounces == max_bounces;
  if (tuning.rounds == 0 && rounds_known) tuning.rounds = b->auto_rounds;
  const bool choose_rounds = b->tuning.rounds == 0 && !rounds_known && frame_count != 0;
  const uint32_t rounds = wavefront_rounds(max_bounces, false, tuning.rounds);
  if (!b->graph || b->graph_layout != layout || b->graph_bounces != max_bounces || b->graph_rounds != rounds) {
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    cudaGraph_t g;
    if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return fail(std::string("graph capture: ") + cudaGetErrorString(e), true);
    launch_wavefront_batch(B, max_bounces, b->P, Q, b->accum, b->color, b->totals, s, tuning);
    if ((e = cudaStreamEndCapture(s, &g)) != cudaSuccess)
      return fail(std::string("graph capture: ") + cudaGetErrorString(e), true);
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(std::string("graph instantiate: ") + cudaGetErrorString(e), true);
    b->graph_layout = layout;
    b->graph_bounces = max_bounces;
    b->graph_rounds = rounds;
  }
  // Two samples in flight (as lotus_cuda_render keeps them): the second on
  // its own path state, queues, frame constants and stream, resolving after
  // the first.
  const bool pairs = frame_count >= 2;
  if (pairs && (e = ensure_pair_buffers(*b)) != cudaSuccess)
    return fail(std::string("batch buffers: ") + cudaGetErrorString(e), true);
  Queues Q2 = b->Q2;
  Q2.capacity = base[count];
  if (pairs && (!b->graph_pair || b->pair_layout != layout || b->pair_bounces != max_bounces ||
                   b->pair_rounds != rounds)) {
    if (b->graph_pair) {
      cudaGraphExecDestroy(b->graph_pair);
      b->graph_pair = nullptr;
    }
    SceneTable B2 = B;
    B2.frames = b->frames2;
    cudaGraph_t g;
    if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return fail(std::string("graph capture: ") + cudaGetErrorString(e), true);
    launch_next_frames(b->frames, b->frames2, count, s);
    cudaEventRecord(b->ev_fork, s);
    cudaStreamWaitEvent(b->stream2, b->ev_fork, 0);
    launch_wavefront_batch(B, max_bounces, b->P, Q, b->accum, b->color, b->totals, s, tuning);
    cudaEventRecord(b->ev_first, s);
    launch_wavefront_batch(B2, max_bounces, b->P2, Q2, b->accum, b->color, b->totals, b->stream2, tuning,
        b->ev_first);
    cudaEventRecord(b->ev_join, b->stream2);
    cudaStreamWaitEvent(s, b->ev_join, 0);
    launch_advance_batch(B, s);
    if ((e = cudaStreamEndCapture(s, &g)) != cudaSuccess)
      return fail(std::string("graph capture: ") + cudaGetErrorString(e), true);
    e = cudaGraphInstantiate(&b->graph_pair, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(std::string("graph instantiate: ") + cudaGetErrorString(e), true);
    b->pair_layout = layout;
    b->pair_bounces = max_bounces;
    b->pair_rounds = rounds;
  }
  bool last_pair = false;
  cudaEventRecord(b->ev_start, s);
  for (uint32_t i = 0; i < frame_count;) {
    last_pair = i + 2 <= frame_count;
    if ((e = cudaGraphLaunch(last_pair ? b->graph_pair : b->graph, s)) != cudaSuccess)
      return fail(std::string("graph launch: ") + cudaGetErrorString(e), true);
    i += last_pair ? 2 : 1;
  }
  cudaEventRecord(b->ev_stop, s);
  RayTotals totals{};
  cudaMemcpyAsync(&totals, b->totals, sizeof(totals), cudaMemcpyDeviceToHost, s);
  uint32_t walks[2] = {0, 0};
  cudaMemcpyAsync(walks, walk_failure, sizeof(walks), cudaMemcpyDeviceToHost, s);
  std::vector<uint32_t> counts;
  if (choose_rounds) {
    counts.assign(3 * (size_t)(max_bounces + 2), 0u);
    cudaMemcpyAsync(counts.data(), last_pair ? Q2.counts : Q.counts, counts.size() * 4, cudaMemcpyDeviceToHost, s);
  }
  for (uint32_t k = 0; colors && k < count; ++k)
    if (colors[k] && frames[k].target.read_back)
      cudaMemcpyAsync(colors[k], b->color + base[k], sizeof(float4) * (base[k + 1] - base[k]),
          cudaMemcpyDeviceToHost, s);
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess)
    return fail(std::string("batch render: ") + cudaGetErrorString(e), true);
  if (walks[0]) return fail(walk_failure_detail(walks, step_limit), true);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, b->ev_start, b->ev_stop);
  if (choose_rounds) {
    b->rounds_layout = layout;
    b->rounds_bounces = max_bounces;
    b->auto_rounds = choose_wavefront_rounds(counts.data(), extension_resident_threads(), max_bounces);
  }
  for (uint32_t k = 0; k < count; ++k) {
    b->accumulated[k] += frame_count;
    b->completion[k] += frame_count;
    if (results) {
      lotus_frame_result& r = results[k];
      std::memset(&r, 0, sizeof(r));
      r.status = LOTUS_PASS;
      r.frames_rendered = frame_count;
      r.samples_per_pixel = b->accumulated[k];
      r.completion = b->completion[k];
      r.gpu_ms = ms;
    }
  }
  tot.status = LOTUS_PASS;
  tot.frames_rendered = frame_count;
  tot.camera_rays = totals.camera;
  tot.extension_rays = totals.extension;
  tot.shadow_rays = totals.shadow;
  tot.gpu_ms = ms;
  return LOTUS_PASS;
}
