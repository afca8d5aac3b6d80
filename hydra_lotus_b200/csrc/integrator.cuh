// SPDX-License-Identifier: Apache-2.0
// Path state, queues and kernel entry points of the two integrators.
#pragma once

#include "radiance_cache.cuh"
#include "transport.cuh"

namespace lotus {

// The wavefront integrator's path state, one slot per target pixel, in
// 16-byte sections (backend/vulkan/shaders/common/path_state.slang in
// hydra-lotus): a kernel loads only the sections it uses, as coalesced
// 16-byte loads.
struct PathState {
  float4* origin;      // ray origin, tmin
  float4* direction;   // ray direction, tmax
  float4* throughput;  // throughput, last pdf (-1: the light found is unweighted)
  float4* radiance;    // radiance, random state; once ended: the sample (rgb, hit)
  uint4* hit;          // instance, leaf-ordered triangle, barycentrics
};

// Shadow queue entries: the part of ShadowedLight (transport.slang:82-115)
// left after the shadow ray, split into four 16-byte sections.
struct ShadowQueue {
  float4* ray_o;     // origin, tmax
  float4* ray_d;     // direction, MIS weight
  float4* fl;        // f * light radiance, light pdf
  float4* thr;       // path throughput, slot (bits)
};

// Per-bounce queue counters: [3 * b] rays entering bounce b's extension
// (b = 0: camera rays), [3 * b + 1] hits shaded at bounce b, [3 * b + 2]
// shadow rays from bounce b. After the 3 * (max_bounces + 2) counts come
// the persistent kernels' fetch cursors, two per bounce (extension,
// shadow): kQueueCounterWords words per bounce in all, cleared per sample.
constexpr uint32_t kQueueCounterWords = 5;

struct Queues {
  uint32_t* ray[2];
  uint32_t* hit;
  ShadowQueue shadow;
  uint32_t* counts;
  uint32_t capacity;
  // The extension queues of bounces 1 and on in key order (origin cell,
  // then direction octant): the shading pass writes each queued ray's key
  // beside it (`keys`) and counts the keys per bin (`bins`: kSortBins
  // counters, then kSortBlocks block totals); a scan and a scatter write
  // the queue in key order to `sorted`, which the extension pass reads.
  // Null `keys`: the queues keep their append order.
  uint32_t* keys = nullptr;
  uint32_t* sorted = nullptr;
  uint32_t* bins = nullptr;
};

// The reordering key: kSortAxisBits per axis of the origin's cell in a grid
// over the scene's box, interleaved (a Morton code), above the direction's
// octant. The histogram is scanned in blocks of kSortScanBlock bins.
constexpr uint32_t kSortAxisBits = 5;
constexpr uint32_t kSortBins = 1u << (3 * kSortAxisBits + 3);
constexpr uint32_t kSortScanBlock = 1024;
constexpr uint32_t kSortBlocks = kSortBins / kSortScanBlock;
constexpr uint32_t kSortBinWords = kSortBins + kSortBlocks;

// The radiance cache's per-sample queues: queries (paths that end into the
// cache at their second vertex) and training records, with their counts in
// counters[0] and counters[1].
struct CacheQueues {
  bool enabled = false;
  uint32_t stride = 32;           // one path in `stride` trains
  uint32_t steps = 1;             // training steps per sample
  uint32_t bounce = 1;            // paths end into the cache at this bounce's vertex
  RadianceCache* cache = nullptr;
  CacheRecord* queries = nullptr;
  uint32_t* query_slots = nullptr;
  float4* query_throughput = nullptr;
  uint32_t query_capacity = 0;
  CacheRecord* train = nullptr;
  uint32_t* train_slots = nullptr;
  float4* train_base = nullptr;        // radiance after the second vertex's emission
  float4* train_throughput = nullptr;  // throughput on arrival at the second vertex
  float4* train_targets = nullptr;
  uint32_t train_capacity = 0;
  uint32_t* counters = nullptr;
  // The queries in spatial order: the shading pass writes each query's key
  // (its position's cell, kQuerySortAxisBits per axis over the cache's
  // grid box, interleaved) and counts the keys per bin; a scan and a
  // scatter write the queries' indices in key order to `query_order`, and
  // inference takes its queries in that order, so that neighbouring
  // threads gather neighbouring hash-grid entries. Null keys: append order.
  uint32_t* query_keys = nullptr;
  uint32_t* query_order = nullptr;
  uint32_t* query_bins = nullptr;  // kSortBinWords
  float grid_lo[3] = {0.0f, 0.0f, 0.0f};
  float grid_scale[3] = {0.0f, 0.0f, 0.0f};  // cells per unit length
};

constexpr uint32_t kQuerySortAxisBits = 6;
static_assert((1u << (3 * kQuerySortAxisBits)) == kSortBins, "query keys fill the histogram");

// Several scenes rendered as one wavefront: scene k owns the path slots
// [slot_base[k], slot_base[k + 1]), in its image's row order, with its own
// scene view and frame constants (device arrays of `count` entries).
struct SceneTable {
  const SceneView* views = nullptr;
  FrameConst* frames = nullptr;
  const uint32_t* slot_base = nullptr;  // count + 1 entries
  uint32_t count = 0;
  uint32_t total_slots = 0;
  bool analytic = false;  // some scene has analytic lights
  bool full_shading = false;  // some scene has texture lookups or glTF PBR materials
  // The camera pass's order within each scene: 0, each image's rows; k,
  // warp tiles 2^k pixels wide and 32 / 2^k high (every scene's size a
  // multiple of the tile).
  uint32_t camera_tile = 0;
};

// Launch shape of the persistent tracing kernels: a lane takes a new ray
// when fewer than `refill_below` lanes of its warp still hold one. Zero
// picks the default.
struct TraceTuning {
  uint32_t refill_below = 0;
  uint32_t blocks_per_sm = 0;  // 0: as many as fit
  uint32_t rounds = 0;         // wavefront rounds before the tail; 0: the default
  uint32_t camera_tile = 0;    // a batch's camera order (LOTUS_CAMERA_TILE_*); 0: the default
};

// Ray totals over a RenderScene call.
struct RayTotals {
  unsigned long long camera;
  unsigned long long extension;
  unsigned long long shadow;
  unsigned long long error;  // traversal or bookkeeping errors
};

// BVH visits by ray kind (camera, extension, shadow), for roofline
// accounting.
struct VisitCounters {
  unsigned long long rays[3];
  unsigned long long nodes[3];
  unsigned long long triangles[3];
  unsigned long long instances[3];
};

// Optional per-sample instrumentation: events around each kernel (its
// class in `kinds`: 0 camera, 1 extend, 2 shade, 3 shadow, 4 resolve,
// 5 radiance-cache inference, 6 tail, 7 queue reordering, 8 radiance-cache
// training) and
// visit counting variants of the tracing kernels.
struct SampleProfile {
  cudaEvent_t* events = nullptr;  // 2 per timed launch
  int* kinds = nullptr;
  int capacity = 0;               // timed launches that fit
  int count = 0;
  VisitCounters* visits = nullptr;  // non-null: count visits
};

void launch_reference_pt(const SceneView& S, const FrameConst* fc, const uint32_t rect[4],
    double4* accum, float4* color, RayTotals* totals, cudaStream_t stream,
    SampleProfile* profile = nullptr);

// The bounces the wavefront integrator runs as rounds (`requested`, or by
// default LOTUS_WAVEFRONT_ROUNDS), the tail kernel taking the rest; all of
// them when visits are counted, and with the radiance cache at least
// bounces 0 and 1 (its vertex is shaded in round 1).
uint32_t wavefront_rounds(uint32_t max_bounces, bool count_visits, uint32_t requested, uint32_t cache_bounce = 0);

// The rounds a sample (or wave) should run, from its queue counts (the
// wavefront kernels' per-bounce words, 3 per bounce): the first bounce whose
// queue held fewer paths than the extension kernel keeps resident on the
// device at once (`resident`, at least 65,536), else every bounce. A round
// over a queue that cannot fill the device once costs more than the tail
// kernel's share of it (the reference's round scheduler stops at a
// sixteenth of the camera rays instead). Results do not depend on it; only
// the launch count does.
uint32_t choose_wavefront_rounds(const uint32_t* counts, uint32_t resident, uint32_t max_bounces);

// Threads of the extension kernel resident on the device at once.
uint32_t extension_resident_threads();

void launch_wavefront_sample(const SceneView& S, const FrameConst* fc, const uint32_t rect[4],
    uint32_t width, uint32_t height, uint32_t max_bounces, const PathState& P, const Queues& Q,
    double4* accum, float4* color, RayTotals* totals, cudaStream_t stream,
    SampleProfile* profile = nullptr, const TraceTuning& tuning = TraceTuning(),
    const CacheQueues* cache = nullptr, cudaEvent_t before_resolve = nullptr, uint32_t wave = 1);
// Frame constants for a wave: `frame`'s advanced by `offset` samples,
// covering `wave` samples whose path slots lie `stride` apart.
void launch_wave_frame(const FrameConst* frame, FrameConst* out, uint32_t offset, uint32_t wave, uint32_t stride,
    cudaStream_t stream);
// Advances the frame constants by `samples` samples.
void launch_advance_by(FrameConst* fc, uint32_t samples, cudaStream_t stream);

// The frame constants of the sample after fc's: a copy of *fc advanced by
// one sample (for two samples in flight at once, each with its own).
void launch_next_frame(const FrameConst* fc, FrameConst* next, cudaStream_t stream);

// One sample of every scene of a batch, as one set of wavefront launches
// over all scenes' paths (the wavefront integrator, no radiance cache).
void launch_wavefront_batch(const SceneTable& B, uint32_t max_bounces, const PathState& P, const Queues& Q,
    double4* accum, float4* color, RayTotals* totals, cudaStream_t stream, const TraceTuning& tuning,
    cudaEvent_t before_resolve = nullptr);

// Every scene's frame constants advanced by one sample into `next` (the
// batch's second sample in flight), and every scene's sample advanced.
void launch_next_frames(const FrameConst* frames, FrameConst* next, uint32_t count, cudaStream_t stream);
void launch_advance_batch(const SceneTable& B, cudaStream_t stream);

// Deferred visibility of the ReSTIR passes. Each pass queues the shadow
// ray of every pixel whose selected sample needs one (origin and distance,
// direction, pixel) and keeps the pixel's unshadowed contribution and
// normalization in `pending`; one persistent any-hit launch per pass then
// traces the queue and completes the pixels' records. counters[2 p] and
// counters[2 p + 1] are pass p's queued rays and fetch cursor.
struct VisibilityQueue {
  float4* origin;     // origin, distance
  float4* direction;
  uint32_t* slot;
  float4* pending;    // per pixel
  uint32_t* counters;
  uint32_t capacity;
  // Per pass, the smallest pixel whose record's arithmetic failed (flag 2),
  // or ~0: the frame then Fails as the reference's record readback does
  // (vulkan_backend.cpp:1650-1705).
  uint32_t* failed;
};
constexpr uint32_t kVisibilityPasses = 3;

// Traces pass `pass`'s queue and completes the RestirPixel at `records +
// slot * stride` of each ray: contribution = (unshadowed * (visibility *
// normalization), visibility), or flag 2 when the normalization is not
// finite (or, with `positive`, not above zero) or the estimate is not
// finite (restir.slang:225-232, 380-386, 484-490).
void launch_visibility(const SceneView& S, const VisibilityQueue& queue, uint32_t pass, unsigned char* records,
    uint32_t stride, bool positive, cudaStream_t stream, const TraceTuning& tuning = TraceTuning());

// The diagnostic outputs, numbered as lotus_settings::output.
constexpr uint32_t kOutputBarycentrics = 1, kOutputShadingNormal = 2, kOutputAlbedo = 3,
                   kOutputRoughnessMetallic = 4;

// A diagnostic output (kOutputBarycentrics .. kOutputRoughnessMetallic) of
// the pixels in `rect` into `color`; misses leave their pixels as they are.
void launch_diagnostic(const SceneView& S, const FrameConst* fc, const uint32_t rect[4], uint32_t output,
    float4* color, cudaStream_t stream);

void launch_advance(FrameConst* fc, cudaStream_t stream);

void launch_clear_color(float4* color, uint32_t pixels, float4 value, cudaStream_t stream);
// The depth product of the pixel centres' closest hits in `rect`; with
// `clear`, every pixel first takes `clear_depth`.
void launch_depth(const SceneView& S, const FrameConst* fc, const uint32_t rect[4], float* depth, uint32_t pixels,
    bool clear, float clear_depth, cudaStream_t stream);

}  // namespace lotus
