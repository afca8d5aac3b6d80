// SPDX-License-Identifier: Apache-2.0
// The learned radiance cache: a multiresolution hash-grid encoding of
// position plus spherical harmonics of direction and the surface's normal,
// roughness and albedo, fed to an MLP of five 64-wide ReLU layers and an
// RGB output, run on the tensor cores (BF16 operands, FP32 accumulation).
// It is trained online, with Adam, on radiance the path tracer itself
// produces, and answers for the paths that end into it. The design follows
// Mueller et al., "Real-time Neural Radiance Caching for Path Tracing"
// (2021) and "Instant Neural Graphics Primitives with a Multiresolution
// Hash Encoding" (2022); it has no counterpart in hydra-lotus.
#pragma once

#include <cuda_fp16.h>

#include "common.cuh"

namespace lotus {

constexpr int kCacheInputs = 64;     // encoded features per query
constexpr int kCacheWidth = 64;      // hidden layer width
constexpr int kCacheOutputs = 16;    // output columns (RGB in the first three)
constexpr int kCacheLayers = 6;      // five hidden layers and the output layer
constexpr int kCacheMaxLevels = 16;  // hash-grid levels (two features each)
constexpr int kCacheGridFeatures = 2 * kCacheMaxLevels;
constexpr int kCacheSh = 16;         // spherical-harmonic coefficients (degree 4)
// FP32 master weights: layer l < 5 is W[in][out], 64 x 64; layer 5 64 x 16.
constexpr uint32_t kCacheWeights = 5 * 64 * 64 + 64 * 16;
// BF16 operand images of all six layers in the tensor-core layout.
constexpr uint32_t kCacheOperandBytes = 5 * 8192 + 2048;

// The raw features of one cache query or training record (64 bytes):
// world position and roughness, the direction toward the previous vertex,
// the shading normal and the albedo.
struct CacheRecord {
  float4 pos_rough;
  float4 dir;
  float4 normal;
  float4 albedo;
};

// The hash grid: `levels` levels of 2^log2_size half2 entries, resolution
// floor(base * growth^l) at level l over the scene box.
struct CacheGrid {
  __half2* table;
  float* grad;          // 2 floats per entry
  uint32_t levels;
  uint32_t log2_size;
  float res[kCacheMaxLevels];  // grid resolution per level
  float lo[3];
  float inv_extent[3];
};

// Device state of one cache.
struct CacheNet {
  const uint4* forward;   // kCacheOperandBytes: layer l's B operand (out x in)
  const uint4* backward;  // kCacheOperandBytes: layer l's transposed operand (in x out)
  float* grad;            // kCacheWeights FP32 weight gradients
  float* loss;            // sum of the per-sample losses
  uint32_t* error;        // set when a tensor-core wait gave up
};

// Host side of the cache's network (radiance_cache.cu).
struct CacheConfig {
  uint32_t levels = 16;
  uint32_t log2_size = 19;
  uint32_t min_resolution = 16;
  uint32_t max_resolution = 2048;
  float learning_rate = 1e-2f;
  uint32_t seed = 1;
};

cudaError_t launch_cache_infer_records(const CacheNet& net, const CacheGrid& grid, const CacheRecord* records,
    const uint32_t* slots, const float4* throughput, float4* radiance, const uint32_t* count, uint32_t capacity,
    cudaStream_t s, const uint32_t* order = nullptr);
cudaError_t launch_cache_train_records(const CacheNet& net, const CacheGrid& grid, const CacheRecord* records,
    const float4* targets, const uint32_t* count, uint32_t capacity, cudaStream_t s);

class RadianceCache {
 public:
  ~RadianceCache() { release(); }
  cudaError_t configure(const CacheConfig& config, const float lo[3], const float hi[3], cudaStream_t s);
  bool ready() const { return master_ != nullptr; }
  void release();

  // Test entry points: a forward pass over encoded inputs (n x 64), and the
  // gradients of the relative L2 loss against targets (n x 3).
  cudaError_t infer_encoded(const float* inputs, uint32_t n, float* outputs, cudaStream_t s);
  cudaError_t gradient_encoded(const float* inputs, const float* targets, uint32_t n, float* weight_grad,
      float* input_grad, float* loss, cudaStream_t s);
  // The hash-grid and direction encoding of raw records (n x 64 outputs).
  cudaError_t encode(const CacheRecord* records, uint32_t n, float* inputs, cudaStream_t s);
  // `steps` training steps (the training pass over all n records, then
  // Adam) on host records and RGB targets; the loss before each step.
  cudaError_t train_records(const CacheRecord* records, const float* targets, uint32_t n, uint32_t steps,
      float* losses, cudaStream_t s);
  // One Adam step over the gradients accumulated since the last one,
  // averaged over `samples` samples.
  cudaError_t adam_step(uint32_t samples, cudaStream_t s);
  // The same with the sample count read on the device (min(*count,
  // capacity)) and the step counter kept there, so that it can be captured
  // in a CUDA graph.
  cudaError_t adam_step_device(const uint32_t* count, uint32_t capacity, cudaStream_t s);

  cudaError_t read_weights(float* host, cudaStream_t s);
  cudaError_t write_weights(const float* host, cudaStream_t s);
  uint32_t error_flag(cudaStream_t s);

  CacheNet net() const;
  CacheGrid grid() const { return grid_; }
  float* master() const { return master_; }

 private:
  cudaError_t pack(cudaStream_t s);
  cudaError_t adam_kernels(cudaStream_t s);

  CacheConfig config_;
  CacheGrid grid_{};
  float* master_ = nullptr;     // FP32 weights
  float* adam_m_ = nullptr;     // moments of weights, then of the grid
  float* adam_v_ = nullptr;
  float* grid_master_ = nullptr;  // FP32 grid features
  uint4* operands_ = nullptr;   // forward then backward images
  float* grad_ = nullptr;
  float* loss_ = nullptr;
  uint32_t* error_ = nullptr;
  float* adam_consts_ = nullptr;  // device: step count, bias corrections, scale
  size_t grid_entries_ = 0;
};

}  // namespace lotus
