// SPDX-License-Identifier: Apache-2.0
// On-device BVH builders: per-CTA binned SAH and LBVH (see bvh_build.cu).
#pragma once

#include <vector>

#include "scene.cuh"

namespace lotus {

// One geometry of a batched build: its triangles in the concatenated
// arrays and its slots in the node and triangle pools.
struct BatchGeometry {
  uint64_t vertex_offset;
  uint32_t tri_base;
  uint32_t count;
  uint32_t node_base;
};

// Geometries up to this many triangles build with the per-CTA binned-SAH
// builder; larger ones with the LBVH.
constexpr uint32_t kSahMaxTriangles = 65536;

// Scratch for building BVHs, grown to the largest primitive count seen. A
// BVH over n > 1 primitives has at most n - 1 nodes; over one, one.
class BvhBuilder {
 public:
  // Binned-SAH BLASes of many geometries in one launch (one CTA each).
  cudaError_t build_triangle_batch(const float* positions, const uint32_t* triangles,
      const std::vector<BatchGeometry>& geometries, BvhNode* nodes, float4* tri_pool, cudaStream_t stream,
      uint32_t leaf_size);
  // The binned-SAH TLAS (one instance per leaf).
  cudaError_t build_instances_sah(const InstanceShading* shade, const InstanceTraversal* trav,
      const BvhNode* blas, uint32_t n, BvhNode* nodes, cudaStream_t stream);
  ~BvhBuilder() { release(); }
  // One BLAS: nodes at nodes[node_base ...], leaf-ordered triangles at
  // tri_pool[kTriStride * tri_base ...]. Positions and triangles are device arrays.
  cudaError_t build_triangles(const float* positions, const uint32_t* triangles, uint32_t n,
      BvhNode* nodes, uint32_t node_base, float4* tri_pool, uint32_t tri_base,
      cudaStream_t stream);
  // Refits one BLAS built over the same triangles (a point edit): its
  // leaf-ordered triangle records take the new positions and its binary
  // nodes' boxes are recomputed bottom-up; the topology is kept.
  cudaError_t refit_triangles(const float* positions, const uint32_t* triangles, uint32_t n,
      BvhNode* nodes, uint32_t node_base, float4* tri_pool, uint32_t tri_base, cudaStream_t stream);
  // The TLAS over the instances' world boxes; leaves hold instance indices.
  cudaError_t build_instances(const InstanceShading* shade, const InstanceTraversal* trav,
      const BvhNode* blas, uint32_t n, BvhNode* nodes, cudaStream_t stream);
  // The 4-wide pool the traversal reads: wide[i] for every binary node i
  // (node references keep their meaning; BLAS leaves take their counts into
  // their references). One launch over the whole pool.
  static cudaError_t collapse(const BvhNode* binary, uint32_t n, Bvh4Node* wide, bool leaves_are_instances,
      cudaStream_t stream);
  // The same over binary nodes [first, first + count) of a pool of n (one
  // geometry's BLAS after it was rebuilt in place).
  static cudaError_t collapse_range(const BvhNode* binary, uint32_t first, uint32_t count, uint32_t n,
      Bvh4Node* wide, bool leaves_are_instances, cudaStream_t stream);
  void release();

  static uint32_t node_count(uint32_t n) { return n > 1 ? n - 1 : n; }

 private:
  cudaError_t reserve(uint32_t n, cudaStream_t stream);
  cudaError_t build_common(uint32_t n, BvhNode* nodes, uint32_t node_base, uint32_t leaf_base,
      bool leaves_are_values, cudaStream_t stream, const uint32_t** sorted);

  uint32_t capacity_ = 0;
  size_t temp_bytes_ = 0;
  uint64_t* keys_ = nullptr;
  uint64_t* keys_alt_ = nullptr;
  uint32_t* values_ = nullptr;
  uint32_t* values_alt_ = nullptr;
  float4* plo_ = nullptr;
  float4* phi_ = nullptr;
  float4* nlo_ = nullptr;
  float4* nhi_ = nullptr;
  uint32_t* left_ = nullptr;
  uint32_t* right_ = nullptr;
  uint32_t* parent_internal_ = nullptr;
  uint32_t* parent_leaf_ = nullptr;
  uint32_t* flags_ = nullptr;
  uint32_t* bounds_ = nullptr;
  void* temp_ = nullptr;
};

}  // namespace lotus
