// SPDX-License-Identifier: Apache-2.0
// On-device BVH construction: a linear BVH (Karras, "Maximizing Parallelism
// in the Construction of BVHs, Octrees, and k-d Trees", HPG 2012) over
// 63-bit Morton codes of the primitives' centroids, sorted by CUB's radix
// sort, with bounds fitted bottom-up. It replaces the driver's BLAS/TLAS
// builds (backend/vulkan/gpu_scene.cpp:1899-1950, 2240-2322 in
// hydra-lotus).
#include "bvh_build.cuh"

#include <cub/device/device_radix_sort.cuh>

namespace lotus {

namespace {

constexpr int kBuildBlock = 256;

__device__ __forceinline__ uint32_t ordered(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float unordered(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// Triangle boxes in object space from the geometry's positions.
__global__ void k_triangle_boxes(const float* __restrict__ positions,
    const uint32_t* __restrict__ triangles, uint32_t n, float4* __restrict__ lo,
    float4* __restrict__ hi, uint32_t* __restrict__ centroid_bounds) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float l[3] = {kFloatMax, kFloatMax, kFloatMax}, h[3] = {-kFloatMax, -kFloatMax, -kFloatMax};
  for (int k = 0; k < 3; ++k) {
    const uint32_t v = triangles[3 * i + k];
    for (int a = 0; a < 3; ++a) {
      const float p = positions[3 * (size_t)v + a];
      l[a] = fminf(l[a], p);
      h[a] = fmaxf(h[a], p);
    }
  }
  lo[i] = make_float4(l[0], l[1], l[2], 0.0f);
  hi[i] = make_float4(h[0], h[1], h[2], 0.0f);
  for (int a = 0; a < 3; ++a) {
    const float c = 0.5f * (l[a] + h[a]);
    atomicMin(&centroid_bounds[a], ordered(c));
    atomicMax(&centroid_bounds[3 + a], ordered(c));
  }
}

// Instance world boxes: the BLAS root box's corners through
// world_from_object, widened by a relative margin.
__global__ void k_instance_boxes(const InstanceShading* __restrict__ shade,
    const InstanceTraversal* __restrict__ trav, const BvhNode* __restrict__ blas, uint32_t n,
    float4* __restrict__ lo, float4* __restrict__ hi, uint32_t* __restrict__ centroid_bounds) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float l[3] = {kFloatMax, kFloatMax, kFloatMax}, h[3] = {-kFloatMax, -kFloatMax, -kFloatMax};
  const uint32_t root = trav[i].blas_root;
  if (root != (uint32_t)kEmptyChild) {
    const BvhNode nd = blas[root];
    float bl[3] = {nd.x.x, nd.y.x, nd.z.x}, bh[3] = {nd.x.y, nd.y.y, nd.z.y};
    if (nd.c.y != kEmptyChild) {
      bl[0] = fminf(bl[0], nd.x.z); bl[1] = fminf(bl[1], nd.y.z); bl[2] = fminf(bl[2], nd.z.z);
      bh[0] = fmaxf(bh[0], nd.x.w); bh[1] = fmaxf(bh[1], nd.y.w); bh[2] = fmaxf(bh[2], nd.z.w);
    }
    const InstanceShading s = shade[i];
    for (int corner = 0; corner < 8; ++corner) {
      const F3 c = V((corner & 1) ? bh[0] : bl[0], (corner & 2) ? bh[1] : bl[1],
          (corner & 4) ? bh[2] : bl[2]);
      const F3 w = row_point(s.m, c);
      l[0] = fminf(l[0], w.x); l[1] = fminf(l[1], w.y); l[2] = fminf(l[2], w.z);
      h[0] = fmaxf(h[0], w.x); h[1] = fmaxf(h[1], w.y); h[2] = fmaxf(h[2], w.z);
    }
    for (int a = 0; a < 3; ++a) {
      const float pad = 1e-6f * fmaxf(fabsf(l[a]), fabsf(h[a])) + 1e-7f;
      l[a] -= pad;
      h[a] += pad;
    }
  } else {
    // An empty instance: a point box that no ray enters deeply.
    for (int a = 0; a < 3; ++a) l[a] = h[a] = 0.0f;
  }
  lo[i] = make_float4(l[0], l[1], l[2], 0.0f);
  hi[i] = make_float4(h[0], h[1], h[2], 0.0f);
  for (int a = 0; a < 3; ++a) {
    const float c = 0.5f * (l[a] + h[a]);
    atomicMin(&centroid_bounds[a], ordered(c));
    atomicMax(&centroid_bounds[3 + a], ordered(c));
  }
}

__device__ __forceinline__ uint64_t spread21(uint64_t x) {
  x &= 0x1FFFFFull;
  x = (x | (x << 32)) & 0x1F00000000FFFFull;
  x = (x | (x << 16)) & 0x1F0000FF0000FFull;
  x = (x | (x << 8)) & 0x100F00F00F00F00Full;
  x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

__global__ void k_morton(const float4* __restrict__ lo, const float4* __restrict__ hi, uint32_t n,
    const uint32_t* __restrict__ cb, uint64_t* __restrict__ keys, uint32_t* __restrict__ values) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float l[3] = {lo[i].x, lo[i].y, lo[i].z}, h[3] = {hi[i].x, hi[i].y, hi[i].z};
  uint64_t q[3];
  for (int a = 0; a < 3; ++a) {
    const float cmin = unordered(cb[a]), cmax = unordered(cb[3 + a]);
    const float c = 0.5f * (l[a] + h[a]);
    const float extent = cmax - cmin;
    float t = extent > 0.0f ? (c - cmin) / extent : 0.5f;
    t = fminf(fmaxf(t, 0.0f), 1.0f);
    q[a] = (uint64_t)fminf(t * 2097152.0f, 2097151.0f);
  }
  keys[i] = spread21(q[0]) | (spread21(q[1]) << 1) | (spread21(q[2]) << 2);
  values[i] = i;
}

__device__ __forceinline__ int delta(const uint64_t* __restrict__ keys, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  const uint64_t a = keys[i], b = keys[j];
  if (a == b) return 64 + __clz((uint32_t)i ^ (uint32_t)j);
  return __clzll(a ^ b);
}

// Karras's hierarchy: internal node i's children. Leaves are encoded as
// (leaf | kLeafBit).
constexpr uint32_t kLeafBit = 0x80000000u;

__global__ void k_karras(const uint64_t* __restrict__ keys, int n, uint32_t* __restrict__ left,
    uint32_t* __restrict__ right, uint32_t* __restrict__ parent_internal,
    uint32_t* __restrict__ parent_leaf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = delta(keys, n, i, i - d);
  int lmax = 2;
  while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = delta(keys, n, i, j);
  int s = 0;
  int t = l;
  do {
    t = (t + 1) >> 1;
    if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  const int gamma = i + s * d + min(d, 0);
  const uint32_t lc = (min(i, j) == gamma) ? ((uint32_t)gamma | kLeafBit) : (uint32_t)gamma;
  const uint32_t rc = (max(i, j) == gamma + 1) ? ((uint32_t)(gamma + 1) | kLeafBit) : (uint32_t)(gamma + 1);
  left[i] = lc;
  right[i] = rc;
  if (lc & kLeafBit) parent_leaf[lc & ~kLeafBit] = (uint32_t)i; else parent_internal[lc] = (uint32_t)i;
  if (rc & kLeafBit) parent_leaf[rc & ~kLeafBit] = (uint32_t)i; else parent_internal[rc] = (uint32_t)i;
}

// Bottom-up bounds: the second child to arrive at a node fits it and
// carries on to its parent.
__global__ void k_fit(const uint32_t* __restrict__ values, const float4* __restrict__ plo,
    const float4* __restrict__ phi, int n, const uint32_t* __restrict__ left,
    const uint32_t* __restrict__ right, const uint32_t* __restrict__ parent_internal,
    const uint32_t* __restrict__ parent_leaf, float4* nlo, float4* nhi, uint32_t* flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t node = parent_leaf[i];
  // A tree over n < 2^31 primitives with 63-bit keys and index tie-breaks
  // is at most 96 levels deep; the bound only guards against corrupt input.
  for (int level = 0; level < 256; ++level) {
    __threadfence();
    if (atomicAdd(&flags[node], 1u) == 0) return;
    __threadfence();
    float4 l[2], h[2];
    const uint32_t ch[2] = {left[node], right[node]};
    for (int k = 0; k < 2; ++k) {
      if (ch[k] & kLeafBit) {
        const uint32_t p = values[ch[k] & ~kLeafBit];
        l[k] = plo[p];
        h[k] = phi[p];
      } else {
        l[k] = __ldcg(&nlo[ch[k]]);
        h[k] = __ldcg(&nhi[ch[k]]);
      }
    }
    nlo[node] = make_float4(fminf(l[0].x, l[1].x), fminf(l[0].y, l[1].y), fminf(l[0].z, l[1].z), 0.0f);
    nhi[node] = make_float4(fmaxf(h[0].x, h[1].x), fmaxf(h[0].y, h[1].y), fmaxf(h[0].z, h[1].z), 0.0f);
    if (node == 0) return;
    node = parent_internal[node];
  }
}

// The 64-byte nodes. Child leaves point into the primitive pool at
// `leaf_base` + sorted position (BLAS), or at the sorted value itself (TLAS).
__global__ void k_write_nodes(const uint32_t* __restrict__ values, const float4* __restrict__ plo,
    const float4* __restrict__ phi, int n, const uint32_t* __restrict__ left,
    const uint32_t* __restrict__ right, const float4* __restrict__ nlo,
    const float4* __restrict__ nhi, BvhNode* __restrict__ out, uint32_t node_base,
    uint32_t leaf_base, int leaves_are_values) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const uint32_t ch[2] = {left[i], right[i]};
  float4 l[2], h[2];
  int32_t c[2];
  for (int k = 0; k < 2; ++k) {
    if (ch[k] & kLeafBit) {
      const uint32_t pos = ch[k] & ~kLeafBit;
      const uint32_t p = values[pos];
      l[k] = plo[p];
      h[k] = phi[p];
      c[k] = ~(int32_t)(leaves_are_values ? p : leaf_base + pos);
    } else {
      l[k] = nlo[ch[k]];
      h[k] = nhi[ch[k]];
      c[k] = (int32_t)(node_base + ch[k]);
    }
  }
  BvhNode nd;
  nd.x = make_float4(l[0].x, h[0].x, l[1].x, h[1].x);
  nd.y = make_float4(l[0].y, h[0].y, l[1].y, h[1].y);
  nd.z = make_float4(l[0].z, h[0].z, l[1].z, h[1].z);
  nd.c = make_int4(c[0], c[1], 1, 1);
  out[node_base + i] = nd;
}

// A one-primitive BVH: a root with one leaf child and an empty one.
__global__ void k_single_root(const float4* __restrict__ plo, const float4* __restrict__ phi,
    BvhNode* __restrict__ out, uint32_t node_base, uint32_t leaf_base, int leaves_are_values) {
  BvhNode nd;
  const float4 l = plo[0], h = phi[0];
  nd.x = make_float4(l.x, h.x, 0.0f, 0.0f);
  nd.y = make_float4(l.y, h.y, 0.0f, 0.0f);
  nd.z = make_float4(l.z, h.z, 0.0f, 0.0f);
  nd.c = make_int4(~(int32_t)(leaves_are_values ? 0u : leaf_base), kEmptyChild, 1, 0);
  out[node_base] = nd;
}

// The leaf-ordered triangle pool: three object-space corners, the original
// primitive index in the first corner's w.
__global__ void k_write_triangles(const uint32_t* __restrict__ values,
    const float* __restrict__ positions, const uint32_t* __restrict__ triangles, uint32_t n,
    float4* __restrict__ pool, uint32_t base) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = values[i];
  float4* out = pool + 3 * (size_t)(base + i);
  for (int k = 0; k < 3; ++k) {
    const uint32_t v = triangles[3 * (size_t)p + k];
    out[k] = make_float4(positions[3 * (size_t)v], positions[3 * (size_t)v + 1],
        positions[3 * (size_t)v + 2], k == 0 ? __uint_as_float(p) : 0.0f);
  }
}

inline uint32_t blocks(uint64_t n) { return (uint32_t)((n + kBuildBlock - 1) / kBuildBlock); }

}  // namespace

cudaError_t BvhBuilder::reserve(uint32_t n, cudaStream_t stream) {
  if (n <= capacity_) return cudaSuccess;
  release();
  cudaError_t e;
  const size_t nn = n;
  auto alloc = [&](void** p, size_t bytes) {
    if ((e = cudaMalloc(p, bytes)) != cudaSuccess) return false;
    return true;
  };
  if (!alloc((void**)&keys_, nn * 8) || !alloc((void**)&keys_alt_, nn * 8) ||
      !alloc((void**)&values_, nn * 4) || !alloc((void**)&values_alt_, nn * 4) ||
      !alloc((void**)&plo_, nn * 16) || !alloc((void**)&phi_, nn * 16) ||
      !alloc((void**)&nlo_, nn * 16) || !alloc((void**)&nhi_, nn * 16) ||
      !alloc((void**)&left_, nn * 4) || !alloc((void**)&right_, nn * 4) ||
      !alloc((void**)&parent_internal_, nn * 4) || !alloc((void**)&parent_leaf_, nn * 4) ||
      !alloc((void**)&flags_, nn * 4) || !alloc((void**)&bounds_, 6 * 4))
    return e;
  size_t temp = 0;
  cub::DoubleBuffer<uint64_t> k(keys_, keys_alt_);
  cub::DoubleBuffer<uint32_t> v(values_, values_alt_);
  cub::DeviceRadixSort::SortPairs(nullptr, temp, k, v, (int)n, 0, 63, stream);
  if (!alloc(&temp_, temp)) return e;
  temp_bytes_ = temp;
  capacity_ = n;
  return cudaSuccess;
}

void BvhBuilder::release() {
  void* ptrs[] = {keys_, keys_alt_, values_, values_alt_, plo_, phi_, nlo_, nhi_, left_, right_,
      parent_internal_, parent_leaf_, flags_, bounds_, temp_};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  keys_ = keys_alt_ = nullptr;
  values_ = values_alt_ = nullptr;
  plo_ = phi_ = nlo_ = nhi_ = nullptr;
  left_ = right_ = parent_internal_ = parent_leaf_ = flags_ = bounds_ = nullptr;
  temp_ = nullptr;
  capacity_ = 0;
  temp_bytes_ = 0;
}

cudaError_t BvhBuilder::build_common(uint32_t n, BvhNode* nodes, uint32_t node_base,
    uint32_t leaf_base, bool leaves_are_values, cudaStream_t stream, const uint32_t** sorted) {
  k_morton<<<blocks(n), kBuildBlock, 0, stream>>>(plo_, phi_, n, bounds_, keys_, values_);
  cub::DoubleBuffer<uint64_t> k(keys_, keys_alt_);
  cub::DoubleBuffer<uint32_t> v(values_, values_alt_);
  size_t temp = temp_bytes_;
  cudaError_t e = cub::DeviceRadixSort::SortPairs(temp_, temp, k, v, (int)n, 0, 63, stream);
  if (e != cudaSuccess) return e;
  const uint64_t* skeys = k.Current();
  const uint32_t* svalues = v.Current();
  *sorted = svalues;
  if (n == 1) {
    k_single_root<<<1, 1, 0, stream>>>(plo_, phi_, nodes, node_base, leaf_base, leaves_are_values);
    return cudaGetLastError();
  }
  k_karras<<<blocks(n - 1), kBuildBlock, 0, stream>>>(skeys, (int)n, left_, right_,
      parent_internal_, parent_leaf_);
  cudaMemsetAsync(flags_, 0, sizeof(uint32_t) * n, stream);
  k_fit<<<blocks(n), kBuildBlock, 0, stream>>>(svalues, plo_, phi_, (int)n, left_, right_,
      parent_internal_, parent_leaf_, nlo_, nhi_, flags_);
  k_write_nodes<<<blocks(n - 1), kBuildBlock, 0, stream>>>(svalues, plo_, phi_, (int)n, left_,
      right_, nlo_, nhi_, nodes, node_base, leaf_base, leaves_are_values ? 1 : 0);
  return cudaGetLastError();
}

static void init_bounds(uint32_t* bounds, cudaStream_t stream) {
  const uint32_t init[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
  cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, stream);
}

cudaError_t BvhBuilder::build_triangles(const float* positions, const uint32_t* triangles,
    uint32_t n, BvhNode* nodes, uint32_t node_base, float4* tri_pool, uint32_t tri_base,
    cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  cudaError_t e = reserve(n, stream);
  if (e != cudaSuccess) return e;
  init_bounds(bounds_, stream);
  k_triangle_boxes<<<blocks(n), kBuildBlock, 0, stream>>>(positions, triangles, n, plo_, phi_, bounds_);
  const uint32_t* sorted = nullptr;
  if ((e = build_common(n, nodes, node_base, tri_base, false, stream, &sorted)) != cudaSuccess) return e;
  k_write_triangles<<<blocks(n), kBuildBlock, 0, stream>>>(sorted, positions, triangles, n, tri_pool, tri_base);
  return cudaGetLastError();
}

cudaError_t BvhBuilder::build_instances(const InstanceShading* shade,
    const InstanceTraversal* trav, const BvhNode* blas, uint32_t n, BvhNode* nodes,
    cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  cudaError_t e = reserve(n, stream);
  if (e != cudaSuccess) return e;
  init_bounds(bounds_, stream);
  k_instance_boxes<<<blocks(n), kBuildBlock, 0, stream>>>(shade, trav, blas, n, plo_, phi_, bounds_);
  const uint32_t* sorted = nullptr;
  return build_common(n, nodes, 0, 0, true, stream, &sorted);
}

}  // namespace lotus
