// SPDX-License-Identifier: Apache-2.0
// On-device BVH construction, replacing the driver's BLAS/TLAS builds. Two
// builders: a binned-SAH builder that runs one BVH per CTA (all of a
// scene's BLASes in one launch, and the TLAS), and, for meshes too large
// for one CTA, a linear BVH (Karras, "Maximizing Parallelism in the
// Construction of BVHs, Octrees, and k-d Trees", HPG 2012) over 63-bit
// Morton codes of the primitives' centroids, sorted by CUB's radix sort,
// with bounds fitted bottom-up. The reference's builds are (backend/vulkan/gpu_scene.cpp:1899-1950, 2240-2322 in
// hydra-lotus).
#include "bvh_build.cuh"

#include <cub/block/block_scan.cuh>
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
// Folds a warp's primitive centroids into the centroid bounds with one
// atomic per bound (lanes without a primitive add the identities); every
// lane of the warp takes part.
__device__ __forceinline__ void warp_centroid_bounds(uint32_t* bounds, bool valid, const float* l,
    const float* h) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const uint32_t o = ordered(0.5f * (l[a] + h[a]));
    const uint32_t lo = __reduce_min_sync(0xFFFFFFFFu, valid ? o : 0xFFFFFFFFu);
    const uint32_t hi = __reduce_max_sync(0xFFFFFFFFu, valid ? o : 0u);
    if ((threadIdx.x & 31u) == 0) {
      atomicMin(&bounds[a], lo);
      atomicMax(&bounds[3 + a], hi);
    }
  }
}

__global__ void k_triangle_boxes(const float* __restrict__ positions,
    const uint32_t* __restrict__ triangles, uint32_t n, float4* __restrict__ lo,
    float4* __restrict__ hi, uint32_t* __restrict__ centroid_bounds) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  float l[3] = {kFloatMax, kFloatMax, kFloatMax}, h[3] = {-kFloatMax, -kFloatMax, -kFloatMax};
  if (valid) {
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
  }
  warp_centroid_bounds(centroid_bounds, valid, l, h);
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
  float4* out = pool + kTriStride * (size_t)(base + i);
  for (int k = 0; k < 3; ++k) {
    const uint32_t v = triangles[3 * (size_t)p + k];
    out[k] = make_float4(positions[3 * (size_t)v], positions[3 * (size_t)v + 1],
        positions[3 * (size_t)v + 2], k == 0 ? __uint_as_float(p) : 0.0f);
  }
  out[3] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}


// ---------------------------------------------------------------------------
// Binned-SAH builder: one CTA builds one BVH top-down (Wald, "On fast
// Construction of SAH-based Bounding Volume Hierarchies", 2007), binning
// centroids into 16 bins per axis in shared memory and partitioning the
// primitive indices with a block-wide scan. Every BVH of a batch builds in
// its own CTA, so a scene's BLASes build concurrently across the SMs.

constexpr int kSahBlock = 256;
constexpr int kSahBins = 16;
constexpr int kSahStack = 128;

struct SahJob {
  uint32_t prim_offset;  // first primitive in the batch's arrays
  uint32_t count;
  uint32_t node_base;    // first node slot
  uint32_t leaf_base;    // first triangle-pool slot (BLAS)
  uint32_t leaf_size;    // most primitives per leaf
  uint32_t leaves_are_values;  // TLAS: leaves hold the primitive index itself
};

struct SahShared {
  uint32_t bin_count[3][kSahBins];
  uint32_t bin_lo[3][kSahBins][3];
  uint32_t bin_hi[3][kSahBins][3];
  uint32_t cb[6];        // centroid bounds (ordered)
  uint32_t nb[6];        // node bounds (ordered)
  uint32_t stack_begin[kSahStack], stack_end[kSahStack], stack_node[kSahStack];
  int sp;
  uint32_t next_node;
  uint32_t begin, end, node;
  int best_axis, best_split;
  float best_cost[3];
  int split_at[3];
  uint32_t left_total;
  uint32_t error;
  uint32_t done;
};

__global__ void __launch_bounds__(kSahBlock) k_sah_build(const SahJob* __restrict__ jobs,
    const float4* __restrict__ plo, const float4* __restrict__ phi, uint32_t* __restrict__ idx,
    uint32_t* __restrict__ scratch, BvhNode* __restrict__ nodes, uint32_t* __restrict__ errors) {
  using BlockScan = cub::BlockScan<uint32_t, kSahBlock>;
  __shared__ typename BlockScan::TempStorage scan_storage;
  __shared__ SahShared sh;
  const SahJob job = jobs[blockIdx.x];
  const uint32_t tid = threadIdx.x;
  uint32_t* index = idx + job.prim_offset;
  uint32_t* tmp = scratch + job.prim_offset;
  if (job.count == 0) return;
  if (tid == 0) {
    sh.sp = 0;
    sh.next_node = 1;
    sh.error = 0;
    sh.stack_begin[0] = 0;
    sh.stack_end[0] = job.count;
    sh.stack_node[0] = 0;
    sh.sp = 1;
  }
  __syncthreads();
  // Small sets: one leaf under the root, its second child empty.
  if (job.count <= job.leaf_size) {
    if (tid < 6) sh.nb[tid] = tid < 3 ? 0xFFFFFFFFu : 0u;
    __syncthreads();
    for (uint32_t i = tid; i < job.count; i += blockDim.x) {
      const float4 l = plo[job.prim_offset + index[i]], h = phi[job.prim_offset + index[i]];
      atomicMin(&sh.nb[0], ordered(l.x)); atomicMin(&sh.nb[1], ordered(l.y)); atomicMin(&sh.nb[2], ordered(l.z));
      atomicMax(&sh.nb[3], ordered(h.x)); atomicMax(&sh.nb[4], ordered(h.y)); atomicMax(&sh.nb[5], ordered(h.z));
    }
    __syncthreads();
    if (tid == 0) {
      BvhNode nd;
      nd.x = make_float4(unordered(sh.nb[0]), unordered(sh.nb[3]), 0.0f, 0.0f);
      nd.y = make_float4(unordered(sh.nb[1]), unordered(sh.nb[4]), 0.0f, 0.0f);
      nd.z = make_float4(unordered(sh.nb[2]), unordered(sh.nb[5]), 0.0f, 0.0f);
      const int32_t leaf = job.leaves_are_values ? ~(int32_t)index[0] : ~(int32_t)job.leaf_base;
      nd.c = make_int4(leaf, kEmptyChild, (int32_t)job.count, 0);
      nodes[job.node_base] = nd;
    }
    return;
  }
  for (int guard = 0; guard < (int)(2 * job.count + 8); ++guard) {
    // Thread 0 pops the next range; the barrier publishes it (and orders
    // the pop after every thread's use of the previous node's state).
    if (tid == 0) {
      sh.done = sh.sp == 0 ? 1u : 0u;
      if (sh.sp > 0) {
        --sh.sp;
        sh.begin = sh.stack_begin[sh.sp];
        sh.end = sh.stack_end[sh.sp];
        sh.node = sh.stack_node[sh.sp];
      }
    }
    __syncthreads();
    if (sh.done) break;
    if (tid < 6) sh.cb[tid] = tid < 3 ? 0xFFFFFFFFu : 0u;
    for (uint32_t k = tid; k < 3 * kSahBins; k += blockDim.x) {
      const uint32_t a = k / kSahBins, b = k % kSahBins;
      sh.bin_count[a][b] = 0;
      for (int c = 0; c < 3; ++c) {
        sh.bin_lo[a][b][c] = 0xFFFFFFFFu;
        sh.bin_hi[a][b][c] = 0u;
      }
    }
    __syncthreads();
    const uint32_t begin = sh.begin, end = sh.end;
    // Centroid bounds.
    for (uint32_t i = begin + tid; i < end; i += blockDim.x) {
      const uint32_t p = job.prim_offset + index[i];
      const float4 l = plo[p], h = phi[p];
      const float cx = 0.5f * (l.x + h.x), cy = 0.5f * (l.y + h.y), cz = 0.5f * (l.z + h.z);
      atomicMin(&sh.cb[0], ordered(cx)); atomicMin(&sh.cb[1], ordered(cy)); atomicMin(&sh.cb[2], ordered(cz));
      atomicMax(&sh.cb[3], ordered(cx)); atomicMax(&sh.cb[4], ordered(cy)); atomicMax(&sh.cb[5], ordered(cz));
    }
    __syncthreads();
    float cmin[3], scale[3];
    for (int a = 0; a < 3; ++a) {
      cmin[a] = unordered(sh.cb[a]);
      const float extent = unordered(sh.cb[3 + a]) - cmin[a];
      scale[a] = extent > 0.0f ? float(kSahBins) / extent : 0.0f;
    }
    // Binning on all three axes.
    for (uint32_t i = begin + tid; i < end; i += blockDim.x) {
      const uint32_t p = job.prim_offset + index[i];
      const float4 l = plo[p], h = phi[p];
      const float c[3] = {0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z)};
      for (int a = 0; a < 3; ++a) {
        const int b = min(kSahBins - 1, max(0, (int)((c[a] - cmin[a]) * scale[a])));
        atomicAdd(&sh.bin_count[a][b], 1u);
        atomicMin(&sh.bin_lo[a][b][0], ordered(l.x)); atomicMin(&sh.bin_lo[a][b][1], ordered(l.y));
        atomicMin(&sh.bin_lo[a][b][2], ordered(l.z));
        atomicMax(&sh.bin_hi[a][b][0], ordered(h.x)); atomicMax(&sh.bin_hi[a][b][1], ordered(h.y));
        atomicMax(&sh.bin_hi[a][b][2], ordered(h.z));
      }
    }
    __syncthreads();
    // The SAH sweep, one axis per thread.
    if (tid < 3) {
      const int a = tid;
      float best = INFINITY;
      int split = -1;
      if (scale[a] > 0.0f) {
        float right_area[kSahBins];
        uint32_t right_count[kSahBins];
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t cnt = 0;
        for (int b = kSahBins - 1; b > 0; --b) {
          if (sh.bin_count[a][b]) {
            for (int c = 0; c < 3; ++c) {
              lo[c] = fminf(lo[c], unordered(sh.bin_lo[a][b][c]));
              hi[c] = fmaxf(hi[c], unordered(sh.bin_hi[a][b][c]));
            }
          }
          cnt += sh.bin_count[a][b];
          const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
          right_area[b] = cnt ? 2.0f * (dx * dy + dy * dz + dz * dx) : 0.0f;
          right_count[b] = cnt;
        }
        lo[0] = lo[1] = lo[2] = INFINITY;
        hi[0] = hi[1] = hi[2] = -INFINITY;
        cnt = 0;
        for (int b = 0; b < kSahBins - 1; ++b) {
          if (sh.bin_count[a][b]) {
            for (int c = 0; c < 3; ++c) {
              lo[c] = fminf(lo[c], unordered(sh.bin_lo[a][b][c]));
              hi[c] = fmaxf(hi[c], unordered(sh.bin_hi[a][b][c]));
            }
          }
          cnt += sh.bin_count[a][b];
          if (cnt == 0 || right_count[b + 1] == 0) continue;
          const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
          const float cost = 2.0f * (dx * dy + dy * dz + dz * dx) * cnt + right_area[b + 1] * right_count[b + 1];
          if (cost < best) {
            best = cost;
            split = b;
          }
        }
      }
      sh.best_cost[a] = best;
      sh.split_at[a] = split;
    }
    __syncthreads();
    if (tid == 0) {
      int axis = -1;
      float best = INFINITY;
      for (int a = 0; a < 3; ++a)
        if (sh.split_at[a] >= 0 && sh.best_cost[a] < best) {
          best = sh.best_cost[a];
          axis = a;
        }
      sh.best_axis = axis;
      sh.best_split = axis >= 0 ? sh.split_at[axis] : -1;
    }
    __syncthreads();
    const int axis = sh.best_axis, split = sh.best_split;
    const uint32_t count = end - begin;
    uint32_t mid;
    if (axis < 0) {
      mid = begin + count / 2;  // coincident centroids: split the list
    } else {
      // Stable partition: lefts to the front of tmp's range, rights after.
      uint32_t left_base = 0;
      uint32_t left_total = 0;
      for (uint32_t t0 = begin; t0 < end; t0 += blockDim.x) {
        const uint32_t i = t0 + tid;
        uint32_t goes_left = 0;
        uint32_t v = 0;
        if (i < end) {
          v = index[i];
          const float4 l = plo[job.prim_offset + v], h = phi[job.prim_offset + v];
          const float c = 0.5f * ((&l.x)[axis] + (&h.x)[axis]);
          const int b = min(kSahBins - 1, max(0, (int)((c - cmin[axis]) * scale[axis])));
          goes_left = b <= split ? 1u : 0u;
        }
        uint32_t prefix, tile_total;
        BlockScan(scan_storage).ExclusiveSum(goes_left, prefix, tile_total);
        __syncthreads();
        if (i < end) {
          if (goes_left) tmp[begin + left_base + prefix] = v;
          else tmp[begin + (count - 1) - ((i - begin) - (left_base + prefix))] = v;
        }
        left_base += tile_total;
        left_total = left_base;
      }
      __syncthreads();
      // Rights were written back to front; copy both halves in order.
      for (uint32_t i = begin + tid; i < end; i += blockDim.x) {
        const uint32_t k = i - begin;
        index[i] = k < left_total ? tmp[i] : tmp[begin + (count - 1) - (k - left_total)];
      }
      mid = begin + left_total;
      if (mid == begin || mid == end) mid = begin + count / 2;
    }
    __syncthreads();
    // Children bounds: a reduction over each half.
    if (tid < 6) sh.nb[tid] = tid < 3 ? 0xFFFFFFFFu : 0u;
    if (tid < 6) sh.cb[tid] = tid < 3 ? 0xFFFFFFFFu : 0u;  // reused for the right child
    __syncthreads();
    for (uint32_t i = begin + tid; i < end; i += blockDim.x) {
      const float4 l = plo[job.prim_offset + index[i]], h = phi[job.prim_offset + index[i]];
      uint32_t* b = i < mid ? sh.nb : sh.cb;
      atomicMin(&b[0], ordered(l.x)); atomicMin(&b[1], ordered(l.y)); atomicMin(&b[2], ordered(l.z));
      atomicMax(&b[3], ordered(h.x)); atomicMax(&b[4], ordered(h.y)); atomicMax(&b[5], ordered(h.z));
    }
    __syncthreads();
    if (tid == 0) {
      const uint32_t ranges[2][2] = {{begin, mid}, {mid, end}};
      const uint32_t* bounds[2] = {sh.nb, sh.cb};
      int32_t child[2], ccount[2];
      for (int k = 0; k < 2; ++k) {
        const uint32_t n = ranges[k][1] - ranges[k][0];
        if (n <= job.leaf_size) {
          child[k] = job.leaves_are_values ? ~(int32_t)index[ranges[k][0]]
                                           : ~(int32_t)(job.leaf_base + ranges[k][0]);
          ccount[k] = (int32_t)n;
        } else {
          const uint32_t slot = sh.next_node++;
          if (sh.sp >= kSahStack || slot >= job.count) {
            sh.error = 1;
            child[k] = kEmptyChild;
            ccount[k] = 0;
            continue;
          }
          sh.stack_begin[sh.sp] = ranges[k][0];
          sh.stack_end[sh.sp] = ranges[k][1];
          sh.stack_node[sh.sp] = slot;
          ++sh.sp;
          child[k] = (int32_t)(job.node_base + slot);
          ccount[k] = 0;
        }
      }
      BvhNode nd;
      nd.x = make_float4(unordered(bounds[0][0]), unordered(bounds[0][3]), unordered(bounds[1][0]), unordered(bounds[1][3]));
      nd.y = make_float4(unordered(bounds[0][1]), unordered(bounds[0][4]), unordered(bounds[1][1]), unordered(bounds[1][4]));
      nd.z = make_float4(unordered(bounds[0][2]), unordered(bounds[0][5]), unordered(bounds[1][2]), unordered(bounds[1][5]));
      nd.c = make_int4(child[0], child[1], ccount[0], ccount[1]);
      nodes[job.node_base + sh.node] = nd;
    }
  }
  __syncthreads();
  if (tid == 0 && (sh.error || sh.sp != 0)) atomicAdd(errors, 1u);
}

// Triangle boxes of every geometry of a batch: primitive i of job j at
// prim_offset + i, its positions and triangles at the job's offsets.
__global__ void k_batch_triangle_boxes(const float* __restrict__ positions, const uint32_t* __restrict__ triangles,
    const uint64_t* __restrict__ vbase, const uint32_t* __restrict__ prim_job, const SahJob* __restrict__ jobs,
    uint32_t total, float4* __restrict__ lo, float4* __restrict__ hi, uint32_t* __restrict__ idx) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const uint32_t j = prim_job[g];
  const uint32_t local = g - jobs[j].prim_offset;
  const float* P = positions + 3 * vbase[j];
  float l[3] = {kFloatMax, kFloatMax, kFloatMax}, h[3] = {-kFloatMax, -kFloatMax, -kFloatMax};
  for (int k = 0; k < 3; ++k) {
    const uint32_t v = triangles[3 * (size_t)g + k];
    for (int a = 0; a < 3; ++a) {
      const float p = P[3 * (size_t)v + a];
      l[a] = fminf(l[a], p);
      h[a] = fmaxf(h[a], p);
    }
  }
  lo[g] = make_float4(l[0], l[1], l[2], 0.0f);
  hi[g] = make_float4(h[0], h[1], h[2], 0.0f);
  idx[g] = local;
}

// The leaf-ordered triangle pool of a batch: pool slot leaf_base + i holds
// triangle idx[prim_offset + i] of job j.
__global__ void k_batch_write_triangles(const float* __restrict__ positions, const uint32_t* __restrict__ triangles,
    const uint64_t* __restrict__ vbase, const uint64_t* __restrict__ tbase, const uint32_t* __restrict__ prim_job,
    const SahJob* __restrict__ jobs, const uint32_t* __restrict__ idx, uint32_t total, float4* __restrict__ pool) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const uint32_t j = prim_job[g];
  const SahJob job = jobs[j];
  const uint32_t local = g - job.prim_offset;
  const uint32_t p = idx[g];
  const float* P = positions + 3 * vbase[j];
  const uint32_t* T = triangles + 3 * tbase[j];
  float4* out = pool + kTriStride * (size_t)(job.leaf_base + local);
  for (int k = 0; k < 3; ++k) {
    const uint32_t v = T[3 * (size_t)p + k];
    out[k] = make_float4(P[3 * (size_t)v], P[3 * (size_t)v + 1], P[3 * (size_t)v + 2],
        k == 0 ? __uint_as_float(p) : 0.0f);
  }
  out[3] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// The 4-wide nodes: wide node i holds binary node i's subtree cut at four
// children, opening the interior child with the largest surface area until
// there are four (the greedy collapse of Wald et al., "Getting Rid of
// Packets", 2008). Every binary node gets a wide node at its own index, so
// the collapse is one independent thread per node; a wide node whose binary
// node was opened by its parent is never referenced.
__global__ void k_collapse4(const BvhNode* __restrict__ bin, uint32_t first, uint32_t count, uint32_t n,
    Bvh4Node* __restrict__ wide, int leaves_are_instances) {
  const uint32_t offset = blockIdx.x * blockDim.x + threadIdx.x;
  if (offset >= count) return;
  const uint32_t i = first + offset;
  if (i >= n) return;
  float lo[4][3], hi[4][3];
  int32_t ref[4], cnt[4];
  int k = 0;
  auto take = [&](const BvhNode& nd) {
    const float bx[4] = {nd.x.x, nd.x.y, nd.x.z, nd.x.w}, by[4] = {nd.y.x, nd.y.y, nd.y.z, nd.y.w},
                bz[4] = {nd.z.x, nd.z.y, nd.z.z, nd.z.w};
    const int32_t c[2] = {nd.c.x, nd.c.y}, m[2] = {nd.c.z, nd.c.w};
    for (int j = 0; j < 2; ++j) {
      if (c[j] == kEmptyChild || k >= 4) continue;
      lo[k][0] = bx[2 * j]; hi[k][0] = bx[2 * j + 1];
      lo[k][1] = by[2 * j]; hi[k][1] = by[2 * j + 1];
      lo[k][2] = bz[2 * j]; hi[k][2] = bz[2 * j + 1];
      ref[k] = c[j];
      cnt[k] = m[j];
      ++k;
    }
  };
  take(bin[i]);
  for (int round = 0; round < 2 && k < 4; ++round) {
    int open = -1;
    float best = -1.0f;
    for (int j = 0; j < k; ++j) {
      if (ref[j] < 0 || (uint32_t)ref[j] >= n) continue;
      const float dx = hi[j][0] - lo[j][0], dy = hi[j][1] - lo[j][1], dz = hi[j][2] - lo[j][2];
      const float area = dx * dy + dy * dz + dz * dx;
      if (area > best) {
        best = area;
        open = j;
      }
    }
    if (open < 0) break;
    const BvhNode child = bin[ref[open]];
    // Replace the opened child by the last one, then append its children.
    --k;
    for (int a = 0; a < 3; ++a) {
      lo[open][a] = lo[k][a];
      hi[open][a] = hi[k][a];
    }
    ref[open] = ref[k];
    cnt[open] = cnt[k];
    take(child);
  }
  float ox[4], oX[4], oy[4], oY[4], oz[4], oZ[4];
  int32_t oc[4], on[4];
  for (int j = 0; j < 4; ++j) {
    const bool used = j < k;
    ox[j] = used ? lo[j][0] : 0.0f; oX[j] = used ? hi[j][0] : 0.0f;
    oy[j] = used ? lo[j][1] : 0.0f; oY[j] = used ? hi[j][1] : 0.0f;
    oz[j] = used ? lo[j][2] : 0.0f; oZ[j] = used ? hi[j][2] : 0.0f;
    oc[j] = used ? ref[j] : kEmptyChild;
    on[j] = used ? cnt[j] : 0;
    if (used && ref[j] < 0 && !leaves_are_instances) {
      // BLAS leaf: the count goes into the reference's low bits.
      const uint32_t first = ~(uint32_t)ref[j];
      const uint32_t count = (uint32_t)min(max(cnt[j], 1), 1 << kLeafCountBits);
      oc[j] = (int32_t)~((first << kLeafCountBits) | (count - 1u));
    }
  }
  Bvh4Node w;
  w.lo_x = make_float4(ox[0], ox[1], ox[2], ox[3]); w.hi_x = make_float4(oX[0], oX[1], oX[2], oX[3]);
  w.lo_y = make_float4(oy[0], oy[1], oy[2], oy[3]); w.hi_y = make_float4(oY[0], oY[1], oY[2], oY[3]);
  w.lo_z = make_float4(oz[0], oz[1], oz[2], oz[3]); w.hi_z = make_float4(oZ[0], oZ[1], oZ[2], oZ[3]);
  w.child = make_int4(oc[0], oc[1], oc[2], oc[3]);
  w.count = make_int4(on[0], on[1], on[2], on[3]);
  wide[i] = w;
}

// Refit after a point edit (the reference refits its BLAS there,
// backend/vulkan/gpu_scene.cpp:1899-1950 in hydra-lotus): the topology is
// kept and the boxes follow the new positions. First the leaf-ordered
// triangle pool takes the new corners (the primitive index each record
// keeps in its first corner's w names its triangle).
__global__ void k_refit_triangles(const float* __restrict__ positions, const uint32_t* __restrict__ triangles,
    float4* __restrict__ pool, uint32_t tri_base, uint32_t count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  float4* rec = pool + kTriStride * (size_t)(tri_base + i);
  const uint32_t p = __float_as_uint(rec[0].w);
  for (int k = 0; k < 3; ++k) {
    const uint32_t v = triangles[3 * (size_t)p + k];
    rec[k] = make_float4(positions[3 * (size_t)v], positions[3 * (size_t)v + 1], positions[3 * (size_t)v + 2],
        k == 0 ? __uint_as_float(p) : 0.0f);
  }
}

// Each binary node's parent (the root, node_base, has none) and a cleared
// arrival count.
__global__ void k_refit_parents(const BvhNode* __restrict__ nodes, uint32_t node_base, uint32_t count,
    uint32_t* __restrict__ parent, uint32_t* __restrict__ arrivals) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int4 c = nodes[node_base + i].c;
  if (c.x >= 0 && c.x != kEmptyChild) parent[(uint32_t)c.x - node_base] = node_base + i;
  if (c.y >= 0 && c.y != kEmptyChild) parent[(uint32_t)c.y - node_base] = node_base + i;
  arrivals[i] = 0;
}

__device__ __forceinline__ void store_child_box(BvhNode* node, int slot, float4 lo, float4 hi) {
  float* x = reinterpret_cast<float*>(&node->x);
  float* y = reinterpret_cast<float*>(&node->y);
  float* z = reinterpret_cast<float*>(&node->z);
  x[2 * slot] = lo.x; x[2 * slot + 1] = hi.x;
  y[2 * slot] = lo.y; y[2 * slot + 1] = hi.y;
  z[2 * slot] = lo.z; z[2 * slot + 1] = hi.z;
}

// Bottom-up boxes: each node's thread boxes its leaf children's triangles
// into the node; a node is complete once all its non-empty children have
// arrived (its leaves, then each interior child as it completes), and the
// last arrival writes its box into its parent's slot and carries on there.
__global__ void k_refit_up(BvhNode* nodes, const float4* __restrict__ pool, uint32_t node_base, uint32_t count,
    const uint32_t* __restrict__ parent, uint32_t* arrivals) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint32_t node = node_base + i;
  int4 c = nodes[node].c;
  const int32_t ref[2] = {c.x, c.y};
  const int32_t cnt[2] = {c.z, c.w};
  uint32_t leaves = 0;
  for (int k = 0; k < 2; ++k) {
    if (ref[k] >= 0) continue;  // interior or empty
    const uint32_t first = ~(uint32_t)ref[k];
    float4 lo = make_float4(INFINITY, INFINITY, INFINITY, 0.0f), hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.0f);
    for (int t = 0; t < max(cnt[k], 1); ++t)
      for (int v = 0; v < 3; ++v) {
        const float4 p = pool[kTriStride * (size_t)(first + t) + v];
        lo = make_float4(fminf(lo.x, p.x), fminf(lo.y, p.y), fminf(lo.z, p.z), 0.0f);
        hi = make_float4(fmaxf(hi.x, p.x), fmaxf(hi.y, p.y), fmaxf(hi.z, p.z), 0.0f);
      }
    store_child_box(&nodes[node], k, lo, hi);
    ++leaves;
  }
  if (leaves == 0) return;
  uint32_t arrived = leaves;
  // A tree over the scene's triangles is far shallower than 256 levels; the
  // bound only guards against corrupt input.
  for (int level = 0; level < 256; ++level) {
    __threadfence();
    const uint32_t before = atomicAdd(&arrivals[node - node_base], arrived);
    c = __ldcg(&nodes[node].c);
    const uint32_t needed = (c.x != kEmptyChild ? 1u : 0u) + (c.y != kEmptyChild ? 1u : 0u);
    if (before + arrived < needed) return;
    __threadfence();
    if (node == node_base) return;
    const float4 bx = __ldcg(&nodes[node].x), by = __ldcg(&nodes[node].y), bz = __ldcg(&nodes[node].z);
    float4 lo, hi;
    if (c.y == kEmptyChild) {
      lo = make_float4(bx.x, by.x, bz.x, 0.0f);
      hi = make_float4(bx.y, by.y, bz.y, 0.0f);
    } else {
      lo = make_float4(fminf(bx.x, bx.z), fminf(by.x, by.z), fminf(bz.x, bz.z), 0.0f);
      hi = make_float4(fmaxf(bx.y, bx.w), fmaxf(by.y, by.w), fmaxf(bz.y, bz.w), 0.0f);
    }
    const uint32_t up = parent[node - node_base];
    const int4 pc = __ldcg(&nodes[up].c);
    store_child_box(&nodes[up], pc.x == (int32_t)node ? 0 : 1, lo, hi);
    node = up;
    arrived = 1;
  }
}

inline uint32_t blocks(uint64_t n) { return (uint32_t)((n + kBuildBlock - 1) / kBuildBlock); }

}  // namespace

cudaError_t BvhBuilder::refit_triangles(const float* positions, const uint32_t* triangles, uint32_t n,
    BvhNode* nodes, uint32_t node_base, float4* tri_pool, uint32_t tri_base, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  cudaError_t e = reserve(n, stream);
  if (e != cudaSuccess) return e;
  const uint32_t count = node_count(n);
  k_refit_triangles<<<blocks(n), kBuildBlock, 0, stream>>>(positions, triangles, tri_pool, tri_base, n);
  k_refit_parents<<<blocks(count), kBuildBlock, 0, stream>>>(nodes, node_base, count, parent_internal_, flags_);
  k_refit_up<<<blocks(count), kBuildBlock, 0, stream>>>(nodes, tri_pool, node_base, count, parent_internal_,
      flags_);
  return cudaGetLastError();
}

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

cudaError_t BvhBuilder::build_triangle_batch(const float* positions, const uint32_t* triangles,
    const std::vector<BatchGeometry>& geometries, BvhNode* nodes, float4* tri_pool, cudaStream_t stream,
    uint32_t leaf_size) {
  std::vector<SahJob> jobs;
  std::vector<uint64_t> vbase, tbase;
  uint32_t total = 0;
  for (const BatchGeometry& g : geometries) {
    if (g.count == 0) continue;
    SahJob j;
    j.prim_offset = total;
    j.count = g.count;
    j.node_base = g.node_base;
    j.leaf_base = g.tri_base;
    j.leaf_size = leaf_size;
    j.leaves_are_values = 0;
    jobs.push_back(j);
    vbase.push_back(g.vertex_offset);
    tbase.push_back(g.tri_base);
    total += g.count;
  }
  if (jobs.empty()) return cudaSuccess;
  std::vector<uint32_t> prim_job(total);
  for (uint32_t k = 0; k < jobs.size(); ++k)
    for (uint32_t i = 0; i < jobs[k].count; ++i) prim_job[jobs[k].prim_offset + i] = k;
  cudaError_t e = reserve(total, stream);
  if (e != cudaSuccess) return e;
  SahJob* d_jobs = nullptr;
  uint64_t* d_vbase = nullptr;
  uint64_t* d_tbase = nullptr;
  uint32_t* d_prim_job = nullptr;
  uint32_t* d_tris = nullptr;
  if ((e = cudaMalloc(&d_jobs, jobs.size() * sizeof(SahJob))) != cudaSuccess ||
      (e = cudaMalloc(&d_vbase, jobs.size() * 8)) != cudaSuccess ||
      (e = cudaMalloc(&d_tbase, jobs.size() * 8)) != cudaSuccess ||
      (e = cudaMalloc(&d_prim_job, (size_t)total * 4)) != cudaSuccess ||
      (e = cudaMalloc(&d_tris, (size_t)total * 12)) != cudaSuccess)
    return e;
  cudaMemcpyAsync(d_jobs, jobs.data(), jobs.size() * sizeof(SahJob), cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(d_vbase, vbase.data(), jobs.size() * 8, cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(d_tbase, tbase.data(), jobs.size() * 8, cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(d_prim_job, prim_job.data(), (size_t)total * 4, cudaMemcpyHostToDevice, stream);
  // Each job's triangles, gathered in batch order.
  for (size_t k = 0; k < jobs.size(); ++k)
    cudaMemcpyAsync(d_tris + 3 * (size_t)jobs[k].prim_offset, triangles + 3 * tbase[k], (size_t)jobs[k].count * 12,
        cudaMemcpyDeviceToDevice, stream);
  k_batch_triangle_boxes<<<blocks(total), kBuildBlock, 0, stream>>>(positions, d_tris, d_vbase, d_prim_job,
      d_jobs, total, plo_, phi_, values_);
  cudaMemsetAsync(flags_, 0, 4, stream);
  k_sah_build<<<(uint32_t)jobs.size(), kSahBlock, 0, stream>>>(d_jobs, plo_, phi_, values_, values_alt_, nodes,
      flags_);
  // The pool: leaf_base is the geometry's tri_base, and the batch's
  // triangles are addressed through the gathered copy.
  std::vector<uint64_t> zero(jobs.size());
  for (size_t k = 0; k < jobs.size(); ++k) zero[k] = jobs[k].prim_offset;
  cudaMemcpyAsync(d_tbase, zero.data(), jobs.size() * 8, cudaMemcpyHostToDevice, stream);
  k_batch_write_triangles<<<blocks(total), kBuildBlock, 0, stream>>>(positions, d_tris, d_vbase, d_tbase,
      d_prim_job, d_jobs, values_, total, tri_pool);
  uint32_t errors = 0;
  cudaMemcpyAsync(&errors, flags_, 4, cudaMemcpyDeviceToHost, stream);
  e = cudaStreamSynchronize(stream);
  cudaFree(d_jobs);
  cudaFree(d_vbase);
  cudaFree(d_tbase);
  cudaFree(d_prim_job);
  cudaFree(d_tris);
  if (e != cudaSuccess) return e;
  return errors ? cudaErrorUnknown : cudaSuccess;
}

cudaError_t BvhBuilder::build_instances_sah(const InstanceShading* shade, const InstanceTraversal* trav,
    const BvhNode* blas, uint32_t n, BvhNode* nodes, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  cudaError_t e = reserve(n, stream);
  if (e != cudaSuccess) return e;
  init_bounds(bounds_, stream);
  k_instance_boxes<<<blocks(n), kBuildBlock, 0, stream>>>(shade, trav, blas, n, plo_, phi_, bounds_);
  std::vector<uint32_t> iota(n);
  for (uint32_t i = 0; i < n; ++i) iota[i] = i;
  cudaMemcpyAsync(values_, iota.data(), (size_t)n * 4, cudaMemcpyHostToDevice, stream);
  SahJob job{0, n, 0, 0, 1, 1};
  SahJob* d_job = nullptr;
  if ((e = cudaMalloc(&d_job, sizeof(SahJob))) != cudaSuccess) return e;
  cudaMemcpyAsync(d_job, &job, sizeof(job), cudaMemcpyHostToDevice, stream);
  cudaMemsetAsync(flags_, 0, 4, stream);
  k_sah_build<<<1, kSahBlock, 0, stream>>>(d_job, plo_, phi_, values_, values_alt_, nodes, flags_);
  uint32_t errors = 0;
  cudaMemcpyAsync(&errors, flags_, 4, cudaMemcpyDeviceToHost, stream);
  e = cudaStreamSynchronize(stream);
  cudaFree(d_job);
  if (e != cudaSuccess) return e;
  return errors ? cudaErrorUnknown : cudaSuccess;
}

cudaError_t BvhBuilder::collapse(const BvhNode* binary, uint32_t n, Bvh4Node* wide, bool leaves_are_instances,
    cudaStream_t stream) {
  return collapse_range(binary, 0, n, n, wide, leaves_are_instances, stream);
}

cudaError_t BvhBuilder::collapse_range(const BvhNode* binary, uint32_t first, uint32_t count, uint32_t n,
    Bvh4Node* wide, bool leaves_are_instances, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  k_collapse4<<<blocks(count), kBuildBlock, 0, stream>>>(binary, first, count, n, wide,
      leaves_are_instances ? 1 : 0);
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
