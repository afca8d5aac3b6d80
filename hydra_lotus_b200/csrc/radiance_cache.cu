// SPDX-License-Identifier: Apache-2.0
// The radiance cache's kernels: the query encoding (hash grid, spherical
// harmonics), the fused MLP forward pass and the fused training pass
// (forward, relative-L2 loss, backward, weight and hash-grid gradients) on
// the tensor cores, and Adam. One CTA of 128 threads works on tiles of 128
// queries, one query per thread and per tensor-memory lane; all six layers
// run back to back out of shared memory, so a query's activations never
// leave the SM.
#include "radiance_cache.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "tcgen05.cuh"

namespace lotus {

namespace {

constexpr int kNetThreads = 128;
constexpr uint32_t kWaitPolls = 1u << 22;
constexpr uint32_t kTile = 16384;           // 128 x 64 BF16
constexpr uint32_t kNarrowTile = 4096;      // 128 x 16 BF16
// Tensor-memory columns of the training pass: the layer result, then the
// weight-gradient accumulators (64 columns each, 16 for the output layer).
constexpr uint32_t kTrainColumns = 512;

// Byte offset of layer l's tile in an operand image (8 KB per 64 x 64
// layer; the output layer's tile is 2 KB).
__host__ __device__ constexpr uint32_t layer_offset(int layer) { return (uint32_t)layer * 8192u; }
__host__ __device__ constexpr uint32_t grad_column(int layer) { return 64u + 64u * (uint32_t)layer; }

__host__ __device__ constexpr uint32_t weight_offset(int layer) { return (uint32_t)layer * 4096u; }
__host__ __device__ constexpr uint32_t layer_outputs(int layer) { return layer < 5 ? 64u : 16u; }

__device__ __forceinline__ unsigned char* align1024(unsigned char* p) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  return reinterpret_cast<unsigned char*>((a + 1023) & ~uintptr_t(1023));
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// Row `row` of a 64-column operand tile from 64 floats.
__device__ __forceinline__ void store_row64(unsigned char* tile, uint32_t row, const float* v) {
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    uint4 q;
    q.x = pack_bf16(v[8 * c + 0], v[8 * c + 1]);
    q.y = pack_bf16(v[8 * c + 2], v[8 * c + 3]);
    q.z = pack_bf16(v[8 * c + 4], v[8 * c + 5]);
    q.w = pack_bf16(v[8 * c + 6], v[8 * c + 7]);
    *reinterpret_cast<uint4*>(tile + tc::tile_offset(row, 8 * c)) = q;
  }
}

__device__ __forceinline__ void store_row16(unsigned char* tile, uint32_t row, const float* v) {
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    uint4 q;
    q.x = pack_bf16(v[8 * c + 0], v[8 * c + 1]);
    q.y = pack_bf16(v[8 * c + 2], v[8 * c + 3]);
    q.z = pack_bf16(v[8 * c + 4], v[8 * c + 5]);
    q.w = pack_bf16(v[8 * c + 6], v[8 * c + 7]);
    *reinterpret_cast<uint4*>(tile + tc::tile_offset_n(row, 8 * c, 16)) = q;
  }
}

// Whether element (row, col) of a 64-column BF16 tile is positive.
__device__ __forceinline__ bool tile_positive(const unsigned char* tile, uint32_t row, uint32_t col) {
  const __nv_bfloat16 v = *reinterpret_cast<const __nv_bfloat16*>(tile + tc::tile_offset(row, col));
  return __bfloat162float(v) > 0.0f;
}

// All 64 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void load_lane64(uint32_t taddr, float* v) {
  float c0[16], c1[16], c2[16], c3[16];
  tc::tmem_ld16(taddr, c0);
  tc::tmem_ld16(taddr + 16, c1);
  tc::tmem_ld16(taddr + 32, c2);
  tc::tmem_ld16(taddr + 48, c3);
  tc::tmem_wait_ld();
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    v[i] = c0[i];
    v[16 + i] = c1[i];
    v[32 + i] = c2[i];
    v[48 + i] = c3[i];
  }
}

// ---------------------------------------------------------------------------
// Encoding.

// Real spherical harmonics of bands 0..3 of a unit direction.
__device__ __forceinline__ void sh_basis(float x, float y, float z, float* o) {
  const float xx = x * x, yy = y * y, zz = z * z;
  o[0] = 0.28209479177387814f;
  o[1] = -0.48860251190291987f * y;
  o[2] = 0.48860251190291987f * z;
  o[3] = -0.48860251190291987f * x;
  o[4] = 1.0925484305920792f * x * y;
  o[5] = -1.0925484305920792f * y * z;
  o[6] = 0.94617469575755997f * zz - 0.31539156525251999f;
  o[7] = -1.0925484305920792f * x * z;
  o[8] = 0.54627421529603959f * (xx - yy);
  o[9] = 0.59004358992664352f * y * (-3.0f * xx + yy);
  o[10] = 2.8906114426405538f * x * y * z;
  o[11] = 0.45704579946446572f * y * (1.0f - 5.0f * zz);
  o[12] = 0.3731763325901154f * z * (5.0f * zz - 3.0f);
  o[13] = 0.45704579946446572f * x * (1.0f - 5.0f * zz);
  o[14] = 1.4453057213202769f * z * (xx - yy);
  o[15] = 0.59004358992664352f * x * (-xx + 3.0f * yy);
}

// One hash-grid level's cell: the 8 corners' table indices and trilinear
// weights for a position u in [0, 1]^3.
struct GridCell {
  uint32_t index[8];
  float weight[8];
};

__device__ __forceinline__ GridCell grid_cell(const CacheGrid& g, uint32_t level, const float* u) {
  GridCell c;
  const float res = g.res[level];
  const uint32_t size = 1u << g.log2_size;
  const uint32_t side = (uint32_t)res + 1u;
  const bool dense = (uint64_t)side * side * side <= size;
  int32_t i0[3];
  float f[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float x = fminf(fmaxf(u[a], 0.0f), 1.0f) * res;
    const float fl = floorf(x);
    i0[a] = min((int32_t)fl, (int32_t)res - 1 < 0 ? 0 : (int32_t)res - 1);
    f[a] = x - (float)i0[a];
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t cx = (uint32_t)i0[0] + (k & 1), cy = (uint32_t)i0[1] + ((k >> 1) & 1),
                   cz = (uint32_t)i0[2] + ((k >> 2) & 1);
    uint32_t idx;
    if (dense) idx = cx + side * (cy + side * cz);
    else idx = (cx * 1u) ^ (cy * 2654435761u) ^ (cz * 805459861u);
    c.index[k] = idx & (size - 1u);
    c.weight[k] = ((k & 1) ? f[0] : 1.0f - f[0]) * (((k >> 1) & 1) ? f[1] : 1.0f - f[1]) *
                  (((k >> 2) & 1) ? f[2] : 1.0f - f[2]);
  }
  return c;
}

__device__ __forceinline__ void grid_position(const CacheGrid& g, const CacheRecord& r, float* u) {
  u[0] = (r.pos_rough.x - g.lo[0]) * g.inv_extent[0];
  u[1] = (r.pos_rough.y - g.lo[1]) * g.inv_extent[1];
  u[2] = (r.pos_rough.z - g.lo[2]) * g.inv_extent[2];
}

// The 64 network inputs of a record: 32 hash-grid features, 16 spherical
// harmonics of the direction, normal, roughness, albedo, a constant 1.
__device__ __forceinline__ void encode_record(const CacheGrid& g, const CacheRecord& r, float* x) {
  float u[3];
  grid_position(g, r, u);
#pragma unroll
  for (uint32_t l = 0; l < (uint32_t)kCacheMaxLevels; ++l) {
    float a = 0.0f, b = 0.0f;
    if (l < g.levels) {
      const GridCell c = grid_cell(g, l, u);
      const __half2* t = g.table + ((size_t)l << g.log2_size);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const float2 v = __half22float2(t[c.index[k]]);
        a += c.weight[k] * v.x;
        b += c.weight[k] * v.y;
      }
    }
    x[2 * l] = a;
    x[2 * l + 1] = b;
  }
  sh_basis(r.dir.x, r.dir.y, r.dir.z, x + kCacheGridFeatures);
  x[48] = r.normal.x;
  x[49] = r.normal.y;
  x[50] = r.normal.z;
  x[51] = r.pos_rough.w;
  x[52] = r.albedo.x;
  x[53] = r.albedo.y;
  x[54] = r.albedo.z;
  x[55] = 1.0f;
#pragma unroll
  for (int i = 56; i < 64; ++i) x[i] = 0.0f;
}

// Adds the gradient of the 32 grid features to the levels' entries.
__device__ __forceinline__ void scatter_grid_gradient(const CacheGrid& g, const CacheRecord& r, const float* dx) {
  float u[3];
  grid_position(g, r, u);
#pragma unroll
  for (uint32_t l = 0; l < (uint32_t)kCacheMaxLevels; ++l) {
    const float ga = dx[2 * l], gb = dx[2 * l + 1];
    if (l >= g.levels || (ga == 0.0f && gb == 0.0f)) continue;
    const GridCell c = grid_cell(g, l, u);
    float* base = g.grad + (((size_t)l << g.log2_size) << 1);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      atomicAdd(base + 2 * (size_t)c.index[k], c.weight[k] * ga);
      atomicAdd(base + 2 * (size_t)c.index[k] + 1, c.weight[k] * gb);
    }
  }
}

// ---------------------------------------------------------------------------
// Sources of network inputs and sinks of outputs.

enum : int { kEncodedIO = 0, kRecordIO = 1 };

struct NetIO {
  // kEncodedIO: inputs n x 64, targets n x 3, outputs n x 3, input
  // gradients n x 64.
  const float* inputs;
  const float* targets;
  float* outputs;
  float* input_grad;
  // kRecordIO: records (queries or training records), their targets
  // (float4, training) or the radiance slots and throughputs they add to
  // (queries).
  const CacheRecord* records;
  const float4* record_targets;
  const uint32_t* slots;
  const float4* throughput;
  float4* radiance;
  // Records: the order to take them in (record order[q] for query q), or
  // null for their own order.
  const uint32_t* order;
  // Count: *count when non-null, else n; clamped to capacity.
  const uint32_t* count;
  uint32_t n;
  uint32_t capacity;
};

__device__ __forceinline__ uint32_t io_count(const NetIO& io) {
  const uint32_t n = io.count ? *io.count : io.n;
  return n < io.capacity ? n : io.capacity;
}

template <int kIO>
__device__ __forceinline__ void load_input(const NetIO& io, const CacheGrid& g, uint32_t q, uint32_t n, float* x,
    CacheRecord& rec) {
  if (q >= n) {
#pragma unroll
    for (int i = 0; i < 64; ++i) x[i] = 0.0f;
    return;
  }
  if (kIO == kEncodedIO) {
    const float4* p = reinterpret_cast<const float4*>(io.inputs + (size_t)q * 64);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const float4 v = p[i];
      x[4 * i] = v.x;
      x[4 * i + 1] = v.y;
      x[4 * i + 2] = v.z;
      x[4 * i + 3] = v.w;
    }
  } else {
    rec = io.records[q];
    encode_record(g, rec, x);
  }
}

// Issues D = A * B over K = 16 * ksteps from the K-major tiles a and b.
__device__ __forceinline__ void issue_k_major(uint32_t tmem, uint32_t a, uint32_t a_cols, uint32_t b,
    uint32_t b_cols, uint32_t n, int ksteps) {
  const uint32_t id = tc::idesc_bf16(128, n, 0, 0);
  for (int k = 0; k < ksteps; ++k)
    tc::mma_bf16(tmem, tc::desc_k_major(a, 16 * k, a_cols), tc::desc_k_major(b, 16 * k, b_cols), id, k > 0);
}

struct Barrier {
  uint32_t mbar;
  uint32_t phase = 0;
  // Waits for the last commit; block-uniform result.
  __device__ __forceinline__ bool wait() {
    const bool ok = tc::mbar_wait(mbar, phase, kWaitPolls);
    phase ^= 1u;
    tc::fence_after_sync();
    return __syncthreads_and(ok) != 0;
  }
};

// Publishes this thread's operand writes to the tensor core and orders
// its tensor-memory loads before the next MMA.
__device__ __forceinline__ void operands_ready() {
  tc::fence_async_shared();
  tc::fence_before_sync();
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Inference: outputs of the network for `n` queries. A CTA holds one copy
// of the weights and kInferGroups warpgroups, each working through its own
// tiles with its own activation tile, tensor-memory columns and mbarrier,
// so that several tiles' encodings, MMAs and epilogues overlap on an SM.

constexpr int kInferGroups = 4;
constexpr int kInferThreads = 128 * kInferGroups;

// Barrier of one warpgroup (named barrier 1 + group).
__device__ __forceinline__ void group_sync(uint32_t group) {
  asm volatile("bar.sync %0, 128;" ::"r"(group + 1u) : "memory");
}

// AND of `pred` over one warpgroup.
__device__ __forceinline__ bool group_and(uint32_t group, bool pred) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(out)
      : "r"(pred ? 1u : 0u), "r"(group + 1u)
      : "memory");
  return out != 0;
}

__device__ __forceinline__ void store_pair(unsigned char* tile, uint32_t row, uint32_t col, float a, float b) {
  *reinterpret_cast<uint32_t*>(tile + tc::tile_offset(row, col)) = pack_bf16(a, b);
}

// encode_record written straight into row `row` of an operand tile, a
// level at a time, so that the 64 inputs never sit in registers together.
__device__ __forceinline__ void encode_record_to_tile(const CacheGrid& g, const CacheRecord& r, unsigned char* tile,
    uint32_t row) {
  float u[3];
  grid_position(g, r, u);
  // All levels unrolled, so that their 128 gathers can be in flight
  // together.
#pragma unroll
  for (uint32_t l = 0; l < (uint32_t)kCacheMaxLevels; ++l) {
    float a = 0.0f, b = 0.0f;
    if (l < g.levels) {
      const GridCell c = grid_cell(g, l, u);
      const __half2* t = g.table + ((size_t)l << g.log2_size);
      __half2 v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = t[c.index[k]];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const float2 f = __half22float2(v[k]);
        a += c.weight[k] * f.x;
        b += c.weight[k] * f.y;
      }
    }
    store_pair(tile, row, 2 * l, a, b);
  }
  float x[16];
  sh_basis(r.dir.x, r.dir.y, r.dir.z, x);
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    uint4 q;
    q.x = pack_bf16(x[8 * c + 0], x[8 * c + 1]);
    q.y = pack_bf16(x[8 * c + 2], x[8 * c + 3]);
    q.z = pack_bf16(x[8 * c + 4], x[8 * c + 5]);
    q.w = pack_bf16(x[8 * c + 6], x[8 * c + 7]);
    *reinterpret_cast<uint4*>(tile + tc::tile_offset(row, 32 + 8 * c)) = q;
  }
  uint4 q;
  q.x = pack_bf16(r.normal.x, r.normal.y);
  q.y = pack_bf16(r.normal.z, r.pos_rough.w);
  q.z = pack_bf16(r.albedo.x, r.albedo.y);
  q.w = pack_bf16(r.albedo.z, 1.0f);
  *reinterpret_cast<uint4*>(tile + tc::tile_offset(row, 48)) = q;
  *reinterpret_cast<uint4*>(tile + tc::tile_offset(row, 56)) = make_uint4(0u, 0u, 0u, 0u);
}

// The ReLU of a 64-column accumulator lane into row `row` of a tile, 16
// columns at a time.
__device__ __forceinline__ void relu_lane_to_tile(uint32_t taddr, unsigned char* tile, uint32_t row) {
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    float v[16];
    tc::tmem_ld16(taddr + 16 * c, v);
    tc::tmem_wait_ld();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      uint4 q;
      q.x = pack_bf16(fmaxf(v[8 * h + 0], 0.0f), fmaxf(v[8 * h + 1], 0.0f));
      q.y = pack_bf16(fmaxf(v[8 * h + 2], 0.0f), fmaxf(v[8 * h + 3], 0.0f));
      q.z = pack_bf16(fmaxf(v[8 * h + 4], 0.0f), fmaxf(v[8 * h + 5], 0.0f));
      q.w = pack_bf16(fmaxf(v[8 * h + 6], 0.0f), fmaxf(v[8 * h + 7], 0.0f));
      *reinterpret_cast<uint4*>(tile + tc::tile_offset(row, 16 * c + 8 * h)) = q;
    }
  }
}

template <int kIO>
__global__ void __launch_bounds__(kInferThreads, 1) k_cache_infer(CacheNet net, CacheGrid grid, NetIO io) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = align1024(smem_raw);
  unsigned char* W = smem;
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  const uint32_t group = tid >> 7, row = tid & 127u;
  unsigned char* A = smem + kCacheOperandBytes + group * kTile;
  uint64_t* mbars = reinterpret_cast<uint64_t*>(smem + kCacheOperandBytes + kInferGroups * kTile);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbars + kInferGroups);
  for (uint32_t i = tid; i < kCacheOperandBytes / 16; i += kInferThreads)
    reinterpret_cast<uint4*>(W)[i] = net.forward[i];
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(tslot), 64 * kInferGroups);
  if (tid < (uint32_t)kInferGroups) tc::mbar_init(tc::smem_u32(mbars + tid), 1);
  tc::fence_async_shared();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot + 64u * group;
  const uint32_t lane_addr = tmem + (((warp & 3u) * 32u) << 16);
  const uint32_t mbar = tc::smem_u32(mbars + group);
  uint32_t phase = 0;
  const uint32_t n = io_count(io);
  const uint32_t tiles = (n + 127) / 128;
  const uint32_t stride = gridDim.x * kInferGroups;
  bool ok = true;
  for (uint32_t tile = blockIdx.x * kInferGroups + group; tile < tiles && ok; tile += stride) {
    const uint32_t q = tile * 128 + row;
    if (kIO == kEncodedIO) {
      float x[64];
      CacheRecord rec;
      load_input<kIO>(io, grid, q, n, x, rec);
      store_row64(A, row, x);
    } else if (q < n) {
      encode_record_to_tile(grid, io.records[io.order ? io.order[q] : q], A, row);
    } else {
#pragma unroll
      for (int c = 0; c < 8; ++c)
        *reinterpret_cast<uint4*>(A + tc::tile_offset(row, 8 * c)) = make_uint4(0u, 0u, 0u, 0u);
    }
    tc::fence_async_shared();
    tc::fence_before_sync();
    group_sync(group);
    float y[16];
    for (int l = 0; l < kCacheLayers && ok; ++l) {
      if (row == 0) {
        tc::fence_after_sync();
        issue_k_major(tmem, tc::smem_u32(A), 64, tc::smem_u32(W) + layer_offset(l), 64, layer_outputs(l), 4);
        tc::commit(mbar);
      }
      __syncwarp();
      const bool waited = tc::mbar_wait(mbar, phase, kWaitPolls);
      phase ^= 1u;
      tc::fence_after_sync();
      ok = group_and(group, waited);
      if (l < kCacheLayers - 1) {
        relu_lane_to_tile(lane_addr, A, row);
        tc::fence_async_shared();
      } else {
        tc::tmem_ld16(lane_addr, y);
        tc::tmem_wait_ld();
      }
      tc::fence_before_sync();
      group_sync(group);
    }
    if (!ok || q >= n) continue;
    if (kIO == kEncodedIO) {
      io.outputs[3 * (size_t)q] = y[0];
      io.outputs[3 * (size_t)q + 1] = y[1];
      io.outputs[3 * (size_t)q + 2] = y[2];
    } else {
      // The query's path ends here: its throughput times the cached
      // radiance (clamped at zero) joins the path's radiance.
      const uint32_t record = io.order ? io.order[q] : q;
      const uint32_t slot = io.slots[record];
      const float4 t = io.throughput[record];
      float4 r = io.radiance[slot];
      r.x += t.x * fmaxf(y[0], 0.0f);
      r.y += t.y * fmaxf(y[1], 0.0f);
      r.z += t.z * fmaxf(y[2], 0.0f);
      io.radiance[slot] = r;
    }
  }
  if (!ok && row == 0) atomicExch(net.error, 1u);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(*tslot, 64 * kInferGroups);
}

// ---------------------------------------------------------------------------
// Training: forward, relative L2 loss (Mueller et al.: (y - t)^2 over
// y^2 + 0.01, y held constant in the denominator), backward. Weight
// gradients accumulate in tensor memory over the CTA's tiles and are added
// to net.grad at the end; input gradients go to the hash grid (records) or
// to io.input_grad (encoded inputs). Gradients are of the loss summed over
// samples and channels.
template <int kIO>
__global__ void __launch_bounds__(kNetThreads, 1) k_cache_train(CacheNet net, CacheGrid grid, NetIO io) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = align1024(smem_raw);
  unsigned char* WF = smem;
  unsigned char* WB = WF + kCacheOperandBytes;
  unsigned char* H = WB + kCacheOperandBytes;      // 6 activation tiles
  unsigned char* G = H + kCacheLayers * kTile;     // 2 gradient tiles
  unsigned char* DY = G + 2 * kTile;               // 128 x 16 output gradients
  uint64_t* mbar = reinterpret_cast<uint64_t*>(DY + kNarrowTile);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
  float* loss_sum = reinterpret_cast<float*>(tslot + 1);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  for (uint32_t i = tid; i < kCacheOperandBytes / 16; i += kNetThreads) {
    reinterpret_cast<uint4*>(WF)[i] = net.forward[i];
    reinterpret_cast<uint4*>(WB)[i] = net.backward[i];
  }
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(tslot), kTrainColumns);
  if (tid == 0) {
    tc::mbar_init(tc::smem_u32(mbar), 1);
    *loss_sum = 0.0f;
  }
  operands_ready();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t lane_addr = tmem + ((warp * 32u) << 16);
  Barrier bar{tc::smem_u32(mbar)};
  const uint32_t n = io_count(io);
  const uint32_t tiles = (n + 127) / 128;
  bool ok = true;
  uint32_t done = 0;
  float loss = 0.0f;
  for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x, ++done) {
    const uint32_t q = tile * 128 + tid;
    const bool valid = q < n;
    float x[64];
    CacheRecord rec;
    load_input<kIO>(io, grid, q, n, x, rec);
    float target[3] = {0.0f, 0.0f, 0.0f};
    if (valid) {
      if (kIO == kEncodedIO) {
        target[0] = io.targets[3 * (size_t)q];
        target[1] = io.targets[3 * (size_t)q + 1];
        target[2] = io.targets[3 * (size_t)q + 2];
      } else {
        const float4 t = io.record_targets[q];
        target[0] = t.x;
        target[1] = t.y;
        target[2] = t.z;
      }
    }
    store_row64(H, tid, x);
    operands_ready();
    // Forward.
    float y[16];
    for (int l = 0; l < kCacheLayers && ok; ++l) {
      if (tid == 0) {
        tc::fence_after_sync();
        issue_k_major(tmem, tc::smem_u32(H + l * kTile), 64, tc::smem_u32(WF) + layer_offset(l), 64,
            layer_outputs(l), 4);
        tc::commit(bar.mbar);
      }
      __syncwarp();
      ok = bar.wait();
      if (l < kCacheLayers - 1) {
        load_lane64(lane_addr, x);
#pragma unroll
        for (int i = 0; i < 64; ++i) x[i] = fmaxf(x[i], 0.0f);
        store_row64(H + (l + 1) * kTile, tid, x);
      } else {
        tc::tmem_ld16(lane_addr, y);
        tc::tmem_wait_ld();
      }
      operands_ready();
    }
    if (!ok) break;
    // Loss and its gradient.
    float dy[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) dy[c] = 0.0f;
    if (valid) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float d = y[c] - target[c];
        const float denom = y[c] * y[c] + 0.01f;
        loss += d * d / denom;
        dy[c] = 2.0f * d / denom;
      }
    }
    store_row16(DY, tid, dy);
    operands_ready();
    // Backward, output layer first. `cur` holds the gradient entering
    // layer l's outputs (after the ReLU's mask).
    unsigned char* cur = DY;
    for (int l = kCacheLayers - 1; l >= 0 && ok; --l) {
      const uint32_t outs = layer_outputs(l);
      if (tid == 0) {
        tc::fence_after_sync();
        // Input gradient of layer l: D[s][i] = sum_o cur[s][o] W_l[i][o].
        issue_k_major(tmem, tc::smem_u32(cur), outs, tc::smem_u32(WB) + layer_offset(l), outs, 64,
            (int)(outs / 16));
        // Weight gradient: D[i][o] += sum_s H_l[s][i] cur[s][o] (rows
        // 64..127 of the M = 128 shape are not used).
        const uint32_t id = tc::idesc_bf16(128, outs, 1, 1);
        for (int k = 0; k < 8; ++k)
          tc::mma_bf16(tmem + grad_column(l), tc::desc_mn_major(tc::smem_u32(H + l * kTile), 16 * k, 64),
              tc::desc_mn_major(tc::smem_u32(cur), 16 * k, outs), id, (done > 0 || k > 0) ? 1u : 0u);
        tc::commit(bar.mbar);
      }
      __syncwarp();
      ok = bar.wait();
      load_lane64(lane_addr, x);
      if (l > 0) {
        unsigned char* next = G + ((kCacheLayers - 1 - l) & 1) * kTile;
#pragma unroll
        for (int i = 0; i < 64; ++i) x[i] = tile_positive(H + l * kTile, tid, i) ? x[i] : 0.0f;
        store_row64(next, tid, x);
        cur = next;
      } else if (valid) {
        if (kIO == kEncodedIO) {
          float4* g = reinterpret_cast<float4*>(io.input_grad + (size_t)q * 64);
#pragma unroll
          for (int i = 0; i < 16; ++i) g[i] = make_float4(x[4 * i], x[4 * i + 1], x[4 * i + 2], x[4 * i + 3]);
        } else {
          scatter_grid_gradient(grid, rec, x);
        }
      }
      operands_ready();
    }
  }
  if (!ok && tid == 0) atomicExch(net.error, 1u);
  // Loss.
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_down_sync(0xFFFFFFFFu, loss, o);
  if ((tid & 31u) == 0) atomicAdd(loss_sum, loss);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (tid == 0 && *loss_sum != 0.0f) atomicAdd(net.loss, *loss_sum);
  // Weight gradients: lanes 0..63 hold rows i of every layer's D[i][o].
  if (ok && done > 0 && warp < 2) {
    const uint32_t i = tid;  // input feature
    for (int l = 0; l < kCacheLayers; ++l) {
      const uint32_t outs = layer_outputs(l);
      float g[64];
      if (outs == 64) {
        load_lane64(lane_addr + grad_column(l), g);
      } else {
        float h[16];
        tc::tmem_ld16(lane_addr + grad_column(l), h);
        tc::tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < 16; ++c) g[c] = h[c];
      }
      float* dst = net.grad + weight_offset(l) + i * outs;
      for (uint32_t o = 0; o < outs; ++o) atomicAdd(dst + o, g[o]);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tmem, kTrainColumns);
}

// ---------------------------------------------------------------------------
// Weights: initialisation, packing into the operand images, Adam.

__device__ __forceinline__ float hash_uniform(uint32_t seed, uint32_t i) {
  uint32_t h = pcg_hash(seed * 0x9E3779B9u ^ pcg_hash(i));
  return (float)(h >> 8) * (1.0f / 16777216.0f);
}

// Uniform in +-sqrt(6 / (fan_in + fan_out)) (Glorot), deterministic in seed.
__global__ void k_init_weights(float* w, uint32_t seed) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kCacheWeights) return;
  const int layer = min((int)(i / 4096u), kCacheLayers - 1);
  const float limit = sqrtf(6.0f / (64.0f + (float)layer_outputs(layer)));
  w[i] = (2.0f * hash_uniform(seed, i) - 1.0f) * limit;
}

__global__ void k_init_grid(float* master, __half2* table, size_t entries, uint32_t seed) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= entries) return;
  const float a = (2.0f * hash_uniform(seed + 17u, (uint32_t)(2 * i)) - 1.0f) * 1e-4f;
  const float b = (2.0f * hash_uniform(seed + 17u, (uint32_t)(2 * i + 1)) - 1.0f) * 1e-4f;
  master[2 * i] = a;
  master[2 * i + 1] = b;
  table[i] = __floats2half2_rn(a, b);
}

// The forward image holds layer l as an (outputs x 64) K-major tile of
// W_l[i][o] at (o, i); the backward image as a (64 x outputs) K-major tile
// at (i, o).
__global__ void k_pack_weights(const float* __restrict__ w, unsigned char* __restrict__ forward,
    unsigned char* __restrict__ backward) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kCacheWeights) return;
  const int l = min((int)(e / 4096u), kCacheLayers - 1);
  const uint32_t outs = layer_outputs(l);
  const uint32_t local = e - weight_offset(l);
  const uint32_t i = local / outs, o = local % outs;
  const __nv_bfloat16 v = __float2bfloat16_rn(w[e]);
  *reinterpret_cast<__nv_bfloat16*>(forward + layer_offset(l) + tc::tile_offset_n(o, i, 64)) = v;
  *reinterpret_cast<__nv_bfloat16*>(backward + layer_offset(l) + tc::tile_offset_n(i, o, outs)) = v;
}

// Adam's per-step constants, on the device: [0] the step count, [1] and
// [2] the bias corrections 1 - beta^t, [3] the gradient scale 1 / (3 n)
// for n samples, [4] whether the step runs (n > 0).
constexpr float kBeta1 = 0.9f, kBeta2 = 0.99f, kAdamEps = 1e-15f;

__global__ void k_adam_prepare(float* c, const uint32_t* count, uint32_t capacity, uint32_t samples) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const uint32_t n = count ? min(*count, capacity) : samples;
  if (n == 0) {
    c[4] = 0.0f;
    return;
  }
  const float t = c[0] + 1.0f;
  c[0] = t;
  c[1] = 1.0f - powf(kBeta1, t);
  c[2] = 1.0f - powf(kBeta2, t);
  c[3] = 1.0f / (3.0f * (float)n);
  c[4] = 1.0f;
}

__device__ __forceinline__ float adam_update(float p, float grad, float* m, float* v, float lr, const float* c) {
  if (!isfinite(grad)) grad = 0.0f;
  const float mi = kBeta1 * *m + (1.0f - kBeta1) * grad;
  const float vi = kBeta2 * *v + (1.0f - kBeta2) * grad * grad;
  *m = mi;
  *v = vi;
  return p - lr * (mi / c[1]) / (sqrtf(vi / c[2]) + kAdamEps);
}

// Adam (Kingma and Ba, 2015) with bias correction over the weights; zeroes
// the gradient. The output layer's unused columns stay as they are.
__global__ void k_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
    uint32_t n, float lr, const float* __restrict__ c) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float grad = g[i] * c[3];
  g[i] = 0.0f;
  if (c[4] == 0.0f) return;
  if (i >= weight_offset(kCacheLayers - 1) && (i - weight_offset(kCacheLayers - 1)) % 16u >= 3u) return;
  p[i] = adam_update(p[i], grad, m + i, v + i, lr, c);
}

// The same over the hash grid, one entry (two features) per thread, which
// also refreshes the entry's FP16 copy. Lazy: an entry no sample touched
// in this step (zero gradient) keeps its moments and value, so a step
// costs one read of the gradients plus the touched entries' updates (the
// sparse Adam of embedding tables).
__global__ void k_adam_grid(float2* __restrict__ p, float2* __restrict__ g, float2* __restrict__ m,
    float2* __restrict__ v, size_t entries, float lr, const float* __restrict__ c, __half2* __restrict__ table) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= entries) return;
  const float2 gr = g[e];
  if (gr.x == 0.0f && gr.y == 0.0f) return;
  g[e] = make_float2(0.0f, 0.0f);
  if (c[4] == 0.0f) return;
  float2 pe = p[e], me = m[e], ve = v[e];
  pe.x = adam_update(pe.x, gr.x * c[3], &me.x, &ve.x, lr, c);
  pe.y = adam_update(pe.y, gr.y * c[3], &me.y, &ve.y, lr, c);
  p[e] = pe;
  m[e] = me;
  v[e] = ve;
  table[e] = __floats2half2_rn(pe.x, pe.y);
}

__global__ void k_encode(CacheGrid grid, const CacheRecord* __restrict__ records, uint32_t n, float* out) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  float x[64];
  encode_record(grid, records[q], x);
  for (int i = 0; i < 64; ++i) out[(size_t)q * 64 + i] = x[i];
}

constexpr size_t kInferSmem = kCacheOperandBytes + kInferGroups * kTile + 64 + 1024;
constexpr size_t kTrainSmem = 2 * kCacheOperandBytes + (kCacheLayers + 2) * kTile + kNarrowTile + 64 + 1024;

template <typename Kernel>
cudaError_t allow_smem(Kernel k, size_t bytes) {
  return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

uint32_t sm_count() {
  static int sms = 0;
  if (sms == 0) {
    int device = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  }
  return (uint32_t)std::max(sms, 1);
}

}  // namespace

// ---------------------------------------------------------------------------
// Launchers shared with the integrator.

cudaError_t launch_cache_infer_records(const CacheNet& net, const CacheGrid& grid, const CacheRecord* records,
    const uint32_t* slots, const float4* throughput, float4* radiance, const uint32_t* count, uint32_t capacity,
    cudaStream_t s, const uint32_t* order) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = allow_smem(k_cache_infer<kRecordIO>, kInferSmem);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  NetIO io{};
  io.records = records;
  io.slots = slots;
  io.throughput = throughput;
  io.radiance = radiance;
  io.order = order;
  io.count = count;
  io.capacity = capacity;
  const uint32_t grid_size = std::min(sm_count(), std::max(1u, (capacity + 127) / 128 / kInferGroups + 1));
  k_cache_infer<kRecordIO><<<grid_size, kInferThreads, kInferSmem, s>>>(net, grid, io);
  return cudaGetLastError();
}

cudaError_t launch_cache_train_records(const CacheNet& net, const CacheGrid& grid, const CacheRecord* records,
    const float4* targets, const uint32_t* count, uint32_t capacity, cudaStream_t s) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = allow_smem(k_cache_train<kRecordIO>, kTrainSmem);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  NetIO io{};
  io.records = records;
  io.record_targets = targets;
  io.count = count;
  io.n = capacity;
  io.capacity = capacity;
  const uint32_t grid_size = std::min(sm_count(), std::max(1u, (capacity + 127) / 128));
  k_cache_train<kRecordIO><<<grid_size, kNetThreads, kTrainSmem, s>>>(net, grid, io);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// RadianceCache.

CacheNet RadianceCache::net() const {
  CacheNet n;
  n.forward = operands_;
  n.backward = operands_ + kCacheOperandBytes / 16;
  n.grad = grad_;
  n.loss = loss_;
  n.error = error_;
  return n;
}

void RadianceCache::release() {
  void* ptrs[] = {master_, adam_m_, adam_v_, grid_master_, operands_, grad_, loss_, error_, grid_.table, grid_.grad,
      adam_consts_};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  master_ = adam_m_ = adam_v_ = grid_master_ = grad_ = loss_ = nullptr;
  operands_ = nullptr;
  error_ = nullptr;
  adam_consts_ = nullptr;
  grid_.table = nullptr;
  grid_.grad = nullptr;
  grid_entries_ = 0;
}

cudaError_t RadianceCache::configure(const CacheConfig& config, const float lo[3], const float hi[3],
    cudaStream_t s) {
  release();
  config_ = config;
  grid_ = CacheGrid{};
  grid_.levels = std::min<uint32_t>(config.levels, kCacheMaxLevels);
  grid_.log2_size = config.log2_size;
  const double growth = grid_.levels > 1
      ? std::exp((std::log((double)config.max_resolution) - std::log((double)config.min_resolution)) /
                 (double)(grid_.levels - 1))
      : 1.0;
  for (uint32_t l = 0; l < (uint32_t)kCacheMaxLevels; ++l)
    grid_.res[l] = (float)std::floor((double)config.min_resolution * std::pow(growth, (double)l));
  for (int a = 0; a < 3; ++a) {
    const float extent = std::max(hi[a] - lo[a], 1e-6f);
    // A margin of 1% keeps surfaces on the box's faces inside it.
    grid_.lo[a] = lo[a] - 0.01f * extent;
    grid_.inv_extent[a] = 1.0f / (1.02f * extent);
  }
  grid_entries_ = (size_t)grid_.levels << grid_.log2_size;
  const size_t grid_floats = 2 * grid_entries_;
  const size_t moments = kCacheWeights + grid_floats;
  cudaError_t e;
  if ((e = cudaMalloc(&master_, kCacheWeights * 4)) != cudaSuccess ||
      (e = cudaMalloc(&adam_m_, moments * 4)) != cudaSuccess ||
      (e = cudaMalloc(&adam_v_, moments * 4)) != cudaSuccess ||
      (e = cudaMalloc(&grid_master_, grid_floats * 4)) != cudaSuccess ||
      (e = cudaMalloc(&operands_, 2 * kCacheOperandBytes)) != cudaSuccess ||
      (e = cudaMalloc(&grad_, kCacheWeights * 4)) != cudaSuccess ||
      (e = cudaMalloc(&loss_, 4)) != cudaSuccess || (e = cudaMalloc(&error_, 4)) != cudaSuccess ||
      (e = cudaMalloc(&grid_.table, grid_entries_ * sizeof(__half2))) != cudaSuccess ||
      (e = cudaMalloc(&grid_.grad, grid_floats * 4)) != cudaSuccess ||
      (e = cudaMalloc(&adam_consts_, 8 * 4)) != cudaSuccess) {
    release();
    return e;
  }
  cudaMemsetAsync(adam_m_, 0, moments * 4, s);
  cudaMemsetAsync(adam_v_, 0, moments * 4, s);
  cudaMemsetAsync(grad_, 0, kCacheWeights * 4, s);
  cudaMemsetAsync(grid_.grad, 0, grid_floats * 4, s);
  cudaMemsetAsync(loss_, 0, 4, s);
  cudaMemsetAsync(error_, 0, 4, s);
  cudaMemsetAsync(adam_consts_, 0, 8 * 4, s);
  cudaMemsetAsync(operands_, 0, 2 * kCacheOperandBytes, s);
  k_init_weights<<<(kCacheWeights + 255) / 256, 256, 0, s>>>(master_, config.seed);
  k_init_grid<<<(uint32_t)((grid_entries_ + 255) / 256), 256, 0, s>>>(grid_master_, grid_.table, grid_entries_,
      config.seed);
  if ((e = pack(s)) != cudaSuccess) return e;
  return cudaGetLastError();
}

cudaError_t RadianceCache::pack(cudaStream_t s) {
  unsigned char* f = reinterpret_cast<unsigned char*>(operands_);
  k_pack_weights<<<(kCacheWeights + 255) / 256, 256, 0, s>>>(master_, f, f + kCacheOperandBytes);
  return cudaGetLastError();
}

cudaError_t RadianceCache::adam_step(uint32_t samples, cudaStream_t s) {
  if (!ready() || samples == 0) return cudaSuccess;
  k_adam_prepare<<<1, 32, 0, s>>>(adam_consts_, nullptr, 0, samples);
  return adam_kernels(s);
}

cudaError_t RadianceCache::adam_step_device(const uint32_t* count, uint32_t capacity, cudaStream_t s) {
  if (!ready()) return cudaSuccess;
  k_adam_prepare<<<1, 32, 0, s>>>(adam_consts_, count, capacity, 0);
  return adam_kernels(s);
}

cudaError_t RadianceCache::adam_kernels(cudaStream_t s) {
  k_adam<<<(kCacheWeights + 255) / 256, 256, 0, s>>>(master_, grad_, adam_m_, adam_v_, kCacheWeights,
      config_.learning_rate, adam_consts_);
  k_adam_grid<<<(uint32_t)((grid_entries_ + 255) / 256), 256, 0, s>>>(reinterpret_cast<float2*>(grid_master_),
      reinterpret_cast<float2*>(grid_.grad), reinterpret_cast<float2*>(adam_m_ + kCacheWeights),
      reinterpret_cast<float2*>(adam_v_ + kCacheWeights), grid_entries_, config_.learning_rate, adam_consts_,
      grid_.table);
  return pack(s);
}

cudaError_t RadianceCache::read_weights(float* host, cudaStream_t s) {
  cudaError_t e = cudaMemcpyAsync(host, master_, kCacheWeights * 4, cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(s);
}

cudaError_t RadianceCache::write_weights(const float* host, cudaStream_t s) {
  cudaError_t e = cudaMemcpyAsync(master_, host, kCacheWeights * 4, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  if ((e = pack(s)) != cudaSuccess) return e;
  return cudaStreamSynchronize(s);
}

uint32_t RadianceCache::error_flag(cudaStream_t s) {
  uint32_t v = 0;
  if (!error_) return 0;
  cudaMemcpyAsync(&v, error_, 4, cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  return v;
}

namespace {

template <typename T>
struct Scratch {
  T* ptr = nullptr;
  ~Scratch() {
    if (ptr) cudaFree(ptr);
  }
  cudaError_t alloc(size_t n) { return cudaMalloc(&ptr, std::max<size_t>(n, 1) * sizeof(T)); }
};

}  // namespace

cudaError_t RadianceCache::infer_encoded(const float* inputs, uint32_t n, float* outputs, cudaStream_t s) {
  if (!ready()) return cudaErrorNotReady;
  Scratch<float> din, dout;
  cudaError_t e;
  if ((e = din.alloc((size_t)n * 64)) != cudaSuccess || (e = dout.alloc((size_t)n * 3)) != cudaSuccess) return e;
  cudaMemcpyAsync(din.ptr, inputs, (size_t)n * 64 * 4, cudaMemcpyHostToDevice, s);
  if ((e = allow_smem(k_cache_infer<kEncodedIO>, kInferSmem)) != cudaSuccess) return e;
  NetIO io{};
  io.inputs = din.ptr;
  io.outputs = dout.ptr;
  io.n = n;
  io.capacity = n;
  const uint32_t grid_size = std::min(sm_count(), std::max(1u, (n + 127) / 128 / kInferGroups + 1));
  k_cache_infer<kEncodedIO><<<grid_size, kInferThreads, kInferSmem, s>>>(net(), grid_, io);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  cudaMemcpyAsync(outputs, dout.ptr, (size_t)n * 3 * 4, cudaMemcpyDeviceToHost, s);
  return cudaStreamSynchronize(s);
}

cudaError_t RadianceCache::gradient_encoded(const float* inputs, const float* targets, uint32_t n,
    float* weight_grad, float* input_grad, float* loss, cudaStream_t s) {
  if (!ready()) return cudaErrorNotReady;
  Scratch<float> din, dt, dg;
  cudaError_t e;
  if ((e = din.alloc((size_t)n * 64)) != cudaSuccess || (e = dt.alloc((size_t)n * 3)) != cudaSuccess ||
      (e = dg.alloc((size_t)n * 64)) != cudaSuccess)
    return e;
  cudaMemcpyAsync(din.ptr, inputs, (size_t)n * 64 * 4, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dt.ptr, targets, (size_t)n * 3 * 4, cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(grad_, 0, kCacheWeights * 4, s);
  cudaMemsetAsync(loss_, 0, 4, s);
  if ((e = allow_smem(k_cache_train<kEncodedIO>, kTrainSmem)) != cudaSuccess) return e;
  NetIO io{};
  io.inputs = din.ptr;
  io.targets = dt.ptr;
  io.input_grad = dg.ptr;
  io.n = n;
  io.capacity = n;
  const uint32_t grid_size = std::min(sm_count(), std::max(1u, (n + 127) / 128));
  k_cache_train<kEncodedIO><<<grid_size, kNetThreads, kTrainSmem, s>>>(net(), grid_, io);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (weight_grad) cudaMemcpyAsync(weight_grad, grad_, kCacheWeights * 4, cudaMemcpyDeviceToHost, s);
  if (input_grad) cudaMemcpyAsync(input_grad, dg.ptr, (size_t)n * 64 * 4, cudaMemcpyDeviceToHost, s);
  if (loss) cudaMemcpyAsync(loss, loss_, 4, cudaMemcpyDeviceToHost, s);
  cudaMemsetAsync(grad_, 0, kCacheWeights * 4, s);
  return cudaStreamSynchronize(s);
}

cudaError_t RadianceCache::encode(const CacheRecord* records, uint32_t n, float* inputs, cudaStream_t s) {
  if (!ready()) return cudaErrorNotReady;
  Scratch<CacheRecord> dr;
  Scratch<float> dout;
  cudaError_t e;
  if ((e = dr.alloc(n)) != cudaSuccess || (e = dout.alloc((size_t)n * 64)) != cudaSuccess) return e;
  cudaMemcpyAsync(dr.ptr, records, (size_t)n * sizeof(CacheRecord), cudaMemcpyHostToDevice, s);
  k_encode<<<(n + 127) / 128, 128, 0, s>>>(grid_, dr.ptr, n, dout.ptr);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  cudaMemcpyAsync(inputs, dout.ptr, (size_t)n * 64 * 4, cudaMemcpyDeviceToHost, s);
  return cudaStreamSynchronize(s);
}

cudaError_t RadianceCache::train_records(const CacheRecord* records, const float* targets, uint32_t n,
    uint32_t steps, float* losses, cudaStream_t s) {
  if (!ready()) return cudaErrorNotReady;
  Scratch<CacheRecord> dr;
  Scratch<float4> dt;
  cudaError_t e;
  if ((e = dr.alloc(n)) != cudaSuccess || (e = dt.alloc(n)) != cudaSuccess) return e;
  std::vector<float4> t4(n);
  for (uint32_t i = 0; i < n; ++i) t4[i] = make_float4(targets[3 * i], targets[3 * i + 1], targets[3 * i + 2], 0.0f);
  cudaMemcpyAsync(dr.ptr, records, (size_t)n * sizeof(CacheRecord), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dt.ptr, t4.data(), (size_t)n * sizeof(float4), cudaMemcpyHostToDevice, s);
  for (uint32_t k = 0; k < steps; ++k) {
    cudaMemsetAsync(loss_, 0, 4, s);
    if ((e = launch_cache_train_records(net(), grid_, dr.ptr, dt.ptr, nullptr, n, s)) != cudaSuccess) return e;
    if (losses) cudaMemcpyAsync(losses + k, loss_, 4, cudaMemcpyDeviceToHost, s);
    if ((e = adam_step(n, s)) != cudaSuccess) return e;
  }
  return cudaStreamSynchronize(s);
}

}  // namespace lotus
