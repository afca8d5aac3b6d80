// SPDX-License-Identifier: Apache-2.0
// The C ABI of include/lotus_cuda.h: the renderer that stands in for the
// reference's VulkanOffscreenRenderer (backend/vulkan/vulkan_backend.cpp:721
// in hydra-lotus) and its GpuScene (backend/vulkan/gpu_scene.cpp:1606).
//
// One renderer owns one CUDA stream and every device allocation. Calls are
// synchronous: they return after the GPU work and any readback completed.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../../include/lotus_cuda.h"
#include "albedo.cuh"
#include "bvh_build.cuh"
#include "integrator.cuh"
#include "radiance_cache.cuh"
#include "renderer_internal.cuh"
#include "temporal_passes.cuh"

namespace lotus {
namespace {

template <typename T>
struct DeviceArray {
  T* ptr = nullptr;
  size_t count = 0;
  cudaError_t resize(size_t n) {
    if (n == count && ptr) return cudaSuccess;
    release();
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&ptr, n * sizeof(T));
    if (e == cudaSuccess) count = n;
    return e;
  }
  cudaError_t upload(const T* host, size_t n, cudaStream_t s) {
    cudaError_t e = resize(n);
    if (e != cudaSuccess || n == 0) return e;
    return cudaMemcpyAsync(ptr, host, n * sizeof(T), cudaMemcpyHostToDevice, s);
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    count = 0;
  }
  size_t bytes() const { return count * sizeof(T); }
};

void copy_detail(char* dst, size_t size, const std::string& s) {
  if (dst && size) std::snprintf(dst, size, "%s", s.c_str());
}

// Object-from-world rows by Gauss-Jordan elimination in double of the
// affine part, rounded to float.
bool invert_affine(const float* m, float4 rows[3]) {
  double a[3][4];
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) a[r][c] = m[c * 4 + r];
    a[r][3] = m[12 + r];
  }
  double aug[3][6];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 6; ++c) aug[r][c] = c < 3 ? a[r][c] : (r == c - 3 ? 1.0 : 0.0);
  for (int c = 0; c < 3; ++c) {
    int p = c;
    for (int r = c + 1; r < 3; ++r)
      if (std::fabs(aug[r][c]) > std::fabs(aug[p][c])) p = r;
    if (aug[p][c] == 0.0) return false;
    for (int k = 0; k < 6; ++k) std::swap(aug[c][k], aug[p][k]);
    const double s = aug[c][c];
    for (int k = 0; k < 6; ++k) aug[c][k] /= s;
    for (int r = 0; r < 3; ++r) {
      if (r == c) continue;
      const double f = aug[r][c];
      for (int k = 0; k < 6; ++k) aug[r][k] -= f * aug[c][k];
    }
  }
  float out[3][4];
  for (int r = 0; r < 3; ++r) {
    double t = 0.0;
    for (int c = 0; c < 3; ++c) {
      out[r][c] = (float)aug[r][3 + c];
      t -= aug[r][3 + c] * a[c][3];
    }
    out[r][3] = (float)t;
    if (!std::isfinite(out[r][0]) || !std::isfinite(out[r][1]) || !std::isfinite(out[r][2]) ||
        !std::isfinite(out[r][3]))
      return false;
    rows[r] = make_float4(out[r][0], out[r][1], out[r][2], out[r][3]);
  }
  return true;
}

// Invert (vulkan_backend.cpp:436-470): 4x4 Gauss-Jordan in double.
bool invert4(const float* matrix, float* inverse) {
  double rows[4][8] = {};
  for (int row = 0; row < 4; ++row) {
    for (int column = 0; column < 4; ++column) {
      const float value = matrix[column * 4 + row];
      if (!std::isfinite(value)) return false;
      rows[row][column] = value;
    }
    rows[row][row + 4] = 1.0;
  }
  for (int column = 0; column < 4; ++column) {
    int pivot = column;
    for (int row = column + 1; row < 4; ++row)
      if (std::abs(rows[row][column]) > std::abs(rows[pivot][column])) pivot = row;
    if (rows[pivot][column] == 0.0) return false;
    for (int index = 0; index < 8; ++index) std::swap(rows[column][index], rows[pivot][index]);
    const double scale = rows[column][column];
    for (double& value : rows[column]) value /= scale;
    for (int row = 0; row < 4; ++row) {
      if (row == column) continue;
      const double factor = rows[row][column];
      for (int index = 0; index < 8; ++index) rows[row][index] -= factor * rows[column][index];
    }
  }
  for (int row = 0; row < 4; ++row)
    for (int column = 0; column < 4; ++column) {
      const float value = (float)rows[row][column + 4];
      if (!std::isfinite(value)) return false;
      inverse[column * 4 + row] = value;
    }
  return true;
}

struct HostF3 {
  float x, y, z;
};

// mul(world_from_object, float4(p, 1)).xyz in the kernels' order.
HostF3 host_transform(const float* m, const float* p) {
  return {m[0] * p[0] + m[4] * p[1] + m[8] * p[2] + m[12],
          m[1] * p[0] + m[5] * p[1] + m[9] * p[2] + m[13],
          m[2] * p[0] + m[6] * p[1] + m[10] * p[2] + m[14]};
}

float host_coverage(const lotus_material& m) {
  if (m.opacity_threshold > 0.0f) return m.opacity >= m.opacity_threshold ? 1.0f : 0.0f;
  return m.opacity;
}

// The environment image's sampling distribution (BuildEnvironmentDistribution,
// gpu_scene.cpp:638-711): cells of at most 2048 x 1024, each the mean
// scaled radiance of its texels times sin(theta) at the row's centre; the
// floats are the density per cell, the marginal CDF (rows + 1) and each
// row's conditional CDF (columns + 1), then guide tables of the CDFs.
// The same distribution and guide tables built on the device from the
// resident texels, in the host build's arithmetic and order (each cell's
// texels rows first, each row's cells and the rows' sums one after
// another, in double), so that it gives the host build's floats bit for bit:
// one thread per cell for the cell means, per row for its sum and CDF, one
// for the marginal. Only the rows' sin(theta) comes from the host, whose
// libm the host build uses.
__global__ void k_env_cells(const float4* __restrict__ texels, uint32_t width, uint32_t height,
    uint32_t columns, uint32_t rows, float sx, float sy, float sz, const double* __restrict__ sin_theta,
    double* __restrict__ values) {
  const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= columns * rows) return;
  const uint32_t row = cell / columns, column = cell % columns;
  // The texels whose row (column) maps to this cell's: y * rows / height == row.
  const uint32_t y0 = (uint32_t)(((uint64_t)row * height + rows - 1) / rows);
  const uint32_t y1 = (uint32_t)(((uint64_t)(row + 1) * height + rows - 1) / rows);
  const uint32_t x0 = (uint32_t)(((uint64_t)column * width + columns - 1) / columns);
  const uint32_t x1 = (uint32_t)(((uint64_t)(column + 1) * width + columns - 1) / columns);
  double sum = 0.0;
  uint32_t count = 0;
  const double scale[3] = {(double)sx, (double)sy, (double)sz};
  for (uint32_t y = y0; y < y1; ++y)
    for (uint32_t x = x0; x < x1; ++x) {
      const float4 t = texels[(size_t)y * width + x];
      const double c[3] = {(double)t.x, (double)t.y, (double)t.z};
      double radiance = 0.0;
      for (int k = 0; k < 3; ++k) radiance += (c[k] < 0.0 ? 0.0 : c[k]) * scale[k];
      sum += radiance / 3.0;
      ++count;
    }
  values[cell] = sum / count * sin_theta[row];
}

__global__ void k_env_row_sums(const double* __restrict__ values, uint32_t columns, uint32_t rows,
    double* __restrict__ row_sums) {
  const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= rows) return;
  double sum = 0.0;
  for (uint32_t column = 0; column < columns; ++column) sum += values[(size_t)row * columns + column];
  row_sums[row] = sum;
}

// totals[0]: the rows' sum; totals[1]: the mean over the cells.
__global__ void k_env_total(const double* __restrict__ row_sums, uint32_t columns, uint32_t rows,
    double* __restrict__ totals, float* __restrict__ marginal) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double total = 0.0;
  for (uint32_t row = 0; row < rows; ++row) total += row_sums[row];
  const double mean = total / (double)((size_t)columns * rows);
  totals[0] = total;
  totals[1] = mean;
  if (!(mean > 0.0) || !isfinite(mean)) return;
  double cumulative = 0.0;
  marginal[0] = 0.0f;
  for (uint32_t row = 0; row < rows; ++row) {
    cumulative += row_sums[row];
    marginal[row + 1] = (float)(cumulative / total);
  }
  marginal[rows] = 1.0f;
}

__global__ void k_env_density(const double* __restrict__ values, uint32_t cells, const double* __restrict__ totals,
    float* __restrict__ density) {
  const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= cells) return;
  const double mean = totals[1];
  density[cell] = (mean > 0.0 && isfinite(mean)) ? (float)(values[cell] / mean) : 0.0f;
}

__global__ void k_env_conditional(const double* __restrict__ values, const double* __restrict__ row_sums,
    uint32_t columns, uint32_t rows, float* __restrict__ conditional) {
  const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= rows) return;
  float* cdf = conditional + (size_t)row * (columns + 1);
  const double sum = row_sums[row];
  double along = 0.0;
  cdf[0] = 0.0f;
  for (uint32_t column = 0; column < columns; ++column) {
    along += values[(size_t)row * columns + column];
    cdf[column + 1] = sum > 0.0 ? (float)(along / sum) : (float)(column + 1) / columns;
  }
  cdf[columns] = 1.0f;
}

// Guide entry k of table `table` (0: the marginal; 1 + r: row r's
// conditional): the CDF entries <= k / K (std::upper_bound's count).
__global__ void k_env_guides(const float* __restrict__ marginal, const float* __restrict__ conditional,
    uint32_t columns, uint32_t rows, uint32_t* __restrict__ guides) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t marginal_entries = kEnvGuideMarginal + 1;
  const uint32_t total = marginal_entries + rows * (kEnvGuideConditional + 1);
  if (i >= total) return;
  const float* F;
  uint32_t entries, buckets, k;
  if (i < marginal_entries) {
    F = marginal;
    entries = rows + 1;
    buckets = kEnvGuideMarginal;
    k = i;
  } else {
    const uint32_t j = i - marginal_entries, row = j / (kEnvGuideConditional + 1);
    F = conditional + (size_t)row * (columns + 1);
    entries = columns + 1;
    buckets = kEnvGuideConditional;
    k = j % (kEnvGuideConditional + 1);
  }
  const float x = (float)k / (float)buckets;
  uint32_t lo = 0, hi = entries;  // the first entry above x
  while (lo < hi) {
    const uint32_t mid = (lo + hi) / 2;
    if (x < F[mid]) hi = mid;
    else lo = mid + 1;
  }
  guides[i] = lo;
}

// The light table (BuildLightTable, gpu_scene.cpp:515-610): every emissive
// triangle weighted by its mean emission times its world area, every
// analytic light by its estimated power, then the environment image
// weighted as a distant light over the scene's bounding sphere, chosen by
// Vose's alias method; with the analytic records, the crossing hierarchy
// over the bounded ones and the distant lights' indices.
struct LightTable {
  std::vector<LightRecord> records;
  std::vector<uint32_t> offsets;  // per instance
  std::vector<float4> verts;      // 3 per entry
  std::vector<float4> radiance;   // 1 per entry
  std::vector<AnalyticLight> analytic;
  std::vector<LightNode> nodes;
  std::vector<uint32_t> distant;
  float env_selection = 0.0f;
};

struct HostD3 {
  double x, y, z;
};
HostD3 column3(const float* m, int c) { return HostD3{m[4 * c], m[4 * c + 1], m[4 * c + 2]}; }
double dot3(HostD3 a, HostD3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
HostD3 cross3(HostD3 a, HostD3 b) { return HostD3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
HostD3 scale3(HostD3 a, double s) { return HostD3{a.x * s, a.y * s, a.z * s}; }
float4 store4(HostD3 v, double w) { return make_float4((float)v.x, (float)v.y, (float)v.z, (float)w); }

// MakeAnalyticLight (gpu_scene.cpp:272-369): a light's record and its table
// weight, its estimated power over 2 pi, the scale of an emissive
// triangle's (a distant light's through a disk of the scene's radius).
// False for a light that emits nothing: black, of zero size, or whose
// radiance after normalization is not a finite float.
bool make_analytic_light(const lotus_light& light, double radius_of_scene, double& weight, AnalyticLight& rec) {
  constexpr double kPiD = 3.14159265358979323846;
  const float* m = light.world_from_light;
  const HostD3 x = column3(m, 0), y = column3(m, 1), z = column3(m, 2), origin = column3(m, 3);
  const double determinant = dot3(x, cross3(y, z));
  rec = AnalyticLight{};
  double extent = 0.0, scale = 1.0;
  if (light.shape == LOTUS_LIGHT_SPHERE) {
    const double radius = light.radius * std::cbrt(std::fabs(determinant));
    extent = 4.0 * kPiD * radius * radius;
    rec.shape = kSphereLight;
    rec.position = store4(origin, radius);
    rec.normal = store4(HostD3{0, 0, 0}, extent);
  } else if (light.shape == LOTUS_LIGHT_RECT || light.shape == LOTUS_LIGHT_DISK) {
    const bool rect = light.shape == LOTUS_LIGHT_RECT;
    const HostD3 u = scale3(x, rect ? 0.5 * light.width : light.radius);
    const HostD3 v = scale3(y, rect ? 0.5 * light.height : light.radius);
    const HostD3 normal = cross3(u, v);
    const double length = std::sqrt(dot3(normal, normal));
    extent = (rect ? 4.0 : kPiD) * length;
    rec.shape = rect ? kRectLight : kDiskLight;
    rec.position = store4(origin, 0.0);
    rec.axis_u = store4(u, 0.0);
    rec.axis_v = store4(v, 0.0);
    // The -Z side, where the frame's inverse transpose takes the normal.
    if (length > 0.0) rec.normal = store4(scale3(normal, (determinant < 0.0 ? 1.0 : -1.0) / length), extent);
  } else {
    const double length = std::sqrt(dot3(z, z));
    if (!(length > 0.0)) return false;
    const double theta = std::min(static_cast<double>(light.angle) * kPiD / 360.0, kPiD);
    const double half = std::sin(0.5 * theta);
    const double one_minus_cos = 2.0 * half * half;
    const double sin2 = std::sin(theta) * std::sin(theta);
    rec.axis_u = store4(scale3(z, 1.0 / length), one_minus_cos);
    rec.shape = kParallelLight;
    extent = 1.0;
    if (theta > 0.0) {
      extent = theta <= 0.5 * kPiD ? kPiD * sin2 : kPiD;
      if (light.normalize) scale = 1.0 / (theta <= 0.5 * kPiD ? kPiD * sin2 : (2.0 - sin2) * kPiD);
      if (static_cast<float>(one_minus_cos) >= std::numeric_limits<float>::min()) {
        rec.shape = kDistantLight;
      } else {
        // Too narrow a cone for float densities: its irradiance, from one
        // direction.
        scale *= extent;
        extent = 1.0;
      }
    }
  }
  if (light.normalize && light.shape != LOTUS_LIGHT_DISTANT) scale = 1.0 / extent;
  double radiance[3];
  for (int c = 0; c < 3; ++c) radiance[c] = light.radiance[c] * scale;
  const double mean = (radiance[0] + radiance[1] + radiance[2]) / 3.0;
  constexpr double kFloatMaxD = std::numeric_limits<float>::max();
  if (!(extent > 0.0) || !std::isfinite(extent) || !(mean > 0.0) ||
      !(radiance[0] <= kFloatMaxD && radiance[1] <= kFloatMaxD && radiance[2] <= kFloatMaxD))
    return false;
  rec.radiance = store4(HostD3{radiance[0], radiance[1], radiance[2]}, 0.0);
  weight = mean * extent / 2.0;
  if (light.shape == LOTUS_LIGHT_DISTANT) weight *= radius_of_scene * radius_of_scene;
  if (!std::isfinite(weight)) weight = std::numeric_limits<double>::max();
  return true;
}

// A bounded light's box (BoundLight, gpu_scene.cpp:398-428), widened by
// 1e-4 of its extent plus 1e-5 of its coordinates' magnitude and rounded
// outwards, so that the crossing test's rounding of a grazing ray cannot
// leave the light outside it; and the centre the hierarchy splits by.
struct LightBox {
  float low[3], high[3];
  double centre[3];
  uint32_t index;
};

LightBox bound_light(const AnalyticLight& light, uint32_t index) {
  LightBox b;
  b.index = index;
  const float pos[3] = {light.position.x, light.position.y, light.position.z};
  const float au[3] = {light.axis_u.x, light.axis_u.y, light.axis_u.z};
  const float av[3] = {light.axis_v.x, light.axis_v.y, light.axis_v.z};
  for (int a = 0; a < 3; ++a) {
    const double centre = pos[a], u = au[a], v = av[a];
    const double extent = light.shape == kSphereLight ? (double)light.position.w
        : light.shape == kRectLight                   ? std::fabs(u) + std::fabs(v)
                                                      : std::sqrt(u * u + v * v);
    const double margin = 1e-4 * extent + 1e-5 * (std::fabs(centre) + extent);
    b.centre[a] = centre;
    b.low[a] = std::nextafter((float)(centre - extent - margin), -std::numeric_limits<float>::infinity());
    b.high[a] = std::nextafter((float)(centre + extent + margin), std::numeric_limits<float>::infinity());
  }
  return b;
}

void store_bounds(float4& low, float4& high, const LightBox* first, const LightBox* last, uint32_t child) {
  float lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = std::numeric_limits<float>::max();
    hi[a] = -std::numeric_limits<float>::max();
    for (const LightBox* it = first; it != last; ++it) {
      lo[a] = std::min(lo[a], it->low[a]);
      hi[a] = std::max(hi[a], it->high[a]);
    }
  }
  float w;
  std::memcpy(&w, &child, 4);
  low = make_float4(lo[0], lo[1], lo[2], w);
  high = make_float4(hi[0], hi[1], hi[2], 0.0f);
}

// BuildLightNode (gpu_scene.cpp:438-476): a leaf for one light, otherwise a
// node whose children split the lights at the median centre along the axis
// of widest centre spread (ties by index, so the hierarchy depends only on
// the lights; depth at most ceil(log2(count))). Nodes in preorder.
uint32_t build_light_node(LightBox* first, LightBox* last, std::vector<LightNode>& nodes) {
  if (last - first == 1) return kLightLeaf | first->index;
  const uint32_t node = (uint32_t)nodes.size();
  nodes.emplace_back();
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) lo[a] = hi[a] = first->centre[a];
  for (const LightBox* it = first; it != last; ++it)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], it->centre[a]);
      hi[a] = std::max(hi[a], it->centre[a]);
    }
  int axis = 0;
  for (int c = 1; c < 3; ++c)
    if (hi[c] - lo[c] > hi[axis] - lo[axis]) axis = c;
  LightBox* middle = first + (last - first) / 2;
  std::nth_element(first, middle, last, [axis](const LightBox& a, const LightBox& b) {
    return a.centre[axis] != b.centre[axis] ? a.centre[axis] < b.centre[axis] : a.index < b.index;
  });
  const uint32_t left = build_light_node(first, middle, nodes);
  const uint32_t right = build_light_node(middle, last, nodes);
  LightNode& stored = nodes[node];
  store_bounds(stored.low0, stored.high0, first, middle, left);
  store_bounds(stored.low1, stored.high1, middle, last, right);
  return node;
}

// BuildLightHierarchy (gpu_scene.cpp:478-499): the crossing hierarchy over
// the sphere, rect and disk lights and the distant lights' indices;
// parallel lights, which no ray crosses, are in neither. One bounded light
// gets a root whose second child is empty.
void build_light_hierarchy(LightTable& table) {
  std::vector<LightBox> bounded;
  for (size_t i = 0; i < table.analytic.size(); ++i) {
    const uint32_t shape = table.analytic[i].shape;
    if (shape == kDistantLight)
      table.distant.push_back((uint32_t)i);
    else if (shape != kParallelLight)
      bounded.push_back(bound_light(table.analytic[i], (uint32_t)i));
  }
  if (bounded.size() == 1) {
    LightNode root;
    store_bounds(root.low0, root.high0, bounded.data(), bounded.data() + 1, kLightLeaf | bounded[0].index);
    store_bounds(root.low1, root.high1, nullptr, nullptr, kNoLightChild);
    table.nodes.push_back(root);
  } else if (bounded.size() > 1) {
    build_light_node(bounded.data(), bounded.data() + bounded.size(), table.nodes);
  }
}

double world_triangle_area(const lotus_geometry& g, uint32_t t, const float* m) {
  double corners[3][3];
  for (int k = 0; k < 3; ++k) {
    const float* p = g.positions + 3 * (size_t)g.triangles[3 * (size_t)t + k];
    for (int r = 0; r < 3; ++r)
      corners[k][r] = (double)m[r] * p[0] + (double)m[4 + r] * p[1] + (double)m[8 + r] * p[2] + m[12 + r];
  }
  double a[3], b[3];
  for (int r = 0; r < 3; ++r) {
    a[r] = corners[1][r] - corners[0][r];
    b[r] = corners[2][r] - corners[0][r];
  }
  const double x = a[1] * b[2] - a[2] * b[1], y = a[2] * b[0] - a[0] * b[2], z = a[0] * b[1] - a[1] * b[0];
  const double area = 0.5 * std::sqrt(x * x + y * y + z * z);
  return std::isfinite(area) ? area : 0.0;
}

double scene_radius(const lotus_scene_desc& s) {
  constexpr double kInf = std::numeric_limits<double>::infinity();
  std::vector<std::array<double, 6>> object(s.geometry_count);
  std::vector<char> done(s.geometry_count, 0);
  std::array<double, 6> world{kInf, kInf, kInf, -kInf, -kInf, -kInf};
  for (uint32_t i = 0; i < s.instance_count; ++i) {
    const lotus_instance& inst = s.instances[i];
    auto& b = object[inst.geometry];
    if (!done[inst.geometry]) {
      done[inst.geometry] = 1;
      b = {kInf, kInf, kInf, -kInf, -kInf, -kInf};
      const lotus_geometry& g = s.geometries[inst.geometry];
      for (uint32_t v = 0; v < g.vertex_count; ++v)
        for (int a = 0; a < 3; ++a) {
          b[a] = std::min(b[a], (double)g.positions[3 * (size_t)v + a]);
          b[3 + a] = std::max(b[3 + a], (double)g.positions[3 * (size_t)v + a]);
        }
    }
    if (!(b[0] <= b[3])) continue;
    const float* m = inst.world_from_object;
    for (int corner = 0; corner < 8; ++corner) {
      const double p[3] = {b[(corner & 1) ? 3 : 0], b[(corner & 2) ? 4 : 1], b[(corner & 4) ? 5 : 2]};
      for (int r = 0; r < 3; ++r) {
        const double v = m[r] * p[0] + m[4 + r] * p[1] + m[8 + r] * p[2] + m[12 + r];
        world[r] = std::min(world[r], v);
        world[3 + r] = std::max(world[3 + r], v);
      }
    }
  }
  if (!(world[0] <= world[3])) return 0.0;
  const double d[3] = {world[3] - world[0], world[4] - world[1], world[5] - world[2]};
  const double radius = 0.5 * std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  return std::isfinite(radius) ? radius : 0.0;
}

LightTable build_light_table(const lotus_scene_desc& s, double env_mean) {
  LightTable table;
  table.offsets.assign(s.instance_count, kNoLights);
  std::vector<double> weights;
  for (uint32_t index = 0; index < s.instance_count; ++index) {
    const lotus_instance& inst = s.instances[index];
    const lotus_geometry& g = s.geometries[inst.geometry];
    const lotus_material& mat = s.materials[inst.material];
    // EmissionEstimate (gpu_scene.cpp:144-180): the mean of the constant's
    // RGB, or of a lookup's bound for texels in [0, 1] (its fallback when
    // it names no image).
    // glTF PBR's emissive (the same slot as UsdPreviewSurface's emission)
    // is scaled by its strength.
    const bool gltf = mat.model == LOTUS_MODEL_GLTF_PBR;
    const double factor = gltf ? (double)mat.emissive_strength : 1.0;
    double e = factor * ((double)mat.emission[0] + (double)mat.emission[1] + (double)mat.emission[2]) / 3.0;
    const uint32_t emission_lookup = mat.lookups[LOTUS_SLOT_EMISSION];
    if (emission_lookup != LOTUS_NO_LOOKUP) {
      const lotus_texture_input& in = s.texture_inputs[emission_lookup - 1];
      double c[3];
      for (int k = 0; k < 3; ++k)
        c[k] = in.texture == LOTUS_NO_TEXTURE ? std::max(0.0f, in.fallback[k])
                                              : (double)std::max(0.0f, in.scale[k]) + std::max(0.0f, in.bias[k]);
      e = factor * (c[0] + c[1] + c[2]) / 3.0;
    }
    if (!(std::isfinite(e) && e > 0.0)) e = 0.0;
    if (e <= 0.0 || g.triangle_count == 0) continue;
    table.offsets[index] = (uint32_t)table.records.size();
    const float coverage = host_coverage(mat);
    // Textured emission or opacity: the sample looks it up (radiance w 1).
    const bool looked_up = emission_lookup != LOTUS_NO_LOOKUP || mat.lookups[LOTUS_SLOT_OPACITY] != LOTUS_NO_LOOKUP;
    for (uint32_t t = 0; t < g.triangle_count; ++t) {
      weights.push_back(e * world_triangle_area(g, t, inst.world_from_object));
      table.records.push_back({0.0f, 1.0f, 0u, index});
      for (int k = 0; k < 3; ++k) {
        const HostF3 w = host_transform(inst.world_from_object,
            g.positions + 3 * (size_t)g.triangles[3 * (size_t)t + k]);
        table.verts.push_back(make_float4(w.x, w.y, w.z, 0.0f));
      }
      // Emission(material, st) * Coverage(hit) (scene.slang:655-657): glTF
      // PBR's emissive times its strength.
      const float strength = gltf ? mat.emissive_strength : 1.0f;
      const float e3[3] = {gltf ? mat.emission[0] * strength : mat.emission[0],
                           gltf ? mat.emission[1] * strength : mat.emission[1],
                           gltf ? mat.emission[2] * strength : mat.emission[2]};
      table.radiance.push_back(make_float4(e3[0] * coverage, e3[1] * coverage, e3[2] * coverage,
          looked_up ? 1.0f : 0.0f));
    }
  }
  bool distant = env_mean > 0.0;
  for (uint32_t i = 0; i < s.light_count; ++i) distant = distant || s.lights[i].shape == LOTUS_LIGHT_DISTANT;
  const double r = distant ? scene_radius(s) : 0.0;
  std::vector<uint32_t> analytic_entries;
  for (uint32_t i = 0; i < s.light_count; ++i) {
    double weight = 0.0;
    AnalyticLight rec;
    if (!make_analytic_light(s.lights[i], r, weight, rec)) continue;
    if (weight > 0.0) {
      analytic_entries.push_back((uint32_t)table.records.size());
      weights.push_back(weight);
      table.records.push_back({0.0f, 1.0f, 0u, kAnalyticLight | (uint32_t)table.analytic.size()});
      for (int k = 0; k < 3; ++k) table.verts.push_back(make_float4(0, 0, 0, 0));
      table.radiance.push_back(make_float4(0, 0, 0, 0));
    }
    table.analytic.push_back(rec);
  }
  build_light_hierarchy(table);
  double env_weight = 0.0;
  if (env_mean > 0.0) {
    constexpr double kPiD = 3.14159265358979323846;
    env_weight = kPiD * kPiD * r * r * env_mean;
    if (!std::isfinite(env_weight)) env_weight = std::numeric_limits<double>::max();
  }
  if (env_weight > 0.0) {
    weights.push_back(env_weight);
    table.records.push_back({0.0f, 1.0f, 0u, kEnvironmentLight});
    for (int k = 0; k < 3; ++k) table.verts.push_back(make_float4(0, 0, 0, 0));
    table.radiance.push_back(make_float4(0, 0, 0, 0));
  }
  double total = 0.0;
  for (double w : weights) total += w;
  if (!(total > 0.0) || !std::isfinite(total)) {
    table.offsets.assign(s.instance_count, kNoLights);
    table.records.clear();
    table.verts.clear();
    table.radiance.clear();
    return table;
  }
  const size_t count = table.records.size();
  std::vector<double> scaled(count);
  std::vector<uint32_t> small, large;
  for (size_t i = 0; i < count; ++i) {
    table.records[i].pdf = (float)(weights[i] / total);
    scaled[i] = weights[i] / total * (double)count;
    (scaled[i] < 1.0 ? small : large).push_back((uint32_t)i);
  }
  while (!small.empty() && !large.empty()) {
    const uint32_t less = small.back();
    small.pop_back();
    const uint32_t more = large.back();
    table.records[less].threshold = (float)scaled[less];
    table.records[less].alias = more;
    scaled[more] -= 1.0 - scaled[less];
    if (scaled[more] < 1.0) {
      large.pop_back();
      small.push_back(more);
    }
  }
  for (uint32_t i : small) { table.records[i].threshold = 1.0f; table.records[i].alias = i; }
  for (uint32_t i : large) { table.records[i].threshold = 1.0f; table.records[i].alias = i; }
  // An analytic light's record carries the probability of its table entry:
  // a BSDF-sampled ray that crosses the light needs it for its MIS weight.
  for (uint32_t entry : analytic_entries)
    table.analytic[table.records[entry].instance & ~kAnalyticLight].radiance.w = table.records[entry].pdf;
  if (env_weight > 0.0) table.env_selection = table.records.back().pdf;
  return table;
}

}  // namespace

// The longest chain of samples one RenderScene graph holds (two in flight
// at a time): each sample has its own frame constants.
constexpr uint32_t kMaxChain = 16;
// Samples one wavefront holds (a wave) unless lotus_cuda_options says
// otherwise, and the most it may: the path state and queues have room for
// the renderer's wave size times the target's pixels.
constexpr uint32_t kDefaultWave = 8;
constexpr uint32_t kMaxWave = 8;

// The resident scene as the incremental updates need it: each geometry's
// arrays (owned copies; `geometries` points into them), its box and its
// places in the device arrays and pools, the materials and the
// environment's summary.
struct HostScene {
  std::vector<std::vector<float>> positions, normals;
  std::vector<std::vector<uint32_t>> triangles;
  std::vector<lotus_geometry> geometries;
  std::vector<std::array<float, 6>> boxes;
  std::vector<uint64_t> vertex_base;
  std::vector<uint32_t> node_base, tri_base, normal_base;
  uint64_t nodes = 0;
  std::vector<lotus_material> materials;
  float environment_constant[3] = {0.0f, 0.0f, 0.0f};
  bool env_bound = false;
  double env_mean = 0.0;
  uint32_t env_width = 0, env_height = 0, env_columns = 0, env_rows = 0;
  float env_scale[3] = {0.0f, 0.0f, 0.0f};
  float env_frame[9] = {};
  std::vector<lotus_light> lights;      // the analytic lights
  // Texture lookups: the scene's texture inputs, its texture count, per
  // geometry its texture-coordinate sets and the first (s, t) of its set 0
  // in the device pool.
  std::vector<lotus_texture_input> texture_inputs;
  uint32_t texture_count = 0;
  std::vector<uint64_t> texcoord_base;
  // Per geometry and colour set: its first value in the device's colour
  // array (floats) and whether it is one value for the whole mesh.
  std::vector<std::vector<uint2>> color_sets;
};

static_assert(LOTUS_OUTPUT_BARYCENTRICS == kOutputBarycentrics && LOTUS_OUTPUT_SHADING_NORMAL == kOutputShadingNormal &&
                  LOTUS_OUTPUT_ALBEDO == kOutputAlbedo && LOTUS_OUTPUT_ROUGHNESS_METALLIC == kOutputRoughnessMetallic,
    "diagnostic outputs are numbered as lotus_settings::output");

// The directional albedo tables (albedo_tables_gen.cpp's output, in
// albedo.cuh's layout).
const float kAlbedoTableData[] = {
#include "albedo_tables.inc"
};
static_assert(sizeof(kAlbedoTableData) == albedo::kSize * sizeof(float), "albedo tables");

struct Renderer {
  int device = 0;
  uint32_t bvh_leaf_size = 1;
  TraceTuning tuning;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  std::string failure;
  uint64_t completion = 0;

  // Scene.
  DeviceArray<BvhNode> blas, tlas;      // binary builds (build scratch)
  DeviceArray<Bvh4Node> blas4, tlas4;   // the 4-wide pools the traversal reads
  DeviceArray<float4> tris;
  DeviceArray<InstanceTraversal> inst_trav;
  DeviceArray<InstanceShading> inst_shade;
  DeviceArray<MaterialRecord> materials;
  DeviceArray<float> normals;
  DeviceArray<LightRecord> lights;
  DeviceArray<float4> light_verts, light_radiance;
  DeviceArray<float4> env_texels;
  DeviceArray<float> env_floats;
  DeviceArray<uint32_t> env_guide;
  DeviceArray<AnalyticLight> analytic;
  DeviceArray<LightNode> light_nodes;
  DeviceArray<uint32_t> distant;
  DeviceArray<float4> tex_texels;            // SceneView::tex_texels
  DeviceArray<uint4> tex_info;
  DeviceArray<TextureLookup> tex_lookups;
  DeviceArray<MaterialLookups> mat_lookups;
  DeviceArray<float> albedo_tables;  // the composed closure's (albedo.cuh), uploaded once
  DeviceArray<float2> texcoords;
  DeviceArray<uint32_t> inst_texcoords;
  DeviceArray<float> colors;         // every geometry's colour sets, RGB
  DeviceArray<uint2> inst_colors;    // per instance: (first float, whole-mesh flag) or kNoTexture
  std::vector<LightRecord> host_lights;
  std::vector<uint32_t> host_light_offsets;
  SceneView view{};
  HostScene host;                       // the resident scene's host copy
  DeviceArray<float> scene_pos;         // every geometry's positions, kept for rebuilds
  DeviceArray<uint32_t> scene_tri;      // every geometry's triangles
  bool scene_ready = false;
  uint64_t scene_generation = 0;
  BvhBuilder builder;

  // Targets.
  uint32_t width = 0, height = 0;
  DeviceArray<double4> accum;
  DeviceArray<float4> color;
  DeviceArray<float> depth;   // the D32 depth product (LOTUS_FRAME_DEPTH)
  bool depth_valid = false;   // the latest RenderScene frame wrote it
  bool depth_fresh = true;    // allocated since its last clear: DEPTH_KEEP clears it too
  DeviceArray<float4> path_origin, path_direction, path_throughput, path_radiance;
  DeviceArray<uint4> path_hit;
  DeviceArray<uint32_t> queue_ray0, queue_ray1, queue_hit, counts;
  DeviceArray<float4> sq_o, sq_d, sq_fl, sq_thr;
  DeviceArray<uint32_t> sort_keys, sort_queue, sort_bins;  // Queues::keys, sorted, bins
  DeviceArray<uint32_t> cache_query_keys, cache_query_order, cache_query_bins;  // CacheQueues::query_*
  // A second path state and queue set, for the second of two samples in
  // flight at once (RenderScene with two or more samples to add): its
  // rounds overlap the first one's tail, on a second stream.
  DeviceArray<float4> path_origin2, path_direction2, path_throughput2, path_radiance2;
  DeviceArray<uint4> path_hit2;
  DeviceArray<uint32_t> queue_ray02, queue_ray12, queue_hit2, counts2;
  DeviceArray<float4> sq_o2, sq_d2, sq_fl2, sq_thr2;
  DeviceArray<uint32_t> sort_keys2, sort_queue2, sort_bins2;
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  std::vector<cudaEvent_t> ev_sample_done;  // per sample of a chain: resolved and counted
  DeviceArray<FrameConst> frame_const;
  DeviceArray<RayTotals> totals;
  DeviceArray<VisitCounters> visits;
  // SceneView::walk_failure: failed BVH walks and their causes, cleared
  // before and read after each frame.
  DeviceArray<uint32_t> walk_failure;
  uint32_t step_limit = kMaxTraversalSteps;
  uint32_t wave = kDefaultWave;  // samples per wavefront (lotus_cuda_options::samples_per_wave)
  // Profiling events, created on first use.
  std::vector<cudaEvent_t> profile_events;
  std::vector<int> profile_kinds;

  // Accumulation key (vulkan_backend.cpp:414-431).
  struct Key {
    float world_to_clip[16];
    uint32_t width, height;
    float display_window[4];
    int32_t data_window[4];
    uint32_t integrator, light_sampling, restir_proposal, restir_candidates, sample_index,
        max_bounces;
    uint64_t scene_generation;
    bool operator==(const Key& o) const { return std::memcmp(this, &o, sizeof(Key)) == 0; }
  };
  Key key{};
  bool key_valid = false;
  uint32_t accumulated = 0;

  // Temporal streams (RenderTemporalScene).
  struct Temporal {
    uint32_t width = 0, height = 0;
    DeviceArray<TemporalPixel> surface[2];
    DeviceArray<ValidityPixel> validity;
    DeviceArray<RadiancePixel> radiance[2];
    DeviceArray<float4> batch;
    DeviceArray<float4> filter;
    DeviceArray<RestirPixel> initial;
    DeviceArray<RestirReuse> reuse[2];
    DeviceArray<RestirReuse> spatial;
    DeviceArray<uint4> sources;
    DeviceArray<RestirSurface> surfaces[2];
    DeviceArray<uint4> primary_hit;     // the camera rays' hits, traced once per frame
    DeviceArray<uint32_t> primary_rng;
    // The ReSTIR passes' deferred visibility (VisibilityQueue).
    DeviceArray<float4> vis_origin, vis_direction, vis_pending;
    DeviceArray<uint32_t> vis_slot, vis_counters;
    DeviceArray<TemporalConst> constants;
    DeviceArray<TemporalInstance> instances;
    bool instances_custom = false;
    int surface_write = 0, radiance_write = 0, restir_write = 0;
    int last_surface = 0, last_radiance = 0, last_restir = 0;
    uint32_t frames = 0;          // temporal frames rendered since the last reset
    uint32_t sample_offset = 0;
    bool key_valid = false;
    uint32_t key[18] = {};
    bool restir_ran = false, accumulate_ran = false, spatial_ran = false, filter_ran = false;
    bool moments_half = false;  // the latest frame's radiance records keep FP16 central moments
  } temporal;
  std::vector<lotus_instance> host_instances;
  // World bounds of the resident scene (the radiance cache's grid box).
  float scene_lo[3] = {0.0f, 0.0f, 0.0f}, scene_hi[3] = {1.0f, 1.0f, 1.0f};

  // The learned radiance cache and its per-sample queues.
  RadianceCache cache;
  lotus_cache_desc cache_desc{};
  bool cache_enabled = false;
  DeviceArray<CacheRecord> cache_queries, cache_train;
  DeviceArray<uint32_t> cache_query_slots, cache_train_slots, cache_counters;
  DeviceArray<float4> cache_query_throughput, cache_train_base, cache_train_throughput, cache_train_targets;
  uint32_t cache_pixels = 0;
  uint32_t cache_generation = 0;  // bumped by every configuration

  // The wavefront sample as a CUDA graph, and chains of two samples in
  // flight: one instantiated graph per chain length (2, 4, .. kMaxChain,
  // at index length / 2), all of one key, so that a call whose remainder
  // makes a short chain does not re-instantiate the long one.
  cudaGraphExec_t graph = nullptr;
  cudaGraphExec_t graph_chains[3 * (kMaxChain / 2 + 1)] = {};
  struct GraphKey {
    uint64_t scene_generation;
    uint32_t width, height, max_bounces;
    uint32_t rect[4];
    uint32_t cache;  // the radiance cache's configuration count (0: off)
    uint32_t rounds; // wavefront rounds before the tail kernel
    bool operator==(const GraphKey& o) const { return std::memcmp(this, &o, sizeof(GraphKey)) == 0; }
  } graph_key{}, graph_chain_key{};
  // Rounds before the tail, chosen (choose_wavefront_rounds) from the queue
  // counts of the first sample rendered with `rounds_key` (its rounds field
  // 0), for RenderScene and for the temporal frames.
  GraphKey rounds_key{}, temporal_rounds_key{};
  uint32_t auto_rounds = 0, temporal_auto_rounds = 0;

  ~Renderer() {
    for (cudaEvent_t e : profile_events) cudaEventDestroy(e);
    if (graph) cudaGraphExecDestroy(graph);
    for (cudaGraphExec_t g : graph_chains)
      if (g) cudaGraphExecDestroy(g);
    for (cudaEvent_t e : {ev_fork, ev_join})
      if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ev_sample_done) cudaEventDestroy(e);
    if (stream2) cudaStreamDestroy(stream2);
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_stop) cudaEventDestroy(ev_stop);
    if (stream) cudaStreamDestroy(stream);
  }

  bool ok(cudaError_t e, const char* what, std::string& detail) {
    if (e == cudaSuccess) return true;
    detail = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
  }

  void release_scene() {
    scene_pos.release(); scene_tri.release(); host = HostScene{};
    blas.release(); tlas.release(); blas4.release(); tlas4.release(); tris.release(); inst_trav.release(); inst_shade.release();
    materials.release(); normals.release(); lights.release(); light_verts.release();
    light_radiance.release(); env_texels.release(); env_floats.release(); env_guide.release();
    analytic.release(); light_nodes.release(); distant.release();
    tex_texels.release(); tex_info.release(); tex_lookups.release(); mat_lookups.release(); texcoords.release();
    inst_texcoords.release(); colors.release(); inst_colors.release();
    scene_ready = false;
  }

  uint64_t scene_bytes() const {
    return scene_pos.bytes() + scene_tri.bytes() + blas.bytes() + tlas.bytes() + blas4.bytes() + tlas4.bytes() + tris.bytes() + inst_trav.bytes() + inst_shade.bytes() +
           materials.bytes() + normals.bytes() + lights.bytes() + light_verts.bytes() +
           light_radiance.bytes() + env_texels.bytes() + env_floats.bytes() + env_guide.bytes() +
           analytic.bytes() + light_nodes.bytes() + distant.bytes() + tex_texels.bytes() + tex_info.bytes() +
           tex_lookups.bytes() + mat_lookups.bytes() + texcoords.bytes() + inst_texcoords.bytes() +
           colors.bytes() + inst_colors.bytes();
  }
};

}  // namespace lotus

using lotus::Renderer;

struct lotus_cuda_renderer {
  Renderer r;
};

namespace {

using namespace lotus;

bool validate_scene(const lotus_scene_desc& s, std::string& detail) {
  if (s.material_count == 0 || !s.materials) {
    detail = "the scene has no material table";
    return false;
  }
  if ((s.geometry_count && !s.geometries) || (s.instance_count && !s.instances)) {
    detail = "the scene's geometry or instance array is missing";
    return false;
  }
  if ((s.texture_count && !s.textures) || (s.texture_input_count && !s.texture_inputs)) {
    detail = "the scene's texture or texture-input array is missing";
    return false;
  }
  for (uint32_t i = 0; i < s.texture_count; ++i) {
    const lotus_texture& t = s.textures[i];
    if (t.width == 0 || t.height == 0 || !t.texels || t.format > LOTUS_TEXTURE_RGBA32_FLOAT ||
        (uint64_t)t.width * t.height > (1ull << 28)) {
      detail = "texture " + std::to_string(i) + " is empty, too large or of an unknown format";
      return false;
    }
  }
  for (uint32_t i = 0; i < s.texture_input_count; ++i) {
    const lotus_texture_input& in = s.texture_inputs[i];
    bool finite = true;
    for (int k = 0; k < 4; ++k)
      finite = finite && std::isfinite(in.scale[k]) && std::isfinite(in.bias[k]) && std::isfinite(in.fallback[k]);
    for (int k = 0; k < 6; ++k) finite = finite && std::isfinite(in.st_transform[k]);
    if ((in.texture != LOTUS_NO_TEXTURE && in.texture > s.texture_count) || in.channel > 3 ||
        in.wrap_s > LOTUS_WRAP_MIRROR || in.wrap_t > LOTUS_WRAP_MIRROR || !finite) {
      detail = "texture input " + std::to_string(i) + " names a missing texture or has an invalid field";
      return false;
    }
  }
  for (uint32_t g = 0; g < s.geometry_count; ++g) {
    const lotus_geometry& geo = s.geometries[g];
    if (geo.triangle_count && (!geo.triangles || !geo.positions)) {
      detail = "geometry " + std::to_string(g) + " has triangles without data";
      return false;
    }
    if (geo.texcoord_sets && !geo.texcoords) {
      detail = "geometry " + std::to_string(g) + " has texture-coordinate sets without data";
      return false;
    }
    if (geo.color_sets && (!geo.colors || !geo.color_counts)) {
      detail = "geometry " + std::to_string(g) + " has colour sets without data";
      return false;
    }
    uint64_t color_values = 0;
    for (uint32_t k = 0; k < geo.color_sets; ++k) {
      if (geo.color_counts[k] != 1 && geo.color_counts[k] != 3ull * geo.triangle_count) {
        detail = "geometry " + std::to_string(g) + "'s colour set " + std::to_string(k) +
                 " has neither one value nor one per triangle corner";
        return false;
      }
      color_values += geo.color_counts[k];
    }
    for (uint64_t i = 0; i < 3 * color_values; ++i)
      if (!std::isfinite(geo.colors[i])) {
        detail = "geometry " + std::to_string(g) + " has a non-finite colour";
        return false;
      }
    for (uint64_t i = 0; i < 3ull * geo.triangle_count; ++i)
      if (geo.triangles[i] >= geo.vertex_count) {
        detail = "geometry " + std::to_string(g) + " indexes past its vertices";
        return false;
      }
    for (uint64_t i = 0; i < 3ull * geo.vertex_count; ++i)
      if (!std::isfinite(geo.positions[i])) {
        detail = "geometry " + std::to_string(g) + " has a non-finite position";
        return false;
      }
  }
  for (uint32_t i = 0; i < s.instance_count; ++i) {
    const lotus_instance& inst = s.instances[i];
    if (inst.geometry >= s.geometry_count || inst.material >= s.material_count) {
      detail = "instance " + std::to_string(i) + " names a missing geometry or material";
      return false;
    }
    if (inst.texcoord_set != LOTUS_NO_TEXCOORDS && inst.texcoord_set > s.geometries[inst.geometry].texcoord_sets) {
      detail = "instance " + std::to_string(i) + " names a missing texture-coordinate set";
      return false;
    }
    if (inst.color_set != LOTUS_NO_COLORS && inst.color_set > s.geometries[inst.geometry].color_sets) {
      detail = "instance " + std::to_string(i) + " names a missing colour set";
      return false;
    }
    const float* m = inst.world_from_object;
    if (m[3] != 0.0f || m[7] != 0.0f || m[11] != 0.0f || m[15] != 1.0f) {
      detail = "instance " + std::to_string(i) + " has a projective transform";
      return false;
    }
  }
  for (uint32_t i = 0; i < s.material_count; ++i) {
    const lotus_material& m = s.materials[i];
    const float* f = &m.base_color[0];
    for (int k = 0; k < 18; ++k)
      if (!std::isfinite(f[k])) {
        detail = "material " + std::to_string(i) + " has a non-finite value";
        return false;
      }
    if (!(m.ior >= 1.0f)) {
      detail = "material " + std::to_string(i) + " has an ior below 1";
      return false;
    }
    if (m.model != LOTUS_MODEL_PREVIEW_SURFACE && m.model != LOTUS_MODEL_GLTF_PBR) {
      detail = "material " + std::to_string(i) + " has an unknown model";
      return false;
    }
    if (m.model == LOTUS_MODEL_GLTF_PBR) {
      // ValidGltfPbr (gpu_scene.cpp:853-881).
      const auto unit = [](float v) { return v >= 0.0f && v <= 1.0f; };
      const auto radiance = [](const float* c) {
        return std::isfinite(c[0]) && std::isfinite(c[1]) && std::isfinite(c[2]) && c[0] >= 0.0f &&
            c[1] >= 0.0f && c[2] >= 0.0f;
      };
      const bool valid = unit(m.base_color[0]) && unit(m.base_color[1]) && unit(m.base_color[2]) &&
          unit(m.roughness) && unit(m.metallic) && radiance(m.emission) &&
          std::isfinite(m.emissive_strength) && m.emissive_strength >= 0.0f && unit(m.specular) &&
          radiance(m.specular_color) && unit(m.transmission) && unit(m.clearcoat) &&
          unit(m.clearcoat_roughness) && unit(m.sheen_color[0]) && unit(m.sheen_color[1]) &&
          unit(m.sheen_color[2]) && unit(m.sheen_roughness);
      if (!valid) {
        detail = "material " + std::to_string(i) + " has a glTF PBR input out of its range";
        return false;
      }
    }
    for (uint32_t k = 0; k < LOTUS_TEXTURE_SLOTS; ++k)
      if (m.lookups[k] != LOTUS_NO_LOOKUP && m.lookups[k] > s.texture_input_count) {
        detail = "material " + std::to_string(i) + " names a missing texture input";
        return false;
      }
    if (!std::isfinite(m.texcoord_fallback[0]) || !std::isfinite(m.texcoord_fallback[1]) ||
        !std::isfinite(m.normal[0]) || !std::isfinite(m.normal[1]) || !std::isfinite(m.normal[2])) {
      detail = "material " + std::to_string(i) + " has a non-finite texture-coordinate fallback or normal";
      return false;
    }
  }
  if (s.environment && s.environment->texels == nullptr &&
      (s.environment->width || s.environment->height)) {
    detail = "the environment image has no texels";
    return false;
  }
  if (s.light_count && !s.lights) {
    detail = "light_count without lights";
    return false;
  }
  // The crossing hierarchy's depth, ceil(log2(lights)), must fit the
  // traversal's stack.
  if (s.light_count >= (1u << 30)) {
    detail = "too many analytic lights";
    return false;
  }
  for (uint32_t i = 0; i < s.light_count; ++i) {
    const lotus_light& l = s.lights[i];
    bool finite = std::isfinite(l.radius) && std::isfinite(l.width) && std::isfinite(l.height) &&
        std::isfinite(l.angle);
    for (float v : l.world_from_light) finite = finite && std::isfinite(v);
    for (float v : l.radiance) finite = finite && std::isfinite(v);
    if (l.shape > LOTUS_LIGHT_DISTANT || !finite) {
      detail = "analytic light " + std::to_string(i) + " has an unknown shape or a non-finite value";
      return false;
    }
  }
  return true;
}

// ---------------------------------------------------------------------------
// Scene updates. A full update (UpdateScene) uploads every geometry, builds
// every BLAS, the materials, the environment and the instance state; the
// incremental ones rebuild only what an edit invalidates, from the resident
// scene's host copy and its device position and triangle arrays:
//   - lotus_cuda_update_instances (transform / material-slot edits): the
//     light table, the instance records and the TLAS;
//   - lotus_cuda_update_geometry (point edits of one geometry, topology
//     kept): that geometry's BLAS refitted in place in its own node and
//     triangle ranges, its corner normals, then the instance state.
// The reference refits in both cases (gpu_scene.cpp:2303-2322); the TLAS is
// rebuilt here, which decides the same hits, since hits are decided by
// triangle tests alone.

// Host-side instance state, prepared before any of it goes to the device.
struct InstanceState {
  LightTable table;
  std::vector<InstanceTraversal> trav;
  std::vector<InstanceShading> shade;
  std::vector<uint32_t> texcoords;  // SceneView::inst_texcoords
  std::vector<uint2> colors;        // SceneView::inst_colors
};

lotus_scene_desc host_desc(const Renderer& R) {
  const HostScene& h = R.host;
  lotus_scene_desc d{};
  d.geometries = h.geometries.data();
  d.instances = R.host_instances.data();
  d.materials = h.materials.data();
  d.environment = nullptr;
  d.geometry_count = (uint32_t)h.geometries.size();
  d.instance_count = (uint32_t)R.host_instances.size();
  d.material_count = (uint32_t)h.materials.size();
  for (int k = 0; k < 3; ++k) d.environment_constant[k] = h.environment_constant[k];
  d.lights = h.lights.data();
  d.light_count = (uint32_t)h.lights.size();
  d.texture_inputs = h.texture_inputs.data();
  d.texture_input_count = (uint32_t)h.texture_inputs.size();
  d.texture_count = h.texture_count;
  return d;
}

std::array<float, 6> geometry_box(const lotus_geometry& geo) {
  std::array<float, 6> b = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
  for (uint32_t v = 0; v < geo.vertex_count; ++v)
    for (int a = 0; a < 3; ++a) {
      b[a] = std::min(b[a], geo.positions[3 * (size_t)v + a]);
      b[3 + a] = std::max(b[3 + a], geo.positions[3 * (size_t)v + a]);
    }
  return b;
}

// The light table, world bounds and instance records of the host copy.
bool prepare_instances(Renderer& R, InstanceState& out, std::string& detail) {
  const HostScene& h = R.host;
  const lotus_scene_desc s = host_desc(R);
  out.table = build_light_table(s, h.env_bound ? h.env_mean : 0.0);
  // World bounds: each instance's geometry box through its transform.
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = 0; i < s.instance_count; ++i) {
    const std::array<float, 6>& b = h.boxes[s.instances[i].geometry];
    if (!(b[0] <= b[3])) continue;
    const float* m = s.instances[i].world_from_object;
    for (int c = 0; c < 8; ++c) {
      const float p[3] = {(c & 1) ? b[3] : b[0], (c & 2) ? b[4] : b[1], (c & 4) ? b[5] : b[2]};
      for (int a = 0; a < 3; ++a) {
        const float w = m[a] * p[0] + m[4 + a] * p[1] + m[8 + a] * p[2] + m[12 + a];
        lo[a] = std::min(lo[a], w);
        hi[a] = std::max(hi[a], w);
      }
    }
  }
  for (int a = 0; a < 3; ++a) {
    R.scene_lo[a] = std::isfinite(lo[a]) ? lo[a] : 0.0f;
    R.scene_hi[a] = std::isfinite(hi[a]) ? hi[a] : 1.0f;
  }
  out.trav.resize(s.instance_count);
  out.shade.resize(s.instance_count);
  out.texcoords.resize(s.instance_count);
  out.colors.resize(s.instance_count);
  for (uint32_t i = 0; i < s.instance_count; ++i) {
    const lotus_instance& inst = s.instances[i];
    const float* m = inst.world_from_object;
    InstanceTraversal& t = out.trav[i];
    InstanceShading& sh = out.shade[i];
    if (!invert_affine(m, t.inv)) {
      detail = "instance " + std::to_string(i) + " has a singular transform";
      return false;
    }
    const lotus_geometry& geo = s.geometries[inst.geometry];
    t.blas_root = geo.triangle_count ? h.node_base[inst.geometry] : (uint32_t)kEmptyChild;
    const lotus_material& mat = s.materials[inst.material];
    t.flags = host_coverage(mat) >= 1.0f && mat.lookups[LOTUS_SLOT_OPACITY] == LOTUS_NO_LOOKUP ? kInstanceOpaque : 0u;
    out.texcoords[i] =
        inst.texcoord_set == LOTUS_NO_TEXCOORDS || inst.texcoord_set > geo.texcoord_sets
            ? kNoTexture
            : (uint32_t)(h.texcoord_base[inst.geometry] + 3ull * geo.triangle_count * (inst.texcoord_set - 1));
    out.colors[i] = inst.color_set == LOTUS_NO_COLORS || inst.color_set > geo.color_sets
                        ? make_uint2(kNoTexture, 0u)
                        : h.color_sets[inst.geometry][inst.color_set - 1];
    t.material = inst.material;
    t.light_offset = out.table.offsets[i];
    for (int r = 0; r < 3; ++r) sh.m[r] = make_float4(m[r], m[4 + r], m[8 + r], m[12 + r]);
    sh.material = inst.material;
    sh.light_offset = out.table.offsets[i];
    sh.normals = h.normal_base[inst.geometry];
    // dot(c0, cross(c1, c2)) < 0 (scene.slang:1237-1240).
    const float c0[3] = {m[0], m[1], m[2]}, c1[3] = {m[4], m[5], m[6]}, c2[3] = {m[8], m[9], m[10]};
    const float x = c1[1] * c2[2] - c1[2] * c2[1], y = c1[2] * c2[0] - c1[0] * c2[2],
                z = c1[0] * c2[1] - c1[1] * c2[0];
    sh.mirror = (c0[0] * x + c0[1] * y + c0[2] * z) < 0.0f ? 1u : 0u;
  }
  return true;
}

// Uploads the prepared instance state, builds the TLAS and its 4-wide pool
// and assembles the SceneView.
bool submit_instances(Renderer& R, InstanceState& in, std::string& detail) {
  cudaStream_t st = R.stream;
  const HostScene& h = R.host;
  const uint32_t n = (uint32_t)R.host_instances.size();
  if (!R.ok(R.lights.upload(in.table.records.data(), in.table.records.size(), st), "light table", detail) ||
      !R.ok(R.light_verts.upload(in.table.verts.data(), in.table.verts.size(), st), "light corners", detail) ||
      !R.ok(R.light_radiance.upload(in.table.radiance.data(), in.table.radiance.size(), st), "light radiance",
          detail) ||
      !R.ok(R.analytic.upload(in.table.analytic.data(), in.table.analytic.size(), st), "analytic lights", detail) ||
      !R.ok(R.light_nodes.upload(in.table.nodes.data(), in.table.nodes.size(), st), "light hierarchy", detail) ||
      !R.ok(R.distant.upload(in.table.distant.data(), in.table.distant.size(), st), "distant lights", detail) ||
      !R.ok(R.inst_trav.upload(in.trav.data(), in.trav.size(), st), "instances", detail) ||
      !R.ok(R.inst_shade.upload(in.shade.data(), in.shade.size(), st), "instances", detail) ||
      !R.ok(R.inst_texcoords.upload(in.texcoords.data(), in.texcoords.size(), st), "instances", detail) ||
      !R.ok(R.inst_colors.upload(in.colors.data(), in.colors.size(), st), "instances", detail) ||
      !R.ok(R.tlas.resize(std::max<uint32_t>(BvhBuilder::node_count(n), 1)), "TLAS", detail))
    return false;
  if (!R.ok(n <= kSahMaxTriangles
                ? R.builder.build_instances_sah(R.inst_shade.ptr, R.inst_trav.ptr, R.blas.ptr, n, R.tlas.ptr, st)
                : R.builder.build_instances(R.inst_shade.ptr, R.inst_trav.ptr, R.blas.ptr, n, R.tlas.ptr, st),
          "TLAS build", detail) ||
      !R.ok(R.tlas4.resize(R.tlas.count), "TLAS", detail) ||
      !R.ok(BvhBuilder::collapse(R.tlas.ptr, BvhBuilder::node_count(n), R.tlas4.ptr, true, st), "BVH collapse",
          detail))
    return false;
  R.host_lights = in.table.records;
  R.host_light_offsets = in.table.offsets;
  SceneView& v = R.view;
  v = SceneView{};
  v.tlas = R.tlas4.ptr;
  v.blas = R.blas4.ptr;
  v.tris = R.tris.ptr;
  v.inst_trav = R.inst_trav.ptr;
  v.inst_shade = R.inst_shade.ptr;
  v.materials = R.materials.ptr;
  v.full_shading = 0;
  for (const uint2& c : in.colors) if (c.x != kNoTexture) v.full_shading = 1;
  for (const lotus_material& m : h.materials) {
    bool any = !(m.normal[0] == 0.0f && m.normal[1] == 0.0f && (m.normal[2] == 0.0f || m.normal[2] == 1.0f)) ||
        m.model == LOTUS_MODEL_GLTF_PBR;
    for (uint32_t k = 0; k < LOTUS_TEXTURE_SLOTS; ++k) any = any || m.lookups[k] != LOTUS_NO_LOOKUP;
    if (any) v.full_shading = 1;
  }
  v.tex_texels = R.tex_texels.ptr;
  v.tex_info = R.tex_info.ptr;
  v.lookups = R.tex_lookups.ptr;
  v.mat_lookups = R.mat_lookups.ptr;
  v.albedo_tables = R.albedo_tables.ptr;
  v.texcoords = R.texcoords.ptr;
  v.inst_texcoords = R.inst_texcoords.ptr;
  v.colors = R.colors.ptr;
  v.inst_colors = R.inst_colors.ptr;
  v.normals = R.normals.ptr;
  v.lights = R.lights.ptr;
  v.light_verts = R.light_verts.ptr;
  v.light_radiance = R.light_radiance.ptr;
  v.env_texels = R.env_texels.ptr;
  v.env_floats = R.env_floats.ptr;
  v.env_guide = R.env_guide.ptr;
  v.instance_count = n;
  v.light_count = (uint32_t)in.table.records.size();
  v.env_bound = h.env_bound ? 1u : 0u;
  if (h.env_bound) {
    v.env_width = h.env_width;
    v.env_height = h.env_height;
    v.env_columns = h.env_columns;
    v.env_rows = h.env_rows;
    for (int k = 0; k < 3; ++k) v.env_scale[k] = h.env_scale[k];
    for (int k = 0; k < 9; ++k) v.env_frame[k] = h.env_frame[k];
  }
  v.env_selection = in.table.env_selection;
  for (int k = 0; k < 3; ++k) v.env_constant[k] = h.environment_constant[k];
  v.analytic = R.analytic.ptr;
  v.light_nodes = R.light_nodes.ptr;
  v.distant = R.distant.ptr;
  v.analytic_count = (uint32_t)in.table.analytic.size();
  v.light_node_count = (uint32_t)in.table.nodes.size();
  v.distant_count = (uint32_t)in.table.distant.size();
  v.step_limit = R.step_limit;
  v.walk_failure = R.walk_failure.ptr;
  return true;
}

// Builds the BLASes of the geometries in `which` from the device position
// and triangle arrays: binned SAH for those up to kSahMaxTriangles (one
// launch), LBVH for larger ones; then collapses their node ranges (or, with
// `whole_pool`, the whole pool at once) into the 4-wide pool.
bool build_blases(Renderer& R, const std::vector<uint32_t>& which, bool whole_pool, std::string& detail) {
  cudaStream_t st = R.stream;
  const HostScene& h = R.host;
  std::vector<BatchGeometry> batch;
  for (uint32_t g : which) {
    const lotus_geometry& geo = h.geometries[g];
    if (!geo.triangle_count) continue;
    if (geo.triangle_count <= kSahMaxTriangles) {
      batch.push_back({h.vertex_base[g], h.tri_base[g], geo.triangle_count, h.node_base[g]});
      continue;
    }
    cudaError_t e = R.builder.build_triangles(R.scene_pos.ptr + 3 * h.vertex_base[g],
        R.scene_tri.ptr + 3 * (size_t)h.tri_base[g], geo.triangle_count, R.blas.ptr, h.node_base[g], R.tris.ptr,
        h.tri_base[g], st);
    if (!R.ok(e, "BLAS build", detail)) return false;
  }
  if (!R.ok(R.builder.build_triangle_batch(R.scene_pos.ptr, R.scene_tri.ptr, batch, R.blas.ptr, R.tris.ptr, st,
                R.bvh_leaf_size),
          "BLAS build", detail))
    return false;
  const uint32_t pool = (uint32_t)h.nodes;
  if (whole_pool) return R.ok(BvhBuilder::collapse(R.blas.ptr, pool, R.blas4.ptr, false, st), "BVH collapse", detail);
  for (uint32_t g : which)
    if (!R.ok(BvhBuilder::collapse_range(R.blas.ptr, h.node_base[g],
                  BvhBuilder::node_count(h.geometries[g].triangle_count), pool, R.blas4.ptr, false, st),
            "BVH collapse", detail))
      return false;
  return true;
}

int32_t finish_update(Renderer& R, lotus_scene_result& res, std::string& detail) {
  cudaEventRecord(R.ev_stop, R.stream);
  if (!R.ok(cudaStreamSynchronize(R.stream), "scene update", detail)) return -1;
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, R.ev_start, R.ev_stop);
  R.scene_ready = true;
  ++R.scene_generation;
  const HostScene& h = R.host;
  res.status = LOTUS_PASS;
  uint64_t tris = 0;
  for (const lotus_geometry& g : h.geometries) tris += g.triangle_count;
  res.triangle_count = (uint32_t)tris;
  res.instance_count = (uint32_t)R.host_instances.size();
  res.light_count = (uint32_t)R.host_lights.size();
  res.bvh_node_count = (uint32_t)h.nodes;
  res.tlas_node_count = BvhBuilder::node_count(res.instance_count);
  res.build_gpu_ms = ms;
  res.device_bytes = R.scene_bytes();
  return LOTUS_PASS;
}

// The environment's sampling distribution and guide tables, built on the
// device from the resident texels (the k_env_* kernels); `mean` is the mean
// cell value, positive and finite for an image that can be sampled.
// The sRGB transfer function's inverse for each 8-bit code (IEC 61966-2-1:
// linear below 0.04045, the 2.4 power above), in double, rounded to float.
const float* srgb_to_linear_table() {
  static const std::vector<float> table = [] {
    std::vector<float> t(256);
    for (int v = 0; v < 256; ++v) {
      const double c = v / 255.0;
      t[v] = (float)(c <= 0.04045 ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4));
    }
    return t;
  }();
  return table.data();
}

// The scene's textures decoded to linear RGBA floats, one after another
// (sRGB codes through srgb_to_linear_table, alpha and unorm codes / 255),
// the texture inputs as TextureLookup records, each material's lookups and
// every geometry's texture-coordinate sets in one pool.
bool upload_textures(Renderer& R, const lotus_scene_desc& s, std::string& detail) {
  cudaStream_t st = R.stream;
  HostScene& h = R.host;
  const float* srgb = srgb_to_linear_table();
  std::vector<float4> texels;
  std::vector<uint4> info(s.texture_count);
  uint64_t total = 0;
  for (uint32_t i = 0; i < s.texture_count; ++i) total += (uint64_t)s.textures[i].width * s.textures[i].height;
  if (total >= (1ull << 31)) {
    detail = "the scene's textures hold 2^31 texels or more";
    return false;
  }
  texels.reserve(total);
  for (uint32_t i = 0; i < s.texture_count; ++i) {
    const lotus_texture& t = s.textures[i];
    info[i] = make_uint4((uint32_t)texels.size(), t.width, t.height, t.format);
    const size_t n = (size_t)t.width * t.height;
    if (t.format == LOTUS_TEXTURE_RGBA32_FLOAT) {
      const float* f = static_cast<const float*>(t.texels);
      for (size_t k = 0; k < n; ++k) texels.push_back(make_float4(f[4 * k], f[4 * k + 1], f[4 * k + 2], f[4 * k + 3]));
    } else {
      const uint8_t* b = static_cast<const uint8_t*>(t.texels);
      const bool encoded = t.format == LOTUS_TEXTURE_RGBA8_SRGB;
      for (size_t k = 0; k < n; ++k) {
        const uint8_t* c = b + 4 * k;
        auto channel = [&](int j) { return encoded ? srgb[c[j]] : (float)(c[j] / 255.0); };
        texels.push_back(make_float4(channel(0), channel(1), channel(2), (float)(c[3] / 255.0)));
      }
    }
  }
  std::vector<TextureLookup> lookups(s.texture_input_count);
  for (uint32_t i = 0; i < s.texture_input_count; ++i) {
    const lotus_texture_input& in = s.texture_inputs[i];
    TextureLookup& L = lookups[i];
    L.texture = in.texture == LOTUS_NO_TEXTURE ? kNoTexture : in.texture - 1;
    L.channel = in.channel;
    L.wrap_s = in.wrap_s;
    L.wrap_t = in.wrap_t;
    L.scale = make_float4(in.scale[0], in.scale[1], in.scale[2], in.scale[3]);
    L.bias = make_float4(in.bias[0], in.bias[1], in.bias[2], in.bias[3]);
    L.fallback = make_float4(in.fallback[0], in.fallback[1], in.fallback[2], in.fallback[3]);
    L.st_s = make_float4(in.st_transform[0], in.st_transform[1], in.st_transform[2], 0.0f);
    L.st_t = make_float4(in.st_transform[3], in.st_transform[4], in.st_transform[5], 0.0f);
  }
  std::vector<MaterialLookups> mats(s.material_count);
  for (uint32_t i = 0; i < s.material_count; ++i) {
    const lotus_material& m = s.materials[i];
    MaterialLookups& ml = mats[i];
    for (uint32_t k = 0; k < LOTUS_TEXTURE_SLOTS; ++k)
      ml.slot[k] = m.lookups[k] == LOTUS_NO_LOOKUP ? kNoTexture : m.lookups[k] - 1;
    ml.fallback_s = m.texcoord_fallback[0];
    ml.fallback_t = m.texcoord_fallback[1];
    const bool zero = m.normal[0] == 0.0f && m.normal[1] == 0.0f && m.normal[2] == 0.0f;
    for (int k = 0; k < 3; ++k) ml.normal[k] = zero ? (k == 2 ? 1.0f : 0.0f) : m.normal[k];
    ml.reserved = 0;
  }
  std::vector<float2> coords;
  h.texcoord_base.assign(s.geometry_count, 0);
  for (uint32_t g = 0; g < s.geometry_count; ++g) {
    const lotus_geometry& geo = s.geometries[g];
    h.texcoord_base[g] = coords.size();
    const size_t n = 3ull * geo.triangle_count * geo.texcoord_sets;
    for (size_t k = 0; k < n; ++k) coords.push_back(make_float2(geo.texcoords[2 * k], geo.texcoords[2 * k + 1]));
  }
  if (coords.size() >= (size_t)kNoTexture) {
    detail = "the scene's texture coordinates exceed 2^32 corners";
    return false;
  }
  std::vector<float> colors;
  R.host.color_sets.assign(s.geometry_count, {});
  for (uint32_t g = 0; g < s.geometry_count; ++g) {
    const lotus_geometry& geo = s.geometries[g];
    const float* values = geo.colors;
    for (uint32_t k = 0; k < geo.color_sets; ++k) {
      R.host.color_sets[g].push_back(make_uint2((uint32_t)colors.size(), geo.color_counts[k] == 1 ? 1u : 0u));
      colors.insert(colors.end(), values, values + 3ull * geo.color_counts[k]);
      values += 3ull * geo.color_counts[k];
    }
  }
  if (colors.size() >= (size_t)kNoTexture) {
    detail = "the scene's colour sets exceed 2^32 values";
    return false;
  }
  return R.ok(R.tex_texels.upload(texels.data(), texels.size(), st), "texels", detail) &&
         R.ok(R.tex_info.upload(info.data(), info.size(), st), "textures", detail) &&
         R.ok(R.tex_lookups.upload(lookups.data(), lookups.size(), st), "texture inputs", detail) &&
         R.ok(R.mat_lookups.upload(mats.data(), mats.size(), st), "material lookups", detail) &&
         R.ok(R.texcoords.upload(coords.data(), coords.size(), st), "texture coordinates", detail) &&
         R.ok(R.colors.upload(colors.data(), colors.size(), st), "colour sets", detail);
}

bool build_env_distribution(Renderer& R, const lotus_environment& e, double& mean, std::string& detail) {
  constexpr double kPiD = 3.14159265358979323846;
  cudaStream_t st = R.stream;
  const uint32_t columns = std::min(e.width, 2048u), rows = std::min(e.height, 1024u);
  const uint32_t cells = columns * rows;
  std::vector<double> sin_theta(rows);
  for (uint32_t row = 0; row < rows; ++row) sin_theta[row] = std::sin(kPiD * (row + 0.5) / rows);
  DeviceArray<double> values, row_sums, totals, sines;
  const size_t floats = (size_t)cells + rows + 1 + (size_t)rows * (columns + 1);
  const size_t guides = (kEnvGuideMarginal + 1) + (size_t)rows * (kEnvGuideConditional + 1);
  if (!R.ok(values.resize(cells), "environment distribution", detail) ||
      !R.ok(row_sums.resize(rows), "environment distribution", detail) ||
      !R.ok(totals.resize(2), "environment distribution", detail) ||
      !R.ok(sines.upload(sin_theta.data(), rows, st), "environment distribution", detail) ||
      !R.ok(R.env_floats.resize(floats), "environment distribution", detail) ||
      !R.ok(R.env_guide.resize(guides), "environment guide tables", detail) ||
      !R.ok(cudaMemsetAsync(R.env_floats.ptr, 0, floats * sizeof(float), st), "environment distribution", detail))
    return false;
  float* density = R.env_floats.ptr;
  float* marginal = density + cells;
  float* conditional = marginal + rows + 1;
  const uint32_t b = 256;
  k_env_cells<<<(cells + b - 1) / b, b, 0, st>>>(R.env_texels.ptr, e.width, e.height, columns, rows, e.scale[0],
      e.scale[1], e.scale[2], sines.ptr, values.ptr);
  k_env_row_sums<<<(rows + b - 1) / b, b, 0, st>>>(values.ptr, columns, rows, row_sums.ptr);
  k_env_total<<<1, 32, 0, st>>>(row_sums.ptr, columns, rows, totals.ptr, marginal);
  k_env_density<<<(cells + b - 1) / b, b, 0, st>>>(values.ptr, cells, totals.ptr, density);
  k_env_conditional<<<(rows + b - 1) / b, b, 0, st>>>(values.ptr, row_sums.ptr, columns, rows, conditional);
  k_env_guides<<<(uint32_t)((guides + b - 1) / b), b, 0, st>>>(marginal, conditional, columns, rows,
      R.env_guide.ptr);
  double t[2] = {0.0, 0.0};
  if (!R.ok(cudaGetLastError(), "environment distribution", detail) ||
      !R.ok(cudaMemcpyAsync(t, totals.ptr, sizeof(t), cudaMemcpyDeviceToHost, st), "environment distribution",
          detail) ||
      !R.ok(cudaStreamSynchronize(st), "environment distribution", detail))
    return false;
  mean = t[1];
  return true;
}

int32_t update_scene(Renderer& R, const lotus_scene_desc& s, lotus_scene_result& res) {
  std::string detail;
  if (!validate_scene(s, detail)) {
    copy_detail(res.detail, sizeof(res.detail), detail);
    return res.status = LOTUS_FAIL;
  }
  cudaStream_t st = R.stream;
  auto fail = [&](const std::string& d) {
    R.failure = d;
    R.release_scene();
    copy_detail(res.detail, sizeof(res.detail), d);
    return res.status = LOTUS_FAIL;
  };
  cudaEventRecord(R.ev_start, st);
  // The host copy: every geometry's arrays, the materials, the instances.
  HostScene& h = R.host;
  h = HostScene{};
  const uint32_t ng = s.geometry_count;
  h.positions.resize(ng);
  h.triangles.resize(ng);
  h.normals.resize(ng);
  h.geometries.resize(ng);
  h.boxes.resize(ng);
  h.vertex_base.resize(ng);
  h.node_base.resize(ng);
  h.tri_base.resize(ng);
  h.normal_base.assign(ng, kNoLights);
  uint64_t nodes = 0, tri_total = 0, normal_total = 0, vert_total = 0;
  for (uint32_t g = 0; g < ng; ++g) {
    const lotus_geometry& geo = s.geometries[g];
    h.positions[g].assign(geo.positions, geo.positions + 3ull * geo.vertex_count);
    h.triangles[g].assign(geo.triangles, geo.triangles + 3ull * geo.triangle_count);
    if (geo.normals && geo.triangle_count) h.normals[g].assign(geo.normals, geo.normals + 9ull * geo.triangle_count);
    lotus_geometry& copy = h.geometries[g];
    copy = geo;
    copy.positions = h.positions[g].data();
    copy.triangles = h.triangles[g].data();
    copy.normals = h.normals[g].empty() ? nullptr : h.normals[g].data();
    copy.texcoords = nullptr;  // on the device only
    copy.colors = nullptr;
    copy.color_counts = nullptr;
    h.boxes[g] = geometry_box(copy);
    h.vertex_base[g] = vert_total;
    h.node_base[g] = (uint32_t)nodes;
    h.tri_base[g] = (uint32_t)tri_total;
    nodes += BvhBuilder::node_count(geo.triangle_count);
    tri_total += geo.triangle_count;
    vert_total += geo.vertex_count;
    if (copy.normals) {
      h.normal_base[g] = (uint32_t)normal_total;
      normal_total += geo.triangle_count;
    }
  }
  h.nodes = nodes;
  h.materials.assign(s.materials, s.materials + s.material_count);
  h.texture_inputs.assign(s.texture_inputs, s.texture_inputs + s.texture_input_count);
  h.texture_count = s.texture_count;
  if (!upload_textures(R, s, detail)) return fail(detail);
  for (int k = 0; k < 3; ++k) h.environment_constant[k] = s.environment_constant[k];
  h.lights.assign(s.lights, s.lights + s.light_count);
  R.host_instances.assign(s.instances, s.instances + s.instance_count);
  if (nodes >= kMaxSceneTriangles || tri_total >= kMaxSceneTriangles)
    return fail("the scene holds 2^28 triangles or more");
  if (!R.ok(R.blas.resize(std::max<uint64_t>(nodes, 1)), "BLAS pool", detail) ||
      !R.ok(R.blas4.resize(R.blas.count), "BLAS pool", detail) ||
      !R.ok(R.tris.resize(kTriStride * std::max<uint64_t>(tri_total, 1)), "triangle pool", detail))
    return fail(detail);
  // Every geometry's positions and triangles in one upload each; they stay
  // resident for the incremental updates' rebuilds.
  {
    std::vector<float> h_pos(3 * vert_total);
    std::vector<uint32_t> h_tri(3 * tri_total);
    for (uint32_t g = 0; g < ng; ++g) {
      if (!h.positions[g].empty())
        std::memcpy(&h_pos[3 * h.vertex_base[g]], h.positions[g].data(), 4 * h.positions[g].size());
      if (!h.triangles[g].empty())
        std::memcpy(&h_tri[3 * (size_t)h.tri_base[g]], h.triangles[g].data(), 4 * h.triangles[g].size());
    }
    if (!R.ok(R.scene_pos.upload(h_pos.data(), h_pos.size(), st), "positions", detail) ||
        !R.ok(R.scene_tri.upload(h_tri.data(), h_tri.size(), st), "triangles", detail))
      return fail(detail);
  }
  std::vector<uint32_t> all(ng);
  for (uint32_t g = 0; g < ng; ++g) all[g] = g;
  if (!build_blases(R, all, true, detail)) return fail(detail);
  // Corner normals.
  if (normal_total) {
    std::vector<float> h_n(9 * normal_total);
    for (uint32_t g = 0; g < ng; ++g)
      if (h.normal_base[g] != kNoLights)
        std::memcpy(&h_n[9 * (size_t)h.normal_base[g]], h.normals[g].data(), 4 * h.normals[g].size());
    if (!R.ok(R.normals.upload(h_n.data(), h_n.size(), st), "normals", detail)) return fail(detail);
  } else {
    R.normals.release();
  }
  // Materials.
  std::vector<MaterialRecord> h_mat(s.material_count);
  for (uint32_t i = 0; i < s.material_count; ++i) {
    const lotus_material& m = s.materials[i];
    MaterialRecord& r = h_mat[i];
    r.base_roughness = make_float4(m.base_color[0], m.base_color[1], m.base_color[2], m.roughness);
    r.emission_metallic = make_float4(m.emission[0], m.emission[1], m.emission[2], m.metallic);
    r.specular_ior = make_float4(m.specular_color[0], m.specular_color[1], m.specular_color[2], m.ior);
    r.transmission = make_float4(m.transmission_color[0], m.transmission_color[1],
        m.transmission_color[2], m.transmission);
    const bool gltf = m.model == LOTUS_MODEL_GLTF_PBR;
    uint32_t flags = gltf ? kMaterialGltf : m.flags & (LOTUS_MATERIAL_SPECULAR_WORKFLOW | LOTUS_MATERIAL_THIN_WALLED);
    // glTF PBR: the dielectric's reflectance at normal incidence from its
    // index, in double so that the default index gives the float nearest
    // 0.04 (gpu_scene.cpp:2059-2063).
    const double root = (1.0 - (double)m.ior) / (1.0 + (double)m.ior);
    const float dielectric_f0 = gltf ? (float)(root * root) : 0.0f;
    r.gltf = gltf ? make_float4(m.specular, m.clearcoat, m.clearcoat_roughness, m.emissive_strength)
                  : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    r.sheen = gltf ? make_float4(m.sheen_color[0], m.sheen_color[1], m.sheen_color[2], m.sheen_roughness)
                   : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (uint32_t k = 0; k < LOTUS_TEXTURE_SLOTS; ++k)
      if (m.lookups[k] != LOTUS_NO_LOOKUP) flags |= kMaterialTextured;
    // A constant tangent-space normal other than the identity (all zero
    // stands for the identity).
    if (!(m.normal[0] == 0.0f && m.normal[1] == 0.0f && (m.normal[2] == 0.0f || m.normal[2] == 1.0f)))
      flags |= kMaterialTextured;
    if (m.lookups[LOTUS_SLOT_OPACITY] != LOTUS_NO_LOOKUP) flags |= kMaterialOpacityTextured;
    float fbits;
    std::memcpy(&fbits, &flags, 4);
    r.coverage = make_float4(m.opacity, m.opacity_threshold, fbits, dielectric_f0);
  }
  if (!R.ok(R.materials.upload(h_mat.data(), h_mat.size(), st), "materials", detail)) return fail(detail);
  // The composed closure's albedo tables, once per renderer.
  if (R.albedo_tables.count != albedo::kSize &&
      !R.ok(R.albedo_tables.upload(kAlbedoTableData, albedo::kSize, st), "albedo tables", detail))
    return fail(detail);
  // Environment: the texels go to the device, where its sampling
  // distribution is built (build_env_distribution).
  h.env_bound = false;
  double env_mean = 0.0;
  if (s.environment && s.environment->texels && s.environment->width && s.environment->height) {
    const size_t texels = (size_t)s.environment->width * s.environment->height;
    if (!R.ok(R.env_texels.upload(reinterpret_cast<const float4*>(s.environment->texels), texels, st),
            "environment texels", detail) ||
        !build_env_distribution(R, *s.environment, env_mean, detail))
      return fail(detail);
    h.env_bound = env_mean > 0.0 && std::isfinite(env_mean);
  }
  if (h.env_bound) {
    h.env_mean = env_mean;
    h.env_width = s.environment->width;
    h.env_height = s.environment->height;
    h.env_columns = std::min(s.environment->width, 2048u);
    h.env_rows = std::min(s.environment->height, 1024u);
    for (int k = 0; k < 3; ++k) h.env_scale[k] = s.environment->scale[k];
    for (int k = 0; k < 9; ++k) h.env_frame[k] = s.environment->environment_from_world[k];
  } else {
    R.env_texels.release();
    R.env_floats.release();
    R.env_guide.release();
  }
  InstanceState inst;
  if (!prepare_instances(R, inst, detail) || !submit_instances(R, inst, detail)) return fail(detail);
  // Default temporal identities: index and material slot, static, 6.
  {
    std::vector<TemporalInstance> ids(std::max<uint32_t>(s.instance_count, 1));
    for (uint32_t i = 0; i < s.instance_count; ++i) {
      TemporalInstance& t = ids[i];
      const float* m = s.instances[i].world_from_object;
      for (int r = 0; r < 3; ++r) t.previous[r] = make_float4(m[r], m[4 + r], m[8 + r], m[12 + r]);
      t.instance_id = i;
      t.material_id = s.instances[i].material;
      t.flags = 6u;
    }
    if (!R.ok(R.temporal.instances.upload(ids.data(), ids.size(), st), "temporal identities", detail))
      return fail(detail);
    R.temporal.instances_custom = false;
  }
  if (finish_update(R, res, detail) != LOTUS_PASS) return fail(detail);
  return LOTUS_PASS;
}

// Transform and material-slot edits of the resident scene's instances
// (any count; the geometries, materials and environment stay).
int32_t update_instances(Renderer& R, const lotus_instance* instances, uint32_t count, lotus_scene_result& res) {
  std::string detail;
  auto reject = [&](const std::string& d) {
    copy_detail(res.detail, sizeof(res.detail), d);
    return res.status = LOTUS_FAIL;
  };
  if (!R.scene_ready) return reject("no resident scene to update");
  if (count && !instances) return reject("the instance array is missing");
  for (uint32_t i = 0; i < count; ++i) {
    const lotus_instance& inst = instances[i];
    if (inst.geometry >= R.host.geometries.size() || inst.material >= R.host.materials.size())
      return reject("instance " + std::to_string(i) + " names a missing geometry or material");
    if (inst.texcoord_set != LOTUS_NO_TEXCOORDS &&
        inst.texcoord_set > R.host.geometries[inst.geometry].texcoord_sets)
      return reject("instance " + std::to_string(i) + " names a missing texture-coordinate set");
    if (inst.color_set != LOTUS_NO_COLORS && inst.color_set > R.host.geometries[inst.geometry].color_sets)
      return reject("instance " + std::to_string(i) + " names a missing colour set");
    const float* m = inst.world_from_object;
    if (m[3] != 0.0f || m[7] != 0.0f || m[11] != 0.0f || m[15] != 1.0f)
      return reject("instance " + std::to_string(i) + " has a projective transform");
    float4 rows[3];
    if (!invert_affine(m, rows)) return reject("instance " + std::to_string(i) + " has a singular transform");
  }
  auto fail = [&](const std::string& d) {
    R.failure = d;
    R.release_scene();
    return reject(d);
  };
  const bool same_count = count == R.host_instances.size();
  R.host_instances.assign(instances, instances + count);
  InstanceState inst;
  if (!prepare_instances(R, inst, detail)) return fail(detail);
  cudaEventRecord(R.ev_start, R.stream);
  if (!submit_instances(R, inst, detail)) return fail(detail);
  if (!R.temporal.instances_custom || !same_count) {
    // Default temporal identities follow the new placements (identities a
    // host set for another instance count no longer apply).
    R.temporal.instances_custom = false;
    std::vector<TemporalInstance> ids(std::max<uint32_t>(count, 1));
    for (uint32_t i = 0; i < count; ++i) {
      TemporalInstance& t = ids[i];
      const float* m = instances[i].world_from_object;
      for (int r = 0; r < 3; ++r) t.previous[r] = make_float4(m[r], m[4 + r], m[8 + r], m[12 + r]);
      t.instance_id = i;
      t.material_id = instances[i].material;
      t.flags = 6u;
    }
    if (!R.ok(R.temporal.instances.upload(ids.data(), ids.size(), R.stream), "temporal identities", detail))
      return fail(detail);
  }
  if (finish_update(R, res, detail) != LOTUS_PASS) return fail(detail);
  return LOTUS_PASS;
}

// New positions (and corner normals) of one resident geometry with its
// vertex and triangle counts and its triangles kept.
int32_t update_geometry(Renderer& R, uint32_t geometry, const float* positions, uint32_t vertex_count,
    const float* normals, lotus_scene_result& res) {
  std::string detail;
  auto reject = [&](const std::string& d) {
    copy_detail(res.detail, sizeof(res.detail), d);
    return res.status = LOTUS_FAIL;
  };
  if (!R.scene_ready) return reject("no resident scene to update");
  HostScene& h = R.host;
  if (geometry >= h.geometries.size()) return reject("no geometry " + std::to_string(geometry));
  lotus_geometry& geo = h.geometries[geometry];
  if (vertex_count != geo.vertex_count) return reject("a point edit keeps the geometry's vertex count");
  if (vertex_count && !positions) return reject("the position array is missing");
  if ((normals != nullptr) != (geo.normals != nullptr))
    return reject("a point edit of a geometry with corner normals gives new ones, and none otherwise");
  for (uint64_t i = 0; i < 3ull * vertex_count; ++i)
    if (!std::isfinite(positions[i])) return reject("the geometry has a non-finite position");
  auto fail = [&](const std::string& d) {
    R.failure = d;
    R.release_scene();
    return reject(d);
  };
  cudaStream_t st = R.stream;
  std::copy(positions, positions + 3ull * vertex_count, h.positions[geometry].begin());
  if (normals) std::copy(normals, normals + 9ull * geo.triangle_count, h.normals[geometry].begin());
  h.boxes[geometry] = geometry_box(geo);
  InstanceState inst;
  if (!prepare_instances(R, inst, detail)) return fail(detail);
  cudaEventRecord(R.ev_start, st);
  if (vertex_count &&
      !R.ok(cudaMemcpyAsync(R.scene_pos.ptr + 3 * h.vertex_base[geometry], h.positions[geometry].data(),
                12ull * vertex_count, cudaMemcpyHostToDevice, st),
          "positions", detail))
    return fail(detail);
  if (normals && geo.triangle_count &&
      !R.ok(cudaMemcpyAsync(R.normals.ptr + 9 * (size_t)h.normal_base[geometry], h.normals[geometry].data(),
                36ull * geo.triangle_count, cudaMemcpyHostToDevice, st),
          "normals", detail))
    return fail(detail);
  // The BLAS is refitted in place (the reference refits on point edits,
  // gpu_scene.cpp:1899-1950): its topology kept, its triangle records and
  // boxes following the new positions; then its 4-wide nodes again.
  const uint32_t count = geo.triangle_count;
  if (count &&
      (!R.ok(R.builder.refit_triangles(R.scene_pos.ptr + 3 * h.vertex_base[geometry],
                 R.scene_tri.ptr + 3 * (size_t)h.tri_base[geometry], count, R.blas.ptr, h.node_base[geometry],
                 R.tris.ptr, h.tri_base[geometry], st),
           "BLAS refit", detail) ||
          !R.ok(BvhBuilder::collapse_range(R.blas.ptr, h.node_base[geometry], BvhBuilder::node_count(count),
                    (uint32_t)h.nodes, R.blas4.ptr, false, st),
              "BVH collapse", detail)))
    return fail(detail);
  if (!submit_instances(R, inst, detail)) return fail(detail);
  if (finish_update(R, res, detail) != LOTUS_PASS) return fail(detail);
  return LOTUS_PASS;
}

bool ensure_targets(Renderer& R, uint32_t w, uint32_t h, bool wavefront, std::string& detail) {
  const size_t n = (size_t)w * h;
  if (R.width != w || R.height != h) {
    R.accum.release();
    R.color.release();
    R.depth.release();
    R.depth_valid = false;
    R.depth_fresh = true;
    R.path_origin.release(); R.path_direction.release(); R.path_throughput.release();
    R.path_radiance.release(); R.path_hit.release();
    R.queue_ray0.release(); R.queue_ray1.release(); R.queue_hit.release();
    R.sq_o.release(); R.sq_d.release(); R.sq_fl.release(); R.sq_thr.release();
    R.sort_keys.release(); R.sort_queue.release(); R.sort_bins.release();
    R.path_origin2.release(); R.path_direction2.release(); R.path_throughput2.release();
    R.path_radiance2.release(); R.path_hit2.release();
    R.queue_ray02.release(); R.queue_ray12.release(); R.queue_hit2.release();
    R.sq_o2.release(); R.sq_d2.release(); R.sq_fl2.release(); R.sq_thr2.release();
    R.sort_keys2.release(); R.sort_queue2.release(); R.sort_bins2.release();
    R.width = w;
    R.height = h;
    R.key_valid = false;
  }
  if (!R.ok(R.accum.resize(n), "accumulation", detail) || !R.ok(R.color.resize(n), "colour", detail) ||
      !R.ok(R.depth.resize(n), "depth", detail) ||
      !R.ok(R.counts.resize(kQueueCounterWords * (LOTUS_MAX_BOUNCES + 2)), "queue counts", detail) ||
      !R.ok(R.frame_const.resize(kMaxChain), "frame constants", detail) ||
      !R.ok(R.totals.resize(1), "ray totals", detail))
    return false;
  if (wavefront) {
    // Room for a wave of the renderer's wave size.
    const size_t w = (size_t)R.wave * n;
    if (!R.ok(R.path_origin.resize(w), "path state", detail) ||
        !R.ok(R.path_direction.resize(w), "path state", detail) ||
        !R.ok(R.path_throughput.resize(w), "path state", detail) ||
        !R.ok(R.path_radiance.resize(w), "path state", detail) ||
        !R.ok(R.path_hit.resize(w), "path state", detail) ||
        !R.ok(R.queue_ray0.resize(w), "queues", detail) || !R.ok(R.queue_ray1.resize(w), "queues", detail) ||
        !R.ok(R.queue_hit.resize(w), "queues", detail) || !R.ok(R.sq_o.resize(w), "shadow queue", detail) ||
        !R.ok(R.sq_d.resize(w), "shadow queue", detail) || !R.ok(R.sq_fl.resize(w), "shadow queue", detail) ||
        !R.ok(R.sq_thr.resize(w), "shadow queue", detail) || !R.ok(R.sort_keys.resize(w), "queue keys", detail) ||
        !R.ok(R.sort_queue.resize(w), "queue keys", detail) ||
        !R.ok(R.sort_bins.resize(kSortBinWords), "queue keys", detail))
      return false;
  }
  return true;
}

// The second path state and queue set (two samples in flight).
bool ensure_pair_buffers(Renderer& R, size_t n, std::string& detail) {
  return R.ok(R.path_origin2.resize(n), "path state", detail) && R.ok(R.path_direction2.resize(n), "path state", detail) &&
         R.ok(R.path_throughput2.resize(n), "path state", detail) &&
         R.ok(R.path_radiance2.resize(n), "path state", detail) && R.ok(R.path_hit2.resize(n), "path state", detail) &&
         R.ok(R.queue_ray02.resize(n), "queues", detail) && R.ok(R.queue_ray12.resize(n), "queues", detail) &&
         R.ok(R.queue_hit2.resize(n), "queues", detail) && R.ok(R.sq_o2.resize(n), "shadow queue", detail) &&
         R.ok(R.sq_d2.resize(n), "shadow queue", detail) && R.ok(R.sq_fl2.resize(n), "shadow queue", detail) &&
         R.ok(R.sq_thr2.resize(n), "shadow queue", detail) &&
         R.ok(R.sort_keys2.resize(n), "queue keys", detail) && R.ok(R.sort_queue2.resize(n), "queue keys", detail) &&
         R.ok(R.sort_bins2.resize(kSortBinWords), "queue keys", detail) &&
         R.ok(R.counts2.resize(kQueueCounterWords * (LOTUS_MAX_BOUNCES + 2)), "queue counts", detail);
}

// The radiance cache's queues for targets of `pixels` pixels: a query per
// pixel, and training records for one pixel in `stride` with a margin for
// the per-sample random choice.
bool ensure_cache_queues(Renderer& R, uint32_t pixels, std::string& detail) {
  const uint32_t stride = R.cache_desc.training_stride ? R.cache_desc.training_stride : 32u;
  const uint32_t train = pixels / stride + pixels / (4 * stride) + 1024;
  if (R.cache_pixels == pixels && R.cache_train.count == train) return true;
  R.cache_pixels = 0;
  if (!R.ok(R.cache_queries.resize(pixels), "cache queries", detail) ||
      !R.ok(R.cache_query_slots.resize(pixels), "cache queries", detail) ||
      !R.ok(R.cache_query_throughput.resize(pixels), "cache queries", detail) ||
      !R.ok(R.cache_query_keys.resize(pixels), "cache queries", detail) ||
      !R.ok(R.cache_query_order.resize(pixels), "cache queries", detail) ||
      !R.ok(R.cache_query_bins.resize(kSortBinWords), "cache queries", detail) ||
      !R.ok(R.cache_train.resize(train), "cache training records", detail) ||
      !R.ok(R.cache_train_slots.resize(train), "cache training records", detail) ||
      !R.ok(R.cache_train_base.resize(train), "cache training records", detail) ||
      !R.ok(R.cache_train_throughput.resize(train), "cache training records", detail) ||
      !R.ok(R.cache_train_targets.resize(train), "cache training records", detail) ||
      !R.ok(R.cache_counters.resize(2), "cache counters", detail))
    return false;
  R.cache_pixels = pixels;
  return true;
}

CacheQueues cache_queues(Renderer& R) {
  CacheQueues C;
  C.enabled = R.cache_enabled && R.cache.ready() && R.cache_pixels != 0;
  if (!C.enabled) return C;
  C.stride = R.cache_desc.training_stride ? R.cache_desc.training_stride : 32u;
  C.steps = R.cache_desc.training_steps ? R.cache_desc.training_steps : 1u;
  C.bounce = R.cache_desc.terminate_bounce ? R.cache_desc.terminate_bounce : 1u;
  C.cache = &R.cache;
  C.queries = R.cache_queries.ptr;
  C.query_slots = R.cache_query_slots.ptr;
  C.query_throughput = R.cache_query_throughput.ptr;
  C.query_keys = R.cache_query_keys.ptr;
  C.query_order = R.cache_query_order.ptr;
  C.query_bins = R.cache_query_bins.ptr;
  {
    const CacheGrid g = R.cache.grid();
    for (int a = 0; a < 3; ++a) {
      C.grid_lo[a] = g.lo[a];
      C.grid_scale[a] = g.inv_extent[a] * (float)(1u << kQuerySortAxisBits);
    }
  }
  C.query_capacity = (uint32_t)R.cache_queries.count;
  C.train = R.cache_train.ptr;
  C.train_slots = R.cache_train_slots.ptr;
  C.train_base = R.cache_train_base.ptr;
  C.train_throughput = R.cache_train_throughput.ptr;
  C.train_targets = R.cache_train_targets.ptr;
  C.train_capacity = (uint32_t)R.cache_train.count;
  C.counters = R.cache_counters.ptr;
  return C;
}

}  // namespace

namespace lotus {

// The detail for a frame whose BVH walks failed (the two words of
// SceneView::walk_failure), or "" when none did.
std::string walk_failure_detail(const uint32_t words[2], uint32_t step_limit) {
  if (words[0] == 0) return std::string();
  std::string causes;
  if (words[1] & kWalkFailedStack)
    causes += "a traversal stack overflowed (" + std::to_string(kStackSize) + " entries)";
  if (words[1] & kWalkFailedSteps) {
    if (!causes.empty()) causes += " and ";
    causes += "a walk ran out of its " + std::to_string(step_limit) + " steps";
  }
  return std::to_string(words[0]) + " BVH walk(s) ended early, so the frame's hits are incomplete: " + causes;
}

}  // namespace lotus

namespace {

using namespace lotus;

int32_t render(Renderer& R, const lotus_frame_desc& d, lotus_frame_result& res, float* color_out) {
  std::string detail;
  auto fail = [&](const std::string& msg) {
    copy_detail(res.detail, sizeof(res.detail), msg);
    return res.status = LOTUS_FAIL;
  };
  auto poison = [&](const std::string& msg) {
    R.failure = msg;
    return fail(msg);
  };
  const lotus_settings& st = d.settings;
  const lotus_target& t = d.target;
  if (!R.scene_ready) return fail("no scene has been uploaded");
  if (d.frame_count == 0) return fail("frame_count must be at least 1");
  if (t.width == 0 || t.height == 0) return fail("the offscreen target is empty");
  if (t.width > 32768 || t.height > 32768) return fail("the offscreen target exceeds 32768 pixels a side");
  for (int k = 0; k < 4; ++k)
    if (!std::isfinite(t.clear_color[k])) return fail("invalid offscreen clear values");
  if (st.integrator > LOTUS_INTEGRATOR_WAVEFRONT) return fail("unknown integrator");
  if (st.light_sampling > LOTUS_LIGHT_SAMPLING_RESTIR_INITIAL) return fail("unknown light sampling");
  if (st.light_sampling == LOTUS_LIGHT_SAMPLING_RESTIR_INITIAL)
    return fail("RestirInitial light sampling runs through the temporal entry point");
  if (st.max_bounces > LOTUS_MAX_BOUNCES)
    return fail("max_bounces " + std::to_string(st.max_bounces) + " exceeds " +
                std::to_string(LOTUS_MAX_BOUNCES));
  // VulkanWorldToClip (vulkan_internal.hpp:326-336) and Invert.
  float vulkan[16];
  std::memcpy(vulkan, d.world_to_clip, sizeof(vulkan));
  for (int c = 0; c < 4; ++c) {
    const float y = d.world_to_clip[c * 4 + 1], z = d.world_to_clip[c * 4 + 2], w = d.world_to_clip[c * 4 + 3];
    vulkan[c * 4 + 1] = -y;
    vulkan[c * 4 + 2] = 0.5f * (z + w);
  }
  FrameConst fc{};
  if (!invert4(vulkan, fc.clip_to_world)) return fail("ray-query camera is singular or non-finite");
  std::memcpy(fc.world_to_clip, vulkan, sizeof(vulkan));
  const bool want_depth = (d.flags & LOTUS_FRAME_DEPTH) != 0;
  if (want_depth && !(t.clear_depth >= 0.0f && t.clear_depth <= 1.0f))
    return fail("invalid offscreen clear values");
  const bool wavefront = st.integrator == LOTUS_INTEGRATOR_WAVEFRONT;
  // The reference integrator's paths run on the wavefront's compacted
  // queues too when one launch holds at least as many as the extension
  // kernel keeps resident (the target's pixels times the samples of a
  // wave): each path is computed as in the per-thread loop, bit for bit,
  // and the sorted queues keep software traversal coherent. Below that the
  // frame is latency-bound and the per-thread loop (k_reference_pt) is
  // faster. The frame's evidence stays the reference integrator's.
  const uint64_t launch_paths = (uint64_t)t.width * t.height *
      std::min(std::max(d.frame_count, 1u), std::max(R.wave, 1u));
  const bool queued = wavefront ||
      (st.integrator == LOTUS_INTEGRATOR_REFERENCE && st.light_sampling <= LOTUS_LIGHT_SAMPLING_MIS &&
       st.output == LOTUS_OUTPUT_RADIANCE && launch_paths >= extension_resident_threads());
  if (!ensure_targets(R, t.width, t.height, queued, detail)) return poison(detail);
  // The radiance cache serves the wavefront integrator's samples.
  const bool use_cache = wavefront && R.cache_enabled && R.cache.ready();
  if (use_cache && !ensure_cache_queues(R, t.width * t.height, detail)) return poison(detail);
  const CacheQueues cq = use_cache ? cache_queues(R) : CacheQueues();
  // DisplayViewport and DataScissor (vulkan_backend.cpp:651-677).
  float vx = 0.0f, vy = 0.0f, vw = (float)t.width, vh = (float)t.height;
  if (t.display_window[2] > 0.0f && t.display_window[3] > 0.0f) {
    vx = t.display_window[0]; vy = t.display_window[1]; vw = t.display_window[2]; vh = t.display_window[3];
  }
  fc.ndc[0] = 2.0f / vw;
  fc.ndc[1] = 2.0f / vh;
  fc.ndc[2] = -2.0f * vx / vw - 1.0f;
  fc.ndc[3] = -2.0f * vy / vh - 1.0f;
  uint32_t rect[4] = {0, 0, t.width, t.height};
  if (t.data_window[2] > 0 && t.data_window[3] > 0) {
    const int64_t x0 = std::max<int64_t>(t.data_window[0], 0), y0 = std::max<int64_t>(t.data_window[1], 0);
    const int64_t x1 = std::min<int64_t>((int64_t)t.data_window[0] + t.data_window[2], t.width);
    const int64_t y1 = std::min<int64_t>((int64_t)t.data_window[1] + t.data_window[3], t.height);
    if (x1 <= x0 || y1 <= y0) {
      rect[0] = rect[1] = rect[2] = rect[3] = 0;
    } else {
      rect[0] = (uint32_t)x0; rect[1] = (uint32_t)y0;
      rect[2] = (uint32_t)(x1 - x0); rect[3] = (uint32_t)(y1 - y0);
    }
  }
  for (int k = 0; k < 4; ++k) {
    fc.rect[k] = rect[k];
    fc.background[k] = t.clear_color[k];
  }
  fc.width = t.width;
  fc.height = t.height;
  fc.max_bounces = st.max_bounces;
  fc.sample_lights = st.light_sampling != LOTUS_LIGHT_SAMPLING_BSDF ? 1u : 0u;
  fc.environment_background = st.environment_background ? 1u : 0u;
  if (st.output > LOTUS_OUTPUT_ROUGHNESS_METALLIC) return fail("unknown scene output");
  if (st.output != LOTUS_OUTPUT_RADIANCE) {
    // A diagnostic of the pixel centres' closest hits: not accumulated, the
    // radiance accumulation untouched.
    cudaStream_t s = R.stream;
    if (!R.ok(cudaMemcpyAsync(R.frame_const.ptr, &fc, sizeof(fc), cudaMemcpyHostToDevice, s), "frame constants",
            detail))
      return poison(detail);
    if (!R.ok(cudaMemsetAsync(R.walk_failure.ptr, 0, 2 * sizeof(uint32_t), s), "walk failure words", detail))
      return poison(detail);
    launch_clear_color(R.color.ptr, t.width * t.height,
        make_float4(t.clear_color[0], t.clear_color[1], t.clear_color[2], t.clear_color[3]), s);
    cudaEventRecord(R.ev_start, s);
    launch_diagnostic(R.view, R.frame_const.ptr, rect, st.output, R.color.ptr, s);
    if (want_depth)
      launch_depth(R.view, R.frame_const.ptr, rect, R.depth.ptr, t.width * t.height,
          (d.flags & LOTUS_FRAME_DEPTH_KEEP) == 0 || R.depth_fresh, t.clear_depth, s);
    R.depth_valid = want_depth;
  if (want_depth) R.depth_fresh = false;
    cudaEventRecord(R.ev_stop, s);
    uint32_t walks[2] = {0, 0};
    cudaMemcpyAsync(walks, R.walk_failure.ptr, sizeof(walks), cudaMemcpyDeviceToHost, s);
    if (!R.ok(cudaGetLastError(), "diagnostic output", detail) ||
        !R.ok(cudaStreamSynchronize(s), "diagnostic output", detail))
      return poison(detail);
    if (walks[0]) return poison(walk_failure_detail(walks, R.step_limit));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, R.ev_start, R.ev_stop);
    if (t.read_back && color_out) {
      if (!R.ok(cudaMemcpy(color_out, R.color.ptr, sizeof(float4) * (size_t)t.width * t.height,
                    cudaMemcpyDeviceToHost), "colour readback", detail))
        return poison(detail);
    }
    R.completion += 1;
    res.status = LOTUS_PASS;
    res.frames_rendered = 1;
    res.samples_per_pixel = 0;
    res.completion = R.completion;
    res.camera_rays = (uint64_t)rect[2] * rect[3];
    res.gpu_ms = ms;
    return LOTUS_PASS;
  }
  // The accumulation key (vulkan_backend.cpp:1188-1205).
  Renderer::Key key{};
  std::memcpy(key.world_to_clip, vulkan, sizeof(vulkan));
  key.width = t.width;
  key.height = t.height;
  std::memcpy(key.display_window, t.display_window, sizeof(key.display_window));
  std::memcpy(key.data_window, t.data_window, sizeof(key.data_window));
  key.integrator = st.integrator;
  key.light_sampling = st.light_sampling;
  key.restir_proposal = st.restir_proposal;
  key.restir_candidates = st.restir_candidates;
  key.sample_index = st.sample_index;
  key.max_bounces = st.max_bounces;
  key.scene_generation = R.scene_generation;
  if (!R.key_valid || !(R.key == key)) {
    R.key = key;
    R.key_valid = true;
    R.accumulated = 0;
  }
  const uint32_t room = st.max_samples == 0 ? d.frame_count
                                            : st.max_samples - std::min(st.max_samples, R.accumulated);
  const uint32_t to_add = std::min(d.frame_count, room);
  const uint32_t submissions = std::max(to_add, 1u);
  fc.sample_index = st.sample_index + R.accumulated;
  fc.accumulated = R.accumulated;
  fc.add_sample = to_add > 0 ? 1u : 0u;
  cudaStream_t s = R.stream;
  if (!R.ok(cudaMemcpyAsync(R.frame_const.ptr, &fc, sizeof(fc), cudaMemcpyHostToDevice, s), "frame constants", detail) ||
      !R.ok(cudaMemsetAsync(R.totals.ptr, 0, sizeof(RayTotals), s), "ray totals", detail) ||
      !R.ok(cudaMemsetAsync(R.walk_failure.ptr, 0, 2 * sizeof(uint32_t), s), "walk failure words", detail))
    return poison(detail);
  if (rect[2] < t.width || rect[3] < t.height || rect[2] == 0)
    launch_clear_color(R.color.ptr, t.width * t.height,
        make_float4(t.clear_color[0], t.clear_color[1], t.clear_color[2], t.clear_color[3]), s);
  // The camera pass's depth, once per call (the frame constants' camera and
  // window, sample 0's coverage sequence).
  if (want_depth)
    launch_depth(R.view, R.frame_const.ptr, rect, R.depth.ptr, t.width * t.height,
        (d.flags & LOTUS_FRAME_DEPTH_KEEP) == 0 || R.depth_fresh, t.clear_depth, s);
  R.depth_valid = want_depth;
  if (want_depth) R.depth_fresh = false;
  PathState P{R.path_origin.ptr, R.path_direction.ptr, R.path_throughput.ptr, R.path_radiance.ptr, R.path_hit.ptr};
  Queues Q;
  Q.ray[0] = R.queue_ray0.ptr;
  Q.ray[1] = R.queue_ray1.ptr;
  Q.hit = R.queue_hit.ptr;
  Q.shadow = ShadowQueue{R.sq_o.ptr, R.sq_d.ptr, R.sq_fl.ptr, R.sq_thr.ptr};
  Q.counts = R.counts.ptr;
  Q.capacity = t.width * t.height;
  Q.keys = R.sort_keys.ptr;
  Q.sorted = R.sort_queue.ptr;
  Q.bins = R.sort_bins.ptr;
  const bool want_timings = (d.flags & LOTUS_FRAME_TIMINGS) != 0;
  const bool want_visits = (d.flags & LOTUS_FRAME_COUNT_VISITS) != 0;
  SampleProfile profile;
  if (want_timings || want_visits) {
    const int capacity = 512;
    if (want_timings && R.profile_events.size() < 2 * (size_t)capacity) {
      while (R.profile_events.size() < 2 * (size_t)capacity) {
        cudaEvent_t e;
        if (!R.ok(cudaEventCreate(&e), "profiling event", detail)) return poison(detail);
        R.profile_events.push_back(e);
      }
    }
    R.profile_kinds.assign(capacity, 0);
    if (want_timings) {
      profile.events = R.profile_events.data();
      profile.kinds = R.profile_kinds.data();
      profile.capacity = capacity;
    }
    if (want_visits) {
      if (!R.ok(R.visits.resize(1), "visit counters", detail) ||
          !R.ok(cudaMemsetAsync(R.visits.ptr, 0, sizeof(VisitCounters), s), "visit counters", detail))
        return poison(detail);
      profile.visits = R.visits.ptr;
    }
  }
  // The graph's key without its rounds, and the rounds this call runs.
  Renderer::GraphKey gk{};
  gk.scene_generation = R.scene_generation;
  gk.width = t.width;
  gk.height = t.height;
  gk.max_bounces = st.max_bounces;
  std::memcpy(gk.rect, rect, sizeof(rect));
  gk.cache = use_cache ? R.cache_generation : 0u;
  TraceTuning tuning = R.tuning;
  if (tuning.rounds == 0 && R.auto_rounds != 0 && R.rounds_key == gk) tuning.rounds = R.auto_rounds;
  // The rounds the call's last sample ran (the frame result reports them).
  uint32_t last_rounds = wavefront_rounds(st.max_bounces, want_visits, tuning.rounds, use_cache ? cq.bounce : 0u);
  const bool choose_rounds = queued && R.tuning.rounds == 0 && !(R.rounds_key == gk);
  // Samples in waves: where two or more are added without the radiance
  // cache (which trains between samples), the wavefront runs `wave` samples
  // (the renderer's wave size, halved while the call adds fewer) as one
  // wave, their paths in slots k * pixels + pixel of a path state R.wave
  // times the target's size, so that every launch holds the wave's paths
  // and pays its ramp-up and drain once for them. Chains of up to kMaxChain samples run two
  // waves in flight: wave j on path state j % 2 and stream j % 2, each
  // resolving (its samples in order) after wave j - 1, so that only the
  // chain's last tail runs alone. A call's profiled part (timings or visit
  // counts) is its last wave (or sample), run alone.
  const uint32_t pixels = t.width * t.height;
  uint32_t wave = std::max(R.wave, 1u);
  while (wave > 1 && wave > to_add) wave /= 2;
  const bool waves = queued && !use_cache && to_add >= 2 && wave >= 2;
  const uint32_t profiled_samples = (want_timings || want_visits) ? (waves ? wave : 1u) : 0u;
  const uint32_t chainable = waves ? submissions - profiled_samples : 0u;
  while (R.ev_sample_done.size() < kMaxChain) {
    cudaEvent_t e;
    if (!R.ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event", detail)) return poison(detail);
    R.ev_sample_done.push_back(e);
  }
  if (chainable >= 2 * wave && !ensure_pair_buffers(R, (size_t)R.wave * pixels, detail)) return poison(detail);
  PathState P2{R.path_origin2.ptr, R.path_direction2.ptr, R.path_throughput2.ptr, R.path_radiance2.ptr,
      R.path_hit2.ptr};
  Queues Q2 = Q;
  Q2.ray[0] = R.queue_ray02.ptr;
  Q2.ray[1] = R.queue_ray12.ptr;
  Q2.hit = R.queue_hit2.ptr;
  Q2.shadow = ShadowQueue{R.sq_o2.ptr, R.sq_d2.ptr, R.sq_fl2.ptr, R.sq_thr2.ptr};
  Q2.counts = R.counts2.ptr;
  Q2.keys = R.sort_keys2.ptr;
  Q2.sorted = R.sort_queue2.ptr;
  Q2.bins = R.sort_bins2.ptr;
  // A wave's queues hold both samples' paths.
  Queues QW = Q, QW2 = Q2;
  QW.capacity = QW2.capacity = wave * pixels;
  const uint32_t* last_counts = R.counts.ptr;  // the call's last launch's queue counts
  uint32_t last_wave = 1;                      // and the samples it held
  FrameConst* fc0 = R.frame_const.ptr;
  cudaEventRecord(R.ev_start, s);
  for (uint32_t k = 0; k < submissions;) {
    if (k + wave <= chainable) {
      // A chain of `length` samples (a multiple of the wave, at most
      // kMaxChain) in length / wave waves; wave j's frame constants are
      // fc0's advanced by j waves.
      const uint32_t length = std::min(kMaxChain, (chainable - k) / wave * wave);
      const uint32_t count = length / wave;
      gk.rounds = wavefront_rounds(st.max_bounces, false, tuning.rounds, 0u);
      if (!(R.graph_chain_key == gk)) {
        for (cudaGraphExec_t& old : R.graph_chains)
          if (old) {
            cudaGraphExecDestroy(old);
            old = nullptr;
          }
        R.graph_chain_key = gk;
      }
      // One graph per chain length and wave size (2, 4, 8).
      const uint32_t shape = wave >= 8 ? 2u : wave >= 4 ? 1u : 0u;
      cudaGraphExec_t& chain = R.graph_chains[shape * (kMaxChain / 2 + 1) + count];
      if (!chain) {
        cudaGraph_t g;
        if (!R.ok(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "graph capture", detail))
          return poison(detail);
        for (uint32_t j = 0; j < count; ++j) launch_wave_frame(fc0, fc0 + 1 + j, wave * j, wave, pixels, s);
        cudaEventRecord(R.ev_fork, s);
        cudaStreamWaitEvent(R.stream2, R.ev_fork, 0);
        for (uint32_t j = 0; j < count; ++j) {
          const bool second = (j & 1u) != 0;
          launch_wavefront_sample(R.view, fc0 + 1 + j, rect, t.width, t.height, st.max_bounces, second ? P2 : P,
              second ? QW2 : QW, R.accum.ptr, R.color.ptr, R.totals.ptr, second ? R.stream2 : s, nullptr, tuning,
              nullptr, j ? R.ev_sample_done[j - 1] : nullptr, wave);
          cudaEventRecord(R.ev_sample_done[j], second ? R.stream2 : s);
        }
        cudaEventRecord(R.ev_join, R.stream2);
        cudaStreamWaitEvent(s, R.ev_join, 0);
        launch_advance_by(fc0, length, s);
        if (!R.ok(cudaStreamEndCapture(s, &g), "graph capture", detail)) return poison(detail);
        cudaError_t e = cudaGraphInstantiate(&chain, g, 0);
        cudaGraphDestroy(g);
        if (!R.ok(e, "graph instantiate", detail)) return poison(detail);
      }
      if (!R.ok(cudaGraphLaunch(chain, s), "graph launch", detail)) return poison(detail);
      k += length;
      last_counts = ((count - 1) & 1u) ? R.counts2.ptr : R.counts.ptr;
      last_wave = wave;
      last_rounds = gk.rounds;
      continue;
    }
    const bool profiled = profiled_samples != 0 && k + profiled_samples == submissions;
    last_rounds = wavefront_rounds(st.max_bounces, profiled && want_visits, tuning.rounds, use_cache ? cq.bounce : 0u);
    last_counts = R.counts.ptr;
    if (profiled && profiled_samples > 1) {
      // The profiled last wave, run alone.
      launch_wave_frame(fc0, fc0 + 1, 0, wave, pixels, s);
      launch_wavefront_sample(R.view, fc0 + 1, rect, t.width, t.height, st.max_bounces, P, QW, R.accum.ptr,
          R.color.ptr, R.totals.ptr, s, &profile, tuning, &cq, nullptr, wave);
      launch_advance_by(fc0, wave, s);
      k += wave;
      last_wave = wave;
      continue;
    }
    last_wave = 1;
    ++k;
    if (profiled) {
      if (queued)
        launch_wavefront_sample(R.view, R.frame_const.ptr, rect, t.width, t.height, st.max_bounces, P, Q,
            R.accum.ptr, R.color.ptr, R.totals.ptr, s, &profile, tuning, &cq);
      else
        launch_reference_pt(R.view, R.frame_const.ptr, rect, R.accum.ptr, R.color.ptr, R.totals.ptr, s,
            &profile);
      launch_advance(R.frame_const.ptr, s);
    } else if (queued) {
      gk.rounds = wavefront_rounds(st.max_bounces, false, tuning.rounds, use_cache ? cq.bounce : 0u);
      if (!R.graph || !(R.graph_key == gk)) {
        if (R.graph) {
          cudaGraphExecDestroy(R.graph);
          R.graph = nullptr;
        }
        cudaGraph_t g;
        if (!R.ok(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "graph capture", detail))
          return poison(detail);
        launch_wavefront_sample(R.view, R.frame_const.ptr, rect, t.width, t.height, st.max_bounces, P, Q,
            R.accum.ptr, R.color.ptr, R.totals.ptr, s, nullptr, tuning, &cq);
        launch_advance(R.frame_const.ptr, s);
        if (!R.ok(cudaStreamEndCapture(s, &g), "graph capture", detail)) return poison(detail);
        cudaError_t e = cudaGraphInstantiate(&R.graph, g, 0);
        cudaGraphDestroy(g);
        if (!R.ok(e, "graph instantiate", detail)) return poison(detail);
        R.graph_key = gk;
      }
      if (!R.ok(cudaGraphLaunch(R.graph, s), "graph launch", detail)) return poison(detail);
    } else {
      launch_reference_pt(R.view, R.frame_const.ptr, rect, R.accum.ptr, R.color.ptr, R.totals.ptr, s);
      launch_advance(R.frame_const.ptr, s);
    }
  }
  cudaEventRecord(R.ev_stop, s);
  RayTotals totals{};
  uint32_t walks[2] = {0, 0};
  std::vector<uint32_t> counts(3 * (size_t)(st.max_bounces + 2), 0);
  cudaMemcpyAsync(&totals, R.totals.ptr, sizeof(totals), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(walks, R.walk_failure.ptr, sizeof(walks), cudaMemcpyDeviceToHost, s);
  if (queued)
    cudaMemcpyAsync(counts.data(), last_counts, counts.size() * 4,
        cudaMemcpyDeviceToHost, s);
  if (!R.ok(cudaStreamSynchronize(s), "render", detail)) return poison(detail);
  if (walks[0]) return poison(walk_failure_detail(walks, R.step_limit));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, R.ev_start, R.ev_stop);
  if (use_cache) {
    uint32_t cc[2] = {0, 0};
    if (R.ok(cudaMemcpy(cc, R.cache_counters.ptr, sizeof(cc), cudaMemcpyDeviceToHost), "cache counters", detail)) {
      res.cache_queries = std::min<uint32_t>(cc[0], (uint32_t)R.cache_queries.count);
      res.cache_training_records = std::min<uint32_t>(cc[1], (uint32_t)R.cache_train.count);
    }
    if (R.cache.error_flag(s) != 0) return poison("a radiance-cache kernel's tensor-core wait gave up");
  }
  if (want_timings) {
    double by_kind[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t launches[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = 0; i < profile.count; ++i) {
      float kms = 0.0f;
      cudaEventElapsedTime(&kms, R.profile_events[2 * i], R.profile_events[2 * i + 1]);
      by_kind[R.profile_kinds[i]] += kms;
      ++launches[R.profile_kinds[i]];
    }
    res.timings_available = 1;
    res.camera_gpu_ms = by_kind[0];
    res.extend_gpu_ms = by_kind[1];
    res.shade_gpu_ms = by_kind[2];
    res.shadow_gpu_ms = by_kind[3];
    res.resolve_gpu_ms = by_kind[4];
    res.cache_gpu_ms = by_kind[5] + by_kind[8];
    res.cache_infer_gpu_ms = by_kind[5];
    res.cache_train_gpu_ms = by_kind[8];
    res.tail_gpu_ms = by_kind[6];
    res.sort_gpu_ms = by_kind[7];
    res.extend_launches = launches[1];
    res.shadow_launches = launches[3];
  }
  if (want_visits) {
    VisitCounters v{};
    if (!R.ok(cudaMemcpy(&v, R.visits.ptr, sizeof(v), cudaMemcpyDeviceToHost), "visit counters", detail))
      return poison(detail);
    for (int k = 0; k < 3; ++k) {
      res.visit_rays[k] = v.rays[k];
      res.node_visits[k] = v.nodes[k];
      res.triangle_visits[k] = v.triangles[k];
      res.instance_visits[k] = v.instances[k];
    }
  }
  R.accumulated += to_add;
  R.completion += submissions;
  if (t.read_back && color_out) {
    if (!R.ok(cudaMemcpyAsync(color_out, R.color.ptr, sizeof(float4) * (size_t)t.width * t.height,
                  cudaMemcpyDeviceToHost, s), "colour readback", detail) ||
        !R.ok(cudaStreamSynchronize(s), "colour readback", detail))
      return poison(detail);
  }
  res.status = LOTUS_PASS;
  res.frames_rendered = submissions;
  res.samples_per_pixel = R.accumulated;
  res.completion = R.completion;
  res.camera_rays = totals.camera;
  res.extension_rays = totals.extension;
  res.shadow_rays = totals.shadow;
  res.gpu_ms = ms;
  res.wavefront_rounds = 0;
  res.wavefront_path_count_size = 0;
  if (wavefront && to_add > 0) {
    uint32_t last = 0;
    for (uint32_t b = 0; b <= st.max_bounces && b < LOTUS_MAX_REPORTED_BOUNCES; ++b) {
      const uint32_t c = b == 0 ? rect[2] * rect[3] * last_wave : counts[3 * b];
      res.wavefront_path_counts[b] = c;
      if (c) last = b + 1;
    }
    res.wavefront_path_count_size = last;
    res.wavefront_rounds = last_rounds;
    res.last_wave_samples = last_wave;
  }
  if (queued && to_add > 0) {
    if (choose_rounds) {
      gk.rounds = 0;
      R.rounds_key = gk;
      R.auto_rounds = choose_wavefront_rounds(counts.data(), extension_resident_threads(), st.max_bounces);
    }
  }
  return LOTUS_PASS;
}

}  // namespace

extern "C" {

uint32_t lotus_cuda_abi_version(void) { return LOTUS_CUDA_ABI_VERSION; }

uint32_t lotus_cuda_struct_sizes(uint64_t* sizes, uint32_t capacity) {
  const uint64_t s[] = {sizeof(lotus_geometry), sizeof(lotus_instance), sizeof(lotus_texture),
      sizeof(lotus_texture_input), sizeof(lotus_material),
      sizeof(lotus_environment), sizeof(lotus_light), sizeof(lotus_scene_desc), sizeof(lotus_scene_result),
      sizeof(lotus_target), sizeof(lotus_settings), sizeof(lotus_frame_desc),
      sizeof(lotus_frame_result), sizeof(lotus_cuda_options), sizeof(lotus_temporal_desc),
      sizeof(lotus_temporal_instance), sizeof(lotus_cache_desc)};
  const uint32_t n = sizeof(s) / sizeof(s[0]);
  for (uint32_t i = 0; i < n && i < capacity; ++i) sizes[i] = s[i];
  return n;
}

int32_t lotus_cuda_capability(int32_t device, char* detail, size_t detail_size) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    copy_detail(detail, detail_size, std::string("no CUDA device: ") + cudaGetErrorString(e));
    return LOTUS_SKIP;
  }
  if (device < 0 || device >= count) {
    copy_detail(detail, detail_size, "no CUDA device " + std::to_string(device));
    return LOTUS_SKIP;
  }
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess || p.major != 10) {
    copy_detail(detail, detail_size, "the device is not sm_100 (built for sm_100a only)");
    return LOTUS_SKIP;
  }
  copy_detail(detail, detail_size, p.name);
  return LOTUS_PASS;
}

int32_t lotus_cuda_create(const lotus_cuda_options* options, lotus_cuda_renderer** out, char* error,
    size_t error_size) {
  if (!out) return LOTUS_FAIL;
  *out = nullptr;
  const int device = options ? options->device : 0;
  const int32_t cap = lotus_cuda_capability(device, error, error_size);
  if (cap != LOTUS_PASS) return cap;
  auto* h = new (std::nothrow) lotus_cuda_renderer();
  if (!h) {
    copy_detail(error, error_size, "out of host memory");
    return LOTUS_FAIL;
  }
  Renderer& R = h->r;
  R.device = device;
  if (options && options->bvh_leaf_size) {
    if (options->bvh_leaf_size > 8) {
      copy_detail(error, error_size, "bvh_leaf_size must be in 1..8");
      delete h;
      return LOTUS_FAIL;
    }
    R.bvh_leaf_size = options->bvh_leaf_size;
  }
  if (options && (options->trace_refill_below > 32 || options->trace_blocks_per_sm > 64 ||
                     options->wavefront_rounds > LOTUS_MAX_BOUNCES + 1 ||
                     (options->samples_per_wave != 0 && options->samples_per_wave != 1 &&
                      options->samples_per_wave != 2 && options->samples_per_wave != 4 &&
                      options->samples_per_wave != kMaxWave))) {
    copy_detail(error, error_size,
        "trace_refill_below must be in 0..32, trace_blocks_per_sm in 0..64, wavefront_rounds in 0..1025 "
        "and samples_per_wave 0, 1, 2, 4 or 8");
    delete h;
    return LOTUS_FAIL;
  }
  if (options) {
    R.tuning.refill_below = options->trace_refill_below;
    R.tuning.blocks_per_sm = options->trace_blocks_per_sm;
    R.tuning.rounds = options->wavefront_rounds;
    if (options->traversal_step_limit) R.step_limit = options->traversal_step_limit;
    if (options->samples_per_wave) R.wave = options->samples_per_wave;
  }
  std::string detail;
  if (!R.ok(cudaSetDevice(device), "cudaSetDevice", detail) ||
      !R.ok(R.walk_failure.resize(2), "walk failure words", detail) ||
      !R.ok(cudaMemset(R.walk_failure.ptr, 0, 2 * sizeof(uint32_t)), "walk failure words", detail) ||
      !R.ok(cudaStreamCreateWithFlags(&R.stream, cudaStreamNonBlocking), "stream", detail) ||
      !R.ok(cudaStreamCreateWithFlags(&R.stream2, cudaStreamNonBlocking), "stream", detail) ||
      !R.ok(cudaEventCreateWithFlags(&R.ev_fork, cudaEventDisableTiming), "event", detail) ||
      !R.ok(cudaEventCreateWithFlags(&R.ev_join, cudaEventDisableTiming), "event", detail) ||
      !R.ok(cudaEventCreate(&R.ev_start), "event", detail) || !R.ok(cudaEventCreate(&R.ev_stop), "event", detail)) {
    copy_detail(error, error_size, detail);
    delete h;
    return LOTUS_FAIL;
  }
  *out = h;
  return LOTUS_PASS;
}

void lotus_cuda_destroy(lotus_cuda_renderer* r) {
  if (!r) return;
  cudaSetDevice(r->r.device);
  cudaStreamSynchronize(r->r.stream);
  delete r;
}

int32_t lotus_cuda_update_scene(lotus_cuda_renderer* r, const lotus_scene_desc* scene,
    lotus_scene_result* result) {
  lotus_scene_result local{};
  lotus_scene_result& res = result ? *result : local;
  std::memset(&res, 0, sizeof(res));
  if (!r || !scene) {
    copy_detail(res.detail, sizeof(res.detail), "no renderer or scene");
    return res.status = LOTUS_FAIL;
  }
  Renderer& R = r->r;
  if (!R.failure.empty()) {
    copy_detail(res.detail, sizeof(res.detail), "the renderer failed earlier: " + R.failure);
    return res.status = LOTUS_FAIL;
  }
  cudaSetDevice(R.device);
  return update_scene(R, *scene, res);
}

int32_t lotus_cuda_update_instances(lotus_cuda_renderer* r, const lotus_instance* instances, uint32_t count,
    lotus_scene_result* result) {
  lotus_scene_result local{};
  lotus_scene_result& res = result ? *result : local;
  std::memset(&res, 0, sizeof(res));
  if (!r) {
    copy_detail(res.detail, sizeof(res.detail), "no renderer");
    return res.status = LOTUS_FAIL;
  }
  Renderer& R = r->r;
  if (!R.failure.empty()) {
    copy_detail(res.detail, sizeof(res.detail), "the renderer failed earlier: " + R.failure);
    return res.status = LOTUS_FAIL;
  }
  cudaSetDevice(R.device);
  return update_instances(R, instances, count, res);
}

int32_t lotus_cuda_update_geometry(lotus_cuda_renderer* r, uint32_t geometry, const float* positions,
    uint32_t vertex_count, const float* normals, lotus_scene_result* result) {
  lotus_scene_result local{};
  lotus_scene_result& res = result ? *result : local;
  std::memset(&res, 0, sizeof(res));
  if (!r) {
    copy_detail(res.detail, sizeof(res.detail), "no renderer");
    return res.status = LOTUS_FAIL;
  }
  Renderer& R = r->r;
  if (!R.failure.empty()) {
    copy_detail(res.detail, sizeof(res.detail), "the renderer failed earlier: " + R.failure);
    return res.status = LOTUS_FAIL;
  }
  cudaSetDevice(R.device);
  return update_geometry(R, geometry, positions, vertex_count, normals, res);
}

int32_t lotus_cuda_render(lotus_cuda_renderer* r, const lotus_frame_desc* frame, lotus_frame_result* result,
    float* color) {
  lotus_frame_result local{};
  lotus_frame_result& res = result ? *result : local;
  std::memset(&res, 0, sizeof(res));
  if (!r || !frame) {
    copy_detail(res.detail, sizeof(res.detail), "no renderer or frame");
    return res.status = LOTUS_FAIL;
  }
  Renderer& R = r->r;
  if (!R.failure.empty()) {
    copy_detail(res.detail, sizeof(res.detail), "the renderer failed earlier: " + R.failure);
    return res.status = LOTUS_FAIL;
  }
  cudaSetDevice(R.device);
  return render(R, *frame, res, color);
}

int32_t lotus_cuda_read_color(lotus_cuda_renderer* r, float* color, uint64_t capacity_floats) {
  if (!r || !color) return LOTUS_FAIL;
  Renderer& R = r->r;
  const uint64_t n = 4ull * R.width * R.height;
  if (n == 0 || capacity_floats < n || !R.color.ptr) return LOTUS_FAIL;
  cudaSetDevice(R.device);
  if (cudaMemcpyAsync(color, R.color.ptr, n * 4, cudaMemcpyDeviceToHost, R.stream) != cudaSuccess ||
      cudaStreamSynchronize(R.stream) != cudaSuccess)
    return LOTUS_FAIL;
  return LOTUS_PASS;
}

int64_t lotus_cuda_read_scene(lotus_cuda_renderer* r, uint32_t what, uint32_t index, void* out,
    uint64_t capacity) {
  if (!r) return -1;
  Renderer& R = r->r;
  if (!R.scene_ready || !R.failure.empty()) return -1;
  const HostScene& h = R.host;
  const bool per_geometry = what == LOTUS_SCENE_POSITIONS || what == LOTUS_SCENE_TRIANGLES ||
      what == LOTUS_SCENE_NORMALS;
  if (per_geometry && index >= h.geometries.size()) return -1;
  const uint32_t n_inst = (uint32_t)R.host_instances.size();
  uint64_t bytes = 0;
  switch (what) {
    case LOTUS_SCENE_POSITIONS: bytes = 12ull * h.geometries[index].vertex_count; break;
    case LOTUS_SCENE_TRIANGLES: bytes = 12ull * h.geometries[index].triangle_count; break;
    case LOTUS_SCENE_NORMALS:
      bytes = h.normal_base[index] == kNoLights ? 0 : 36ull * h.geometries[index].triangle_count;
      break;
    case LOTUS_SCENE_INSTANCES: bytes = sizeof(lotus_instance) * (uint64_t)n_inst; break;
    case LOTUS_SCENE_MATERIALS: bytes = sizeof(lotus_material) * (uint64_t)R.materials.count; break;
    case LOTUS_SCENE_ENVIRONMENT: bytes = 12; break;
    default: return -1;
  }
  if (!out) return (int64_t)bytes;
  if (capacity < bytes) return -1;
  if (bytes == 0) return 0;
  cudaSetDevice(R.device);
  auto copy = [&](const void* src) {
    return cudaMemcpy(out, src, bytes, cudaMemcpyDeviceToHost) == cudaSuccess;
  };
  switch (what) {
    case LOTUS_SCENE_POSITIONS:
      return copy(R.scene_pos.ptr + 3 * h.vertex_base[index]) ? (int64_t)bytes : -1;
    case LOTUS_SCENE_TRIANGLES:
      return copy(R.scene_tri.ptr + 3 * (size_t)h.tri_base[index]) ? (int64_t)bytes : -1;
    case LOTUS_SCENE_NORMALS:
      return copy(R.normals.ptr + 9 * (size_t)h.normal_base[index]) ? (int64_t)bytes : -1;
    case LOTUS_SCENE_INSTANCES: {
      // The shading records hold world_from_object's rows and the material
      // slot; the traversal records the BLAS root, which names the geometry.
      std::vector<InstanceShading> shade(n_inst);
      std::vector<InstanceTraversal> trav(n_inst);
      if (n_inst &&
          (cudaMemcpy(shade.data(), R.inst_shade.ptr, n_inst * sizeof(InstanceShading), cudaMemcpyDeviceToHost) !=
               cudaSuccess ||
           cudaMemcpy(trav.data(), R.inst_trav.ptr, n_inst * sizeof(InstanceTraversal), cudaMemcpyDeviceToHost) !=
               cudaSuccess))
        return -1;
      lotus_instance* o = static_cast<lotus_instance*>(out);
      for (uint32_t i = 0; i < n_inst; ++i) {
        std::memset(&o[i], 0, sizeof(o[i]));
        const float4* m = shade[i].m;
        const float rows[3][4] = {{m[0].x, m[0].y, m[0].z, m[0].w}, {m[1].x, m[1].y, m[1].z, m[1].w},
            {m[2].x, m[2].y, m[2].z, m[2].w}};
        for (int c = 0; c < 4; ++c) {
          for (int rr = 0; rr < 3; ++rr) o[i].world_from_object[c * 4 + rr] = rows[rr][c];
          o[i].world_from_object[c * 4 + 3] = c == 3 ? 1.0f : 0.0f;
        }
        o[i].material = shade[i].material;
        // The resident host copy keeps each instance's geometry; the device
        // record's BLAS root must name the same one (or none, for a
        // geometry without triangles).
        const uint32_t g = R.host_instances[i].geometry;
        const uint32_t want = h.geometries[g].triangle_count ? h.node_base[g] : (uint32_t)kEmptyChild;
        if (trav[i].blas_root != want) return -1;
        o[i].geometry = g;
      }
      return (int64_t)bytes;
    }
    case LOTUS_SCENE_MATERIALS: {
      std::vector<MaterialRecord> rec(R.materials.count);
      if (cudaMemcpy(rec.data(), R.materials.ptr, rec.size() * sizeof(MaterialRecord), cudaMemcpyDeviceToHost) !=
          cudaSuccess)
        return -1;
      lotus_material* o = static_cast<lotus_material*>(out);
      for (size_t i = 0; i < rec.size(); ++i) {
        const MaterialRecord& m = rec[i];
        std::memset(&o[i], 0, sizeof(o[i]));
        o[i].base_color[0] = m.base_roughness.x; o[i].base_color[1] = m.base_roughness.y;
        o[i].base_color[2] = m.base_roughness.z; o[i].roughness = m.base_roughness.w;
        o[i].emission[0] = m.emission_metallic.x; o[i].emission[1] = m.emission_metallic.y;
        o[i].emission[2] = m.emission_metallic.z; o[i].metallic = m.emission_metallic.w;
        o[i].specular_color[0] = m.specular_ior.x; o[i].specular_color[1] = m.specular_ior.y;
        o[i].specular_color[2] = m.specular_ior.z; o[i].ior = m.specular_ior.w;
        o[i].transmission_color[0] = m.transmission.x; o[i].transmission_color[1] = m.transmission.y;
        o[i].transmission_color[2] = m.transmission.z; o[i].transmission = m.transmission.w;
        o[i].opacity = m.coverage.x;
        o[i].opacity_threshold = m.coverage.y;
        uint32_t flags;
        std::memcpy(&flags, &m.coverage.z, 4);
        o[i].flags = flags & (LOTUS_MATERIAL_SPECULAR_WORKFLOW | LOTUS_MATERIAL_THIN_WALLED);
        if (flags & kMaterialGltf) {
          o[i].model = LOTUS_MODEL_GLTF_PBR;
          o[i].specular = m.gltf.x;
          o[i].clearcoat = m.gltf.y;
          o[i].clearcoat_roughness = m.gltf.z;
          o[i].emissive_strength = m.gltf.w;
          o[i].sheen_color[0] = m.sheen.x; o[i].sheen_color[1] = m.sheen.y; o[i].sheen_color[2] = m.sheen.z;
          o[i].sheen_roughness = m.sheen.w;
        }
      }
      return (int64_t)bytes;
    }
    case LOTUS_SCENE_ENVIRONMENT:
      std::memcpy(out, R.view.env_constant, 12);
      return 12;
    default:
      return -1;
  }
}

int32_t lotus_cuda_read_depth(lotus_cuda_renderer* r, float* depth, uint64_t capacity_floats) {
  if (!r || !depth) return LOTUS_FAIL;
  Renderer& R = r->r;
  const uint64_t n = (uint64_t)R.width * R.height;
  if (n == 0 || capacity_floats < n || !R.depth.ptr || !R.depth_valid) return LOTUS_FAIL;
  cudaSetDevice(R.device);
  if (cudaMemcpyAsync(depth, R.depth.ptr, n * 4, cudaMemcpyDeviceToHost, R.stream) != cudaSuccess ||
      cudaStreamSynchronize(R.stream) != cudaSuccess)
    return LOTUS_FAIL;
  return LOTUS_PASS;
}

void* lotus_cuda_stream(lotus_cuda_renderer* r) { return r ? (void*)r->r.stream : nullptr; }

int64_t lotus_cuda_read_light_table(lotus_cuda_renderer* r, uint32_t* records, uint64_t record_capacity,
    uint32_t* offsets, uint64_t offset_capacity) {
  if (!r) return -1;
  Renderer& R = r->r;
  const uint64_t n = R.host_lights.size();
  if (records) {
    std::vector<LightRecord> dev(n);
    if (n) {
      cudaSetDevice(R.device);
      if (cudaMemcpy(dev.data(), R.lights.ptr, n * sizeof(LightRecord), cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1;
    }
    for (uint64_t i = 0; i < n && i < record_capacity; ++i) std::memcpy(records + 4 * i, &dev[i], 16);
  }
  if (offsets)
    for (uint64_t i = 0; i < R.host_light_offsets.size() && i < offset_capacity; ++i)
      offsets[i] = R.host_light_offsets[i];
  return (int64_t)n;
}

}  // extern "C"

namespace lotus {

bool renderer_access(lotus_cuda_renderer* r, RendererAccess& out, std::string& detail) {
  Renderer& R = r->r;
  if (!R.failure.empty()) {
    detail = "the renderer failed earlier: " + R.failure;
    return false;
  }
  if (!R.scene_ready) {
    detail = "no scene has been uploaded";
    return false;
  }
  out.device = R.device;
  out.stream = R.stream;
  out.view = &R.view;
  out.tuning = R.tuning;
  out.step_limit = R.step_limit;
  out.cache_enabled = R.cache_enabled;
  return true;
}

void renderer_poison(lotus_cuda_renderer* r, const std::string& detail) {
  if (r && r->r.failure.empty()) r->r.failure = detail;
}

bool make_frame_constants(const lotus_frame_desc& d, FrameConst& fc, uint32_t rect[4],
    std::string& detail) {
  const lotus_settings& st = d.settings;
  const lotus_target& t = d.target;
  if (t.width == 0 || t.height == 0) {
    detail = "the offscreen target is empty";
    return false;
  }
  for (int k = 0; k < 4; ++k)
    if (!std::isfinite(t.clear_color[k])) {
      detail = "invalid offscreen clear values";
      return false;
    }
  if (st.output != LOTUS_OUTPUT_RADIANCE) {
    detail = "only lotus_cuda_render renders the diagnostic outputs";
    return false;
  }
  if (st.integrator > LOTUS_INTEGRATOR_WAVEFRONT || st.light_sampling > LOTUS_LIGHT_SAMPLING_MIS) {
    detail = "unsupported integrator or light sampling";
    return false;
  }
  if (st.max_bounces > LOTUS_MAX_BOUNCES) {
    detail = "max_bounces exceeds " + std::to_string(LOTUS_MAX_BOUNCES);
    return false;
  }
  float vulkan[16];
  std::memcpy(vulkan, d.world_to_clip, sizeof(vulkan));
  for (int c = 0; c < 4; ++c) {
    const float z = d.world_to_clip[c * 4 + 2], w = d.world_to_clip[c * 4 + 3];
    vulkan[c * 4 + 1] = -d.world_to_clip[c * 4 + 1];
    vulkan[c * 4 + 2] = 0.5f * (z + w);
  }
  fc = FrameConst{};
  std::memcpy(fc.world_to_clip, vulkan, sizeof(vulkan));
  if (!invert4(vulkan, fc.clip_to_world)) {
    detail = "ray-query camera is singular or non-finite";
    return false;
  }
  float vx = 0.0f, vy = 0.0f, vw = (float)t.width, vh = (float)t.height;
  if (t.display_window[2] > 0.0f && t.display_window[3] > 0.0f) {
    vx = t.display_window[0]; vy = t.display_window[1]; vw = t.display_window[2]; vh = t.display_window[3];
  }
  fc.ndc[0] = 2.0f / vw;
  fc.ndc[1] = 2.0f / vh;
  fc.ndc[2] = -2.0f * vx / vw - 1.0f;
  fc.ndc[3] = -2.0f * vy / vh - 1.0f;
  rect[0] = 0; rect[1] = 0; rect[2] = t.width; rect[3] = t.height;
  if (t.data_window[2] > 0 && t.data_window[3] > 0) {
    const int64_t x0 = std::max<int64_t>(t.data_window[0], 0), y0 = std::max<int64_t>(t.data_window[1], 0);
    const int64_t x1 = std::min<int64_t>((int64_t)t.data_window[0] + t.data_window[2], t.width);
    const int64_t y1 = std::min<int64_t>((int64_t)t.data_window[1] + t.data_window[3], t.height);
    if (x1 <= x0 || y1 <= y0) {
      rect[0] = rect[1] = rect[2] = rect[3] = 0;
    } else {
      rect[0] = (uint32_t)x0; rect[1] = (uint32_t)y0;
      rect[2] = (uint32_t)(x1 - x0); rect[3] = (uint32_t)(y1 - y0);
    }
  }
  for (int k = 0; k < 4; ++k) {
    fc.rect[k] = rect[k];
    fc.background[k] = t.clear_color[k];
  }
  fc.width = t.width;
  fc.height = t.height;
  fc.max_bounces = st.max_bounces;
  fc.sample_lights = st.light_sampling != LOTUS_LIGHT_SAMPLING_BSDF ? 1u : 0u;
  fc.environment_background = st.environment_background ? 1u : 0u;
  return true;
}

}  // namespace lotus

namespace {

using namespace lotus;

// RenderTemporalScene (vulkan_backend.cpp:1711-2100): validation, history
// rules, then the passes in the reference's order.
int32_t render_temporal(Renderer& R, const lotus_temporal_desc& td, lotus_frame_result& res, float* color_out) {
  std::string detail;
  auto fail = [&](const std::string& msg) {
    copy_detail(res.detail, sizeof(res.detail), msg);
    return res.status = LOTUS_FAIL;
  };
  auto poison = [&](const std::string& msg) {
    R.failure = msg;
    return fail(msg);
  };
  const lotus_frame_desc& d = td.frame;
  const lotus_settings& st = d.settings;
  const lotus_target& t = d.target;
  if (!R.scene_ready) return fail("no scene has been uploaded");
  if (d.frame_count == 0) return fail("frame_count must be at least 1");
  const bool reuse = st.restir_temporal != 0;
  const bool reservoirs = reuse || st.restir_spatial != 0;
  const bool restir = st.light_sampling == LOTUS_LIGHT_SAMPLING_RESTIR_INITIAL;
  const bool accumulate = td.accumulate_radiance != 0;
  if (reservoirs && (d.frame_count != 1 || !restir || st.restir_candidates == 0 || st.restir_candidates > 64 ||
                        st.restir_max_history_candidates == 0 || st.restir_max_history_candidates > 65536))
    return fail("temporal reservoirs require Radiance, RestirInitial, one fresh sample, candidates in [1, 64] "
                "and history candidates in [1, 65536]");
  if (restir && (st.restir_candidates == 0 || st.restir_candidates > 64))
    return fail("RestirInitial needs restir_candidates in [1, 64]");
  if (st.restir_spatial && (st.restir_spatial_radius == 0 || st.restir_spatial_radius > 32))
    return fail("restir_spatial_radius must be in [1, 32]");
  if (st.restir_spatial_neighbours > LOTUS_MAX_SPATIAL_NEIGHBOURS)
    return fail("restir_spatial_neighbours must be in [0, " + std::to_string(LOTUS_MAX_SPATIAL_NEIGHBOURS) + "]");
  if (accumulate && (td.max_history_samples == 0 || td.max_history_samples > 65536))
    return fail("temporal radiance requires history samples in [1, 65536]");
  if (td.filter_iterations > 8 || (td.filter_iterations != 0 && !accumulate))
    return fail("temporal filtering requires radiance accumulation and at most 8 iterations");
  if (td.moment_precision > LOTUS_MOMENTS_FP16) return fail("unknown moment precision");
  if (td.history_rectification != 0)
    return fail("history rectification other than None is not built");
  if (st.integrator > LOTUS_INTEGRATOR_WAVEFRONT) return fail("unknown integrator");
  FrameConst fc{};
  uint32_t rect[4];
  lotus_frame_desc checked = d;
  if (restir) checked.settings.light_sampling = LOTUS_LIGHT_SAMPLING_MIS;  // validated as MIS
  if (!make_frame_constants(checked, fc, rect, detail)) return fail(detail);
  float prev_vulkan[16];
  std::memcpy(prev_vulkan, td.previous_world_to_clip, sizeof(prev_vulkan));
  for (int c = 0; c < 4; ++c) {
    const float z = td.previous_world_to_clip[c * 4 + 2], w = td.previous_world_to_clip[c * 4 + 3];
    prev_vulkan[c * 4 + 1] = -td.previous_world_to_clip[c * 4 + 1];
    prev_vulkan[c * 4 + 2] = 0.5f * (z + w);
  }
  Renderer::Temporal& T = R.temporal;
  const bool wavefront = st.integrator == LOTUS_INTEGRATOR_WAVEFRONT;
  if (!ensure_targets(R, t.width, t.height, wavefront, detail)) return poison(detail);
  // Buffers.
  const size_t n = (size_t)t.width * t.height;
  if (T.width != t.width || T.height != t.height) {
    T.width = t.width;
    T.height = t.height;
    T.frames = 0;
    T.surface_write = T.radiance_write = T.restir_write = 0;
    T.key_valid = false;
  }
  bool okb = R.ok(T.surface[0].resize(n), "temporal surface", detail) &&
             R.ok(T.surface[1].resize(n), "temporal surface", detail) &&
             R.ok(T.validity.resize(n), "temporal validity", detail) &&
             R.ok(T.constants.resize(1), "temporal constants", detail);
  if (okb && accumulate)
    okb = R.ok(T.radiance[0].resize(n), "temporal radiance", detail) &&
          R.ok(T.radiance[1].resize(n), "temporal radiance", detail) &&
          R.ok(T.batch.resize(n), "temporal batch", detail) &&
          (td.filter_iterations == 0 || R.ok(T.filter.resize(4 * n), "temporal filter", detail));
  if (okb && restir)
    okb = R.ok(T.initial.resize(n), "reservoirs", detail) && R.ok(T.reuse[0].resize(n), "reservoirs", detail) &&
          R.ok(T.reuse[1].resize(n), "reservoirs", detail) && R.ok(T.spatial.resize(n), "reservoirs", detail) &&
          R.ok(T.sources.resize(n), "reservoirs", detail) &&
          R.ok(T.surfaces[0].resize(n), "reservoir surfaces", detail) &&
          R.ok(T.surfaces[1].resize(n), "reservoir surfaces", detail) &&
          R.ok(T.primary_hit.resize(n), "primary hits", detail) && R.ok(T.primary_rng.resize(n), "primary hits", detail) &&
          R.ok(T.vis_origin.resize(n), "visibility queue", detail) &&
          R.ok(T.vis_direction.resize(n), "visibility queue", detail) &&
          R.ok(T.vis_pending.resize(n), "visibility queue", detail) &&
          R.ok(T.vis_slot.resize(n), "visibility queue", detail) &&
          R.ok(T.vis_counters.resize(3 * kVisibilityPasses), "visibility queue", detail);
  if (!okb) return poison(detail);
  // The transport key: a change drops the history (vulkan_backend.cpp:1766-1781).
  uint32_t key[18] = {st.integrator, st.light_sampling, st.restir_proposal, st.restir_candidates,
      st.restir_temporal, st.restir_max_history_candidates, st.restir_spatial, st.restir_spatial_radius,
      td.accumulate_radiance, st.sample_index, st.max_bounces, st.environment_background, 0, 0, 0, 0,
      st.restir_spatial_neighbours, td.moment_precision};
  std::memcpy(&key[12], t.clear_color, sizeof(t.clear_color));
  const bool fresh_batch = accumulate || reservoirs;
  bool previous = td.history_available != 0 && T.frames > 0;
  if (fresh_batch && previous && (!T.key_valid || std::memcmp(key, T.key, sizeof(key)) != 0)) previous = false;
  std::memcpy(T.key, key, sizeof(key));
  T.key_valid = true;
  if (!previous) T.sample_offset = 0;
  const uint32_t sample_offset = previous ? T.sample_offset : 0u;
  // Constants.
  fc.sample_index = st.sample_index + (fresh_batch ? sample_offset : 0u);
  fc.accumulated = 0;
  fc.add_sample = 1;
  fc.sample_lights = st.light_sampling != LOTUS_LIGHT_SAMPLING_BSDF ? 1u : 0u;
  TemporalConst tc{};
  std::memcpy(tc.current_view, td.current_view, sizeof(tc.current_view));
  if (previous) {
    std::memcpy(tc.previous_view, td.previous_view, sizeof(tc.previous_view));
    std::memcpy(tc.previous_world_to_clip, prev_vulkan, sizeof(prev_vulkan));
  }
  float vx = 0.0f, vy = 0.0f, vw = (float)t.width, vh = (float)t.height;
  if (t.display_window[2] > 0.0f && t.display_window[3] > 0.0f) {
    vx = t.display_window[0]; vy = t.display_window[1]; vw = t.display_window[2]; vh = t.display_window[3];
  }
  tc.previous_display[0] = vx; tc.previous_display[1] = vy; tc.previous_display[2] = vw; tc.previous_display[3] = vh;
  for (int k = 0; k < 4; ++k) {
    tc.previous_data[k] = rect[k];
    tc.validation[k] = td.validation[k];
  }
  tc.history = previous ? 1u : 0u;
  tc.width = t.width;
  tc.height = t.height;
  tc.accumulate = accumulate ? 1u : 0u;
  tc.fresh_samples = d.frame_count;
  tc.history_cap = td.max_history_samples;
  tc.filter_iterations = td.filter_iterations;
  tc.moments_half = td.moment_precision == LOTUS_MOMENTS_FP16 ? 1u : 0u;
  T.moments_half = tc.moments_half != 0;
  tc.restir_candidates = restir ? st.restir_candidates : 0u;
  tc.restir_history = reuse && previous ? 1u : 0u;
  tc.restir_max_history = st.restir_max_history_candidates;
  tc.restir_spatial = st.restir_spatial ? 1u : 0u;
  tc.restir_temporal = reservoirs ? 1u : 0u;
  tc.restir_radius = st.restir_spatial_radius;
  tc.restir_neighbours = st.restir_spatial_neighbours;
  tc.restir_proposal = st.restir_proposal;
  tc.sample_index = fc.sample_index;
  tc.max_bounces = st.max_bounces;
  const int sw = T.surface_write, rs = T.restir_write, rw = T.radiance_write;
  if (restir) {
    fc.restir_primary = 1;
    if (st.restir_candidates != 0) {
      // The initial pass traces the first sample's camera rays; the
      // temporal pass and the path tracer's camera step reuse its hits.
      fc.primary_hit = T.primary_hit.ptr;
      fc.primary_rng = T.primary_rng.ptr;
      fc.primary_sample = fc.sample_index;
    }
    if (st.restir_spatial) {
      fc.restir_final = reinterpret_cast<const unsigned char*>(T.spatial.ptr);
      fc.restir_stride = sizeof(RestirReuse);
    } else if (reservoirs) {
      fc.restir_final = reinterpret_cast<const unsigned char*>(T.reuse[rs].ptr);
      fc.restir_stride = sizeof(RestirReuse);
    } else {
      fc.restir_final = reinterpret_cast<const unsigned char*>(T.initial.ptr);
      fc.restir_stride = sizeof(RestirPixel);
    }
  }
  cudaStream_t s = R.stream;
  if (!R.ok(cudaMemcpyAsync(R.frame_const.ptr, &fc, sizeof(fc), cudaMemcpyHostToDevice, s), "frame constants", detail) ||
      !R.ok(cudaMemcpyAsync(T.constants.ptr, &tc, sizeof(tc), cudaMemcpyHostToDevice, s), "temporal constants", detail) ||
      !R.ok(cudaMemsetAsync(R.totals.ptr, 0, sizeof(RayTotals), s), "ray totals", detail) ||
      !R.ok(cudaMemsetAsync(R.walk_failure.ptr, 0, 2 * sizeof(uint32_t), s), "walk failure words", detail))
    return poison(detail);
  cudaEventRecord(R.ev_start, s);
  const uint32_t pixels = (uint32_t)n;
  launch_temporal_surface(R.view, R.frame_const.ptr, T.constants.ptr, T.instances.ptr, T.surface[sw].ptr, pixels, s);
  launch_reproject(T.constants.ptr, T.surface[sw].ptr, T.surface[1 - sw].ptr, T.validity.ptr, pixels, s);
  if (restir) {
    const VisibilityQueue vq{T.vis_origin.ptr, T.vis_direction.ptr, T.vis_slot.ptr, T.vis_pending.ptr,
        T.vis_counters.ptr, pixels, T.vis_counters.ptr + 2 * kVisibilityPasses};
    if (!R.ok(cudaMemsetAsync(T.vis_counters.ptr, 0, 2 * kVisibilityPasses * sizeof(uint32_t), s),
            "visibility queue", detail) ||
        !R.ok(cudaMemsetAsync(vq.failed, 0xFF, kVisibilityPasses * sizeof(uint32_t), s), "visibility queue", detail))
      return poison(detail);
    launch_restir_initial(R.view, R.frame_const.ptr, T.constants.ptr, T.initial.ptr, T.primary_hit.ptr,
        T.primary_rng.ptr, vq, pixels, s);
    launch_visibility(R.view, vq, 0, reinterpret_cast<unsigned char*>(T.initial.ptr), sizeof(RestirPixel), false,
        s, R.tuning);
    if (reservoirs) {
      launch_restir_temporal(R.view, R.frame_const.ptr, T.constants.ptr, T.primary_hit.ptr, T.instances.ptr,
          T.initial.ptr, T.validity.ptr, T.surface[sw].ptr, T.reuse[1 - rs].ptr, T.surfaces[1 - rs].ptr,
          T.reuse[rs].ptr, T.surfaces[rs].ptr, vq, pixels, s);
      launch_visibility(R.view, vq, 1, reinterpret_cast<unsigned char*>(T.reuse[rs].ptr), sizeof(RestirReuse),
          true, s, R.tuning);
    }
    if (st.restir_spatial) {
      launch_restir_spatial(R.view, R.frame_const.ptr, T.constants.ptr, T.reuse[rs].ptr, T.surfaces[rs].ptr,
          T.spatial.ptr, T.sources.ptr, vq, pixels, s);
      launch_visibility(R.view, vq, 2, reinterpret_cast<unsigned char*>(T.spatial.ptr), sizeof(RestirReuse), true,
          s, R.tuning);
    }
  }
  if (rect[2] < t.width || rect[3] < t.height || rect[2] == 0)
    launch_clear_color(R.color.ptr, pixels, make_float4(t.clear_color[0], t.clear_color[1], t.clear_color[2],
        t.clear_color[3]), s);
  PathState P{R.path_origin.ptr, R.path_direction.ptr, R.path_throughput.ptr, R.path_radiance.ptr, R.path_hit.ptr};
  Queues Q;
  Q.ray[0] = R.queue_ray0.ptr;
  Q.ray[1] = R.queue_ray1.ptr;
  Q.hit = R.queue_hit.ptr;
  Q.shadow = ShadowQueue{R.sq_o.ptr, R.sq_d.ptr, R.sq_fl.ptr, R.sq_thr.ptr};
  Q.counts = R.counts.ptr;
  Q.capacity = pixels;
  Q.keys = R.sort_keys.ptr;
  Q.sorted = R.sort_queue.ptr;
  Q.bins = R.sort_bins.ptr;
  // The radiance cache serves the temporal frames' wavefront samples too.
  const bool use_cache = wavefront && R.cache_enabled && R.cache.ready();
  if (use_cache && !ensure_cache_queues(R, pixels, detail)) return poison(detail);
  const CacheQueues cq = use_cache ? cache_queues(R) : CacheQueues();
  // The wavefront rounds before the tail, as RenderScene chooses them.
  Renderer::GraphKey rk{};
  rk.scene_generation = R.scene_generation;
  rk.width = t.width;
  rk.height = t.height;
  rk.max_bounces = st.max_bounces;
  std::memcpy(rk.rect, rect, sizeof(rect));
  rk.cache = use_cache ? R.cache_generation : 0u;
  TraceTuning tuning = R.tuning;
  if (tuning.rounds == 0 && R.temporal_auto_rounds != 0 && R.temporal_rounds_key == rk)
    tuning.rounds = R.temporal_auto_rounds;
  const bool choose_rounds = wavefront && d.frame_count != 0 && R.tuning.rounds == 0 && !(R.temporal_rounds_key == rk);
  for (uint32_t k = 0; k < d.frame_count; ++k) {
    if (wavefront)
      launch_wavefront_sample(R.view, R.frame_const.ptr, rect, t.width, t.height, st.max_bounces, P, Q,
          R.accum.ptr, R.color.ptr, R.totals.ptr, s, nullptr, tuning, &cq);
    else
      launch_reference_pt(R.view, R.frame_const.ptr, rect, R.accum.ptr, R.color.ptr, R.totals.ptr, s);
    launch_advance(R.frame_const.ptr, s);
  }
  if (accumulate) {
    cudaMemcpyAsync(T.batch.ptr, R.color.ptr, n * sizeof(float4), cudaMemcpyDeviceToDevice, s);
    launch_svgf(T.constants.ptr, tc, T.batch.ptr, T.surface[sw].ptr, T.validity.ptr, T.radiance[1 - rw].ptr,
        T.radiance[rw].ptr, T.filter.ptr, R.color.ptr, pixels, s);
  }
  cudaEventRecord(R.ev_stop, s);
  RayTotals totals{};
  cudaMemcpyAsync(&totals, R.totals.ptr, sizeof(totals), cudaMemcpyDeviceToHost, s);
  uint32_t walks[2] = {0, 0};
  cudaMemcpyAsync(walks, R.walk_failure.ptr, sizeof(walks), cudaMemcpyDeviceToHost, s);
  uint32_t failed[kVisibilityPasses] = {~0u, ~0u, ~0u};
  if (restir)
    cudaMemcpyAsync(failed, T.vis_counters.ptr + 2 * kVisibilityPasses, sizeof(failed), cudaMemcpyDeviceToHost, s);
  std::vector<uint32_t> counts;
  if (choose_rounds) {
    counts.assign(3 * (size_t)(st.max_bounces + 2), 0u);
    cudaMemcpyAsync(counts.data(), R.counts.ptr, counts.size() * 4, cudaMemcpyDeviceToHost, s);
  }
  if (!R.ok(cudaStreamSynchronize(s), "temporal frame", detail)) return poison(detail);
  if (walks[0]) return poison(walk_failure_detail(walks, R.step_limit));
  if (choose_rounds) {
    R.temporal_rounds_key = rk;
    R.temporal_auto_rounds = choose_wavefront_rounds(counts.data(), extension_resident_threads(), st.max_bounces);
  }
  // A reservoir whose arithmetic failed (flag 2) fails the frame and the
  // renderer, as the reference's record readback does
  // (vulkan_backend.cpp:1650-1705): the first failed initial record, else
  // the first pixel whose temporal or spatial record failed.
  if (failed[0] != ~0u) {
    RestirPixel p{};
    cudaMemcpy(&p, T.initial.ptr + failed[0], sizeof(p), cudaMemcpyDeviceToHost);
    char where[320];
    std::snprintf(where, sizeof(where),
        "initial reservoir arithmetic is invalid or exceeds GPU float storage at pixel (%u, %u): light %u, "
        "weight sum %g, target %g, candidates %u, proposal %g",
        failed[0] % t.width, failed[0] / t.width, p.reservoir.sample, (double)p.reservoir.weight_sum,
        (double)p.reservoir.selected_target, p.reservoir.candidate_count, (double)p.proposal);
    return poison(where);
  }
  if (failed[1] != ~0u && failed[1] <= failed[2])
    return poison("temporal reservoir arithmetic is invalid or exceeds GPU float storage");
  if (failed[2] != ~0u) return poison("spatial reservoir arithmetic is invalid or exceeds GPU float storage");
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, R.ev_start, R.ev_stop);
  T.restir_ran = restir;
  T.spatial_ran = restir && st.restir_spatial;
  T.accumulate_ran = accumulate;
  T.filter_ran = accumulate && td.filter_iterations != 0;
  // The products of this frame stay at the indices just written; the next
  // frame writes the other halves.
  T.last_surface = sw;
  T.last_radiance = rw;
  T.last_restir = rs;
  T.surface_write ^= 1;
  if (accumulate) T.radiance_write ^= 1;
  if (reservoirs) T.restir_write ^= 1;
  ++T.frames;
  T.sample_offset = fresh_batch ? sample_offset + d.frame_count : 0u;
  R.key_valid = false;  // the next RenderScene restarts its accumulation
  R.completion += d.frame_count;
  if (t.read_back && color_out) {
    if (!R.ok(cudaMemcpyAsync(color_out, R.color.ptr, sizeof(float4) * n, cudaMemcpyDeviceToHost, s), "colour", detail) ||
        !R.ok(cudaStreamSynchronize(s), "colour", detail))
      return poison(detail);
  }
  res.status = LOTUS_PASS;
  res.frames_rendered = d.frame_count;
  res.samples_per_pixel = d.frame_count;
  res.completion = R.completion;
  res.camera_rays = totals.camera;
  res.extension_rays = totals.extension;
  res.shadow_rays = totals.shadow;
  res.gpu_ms = ms;
  return LOTUS_PASS;
}

}  // namespace

extern "C" {

int32_t lotus_cuda_set_temporal_instances(lotus_cuda_renderer* r, const lotus_temporal_instance* instances,
    uint32_t count) {
  if (!r || (!instances && count)) return LOTUS_FAIL;
  Renderer& R = r->r;
  if (!R.failure.empty() || !R.scene_ready || count != R.view.instance_count) return LOTUS_FAIL;
  cudaSetDevice(R.device);
  std::vector<TemporalInstance> ids(std::max<uint32_t>(count, 1));
  for (uint32_t i = 0; i < count; ++i) {
    const float* m = instances[i].previous_world_from_object;
    for (int k = 0; k < 3; ++k) ids[i].previous[k] = make_float4(m[k], m[4 + k], m[8 + k], m[12 + k]);
    ids[i].instance_id = instances[i].instance_id;
    ids[i].material_id = instances[i].material_id;
    ids[i].flags = instances[i].flags;
  }
  std::string detail;
  if (!R.ok(R.temporal.instances.upload(ids.data(), ids.size(), R.stream), "temporal identities", detail) ||
      !R.ok(cudaStreamSynchronize(R.stream), "temporal identities", detail))
    return LOTUS_FAIL;
  R.temporal.instances_custom = true;
  return LOTUS_PASS;
}

int32_t lotus_cuda_render_temporal(lotus_cuda_renderer* r, const lotus_temporal_desc* temporal,
    lotus_frame_result* result, float* color) {
  lotus_frame_result local{};
  lotus_frame_result& res = result ? *result : local;
  std::memset(&res, 0, sizeof(res));
  if (!r || !temporal) {
    copy_detail(res.detail, sizeof(res.detail), "no renderer or temporal frame");
    return res.status = LOTUS_FAIL;
  }
  Renderer& R = r->r;
  if (!R.failure.empty()) {
    copy_detail(res.detail, sizeof(res.detail), "the renderer failed earlier: " + R.failure);
    return res.status = LOTUS_FAIL;
  }
  cudaSetDevice(R.device);
  return render_temporal(R, *temporal, res, color);
}

int64_t lotus_cuda_read_product(lotus_cuda_renderer* r, uint32_t product, void* out, uint64_t capacity) {
  if (!r || !out) return -1;
  Renderer& R = r->r;
  Renderer::Temporal& T = R.temporal;
  if (T.frames == 0) return -1;
  const size_t n = (size_t)T.width * T.height;
  const void* src = nullptr;
  size_t bytes = 0;
  const int sw = T.last_surface, rw = T.last_radiance, rs = T.last_restir;
  switch (product) {
    case LOTUS_PRODUCT_SURFACE: src = T.surface[sw].ptr; bytes = n * sizeof(TemporalPixel); break;
    case LOTUS_PRODUCT_PREVIOUS_SURFACE: src = T.surface[1 - sw].ptr; bytes = n * sizeof(TemporalPixel); break;
    case LOTUS_PRODUCT_VALIDITY: src = T.validity.ptr; bytes = n * sizeof(ValidityPixel); break;
    case LOTUS_PRODUCT_RADIANCE:
      if (T.accumulate_ran) { src = T.radiance[rw].ptr; bytes = n * sizeof(RadiancePixel); }
      break;
    case LOTUS_PRODUCT_PREVIOUS_RADIANCE:
      if (T.accumulate_ran) { src = T.radiance[1 - rw].ptr; bytes = n * sizeof(RadiancePixel); }
      break;
    case LOTUS_PRODUCT_BATCH:
      if (T.accumulate_ran) { src = T.batch.ptr; bytes = n * sizeof(float4); }
      break;
    case LOTUS_PRODUCT_RESTIR_INITIAL:
      if (T.restir_ran) { src = T.initial.ptr; bytes = n * sizeof(RestirPixel); }
      break;
    case LOTUS_PRODUCT_RESTIR_TEMPORAL:
      if (T.restir_ran) { src = T.reuse[rs].ptr; bytes = n * sizeof(RestirReuse); }
      break;
    case LOTUS_PRODUCT_RESTIR_PREVIOUS:
      if (T.restir_ran) { src = T.reuse[1 - rs].ptr; bytes = n * sizeof(RestirReuse); }
      break;
    case LOTUS_PRODUCT_RESTIR_SPATIAL:
      if (T.spatial_ran) { src = T.spatial.ptr; bytes = n * sizeof(RestirReuse); }
      break;
    case LOTUS_PRODUCT_RESTIR_SOURCES:
      if (T.spatial_ran) { src = T.sources.ptr; bytes = n * sizeof(uint4); }
      break;
    case LOTUS_PRODUCT_RESTIR_SURFACES:
      if (T.restir_ran) { src = T.surfaces[rs].ptr; bytes = n * sizeof(RestirSurface); }
      break;
    case LOTUS_PRODUCT_RESTIR_PREVIOUS_SURFACES:
      if (T.restir_ran) { src = T.surfaces[1 - rs].ptr; bytes = n * sizeof(RestirSurface); }
      break;
    case LOTUS_PRODUCT_FILTER:
      if (T.filter_ran) { src = T.filter.ptr; bytes = 3 * n * sizeof(float4); }
      break;
    default: break;
  }
  if (!src || bytes > capacity) return -1;
  cudaSetDevice(R.device);
  if (cudaMemcpy(out, src, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  if (T.moments_half && (product == LOTUS_PRODUCT_RADIANCE || product == LOTUS_PRODUCT_PREVIOUS_RADIANCE)) {
    // The FP16 moment mode stores the central second moment; the product
    // carries the raw one, as the passes reconstruct it.
    RadiancePixel* p = static_cast<RadiancePixel*>(out);
    for (size_t i = 0; i < n; ++i) p[i].second_moment = p[i].second_moment + p[i].first_moment * p[i].first_moment;
  }
  return (int64_t)bytes;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The learned radiance cache.

namespace {

Renderer* cache_renderer(lotus_cuda_renderer* h, bool need_cache) {
  if (!h || !h->r.failure.empty()) return nullptr;
  if (need_cache && !h->r.cache.ready()) return nullptr;
  cudaSetDevice(h->r.device);
  return &h->r;
}

}  // namespace

extern "C" int32_t lotus_cuda_configure_cache(lotus_cuda_renderer* h, const lotus_cache_desc* d, char* detail,
    size_t detail_size) {
  Renderer* R = cache_renderer(h, false);
  if (!R || !d) {
    copy_detail(detail, detail_size, !d ? "no cache description" : "the renderer has failed");
    return LOTUS_FAIL;
  }
  CacheConfig c;
  c.levels = d->levels ? d->levels : 16u;
  c.log2_size = d->log2_table ? d->log2_table : 19u;
  c.min_resolution = d->min_resolution ? d->min_resolution : 16u;
  c.max_resolution = d->max_resolution ? d->max_resolution : 2048u;
  c.learning_rate = d->learning_rate > 0.0f ? d->learning_rate : 1e-2f;
  c.seed = d->seed;
  if (c.levels > (uint32_t)kCacheMaxLevels || c.log2_size < 10 || c.log2_size > 22 || c.min_resolution < 2 ||
      c.max_resolution < c.min_resolution || !std::isfinite(c.learning_rate) || d->terminate_bounce > 16) {
    copy_detail(detail, detail_size, "cache settings out of range (levels 1..16, log2_table 10..22, "
        "2 <= min_resolution <= max_resolution, terminate_bounce 0..16)");
    return LOTUS_FAIL;
  }
  cudaError_t e = R->cache.configure(c, R->scene_lo, R->scene_hi, R->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(R->stream);
  if (e != cudaSuccess) {
    copy_detail(detail, detail_size, std::string("cache set-up: ") + cudaGetErrorString(e));
    R->cache.release();
    return LOTUS_FAIL;
  }
  R->cache_desc = *d;
  R->cache_enabled = d->enable != 0;
  R->cache_pixels = 0;
  ++R->cache_generation;
  R->key_valid = false;
  return LOTUS_PASS;
}

extern "C" int32_t lotus_cuda_cache_weights(lotus_cuda_renderer* h, float* weights, uint64_t count, int32_t write) {
  Renderer* R = cache_renderer(h, true);
  if (!R || !weights || count != kCacheWeights) return LOTUS_FAIL;
  const cudaError_t e = write ? R->cache.write_weights(weights, R->stream) : R->cache.read_weights(weights, R->stream);
  if (write) R->key_valid = false;
  return e == cudaSuccess ? LOTUS_PASS : LOTUS_FAIL;
}

extern "C" int32_t lotus_cuda_cache_infer(lotus_cuda_renderer* h, const float* inputs, uint32_t n, float* outputs) {
  Renderer* R = cache_renderer(h, true);
  if (!R || !inputs || !outputs) return LOTUS_FAIL;
  if (n == 0) return LOTUS_PASS;
  const cudaError_t e = R->cache.infer_encoded(inputs, n, outputs, R->stream);
  return e == cudaSuccess && R->cache.error_flag(R->stream) == 0 ? LOTUS_PASS : LOTUS_FAIL;
}

extern "C" int32_t lotus_cuda_cache_gradient(lotus_cuda_renderer* h, const float* inputs, const float* targets,
    uint32_t n, float* weight_grad, float* input_grad, float* loss) {
  Renderer* R = cache_renderer(h, true);
  if (!R || !inputs || !targets) return LOTUS_FAIL;
  if (n == 0) return LOTUS_PASS;
  const cudaError_t e = R->cache.gradient_encoded(inputs, targets, n, weight_grad, input_grad, loss, R->stream);
  return e == cudaSuccess && R->cache.error_flag(R->stream) == 0 ? LOTUS_PASS : LOTUS_FAIL;
}

extern "C" int32_t lotus_cuda_cache_encode(lotus_cuda_renderer* h, const float* records, uint32_t n, float* inputs) {
  Renderer* R = cache_renderer(h, true);
  if (!R || !records || !inputs) return LOTUS_FAIL;
  if (n == 0) return LOTUS_PASS;
  const cudaError_t e =
      R->cache.encode(reinterpret_cast<const CacheRecord*>(records), n, inputs, R->stream);
  return e == cudaSuccess ? LOTUS_PASS : LOTUS_FAIL;
}

extern "C" int32_t lotus_cuda_cache_train(lotus_cuda_renderer* h, const float* records, const float* targets,
    uint32_t n, uint32_t steps, float* losses) {
  Renderer* R = cache_renderer(h, true);
  if (!R || !records || !targets) return LOTUS_FAIL;
  if (n == 0 || steps == 0) return LOTUS_PASS;
  const cudaError_t e = R->cache.train_records(reinterpret_cast<const CacheRecord*>(records), targets, n, steps,
      losses, R->stream);
  R->key_valid = false;
  return e == cudaSuccess && R->cache.error_flag(R->stream) == 0 ? LOTUS_PASS : LOTUS_FAIL;
}
