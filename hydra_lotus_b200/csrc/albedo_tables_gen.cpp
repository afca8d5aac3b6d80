// SPDX-License-Identifier: Apache-2.0
// albedo_tables_gen: writes albedo_tables.inc, the directional albedo
// tables albedo.cuh reads (the grid of albedo.slang in hydra-lotus; the
// tables that generator, validation/bsdf-tables.cpp, writes are its
// counterpart). Every node holds the single-scattering albedo of one
// uncompensated, untinted, reflecting lobe at the node's outgoing cosine,
// alpha (or sheen roughness) and relative index:
//
//   E(wo) = integral over [0, 1)^2 of weight(wo, u) du,
//
// weight = f cos(theta_i) / pdf of the lobe's own sampler at u, which is
// the albedo by a change of variables: the sampler flattens the lobe's
// peak, so the integrand is smooth except where the sampled direction
// crosses the horizon. The integral is taken by adaptive cubature: a
// tensor 5-point Gauss-Legendre rule on a panel is compared with the sum
// over its four quarters, and a panel is split until the two agree within
// the tolerance times its area (at least one split, at most eight). The
// lobes are evaluated in double precision.
//
// Usage: albedo_tables_gen <out.inc> [tolerance]
//        albedo_tables_gen --check <in.inc> <stride> [tolerance]
// --check compares every stride-th node with a fresh cubature, and the
// spline (albedo.cuh's lookups) at every stride-th cell centre with a
// cubature there, and prints the largest error of each part.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

#include "albedo.cuh"

namespace {

using lotus::albedo::kAlphas;
using lotus::albedo::kDielectric;
using lotus::albedo::kGgx;
using lotus::albedo::kIndices;
using lotus::albedo::kSchlickShare;
using lotus::albedo::kSheen;
using lotus::albedo::kTables;

constexpr double kPi = 3.14159265358979323846;
constexpr double kDefaultTolerance = 1.0e-5;

struct D3 {
  double x, y, z;
};
D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
D3 normalized(D3 a) { return a * (1.0 / std::sqrt(dot(a, a))); }

// --- The grid's parameters (the inverses of albedo.cuh's coordinates) ------

double log_linear(double v, double slope) { return std::log(v) + slope * v; }

// The value in [low, high] whose normalized log-linear coordinate is x:
// bisection on the increasing scale.
double log_linear_at(double x, double low, double high, double slope) {
  const double target = log_linear(low, slope) +
      std::min(std::max(x, 0.0), 1.0) * (log_linear(high, slope) - log_linear(low, slope));
  double lo = low, hi = high;
  for (int i = 0; i < 200; ++i) {
    const double mid = 0.5 * (lo + hi);
    (log_linear(mid, slope) < target ? lo : hi) = mid;
  }
  return 0.5 * (lo + hi);
}

double cosine_at(double x) {
  return log_linear_at(x, lotus::albedo::kMinCosine, 1.0, lotus::albedo::kCosineSlope);
}
double alpha_at(double x) {
  return log_linear_at(x, lotus::albedo::kMinAlphaAxis, 1.0, lotus::albedo::kAlphaSlope);
}
double sheen_at(double x) {
  return log_linear_at(x, lotus::albedo::kMinSheenAxis, 1.0, lotus::albedo::kAlphaSlope);
}
double index_at(double x) {
  return 1.0 + log_linear_at(x, lotus::albedo::kMinIndex - 1.0, lotus::albedo::kMaxIndex - 1.0,
      lotus::albedo::kIndexSlope);
}

double evanescent_scale(double mu, double index, double critical) {
  const double tau = std::max(index * std::sqrt(std::max(critical * critical - mu * mu, 0.0)),
      double(lotus::albedo::kMinEvanescent));
  return std::log(mu) - std::log(tau) + lotus::albedo::kCosineSlope * mu;
}

// The leaving sheet's outgoing cosine at coordinate x.
double leaving_at(double x, double index) {
  const double split = double(lotus::albedo::kCriticalNode) / double(lotus::albedo::kDielectricCosines - 1);
  const double critical = std::sqrt(std::max(1.0 - 1.0 / (index * index), 0.0));
  if (x <= split) {
    const double low = evanescent_scale(lotus::albedo::kMinCosine, index, critical);
    const double high = evanescent_scale(critical, index, critical);
    const double target = low + (x / split) * (high - low);
    double lo = lotus::albedo::kMinCosine, hi = critical;
    for (int i = 0; i < 200; ++i) {
      const double mid = 0.5 * (lo + hi);
      (evanescent_scale(mid, index, critical) < target ? lo : hi) = mid;
    }
    return 0.5 * (lo + hi);
  }
  const double refracted = cosine_at((x - split) / (1.0 - split));
  return std::sqrt(1.0 - (1.0 - refracted * refracted) / (index * index));
}

// What a table point integrates: the lobe, its outgoing cosine, its alpha
// (or sheen roughness) and its relative index from the outgoing side.
struct Point {
  uint32_t table;
  double cos_theta;
  double alpha;
  double eta;
  bool thin;
};

// The point at grid coordinates in [0, 1] (the dielectric's sheet apart).
Point point_at(uint32_t table, double x_cos, double x_alpha, uint32_t sheet, double x_index) {
  Point p{table, 0.0, 0.0, 1.0, false};
  if (table == kSheen) {
    p.cos_theta = cosine_at(x_cos);
    p.alpha = sheen_at(x_alpha);
    return p;
  }
  p.alpha = alpha_at(x_alpha);
  if (table != kDielectric) {
    p.cos_theta = cosine_at(x_cos);
    return p;
  }
  const double index = index_at(x_index);
  if (sheet == lotus::albedo::kLeaving) {
    p.cos_theta = leaving_at(x_cos, index);
    p.eta = 1.0 / index;
  } else {
    p.cos_theta = cosine_at(x_cos);
    p.eta = index;
    p.thin = sheet == lotus::albedo::kThin;
  }
  return p;
}

// --- The lobes' sample weights ----------------------------------------------

double ggx_lambda(D3 w, double alpha) {
  const double tan2 = std::max(0.0, 1.0 - w.z * w.z) / (w.z * w.z);
  return 0.5 * (std::sqrt(1.0 + alpha * alpha * tan2) - 1.0);
}

// Visible normals by spherical caps (Dupuy and Benyoub 2023), as the lobes
// sample them.
D3 sample_visible_normal(D3 wo, double alpha, double ux, double uy) {
  const D3 wo_std = normalized({wo.x * alpha, wo.y * alpha, wo.z});
  const double phi = 2.0 * kPi * ux;
  const double z = (1.0 - uy) * (1.0 + wo_std.z) - wo_std.z;
  const double sin_theta = std::sqrt(std::min(std::max(1.0 - z * z, 0.0), 1.0));
  const D3 h_std = D3{sin_theta * std::cos(phi), sin_theta * std::sin(phi), z} + wo_std;
  return normalized({h_std.x * alpha, h_std.y * alpha, h_std.z});
}

double fresnel_dielectric(double c, double eta) {
  c = std::min(std::max(c, 0.0), 1.0);
  const double sin2_t = (1.0 - c * c) / (eta * eta);
  if (sin2_t >= 1.0) return 1.0;
  const double cos_t = std::sqrt(1.0 - sin2_t);
  const double parallel = (eta * c - cos_t) / (eta * c + cos_t);
  const double perpendicular = (c - eta * cos_t) / (c + eta * cos_t);
  return 0.5 * (parallel * parallel + perpendicular * perpendicular);
}

// f cos(theta_i) / pdf for the sampler's numbers (ux, uy); 0 where the
// sampler yields no reflected direction.
double sample_weight(const Point& p, D3 wo, double ux, double uy) {
  if (p.table == kSheen) {
    // Uniform hemisphere sampling, pdf 1 / (2 pi).
    const double sin_theta = std::sqrt(std::max(1.0 - ux * ux, 0.0));
    const double phi = 2.0 * kPi * uy;
    const D3 wi{sin_theta * std::cos(phi), sin_theta * std::sin(phi), ux};
    if (!(wi.z > 0.0)) return 0.0;
    const D3 h = normalized(wo + wi);
    const double inverse = 1.0 / p.alpha;
    const double sin2 = std::max(1.0 - h.z * h.z, 0.0);
    const double d = (2.0 + inverse) * std::pow(sin2, 0.5 * inverse) / (2.0 * kPi);
    return 2.0 * kPi * d * wi.z / (4.0 * (wi.z + wo.z - wi.z * wo.z));
  }
  const D3 h = sample_visible_normal(wo, p.alpha, ux, uy);
  const double cos_oh = dot(wo, h);
  if (!(cos_oh > 0.0)) return 0.0;
  const D3 wi = h * (2.0 * cos_oh) + wo * -1.0;
  if (!(wi.z > 0.0)) return 0.0;
  // G2 / G1 of the height-correlated Smith term.
  const double lambda_o = ggx_lambda(wo, p.alpha);
  const double ratio = (1.0 + lambda_o) / (1.0 + lambda_o + ggx_lambda(wi, p.alpha));
  double fresnel = 1.0;
  if (p.table == kSchlickShare) {
    fresnel = std::pow(std::min(std::max(1.0 - cos_oh, 0.0), 1.0), 5.0);
  } else if (p.table == kDielectric) {
    const double r = fresnel_dielectric(cos_oh, p.eta);
    fresnel = p.thin ? 2.0 * r / (1.0 + r) : r;
  }
  return fresnel * ratio;
}

// --- Adaptive cubature ---------------------------------------------------------

constexpr double kGaussNodes[5] = {-0.9061798459386640, -0.5384693101056831, 0.0,
    0.5384693101056831, 0.9061798459386640};
constexpr double kGaussWeights[5] = {0.2369268850561891, 0.4786286704993665, 0.5688888888888889,
    0.4786286704993665, 0.2369268850561891};

struct Cubature {
  Point p;
  D3 wo;
  double tolerance;

  double rule(double x0, double x1, double y0, double y1) const {
    const double cx = 0.5 * (x0 + x1), hx = 0.5 * (x1 - x0);
    const double cy = 0.5 * (y0 + y1), hy = 0.5 * (y1 - y0);
    double sum = 0.0;
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j)
        sum += kGaussWeights[i] * kGaussWeights[j] *
            sample_weight(p, wo, cx + hx * kGaussNodes[i], cy + hy * kGaussNodes[j]);
    return sum * hx * hy;
  }

  double refine(double x0, double x1, double y0, double y1, double whole, int depth) const {
    const double xm = 0.5 * (x0 + x1), ym = 0.5 * (y0 + y1);
    const double q[4] = {rule(x0, xm, y0, ym), rule(xm, x1, y0, ym), rule(x0, xm, ym, y1),
        rule(xm, x1, ym, y1)};
    const double parts = q[0] + q[1] + q[2] + q[3];
    if (depth >= 8 || (depth >= 1 && std::fabs(parts - whole) <= tolerance * (x1 - x0) * (y1 - y0)))
      return parts;
    return refine(x0, xm, y0, ym, q[0], depth + 1) + refine(xm, x1, y0, ym, q[1], depth + 1) +
        refine(x0, xm, ym, y1, q[2], depth + 1) + refine(xm, x1, ym, y1, q[3], depth + 1);
  }

  double integrate() const {
    constexpr int kPanels = 4;
    const double h = 1.0 / kPanels;
    double sum = 0.0;
    for (int i = 0; i < kPanels; ++i)
      for (int j = 0; j < kPanels; ++j) {
        const double x0 = i * h, y0 = j * h;
        sum += refine(x0, x0 + h, y0, y0 + h, rule(x0, x0 + h, y0, y0 + h), 0);
      }
    return sum;
  }
};

double albedo_at(const Point& p, double tolerance) {
  const double c = p.cos_theta;
  Cubature q{p, {std::sqrt(std::max(0.0, 1.0 - c * c)), 0.0, c}, tolerance};
  return q.integrate();
}

// --- The grid ------------------------------------------------------------------

struct Node {
  uint32_t index;  // into the data
  uint32_t table, sheet, c, a, k;
};

std::vector<Node> all_nodes() {
  std::vector<Node> nodes;
  for (uint32_t table = 0; table < kTables; ++table) {
    const uint32_t n_cos = lotus::albedo::cosines(table);
    const uint32_t layers = table == kDielectric ? lotus::albedo::kSheets * kIndices : 1;
    for (uint32_t layer = 0; layer < layers; ++layer)
      for (uint32_t a = 0; a < kAlphas; ++a)
        for (uint32_t c = 0; c < n_cos; ++c) {
          const uint32_t index = lotus::albedo::offset(table) + (layer * kAlphas + a) * n_cos + c;
          nodes.push_back({index, table, layer / kIndices, c, a, layer % kIndices});
        }
  }
  return nodes;
}

// The node's point, or with `centre` the point halfway to the next node
// along every axis.
Point node_point(const Node& n, bool centre) {
  const double half = centre ? 0.5 : 0.0;
  const uint32_t n_cos = lotus::albedo::cosines(n.table);
  return point_at(n.table, (n.c + half) / double(n_cos - 1), (n.a + half) / double(kAlphas - 1),
      n.sheet, (n.k + half) / double(kIndices - 1));
}

template <class F>
void parallel_for(size_t count, F&& f) {
  std::atomic<size_t> next{0};
  const unsigned threads = std::max(1u, std::thread::hardware_concurrency());
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < threads; ++t)
    pool.emplace_back([&] {
      for (size_t i; (i = next.fetch_add(1)) < count;) f(i);
    });
  for (std::thread& t : pool) t.join();
}

int write_tables(const char* path, double tolerance) {
  const std::vector<Node> nodes = all_nodes();
  std::vector<float> data(lotus::albedo::kSize, 0.0f);
  parallel_for(nodes.size(), [&](size_t i) {
    data[nodes[i].index] = float(albedo_at(node_point(nodes[i], false), tolerance));
  });
  std::FILE* f = std::fopen(path, "w");
  if (!f) {
    std::fprintf(stderr, "cannot write %s\n", path);
    return 1;
  }
  std::fprintf(f,
      "// SPDX-License-Identifier: Apache-2.0\n"
      "// Generated by albedo_tables_gen.cpp: the directional albedo tables albedo.cuh\n"
      "// reads, %u floats, adaptive cubature tolerance %g. Regenerate it with the\n"
      "// change that moves a lobe or an axis.\n",
      lotus::albedo::kSize, tolerance);
  for (uint32_t table = 0; table < kTables; ++table) {
    const uint32_t n_cos = lotus::albedo::cosines(table);
    std::fprintf(f, "// table %u at %u\n", table, lotus::albedo::offset(table));
    for (uint32_t i = lotus::albedo::offset(table); i < lotus::albedo::offset(table + 1); ++i)
      std::fprintf(f, "%.8g,%s", data[i], (i - lotus::albedo::offset(table)) % n_cos == n_cos - 1 ? "\n" : "");
  }
  std::fclose(f);
  return 0;
}

std::vector<float> read_tables(const char* path) {
  std::vector<float> data;
  std::FILE* f = std::fopen(path, "r");
  if (!f) return data;
  std::string text;
  char buffer[65536];
  for (size_t n; (n = std::fread(buffer, 1, sizeof buffer, f)) > 0;) text.append(buffer, n);
  std::fclose(f);
  size_t at = 0;
  while (at < text.size()) {
    const size_t end = text.find('\n', at);
    const std::string line = text.substr(at, end == std::string::npos ? std::string::npos : end - at);
    at = end == std::string::npos ? text.size() : end + 1;
    if (line.rfind("//", 0) == 0) continue;
    const char* s = line.c_str();
    while (*s) {
      char* stop = nullptr;
      const float v = std::strtof(s, &stop);
      if (stop == s) break;
      data.push_back(v);
      s = stop;
      while (*s == ',' || *s == ' ') ++s;
    }
  }
  return data;
}

float lookup(const std::vector<float>& data, const Point& p) {
  const float c = float(p.cos_theta), a = float(p.alpha);
  switch (p.table) {
    case kGgx: return lotus::albedo::ggx(data.data(), c, a);
    case kSchlickShare: return lotus::albedo::schlick_share(data.data(), c, a);
    case kSheen: return lotus::albedo::sheen(data.data(), c, a);
    default: return lotus::albedo::dielectric(data.data(), c, a, float(p.eta), p.thin);
  }
}

int check_tables(const char* path, uint32_t stride, double tolerance) {
  const std::vector<float> data = read_tables(path);
  if (data.size() != lotus::albedo::kSize) {
    std::fprintf(stderr, "%s holds %zu floats, not %u\n", path, data.size(), lotus::albedo::kSize);
    return 1;
  }
  const std::vector<Node> nodes = all_nodes();
  // Parts: E1, Eschlick, dielectric entering, leaving, thin, sheen.
  std::vector<double> node_error(6, 0.0), centre_error(6, 0.0);
  std::vector<std::atomic<long long>> counts(6);
  std::vector<size_t> picked;
  for (size_t i = 0; i < nodes.size(); i += stride) picked.push_back(i);
  std::vector<double> errs(picked.size() * 2, 0.0);
  parallel_for(picked.size(), [&](size_t j) {
    const Node& n = nodes[picked[j]];
    // Relative error where the albedo exceeds 1 (the sheen's, toward
    // grazing directions).
    const double fresh = albedo_at(node_point(n, false), tolerance);
    errs[2 * j] = std::fabs(double(data[n.index]) - fresh) / std::max(1.0, std::fabs(fresh));
    const bool inside = n.c + 1 < lotus::albedo::cosines(n.table) && n.a + 1 < kAlphas &&
        (n.table != kDielectric || n.k + 1 < kIndices);
    if (inside) {
      const Point p = node_point(n, true);
      const double centre = albedo_at(p, tolerance);
      errs[2 * j + 1] = std::fabs(double(lookup(data, p)) - centre) / std::max(1.0, std::fabs(centre));
    }
  });
  for (size_t j = 0; j < picked.size(); ++j) {
    const Node& n = nodes[picked[j]];
    const int part = n.table == kSheen ? 5 : (n.table == kDielectric ? 2 + int(n.sheet) : int(n.table));
    node_error[part] = std::max(node_error[part], errs[2 * j]);
    centre_error[part] = std::max(centre_error[part], errs[2 * j + 1]);
    counts[part]++;
  }
  const char* names[6] = {"E1", "Eschlick", "Edielectric entering", "Edielectric leaving",
      "Edielectric thin", "Esheen"};
  for (int part = 0; part < 6; ++part)
    std::printf("%s: points %lld node error %.3g centre error %.3g\n", names[part],
        (long long)counts[part], node_error[part], centre_error[part]);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc >= 4 && std::string(argv[1]) == "--check")
    return check_tables(argv[2], uint32_t(std::max(1, std::atoi(argv[3]))),
        argc >= 5 ? std::atof(argv[4]) : kDefaultTolerance);
  if (argc < 2 || argc > 3) {
    std::fprintf(stderr, "usage: albedo_tables_gen <out.inc> [tolerance]\n"
                         "       albedo_tables_gen --check <in.inc> <stride> [tolerance]\n");
    return 2;
  }
  return write_tables(argv[1], argc == 3 ? std::atof(argv[2]) : kDefaultTolerance);
}
