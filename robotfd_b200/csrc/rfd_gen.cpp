// Seeded synthetic trajectory generators for the benchmark workloads.
//
// The reference repository ships no data (its CLI example names OSM files that
// are not part of it, src/main.cpp:19), so every workload is generated here from
// a counter-based SplitMix64 stream with Box-Muller normals:
//   style 0 ("walk")   : P is a Gaussian random walk (step sigma), Q resamples P
//                        at uniform arc-length positions and adds N(0, noise^2).
//   style 1 ("spline") : P samples a uniform Catmull-Rom spline through random
//                        waypoints U[-scale, scale]^d; Q samples the same spline
//                        under a random monotone piecewise-linear time warp
//                        (20 interior knots) and adds N(0, noise^2).
// Every generated curve passes through the loader's rule that drops a point
// equal to its predecessor (include/txtReader.hpp:37 and :79 of the reference),
// so a curve never holds a zero-length segment.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#include "rfd.h"

namespace {

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed, uint64_t stream) {
    s = seed * 0x9E3779B97F4A7C15ULL + (stream + 1) * 0xD1B54A32D192ED03ULL;
    next();
  }
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  // uniform in [0, 1)
  double uni() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  // uniform in (0, 1]
  double uni_open() { return ((double)(next() >> 11) + 1.0) * (1.0 / 9007199254740992.0); }
  double normal() {
    double u1 = uni_open(), u2 = uni();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

// Drop every point equal (in all d coordinates) to the previously kept point.
int64_t dedupe(double* pts, int64_t n, int d) {
  if (n <= 1) return n;
  int64_t w = 1;
  for (int64_t r = 1; r < n; ++r) {
    bool same = true;
    for (int k = 0; k < d; ++k) same = same && (pts[r * d + k] == pts[(w - 1) * d + k]);
    if (!same) {
      if (w != r) std::memmove(pts + w * d, pts + r * d, sizeof(double) * d);
      ++w;
    }
  }
  return w;
}

void walk(Rng& g, double* out, int64_t n, int d, double sigma) {
  for (int k = 0; k < d; ++k) out[k] = 0.0;
  for (int64_t i = 1; i < n; ++i)
    for (int k = 0; k < d; ++k) out[i * d + k] = out[(i - 1) * d + k] + sigma * g.normal();
}

// m points at uniform arc-length positions of polyline P (n points), plus noise.
void resample(Rng& g, const double* P, int64_t n, int d, double* out, int64_t m, double noise) {
  std::vector<double> cum(n, 0.0);
  for (int64_t i = 1; i < n; ++i) {
    double s = 0.0;
    for (int k = 0; k < d; ++k) {
      double t = P[i * d + k] - P[(i - 1) * d + k];
      s += t * t;
    }
    cum[i] = cum[i - 1] + std::sqrt(s);
  }
  const double L = cum[n - 1];
  int64_t seg = 0;
  for (int64_t q = 0; q < m; ++q) {
    double target = (m > 1) ? L * (double)q / (double)(m - 1) : 0.0;
    while (seg < n - 2 && cum[seg + 1] < target) ++seg;
    double len = (n > 1) ? cum[seg + 1] - cum[seg] : 0.0;
    double u = (len > 0.0) ? (target - cum[seg]) / len : 0.0;
    u = std::min(1.0, std::max(0.0, u));
    int64_t s1 = std::min<int64_t>(seg + 1, n - 1);
    for (int k = 0; k < d; ++k)
      out[q * d + k] = P[seg * d + k] + u * (P[s1 * d + k] - P[seg * d + k]) + noise * g.normal();
  }
}

// Uniform Catmull-Rom spline through W waypoints, evaluated at global parameter U in [0, W-1].
void spline_eval(const double* w, int64_t W, int d, double U, double* out) {
  int64_t k = (int64_t)std::floor(U);
  if (k > W - 2) k = W - 2;
  if (k < 0) k = 0;
  double u = U - (double)k;
  int64_t i0 = std::max<int64_t>(k - 1, 0), i1 = k, i2 = k + 1, i3 = std::min<int64_t>(k + 2, W - 1);
  double u2 = u * u, u3 = u2 * u;
  for (int c = 0; c < d; ++c) {
    double p0 = w[i0 * d + c], p1 = w[i1 * d + c], p2 = w[i2 * d + c], p3 = w[i3 * d + c];
    out[c] = 0.5 * ((2.0 * p1) + (-p0 + p2) * u + (2.0 * p0 - 5.0 * p1 + 4.0 * p2 - p3) * u2 +
                    (-p0 + 3.0 * p1 - 3.0 * p2 + p3) * u3);
  }
}

}  // namespace

extern "C" {

int rfd_gen_pair(int style, int dims, int64_t n1, int64_t n2, double scale, double noise,
                 uint64_t seed, uint64_t stream, double* P, int64_t* out_n1, double* Q,
                 int64_t* out_n2) {
  if ((dims != 2 && dims != 3) || n1 < 2 || n2 < 2 || !P || !Q || !out_n1 || !out_n2)
    return RFD_ERR_ARG;
  Rng g(seed, stream);
  if (style == 0) {
    // walk of n1 points with step sigma = scale; Q = n2 arc-length resamples + noise
    walk(g, P, n1, dims, scale);
    resample(g, P, n1, dims, Q, n2, noise);
  } else if (style == 1) {
    int64_t W = std::max<int64_t>(4, (std::max(n1, n2) + 50) / 100);
    std::vector<double> way(W * dims);
    for (auto& v : way) v = scale * (2.0 * g.uni() - 1.0);
    for (int64_t m = 0; m < n1; ++m)
      spline_eval(way.data(), W, dims, (double)(W - 1) * (double)m / (double)(n1 - 1), P + m * dims);
    // monotone piecewise-linear warp with 20 interior knots at x = k/21
    const int K = 20;
    double ky[K + 2];
    ky[0] = 0.0;
    ky[K + 1] = 1.0;
    for (int k = 1; k <= K; ++k) ky[k] = g.uni();
    std::sort(ky + 1, ky + K + 1);
    for (int64_t m = 0; m < n2; ++m) {
      double x = (double)m / (double)(n2 - 1);
      double xs = x * (K + 1);
      int seg = (int)std::floor(xs);
      if (seg > K) seg = K;
      double f = xs - seg;
      double y = ky[seg] + f * (ky[seg + 1] - ky[seg]);
      spline_eval(way.data(), W, dims, (double)(W - 1) * y, Q + m * dims);
      for (int c = 0; c < dims; ++c) Q[m * dims + c] += noise * g.normal();
    }
  } else {
    return RFD_ERR_ARG;
  }
  *out_n1 = dedupe(P, n1, dims);
  *out_n2 = dedupe(Q, n2, dims);
  return RFD_OK;
}

int rfd_gen_batch_spec(int config, int64_t npairs, uint64_t seed, int* dims, int64_t* n1s,
                       int64_t* n2s, int* styles, double* scales, double* noises) {
  if (npairs < 0 || !dims || !n1s || !n2s || !styles || !scales || !noises) return RFD_ERR_ARG;
  for (int64_t k = 0; k < npairs; ++k) {
    Rng g(seed, 0x5EC0000000ULL + (uint64_t)k);
    if (config == 2 || config == 3) {
      // uneven batch: dim 50/50, lengths lognormal(ln 2000, 1) clipped to [100, 50000],
      // style 50/50 (walk: step 1, noise 0.05; spline: waypoints U[-100,100]^d, noise 0.1)
      dims[k] = (g.uni() < 0.5) ? 2 : 3;
      double a = std::exp(std::log(2000.0) + g.normal());
      double b = std::exp(std::log(2000.0) + g.normal());
      n1s[k] = (int64_t)std::llround(std::min(50000.0, std::max(100.0, a)));
      n2s[k] = (int64_t)std::llround(std::min(50000.0, std::max(100.0, b)));
      styles[k] = (g.uni() < 0.5) ? 0 : 1;
      scales[k] = styles[k] == 0 ? 1.0 : 100.0;
      noises[k] = styles[k] == 0 ? 0.05 : 0.1;
    } else if (config == 4) {
      // large 3D pairs, lengths U[100000, 400000], spline style with waypoints U[-1e4,1e4]^3
      dims[k] = 3;
      n1s[k] = 100000 + (int64_t)(g.uni() * 300001.0);
      n2s[k] = 100000 + (int64_t)(g.uni() * 300001.0);
      if (n1s[k] > 400000) n1s[k] = 400000;
      if (n2s[k] > 400000) n2s[k] = 400000;
      styles[k] = 1;
      scales[k] = 1.0e4;
      noises[k] = 0.1;
    } else if (config == 0) {
      dims[k] = 2; n1s[k] = 2000; n2s[k] = 1900; styles[k] = 0; scales[k] = 1.0; noises[k] = 0.05;
    } else if (config == 1) {
      dims[k] = 3; n1s[k] = 200000; n2s[k] = 200000; styles[k] = 1; scales[k] = 100.0; noises[k] = 0.1;
    } else {
      return RFD_ERR_ARG;
    }
  }
  return RFD_OK;
}

}  // extern "C"
