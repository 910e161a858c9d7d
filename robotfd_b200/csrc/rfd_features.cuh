// Bracket features of one pair, computed by one CTA (blockDim.x = kFeatThreads).
//
// Each curve is resampled at 64 positions uniform in arc length (position k at k/63 of the
// length, linear interpolation inside the segment that contains it), both resampled curves
// are centred on their joint mean and scaled by their largest distance from it, and
// log(endpoint / scale), log(VE-FD / scale) are appended.  2D curves get z = 0.
#pragma once

#include "rfd_mlp.h"

namespace rfd {

constexpr int kFeatThreads = 256;

struct FeatScratch {
  double part[kFeatThreads];
  double total;
  float pts[2 * rfd_mlp::kPoints][3];
};

__device__ __forceinline__ double seg_len(const double* X, int sgi, int d) {
  double l2 = 0.0;
  for (int k = 0; k < d; ++k) {
    const double df = X[(size_t)(sgi + 1) * d + k] - X[(size_t)sgi * d + k];
    l2 += df * df;
  }
  return sqrt(l2);
}

// Resample curve X (n points, d dims) into sh.pts[base .. base+63].  Thread t owns the
// segments [s0, s1) and the targets k with prefix[t] <= k L / 63 < prefix[t+1], so every
// target is written exactly once.
__device__ void resample64(const double* X, int n, int d, FeatScratch& sh, int base) {
  const int T = blockDim.x, t = threadIdx.x;
  const int nseg = n - 1;
  const int per = (nseg + T - 1) / T;
  const int s0 = min(t * per, nseg), s1 = min(s0 + per, nseg);
  double mine = 0.0;
  for (int sgi = s0; sgi < s1; ++sgi) mine += seg_len(X, sgi, d);
  sh.part[t] = mine;
  __syncthreads();
  if (t == 0) {
    double run = 0.0;
    for (int k = 0; k < T; ++k) {
      const double v = sh.part[k];
      sh.part[k] = run;
      run += v;
    }
    sh.total = run;
  }
  __syncthreads();
  const double L = sh.total;
  const double lo = sh.part[t];
  const double hi = t + 1 < T ? sh.part[t + 1] : L;
  if (L > 0.0 && s0 < s1) {
    int kk = max(1, (int)ceil(lo * 63.0 / L) - 1);
    double cum = lo;
    for (int sgi = s0; sgi < s1 && kk <= 62; ++sgi) {
      const double len = seg_len(X, sgi, d);
      while (kk <= 62) {
        const double target = kk * L / 63.0;
        if (target >= hi) { kk = 63; break; }
        if (target < lo) { ++kk; continue; }
        if (target >= cum + len && sgi + 1 < s1) break;
        double u = len > 0.0 ? (target - cum) / len : 0.0;
        u = fmin(1.0, fmax(0.0, u));
        for (int k = 0; k < 3; ++k) {
          const double a = k < d ? X[(size_t)sgi * d + k] : 0.0;
          const double b = k < d ? X[(size_t)(sgi + 1) * d + k] : 0.0;
          sh.pts[base + kk][k] = (float)(a + u * (b - a));
        }
        ++kk;
      }
      cum += len;
    }
  }
  __syncthreads();
  if (t == 0) {
    for (int k = 0; k < 3; ++k) {
      sh.pts[base][k] = k < d ? (float)X[k] : 0.f;
      sh.pts[base + 63][k] = k < d ? (float)X[(size_t)(n - 1) * d + k] : 0.f;
    }
    if (!(L > 0.0))
      for (int p = 1; p < 63; ++p)
        for (int k = 0; k < 3; ++k) sh.pts[base + p][k] = sh.pts[base][k];
  }
  __syncthreads();
}

// Writes kInputWidth floats to out (features then zero padding).
__device__ void pair_features(const double* P, int n1, const double* Q, int n2, int d,
                              double endpoint, double vefd, FeatScratch& sh, float* out) {
  const int t = threadIdx.x;
  resample64(P, n1, d, sh, 0);
  resample64(Q, n2, d, sh, rfd_mlp::kPoints);
  __shared__ float cen[3];
  __shared__ float scale;
  if (t == 0) {
    double c[3] = {0, 0, 0};
    for (int p = 0; p < 2 * rfd_mlp::kPoints; ++p)
      for (int k = 0; k < 3; ++k) c[k] += sh.pts[p][k];
    for (int k = 0; k < 3; ++k) cen[k] = (float)(c[k] / (2 * rfd_mlp::kPoints));
    double r = 0.0;
    for (int p = 0; p < 2 * rfd_mlp::kPoints; ++p) {
      double q = 0.0;
      for (int k = 0; k < 3; ++k) {
        const double dd = sh.pts[p][k] - cen[k];
        q += dd * dd;
      }
      r = fmax(r, q);
    }
    scale = (float)fmax(sqrt(r), 1e-30);
  }
  __syncthreads();
  for (int f = t; f < rfd_mlp::kInputWidth; f += blockDim.x) {
    float v = 0.f;
    if (f < 2 * rfd_mlp::kPoints * 3) {
      const int p = f / 3, k = f % 3;
      v = (sh.pts[p][k] - cen[k]) / scale;
    } else if (f == 2 * rfd_mlp::kPoints * 3) {
      v = (float)fmax(-30.0, fmin(5.0, log(fmax(endpoint, 1e-300) / scale)));
    } else if (f == 2 * rfd_mlp::kPoints * 3 + 1) {
      v = (float)fmax(-30.0, fmin(5.0, log(fmax(vefd, 1e-300) / scale)));
    }
    out[f] = v;
  }
  __syncthreads();
}

}  // namespace rfd
