// Dense discrete Frechet strips (the DFD upper bound, reference
// src/intersection_algorithm_in_parallel.cu:435-641, cell recurrence :608-637).
//
// The DFD is a dense min-max DP with a cheap cell (one squared point distance), so its
// sweep is bound by instruction issue and by the step-to-step latency of the skewed
// wavefront, not by the geometry.  Compared with the generic strip (rfd_device.cuh):
//   - a lane owns K consecutive rows, so a strip is 32*K rows high: per step a lane
//     computes K cells in row order (each one's "from below" input is the previous row's
//     carry of the same step), one shuffle brings the row below the lane's first row, and
//     the strip-to-strip handoff (and its lag of two 32-column chunks) is paid once per
//     32*K rows instead of once per 32;
//   - the points of curve 2 a chunk of 32 steps needs are staged in a per-warp ring of 64
//     columns in shared memory (structure of arrays, conflict-free), loaded into registers
//     one chunk ahead, so no global load sits in a step;
//   - there is no dead-region logic (the DFD is computed unpruned).
// Boundary conditions of the reference (:614-626) are folded into the inputs: strip 0
// reads the row above it as 0 at column 0 and FLT_MAX elsewhere, and every row reads
// FLT_MAX to the left of column 0.  The operations of every cell, and their order, are
// those of cell<K_DFD> in rfd_device.cuh, so results are bit-identical.
#pragma once

#include "rfd_device.cuh"

namespace rfd {

constexpr int kDfdRing = 64;  // columns held per warp (two chunks)

// Returns 0, or 1 on error / timeout (the error word is set).
template <int D, int K>
__device__ int dfd_strip(const WaveArgs& wa, const PairDesc& pd, PairState* st, const int s,
                         double* ring /* [3][kDfdRing] per warp */) {
  const int lane = threadIdx.x & 31;
  const int R = pd.n1, C = pd.n2;
  constexpr int H = 32 * K;
  const int S = (R + H - 1) / H;
  const unsigned E = st->epoch;
  const bool has_prod = s > 0;
  const bool has_cons = s + 1 < S;
  Prog* in_prog = has_prod ? pd.prog + (s - 1) : nullptr;
  Prog* out_prog = has_cons ? pd.prog + s : nullptr;
  const double* in_bnd = has_prod ? pd.bnd + (size_t)(s - 1) * pd.cstride : nullptr;
  double* out_bnd = has_cons ? pd.bnd + (size_t)s * pd.cstride : nullptr;

  Waiter wt;
  wt.start(wa, st, s);

  // rows of this lane (clamped loads beyond the last row: their values are never used)
  const int i0 = s * H + lane * K;
  double p[K][D];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int row = min(i0 + k, R - 1);
#pragma unroll
    for (int e = 0; e < D; ++e) p[k][e] = __ldg(pd.P + (size_t)row * D + e);
  }
  const int rlast = R - 1 - i0;  // index k of the pair's last row when this lane holds it
  const bool holds_last = s == S - 1 && rlast >= 0 && rlast < K;

  double bot[K];
#pragma unroll
  for (int k = 0; k < K; ++k) bot[k] = kFltMax;
  double carry = kFltMax;  // carry of this lane's last row (to the lane above)
  double ob0 = kFltMax, ob1 = kFltMax;
  double res = kFltMax;
  int next_flush = 0;
  const int nout = (C + 31) >> 5;
  const int nsteps = C + 31;
  int status = 0;

  auto flush = [&](int k) {
    const int col = (k << 5) + lane;
    const double v = (k & 1) ? ob1 : ob0;
    if (col < C) __stcg(out_bnd + col, v);
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      st_release(&out_prog->word, ((unsigned long long)E << 32) | (unsigned)min((k + 1) << 5, C));
    }
  };
  auto wait_cols = [&](unsigned need) -> int {
    for (int it = 0;; ++it) {
      const unsigned long long w = bcast(lane == 0 ? ld_acquire(&in_prog->word) : 0ull);
      if ((unsigned)(w >> 32) == E && (unsigned)(w & 0xffffffffu) >= need) return 0;
      const int r = wt.check(it);
      if (r) return r;
    }
  };
  auto stage = [&](int c, const double (&q)[D]) {
    const int slot = ((c << 5) + lane) & (kDfdRing - 1);
#pragma unroll
    for (int e = 0; e < D; ++e) ring[e * kDfdRing + slot] = q[e];
  };
  auto fetch = [&](int c, double (&q)[D]) {
    const int j = min((c << 5) + lane, C - 1);
#pragma unroll
    for (int e = 0; e < D; ++e) q[e] = __ldg(pd.Q + (size_t)j * D + e);
  };

  double qn[D];
  fetch(0, qn);
  stage(0, qn);
  __syncwarp();

  for (int c = 0; (c << 5) < nsteps; ++c) {
    if (has_cons)
      while (next_flush <= c - 2) flush(next_flush++);
    // row above the strip for columns [32c, 32c + 32)
    const int col = (c << 5) + lane;
    double inreg = kFltMax;
    if ((c << 5) < C) {
      if (has_prod) {
        const int r = wait_cols((unsigned)min((c + 1) << 5, C));
        if (r) {  // 1 cannot happen (the DFD has no dead strips); 2: error
          status = 1;
          break;
        }
        if (col < C) inreg = __ldcg(in_bnd + col);
      } else {
        inreg = col == 0 ? 0.0 : kFltMax;
      }
    }
    fetch(c + 1, qn);  // next chunk's points, in flight during this chunk
#pragma unroll 4
    for (int u = 0; u < 32; ++u) {
      const int j = (c << 5) + u - lane;
      const double lin = __shfl_sync(kFull, inreg, u);
      const double lup = __shfl_up_sync(kFull, carry, 1);
      double left = lane == 0 ? lin : lup;
      const int slot = j & (kDfdRing - 1);
      double q[D];
#pragma unroll
      for (int e = 0; e < D; ++e) q[e] = ring[e * kDfdRing + slot];
      const bool j0 = j == 0;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const double dist = dist_sq<D>(p[k], q);
        const double b = j0 ? kFltMax : bot[k];
        const double in = fmin(left, b);
        const double top = fmax(dist, in);
        left = fmin(top, b);
        bot[k] = top;
        if (holds_last && k == rlast && j == C - 1) res = top;
      }
      carry = left;
      const double o = __shfl_sync(kFull, carry, 31);
      if (lane == ((u + 1) & 31)) {  // lane 31 produced column (c << 5) + u - 31
        if (((((c << 5) + u - 31) >> 5) & 1) != 0) ob1 = o;
        else ob0 = o;
      }
    }
    __syncwarp();
    stage(c + 1, qn);
    __syncwarp();
  }
  if (status == 0 && has_cons)
    while (next_flush < nout) flush(next_flush++);
  if (holds_last) st->result = res;
  return status;
}

}  // namespace rfd
