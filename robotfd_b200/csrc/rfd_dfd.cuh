// Dense discrete Frechet strips (the DFD upper bound, reference
// src/intersection_algorithm_in_parallel.cu:435-641, cell recurrence :608-637).
//
// The DFD is a dense min-max DP with a cheap cell (one squared point distance), so its
// sweep is bound by instruction issue and by how fast strips hand rows to each other, not
// by the geometry.  Compared with the generic strip (rfd_device.cuh):
//   - a lane owns K consecutive rows, in one of two layouts.  Skewed (for few, long pairs,
//     where the sweep's latency decides): at step t, row k of lane l is at column
//     t - (lK + k), so row k's "from below" input is row k-1's carry of the previous step
//     and the K cells of a step are independent (ILP K); row k reuses the point row k-1
//     used a step earlier, passed along in registers.  Stacked (for many pairs, where
//     instruction throughput decides): the K rows are at the lane's column and computed in
//     row order, fewer instructions per cell.  Either way a strip is 32K rows high, so K
//     times fewer strips hand rows to each other;
//   - the points of curve 2 a chunk of 32 steps needs are staged in a per-warp ring in
//     shared memory (structure of arrays, conflict-free), loaded into registers one chunk
//     ahead, so no global load sits in a step;
//   - the row handed to the next strip carries its own validity: the rows are filled with
//     an all-ones NaN pattern before the launch (dfd_fill_kernel), lane 31 stores each
//     value of the strip's last row once as it is produced, and the next strip polls the
//     values themselves, one 32-column chunk ahead of use.  A DFD value is never NaN (see
//     dmin / dmax), and each word is written once, so no fence or progress word is needed
//     and the load latency overlaps a chunk of steps;
//   - min / max are compare-and-select: every value is a squared distance of finite points,
//     0 or FLT_MAX, where they equal the reference's fmin / fmax (and a NaN coordinate
//     cannot make a NaN value: a comparison with NaN selects the other operand);
//   - there is no dead-region logic (the DFD is computed unpruned).
// Boundary conditions of the reference (:614-626) are folded into the inputs: strip 0
// reads the row above it as 0 at column 0 and FLT_MAX elsewhere, and every row reads
// FLT_MAX to the left of column 0.  Every cell performs the operations of cell<K_DFD> in
// rfd_device.cuh in the same order, so results are bit-identical.
#pragma once

#include "rfd_device.cuh"

namespace rfd {

// Ring of curve-2 points per warp: at least 32K + 64 columns (a chunk ahead of the widest
// span row 0 of the 32 lanes reads in one chunk, 31K + 32 columns).
template <int K>
struct DfdRing {
  static constexpr int cols = K <= 2 ? 128 : (K <= 4 ? 256 : 512);
  static_assert(cols >= 32 * K + 64, "ring too small");
};

template <bool B>
struct BoolC {
  static constexpr bool value = B;
};


// Cell weight: the squared point distance, or with INFL (the coarse upper bound,
// rfd_options.coarse_ub) the squared sum of the point distance and the two points' inflations
// (stored as coordinate D), each operation rounded to nearest; the bound built from it is
// widened by a relative margin that covers these roundings.
template <int D, bool INFL>
__device__ __forceinline__ double cell_weight(const double* p, const double* q) {
  const double s = dist_sq<D>(p, q);
  if (!INFL) return s;
  const double e = __dadd_rn(__dadd_rn(__dsqrt_rn(s), p[D]), q[D]);
  return __dmul_rn(e, e);
}

// Returns 0, or 1 on error / timeout (the error word is set).
// SKEW: rows of a lane skewed by one column each (latency: independent cells per step), or
// all at the lane's column (throughput: fewer instructions per cell, no point passing).
// INFL: points carry an inflation as coordinate D (stride D + 1) and the weight of a cell is
// cell_weight<D, true>.
template <int D, int K, bool SKEW, bool INFL = false>
__device__ int dfd_strip(const WaveArgs& wa, const PairDesc& pd, PairState* st, const int s,
                         double* ring /* [D + INFL][DfdRing<K>::cols] per warp */) {
  constexpr int DS = D + (INFL ? 1 : 0);  // stride of a point
  constexpr int H = 32 * K;
  constexpr int RC = DfdRing<K>::cols;
  const int lane = threadIdx.x & 31;
  const int R = pd.n1, C = pd.n2;
  const int S = (R + H - 1) / H;
  const bool has_prod = s > 0;
  const bool has_cons = s + 1 < S;
  // rows of the boundary ring, handed on column by column (see "Boundary ring" in
  // rfd_device.cuh): this strip clears each input chunk once read, and writes an output column
  // only where the row's previous reader has cleared it.  clr[w] counts the columns cleared
  // for writer w; its one publisher is the reader of the row's previous writer.
  const int nring = pd.ring;
  const int slot_in = has_prod ? (s - 1) % nring : 0;
  const int slot_out = has_cons ? s % nring : 0;
  if (!ring_check(wa, slot_in >= 0 && slot_in < nring && slot_out >= 0 && slot_out < nring, 8))
    return 1;
  double* in_bnd = has_prod ? pd.bnd + (size_t)slot_in * pd.cstride : nullptr;
  double* out_bnd = has_cons ? pd.bnd + (size_t)slot_out * pd.cstride : nullptr;
  unsigned long long* clr_in = has_prod ? pd.slots + (s - 1) : nullptr;   // writer s - 1's count
  unsigned long long* clr_out = pd.slots + s;                              // this strip's count
  unsigned long long* clr_next =                                           // the next writer's
      has_prod && s - 1 + nring < S ? pd.slots + (s - 1 + nring) : nullptr;
  unsigned in_ok = 0, out_ok = 0;  // leading columns cleared for the input's / this strip's writer
  constexpr int kPublish = 8;      // chunks between releases of the cleared count

  Waiter wt;
  wt.start(wa, st, s);

  // rows of this lane (clamped loads beyond the last row: their values are never used)
  const int base = SKEW ? lane * K : lane;  // row k of this lane is at column t - base - k*SKEW
  const int i0 = s * H + lane * K;
  double p[K][DS];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int row = min(i0 + k, R - 1);
#pragma unroll
    for (int e = 0; e < DS; ++e) p[k][e] = __ldg(pd.P + (size_t)row * DS + e);
  }
  const int rlast = R - 1 - i0;  // index k of the pair's last row when this lane holds it
  const bool holds_last = s == S - 1 && rlast >= 0 && rlast < K;
  // step at which that row reaches column C - 1
  const int tres = C - 1 + base + (SKEW ? rlast : 0);
  constexpr int kOutLag = SKEW ? H - 1 : 31;  // column of the last row = t - kOutLag

  double bot[K], carry[K], qp[K][DS];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    bot[k] = kFltMax;
    carry[k] = kFltMax;
#pragma unroll
    for (int e = 0; e < DS; ++e) qp[k][e] = 0.0;
  }
  double res = kFltMax;
  const int nsteps = C + kOutLag;
  int status = 0;

  auto stage = [&](int c, const double (&q)[DS]) {
    const int slot = ((c << 5) + lane) & (RC - 1);
#pragma unroll
    for (int e = 0; e < DS; ++e) ring[e * RC + slot] = q[e];
  };
  auto fetch = [&](int c, double (&q)[DS]) {
    const int j = min((c << 5) + lane, C - 1);
#pragma unroll
    for (int e = 0; e < DS; ++e) q[e] = __ldg(pd.Q + (size_t)j * DS + e);
  };
  // the row above the strip at column 32c + lane (empty pattern while not yet written, or
  // while the row may still hold its previous writer's words there)
  auto load_in = [&](int c) -> unsigned long long {
    const int col = (c << 5) + lane;
    if (!has_prod) return __double_as_longlong(col == 0 ? 0.0 : kFltMax);
    if ((c << 5) >= C || col >= C) return __double_as_longlong(kFltMax);
    if (in_ok < (unsigned)min((c + 1) << 5, C)) return kBndEmpty;
    return ld_relaxed_u64(in_bnd + col);
  };
  // cleared count of a writer (acquire: the clearing stores are visible)
  auto cleared = [&](unsigned long long* cnt, unsigned have) -> unsigned {
    const unsigned long long w = bcast(lane == 0 ? ld_acquire(cnt) : 0ull);
    __syncwarp();  // every lane's later accesses of the row are ordered after the acquire
    return max(have, (unsigned)w);
  };
  const bool store_out = has_cons && lane == 31;

  // 32 steps of chunk c.  Column 0 (the reference's left boundary, FLT_MAX) only occurs in
  // the first chunks (SKEW: K of them, else one), which alone carry that select.  The steps
  // are unrolled by 8 only (those first chunks: not at all): with K rows, 2 and 3
  // dimensions, a full unroll makes code that no longer fits the instruction cache, and
  // fetch stalls then dominate.
  auto steps = [&](const int c, const double inreg, auto first) {
    constexpr bool FIRST = decltype(first)::value;
    constexpr int kUnroll = FIRST ? 1 : 8;
#pragma unroll kUnroll
    for (int u = 0; u < 32; ++u) {
      const int t = (c << 5) + u;
      const double lin = __shfl_sync(kFull, inreg, u);
      const double lup = __shfl_up_sync(kFull, carry[K - 1], 1);
      const double left0 = lane == 0 ? lin : lup;
      double q0[DS];
      const int slot = (t - base) & (RC - 1);
#pragma unroll
      for (int e = 0; e < DS; ++e) q0[e] = ring[e * RC + slot];
      if (SKEW) {
        // rows in descending order: row k reads row k-1's values of the previous step
#pragma unroll
        for (int k = K - 1; k >= 0; --k) {
          double q[DS];
#pragma unroll
          for (int e = 0; e < DS; ++e) q[e] = k == 0 ? q0[e] : qp[k - 1][e];
          const double left = k == 0 ? left0 : carry[k - 1];
          const double dist = cell_weight<D, INFL>(p[k], q);
          const double b = (FIRST && t - base - k == 0) ? kFltMax : bot[k];
          const double in = dmin(left, b);
          const double top = dmax(dist, in);
          carry[k] = dmin(top, b);
          bot[k] = top;
#pragma unroll
          for (int e = 0; e < DS; ++e) qp[k][e] = q[e];
        }
      } else {
        // rows in ascending order at one column: each takes the row below's carry
        double left = left0;
        const bool j0 = FIRST && t - base == 0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const double dist = cell_weight<D, INFL>(p[k], q0);
          const double b = j0 ? kFltMax : bot[k];
          const double in = dmin(left, b);
          const double top = dmax(dist, in);
          left = dmin(top, b);
          bot[k] = top;
        }
        carry[K - 1] = left;
      }
      if (holds_last && t == tres) {
#pragma unroll
        for (int k = 0; k < K; ++k)
          if (k == rlast) res = bot[k];
      }
      const int jo = t - kOutLag;  // column of the strip's last row at this step
      if (store_out && jo >= 0 && jo < C) st_relaxed_f64(out_bnd + jo, carry[K - 1]);
    }
  };

  double qn[DS];
  fetch(0, qn);
  stage(0, qn);
  __syncwarp();
  unsigned long long nxt = load_in(0);
  constexpr int kFirstChunks = SKEW ? K : 1;

  for (int c = 0; (c << 5) < nsteps; ++c) {
    // wait until every column of this chunk's input row has been written
    unsigned long long cur = nxt;
    const bool reads = has_prod && (c << 5) < C;
    const unsigned need_in = (unsigned)min((c + 1) << 5, C);
    for (int it = 0;; ++it) {
      if (reads && in_ok < need_in) {
        in_ok = cleared(clr_in, in_ok);
        if (in_ok >= need_in) cur = load_in(c);
      }
      if (__all_sync(kFull, cur != kBndEmpty)) break;
      const int r = wt.check(it);
      if (r) {  // 1 cannot happen (the DFD has no dead strips); 2: error
        status = 1;
        break;
      }
      if (cur == kBndEmpty) cur = load_in(c);
    }
    if (status) break;
    if (reads) {
      // read: the chunk's words go back to "not yet written" for the row's next writer
      const int col = (c << 5) + lane;
      if (col < C) st_relaxed_u64(reinterpret_cast<unsigned long long*>(in_bnd) + col, kBndEmpty);
      if ((c & (kPublish - 1)) == kPublish - 1 && clr_next) {
        __syncwarp();
        if (lane == 0) {
          __threadfence();
          st_release(clr_next, need_in);
        }
      }
    }
    if (has_cons) {
      // this chunk's steps store the last row's columns below 32c + 32 - kOutLag
      const unsigned need_out = (unsigned)min(max((c << 5) + 32 - kOutLag, 0), C);
      for (int it = 0; out_ok < need_out; ++it) {
        out_ok = cleared(clr_out, out_ok);
        if (out_ok >= need_out) break;
        if (wt.check(it)) {
          status = 1;
          break;
        }
      }
      if (status) break;
    }
    nxt = load_in(c + 1);  // in flight during this chunk
    fetch(c + 1, qn);
    if (c < kFirstChunks) steps(c, __longlong_as_double(cur), BoolC<true>{});
    else steps(c, __longlong_as_double(cur), BoolC<false>{});
    __syncwarp();
    stage(c + 1, qn);
    __syncwarp();
  }
  if (status == 0 && clr_next) {
    // every input word has been read and cleared: the whole row is the next writer's
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      st_release(clr_next, kSlotAll);
    }
  }
  if (holds_last) st->result = res;
  return status;
}

}  // namespace rfd
