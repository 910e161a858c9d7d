// "Team" strips: one CTA of 8 (or 4) warps per 32-row strip for the VE-FD and decision DPs.
//
// The solo strip (rfd_device.cuh) computes each cell's geometry on the step-to-step
// dependency chain, so a sparse band - a handful of live lanes per step - advances at the
// latency of two FP64 quadratics per step.  Here the geometry leaves that chain:
//   warps 1..7 (helpers)  compute a whole skewed 32x32 tile of step-chunk c - for the
//                          decision the right and top free intervals of every cell, for
//                          VE-FD the two vertex-edge weights - into shared memory;
//   warp 0 (propagator)   runs the same skewed sweep, the same L2 strip handoff and the
//                          same dead-region jumps as the solo strip, but a step is only a
//                          shared-memory read, two shuffles and the min/max propagation.
// Tile c+1 is requested speculatively while tile c is consumed (two slots, mbarrier
// handshakes); a jump cancels the speculative tile.  The arithmetic of every cell is the
// solo strip's (same functions), so results are bit-identical.  The same code, instantiated
// with MIR, sweeps the mirror half of a split pair from the far corner (mirror_interval).
#pragma once

#include <type_traits>

#include "rfd_device.cuh"
#include "rfd_filter.h"

namespace rfd {

// Warps per team: 8 by default (warp 0 propagates, 7 helpers); teams of 4 (3 helpers) are the
// autotuner's other shape (rfd_autotune_search), twice as many teams of half the tile rate.
constexpr int kTeamThreads = 256;
constexpr int kStop = -2;  // request word: strip finished

struct TeamShared {
  unsigned long long full[2];  // helpers -> propagator: tile ready (one arrival per helper)
  unsigned long long req[2];   // propagator -> helpers: chunk requested (1 arrival)
  unsigned long long staged;   // helpers -> helpers: a tile's column records are staged
  int req_chunk[2];
  int cancel[2];
  int item_pair, item_strip, go, quit;
  unsigned long long evaluated;    // cells the helpers computed
  unsigned long long evaluated64;  // of those, cells with an interval computed in FP64
  int status;
  int push;                 // continuous search: this CTA starts the pair's next probe
  int push_req;             // continuous search: 1 the strip's band started (queue a strip),
                            // 2 queued, 3 the strip found no live input (queue the rest)
  // the strip's last row, two 32-column chunks: lane 31 stores each value as it is produced
  // (off the propagation chain), the flush reads a chunk back one column per lane
  double out_row[64];
};

// Continuous search: makes `count` more strips of pair p's running probe available (S per
// probe at most), one queue entry, the pair's index, each.  A taker draws the strip index
// from the pair's next_strip counter, so strips start in order and a strip's predecessor is
// always already running, as with a launch's item list.  One thread.
__device__ __forceinline__ void queue_strips(const WaveArgs& wa, PairState* st, int p, int S,
                                             int count) {
  const int k = atomicAdd(&st->pushed, count);
  const int n = min(count, S - k);
  if (n <= 0) return;
  const unsigned slot = atomicAdd(wa.dyn_tail, (unsigned)n);
  if ((long long)slot + n > wa.dyn_cap) {  // cannot happen: sized for max_probes probes per pair
    atomicExch(wa.error, 1);
    return;
  }
  for (int i = 0; i < n; ++i) st_release(wa.dyn_items + slot + i, (unsigned long long)(unsigned)p);
}

// Column records of one tile, staged by the helpers: the tile of step-chunk c reads the
// columns c*32-31 .. c*32+31, i.e. the points q_{c*32-31} .. q_{c*32+32} and the segments'
// A and 0.5/A, as structure-of-arrays rows of 64 (conflict-free reads along a warp).
constexpr int kStageRow = 64;
constexpr int kStageDoubles = 5 * kStageRow;  // q[3][64], A[64], inv2A[64]

constexpr size_t kTeamHeader = 1024;
static_assert(sizeof(TeamShared) <= kTeamHeader, "team header");

template <int KIND>
struct TileT {
  static constexpr int vals = KIND == K_DEC ? 2 : 1;  // double2 per cell
  static constexpr size_t slot_bytes = (size_t)vals * 1024 * sizeof(double2);
};

template <int KIND>
__host__ __device__ constexpr size_t team_smem_bytes() {
  return kTeamHeader + 2 * TileT<KIND>::slot_bytes + 2 * kStageDoubles * sizeof(double);
}

// ------------------------------------------------------------------ mbarrier helpers

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait (warp-uniform: every lane polls the same barrier phase).  false on timeout
// or when the global error word is set.
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity, const WaveArgs& wa,
                                          long long t0) {
  for (int it = 0;; ++it) {
    if (mbar_try_wait(b, parity)) return true;
    if ((it & 63) == 63) {
      int bad = 0;
      if ((threadIdx.x & 31) == 0)
        bad = ld_volatile(wa.error) || (clock64() - t0 > wa.spin_cycles);
      if (__shfl_sync(kFull, bad, 0)) {
        if ((threadIdx.x & 31) == 0) atomicExch(wa.error, 1);
        return false;
      }
    }
  }
}

// ------------------------------------------------------------------ helpers (warps 1..H)

// Mirror sweep (MIR, meet in the middle): the grid seen from its far corner.  Mirror cell
// (i, j) is cell (a, b) = (mrow - i, C - 1 - j) of the pair, and its tile holds the values of
// that cell's two entry edges - the right edge of cell (a - 1, b) (point p_a against segment
// q_b q_{b+1}) and the top edge of cell (a, b - 1) (point q_b against segment p_a p_{a+1}) -
// computed by the same functions from the same operands as the forward sweep's tiles, so
// they are the same doubles.  VE-FD weights are used as they are (the min-max recurrence runs
// backwards unchanged); a free interval [lo, hi] becomes [-hi, -lo] (exact), so that the
// forward propagation, run on the mirrored grid, computes the negated upper ends of the
// co-reachable parts (points from which the far corner can be reached); an empty interval
// becomes (-3, -4), dead below -1.5.
__device__ __forceinline__ void mirror_interval(double& lo, double& hi) {
  if (lo < 0.0) {
    lo = -3.0;
    hi = -4.0;
  } else {
    const double l = lo;
    lo = -hi;
    hi = -l;
  }
}

template <int KIND, int D, int H /* helper warps */, bool MIR = false>
__device__ void team_helpers(const WaveArgs& wa, const PairDesc& pd, const PairState* st, int s,
                             TeamShared* sh, double2* tiles, double* stage, unsigned& seqH,
                             unsigned& seqS, int hw) {
  const int lane = threadIdx.x & 31;
  const int R = pd.n1 - 1, C = pd.n2 - 1;
  const int i = (s << 5) + lane;
  const bool rowv = i < R;
  const double r2 = st->r2;
  const bool filt = KIND == K_DEC && st->filter;  // FP32 classification first (rfd_filter.h)
  const bool mat = KIND == K_DEC && st->formula == 1;  // materialised path's intervals
  RowData<KIND, D> row;
  if (rowv) row.load(pd, MIR ? pd.mrow - i : i);
  const long long t0 = clock64();
  unsigned long long count = 0, count64 = 0;
  for (;;) {
    const int slot = seqH & 1;
    const long long tw0 = wa.prof ? clock64() : 0;
    if (!mbar_wait(&sh->req[slot], (seqH >> 1) & 1, wa, t0)) break;
    if (wa.prof && lane == 0) atomicAdd(&wa.prof[9], (unsigned long long)(clock64() - tw0));
    const int c = *(volatile int*)&sh->req_chunk[slot];
    if (c == kStop) {
      // every request, the stop included, is answered with one completion, so the
      // propagator's take count and the request count stay equal across strips
      __syncwarp();
      if (lane == 0) mbar_arrive(&sh->full[slot]);
      ++seqH;
      break;
    }
    double2* T0 = tiles + (size_t)slot * TileT<KIND>::vals * 1024;
    double2* T1 = T0 + 1024;
    const long long tc0 = wa.prof ? clock64() : 0;
    // Stage the tile's column records once for all helpers (one round of coalesced loads
    // instead of a dependent load per cell pair), with clamped indices: a clamped record
    // only feeds cells outside the grid, whose results are not stored.  Two buffers: a
    // helper stages tile k+1 while slower ones may still read tile k.
    double* buf = stage + (seqS & 1) * kStageDoubles;
    {
      const int base = (c << 5) - 31;
      const int t = (hw << 5) + lane;
      // (mirror: staged row jj holds point q_{C - base - jj} and the records of segment
      // C - 1 - base - jj, so column j = base + jj reads q_b at jj + 1 and q_{b+1} at jj)
      for (int e = t; e < kStageRow * D; e += 32 * H) {
        const int jj = e / D, k = e - jj * D;
        const int qi = MIR ? min(max(C - (base + jj), 0), C) : min(max(base + jj, 0), C);
        buf[k * kStageRow + jj] = __ldg(pd.Q + (size_t)qi * D + k);
      }
      constexpr int W = RecW<D>::value;
      for (int e = t; e < kStageRow - 1; e += 32 * H) {
        const int j = MIR ? min(max(C - 1 - (base + e), 0), C - 1) : min(max(base + e, 0), C - 1);
        const double2 a = __ldg(pd.colrec + (size_t)j * W + (W - 1));
        buf[3 * kStageRow + e] = a.x;
        buf[4 * kStageRow + e] = a.y;
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&sh->staged);
    if (!mbar_wait(&sh->staged, seqS & 1, wa, t0)) break;
    ++seqS;
    if (wa.prof && lane == 0) atomicAdd(&wa.prof[13], (unsigned long long)(clock64() - tc0));
    // column j = c*32 + u - lane sits at jj = u - lane + 31 of the staged rows
    auto col_at = [&](int u, ColRec<KIND, D>& col) {
      const int jj = u - lane + 31;
#pragma unroll
      for (int k = 0; k < D; ++k) {
        col.qa[k] = buf[k * kStageRow + jj + (MIR ? 1 : 0)];
        col.qb[k] = buf[k * kStageRow + jj + (MIR ? 0 : 1)];
      }
      col.A = buf[3 * kStageRow + jj];
      col.inv2A = buf[4 * kStageRow + jj];
    };
    // Two independent cells (u, u + H) per iteration; results are stored only for
    // cells inside the grid.
    auto one = [&](int u, const ColRec<KIND, D>& col) {
      const int j = (c << 5) + u - lane;
      double qd[D];
#pragma unroll
      for (int k = 0; k < D; ++k) qd[k] = __dsub_rn(col.qb[k], col.qa[k]);
      const bool ok = rowv && j >= 0 && j < C;
      // the right edge's point (p_{i+1}; mirror: p_a) and the top edge's (q_{j+1}; mirror: q_b)
      const double* xr = MIR ? row.a : row.b;
      const double* xt = MIR ? col.qa : col.qb;
      if (KIND == K_DEC) {
        double rLB, rUB, tLB, tUB;
        // with the filter, an edge certainly empty or certainly whole takes the exact value
        // the FP64 code would write; the others are computed in FP64
        int cr = 0, ct = 0;
        if (filt) {
          cr = interval_class32<D>(xr, col.qa, qd, col.A, r2);
          ct = interval_class32<D>(xt, row.a, row.ab, row.A, r2);
        }
        if (cr == 0) {
          free_interval<D>(xr, col.qa, qd, col.A, col.inv2A, r2, rLB, rUB, mat);
        } else {
          rLB = cr == 1 ? -1.0 : 0.0;
          rUB = cr == 1 ? -2.0 : 1.0;
        }
        if (ct == 0) {
          free_interval<D>(xt, row.a, row.ab, row.A, row.inv2A, r2, tLB, tUB, mat);
        } else {
          tLB = ct == 1 ? -1.0 : 0.0;
          tUB = ct == 1 ? -2.0 : 1.0;
        }
        if (MIR) {
          mirror_interval(rLB, rUB);
          mirror_interval(tLB, tUB);
        }
        count64 += (ok && (cr == 0 || ct == 0)) ? 1 : 0;
        if (ok) {
          T0[(u << 5) + lane] = make_double2(rLB, rUB);
          T1[(u << 5) + lane] = make_double2(tLB, tUB);
        }
      } else {
        double wr, wt;
        if constexpr (MIR) {
          wr = pt_seg_sq<D>(row.a, col.qa, qd, col.A);
          wt = pt_seg_sq<D>(col.qa, row.a, row.ab, row.A);
        } else {
          wr = pt_seg_sq<D>(row.b, col.qa, qd, col.A);
          wt = pt_seg_sq<D>(col.qb, row.a, row.ab, row.A);
        }
        if (ok) T0[(u << 5) + lane] = make_double2(wt, wr);
      }
      count += ok ? 1 : 0;
    };
    for (int u0 = hw; u0 < 32; u0 += 2 * H) {
      if (__shfl_sync(kFull, *(volatile int*)&sh->cancel[slot], 0)) break;
      const int u1 = u0 + H;
      ColRec<KIND, D> c0, c1;
      col_at(u0, c0);
      col_at(min(u1, 31), c1);
      one(u0, c0);
      if (u1 < 32) one(u1, c1);
    }
    if (wa.prof && lane == 0) {
      atomicAdd(&wa.prof[8], (unsigned long long)(clock64() - tc0));
      atomicAdd(&wa.prof[10], 1ull);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&sh->full[slot]);
    ++seqH;
    if (wa.dyn_items && hw == 0 && lane == 0 && *(volatile int*)&sh->push_req == 1) {
      // the band reached this strip: queue one more of the probe, once this warp's share of
      // the tile is in (the push's round trips then delay no tile)
      *(volatile int*)&sh->push_req = 2;
      PairState* ps = const_cast<PairState*>(st);
      queue_strips(wa, ps, (int)(ps - wa.st), (R + 31) >> 5, 1);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    count += __shfl_xor_sync(kFull, count, o);
    count64 += __shfl_xor_sync(kFull, count64, o);
  }
  if (lane == 0 && count) atomicAdd(&sh->evaluated, count);
  if (lane == 0 && count64) atomicAdd(&sh->evaluated64, count64);
}

// ------------------------------------------------------------------ propagator (warp 0)

// RFD_PROF trace of the first kTrace strips of the first pair: wall-clock ns (globaltimer,
// comparable across SMs) at strip start, first live input chunk, first live output flush, the
// first live chunk's tile taken, its steps done, and the next chunk's input in hand.
constexpr int kTrace = 512;
constexpr int kTraceW = 6;  // trace words per strip
constexpr int kTraceBase = 16;
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <int KIND, int D, bool MIR = false>
__device__ int team_propagator(const WaveArgs& wa, const PairDesc& pd, PairState* st, const int s,
                               TeamShared* sh, const double2* tiles, unsigned& seqP,
                               unsigned& seqC) {
  const int lane = threadIdx.x & 31;
  const int R = pd.n1 - 1;
  const int C = pd.n2 - 1;
  const int S = (R + 31) >> 5;
  const unsigned E = st->epoch;
  const double U = st->U;
  const bool dense = st->dense != 0;
  const bool has_prod = s > 0;
  // mirror sweep (meet in the middle): decision values live in [-1, 0], dead below -1.5
  // (see mirror_interval); its last strip also hands its row on, to the meet kernel
  constexpr bool mir = MIR;
  const double dthr = mir ? -1.5 : 0.0;
  const double dv = KIND == K_DEC ? (mir ? -3.0 : -1.0) : kFltMax;
  auto isd = [U, dthr](double v) { return KIND == K_DEC ? v < dthr : v > U; };
  const bool has_cons = s + 1 < S || mir;
  // the lane whose row the strip hands on: 31, or, for the mirror's last strip, which may
  // hold fewer than 32 rows, the lane of the grid's last row
  const int olane = MIR ? (s + 1 < S ? 31 : ((R - 1) & 31)) : 31;
  const bool tr = pd.tr != 0;

  // Strip s writes boundary row s % ring (and its tags).  ring >= S - 1 unless the strips run
  // in launch windows of ring - 1 strips (rfd_engine.cu, team_window_fill_kernel): a window's
  // strips then write distinct rows, none of them the row its first strip reads.
  const int rin = has_prod ? (s - 1) % pd.ring : 0;
  const int rout = has_cons ? s % pd.ring : 0;
  Prog* in_prog = has_prod ? pd.prog + (s - 1) : nullptr;
  Prog* out_prog = has_cons ? pd.prog + s : nullptr;
  const double* in_bnd = has_prod ? pd.bnd + (size_t)rin * pd.cstride : nullptr;
  double* out_bnd = has_cons ? pd.bnd + (size_t)rout * pd.cstride : nullptr;
  const unsigned* in_tags = has_prod ? pd.tags + (size_t)rin * pd.tstride : nullptr;
  unsigned* out_tags = has_cons ? pd.tags + (size_t)rout * pd.tstride : nullptr;

  int status = 0;
  Waiter wt;
  wt.start(wa, st, s);
  const long long t0 = clock64();
  if (wa.prof && lane == 0) atomicAdd(&wa.prof[7], 1ull);
  unsigned long long* trace =
      (wa.prof && st == wa.st && s < kTrace) ? wa.prof + kTraceBase + kTraceW * s : nullptr;
  bool traced_in = false;
  int trace_step = 0;  // 1: first live chunk's tile taken, 2: its steps done, 3: next input in
  if (trace && lane == 0) trace[0] = global_ns();

  const int i = (s << 5) + lane;
  const bool rowv = i < R;
  const bool last_row = i == R - 1;
  const int nout = (C + 31) >> 5;
  const int nsteps = C + 31;
  double res = KIND == K_DEC ? -2.0 : kFltMax;
  bool dead_tail = !dense && bcast(lane == 0 ? ld_volatile(&st->dead_from) : 0) <= s;

  if (has_cons && lane == 0) {
    out_prog->first_live = kNone;
    out_prog->last_live = 0;
  }
  double bot;
  // the mirror decision starts at the far corner: through the top edge of the pair's last
  // cell (transposed grid) here, through its right edge as strip 0's input below
  const bool inj = KIND == K_DEC && mir && !tr && st->corner != 0;
  if (KIND == K_DEC) bot = mir ? ((i == 0 && tr && st->corner) ? -1.0 : dv) : (i == 0 ? 0.0 : -1.0);
  else bot = i == 0 ? st->seed : kFltMax;
  double carry = dv;
  double* out_row = sh->out_row;
  out_row[lane] = dv;
  out_row[32 + lane] = dv;
  __syncwarp();
  unsigned first_live_out = kNone;
  int next_flush = 0;
  int wlo = INT_MAX, whi = -1;  // output chunks written (cleared before the pair's next probe)
  int pending = -1;  // chunk of the outstanding tile request (-1: none)

  auto request = [&](int c) {
    const int slot = seqP & 1;
    if (lane == 0) {
      *(volatile int*)&sh->req_chunk[slot] = c;
      *(volatile int*)&sh->cancel[slot] = 0;
      mbar_arrive(&sh->req[slot]);
    }
    __syncwarp();
    ++seqP;
  };
  // Waits for the oldest outstanding tile; returns its slot or -1 on error.
  auto take = [&]() -> int {
    const int slot = seqC & 1;
    const long long tw0 = wa.prof ? clock64() : 0;
    if (!mbar_wait(&sh->full[slot], (seqC >> 1) & 1, wa, t0)) return -1;
    if (wa.prof && lane == 0) atomicAdd(&wa.prof[2], (unsigned long long)(clock64() - tw0));
    ++seqC;
    return slot;
  };
  auto drop_pending = [&]() -> bool {
    if (pending < 0) return true;
    if (lane == 0) *(volatile int*)&sh->cancel[seqC & 1] = 1;
    __syncwarp();
    pending = -1;
    return take() >= 0;
  };
  // Flush of output chunk k: its words, then (lane 0) its tag and the first/last live hints.
  // The progress word is released (after a fence) only when `publish` is set: the next strip
  // reads written words directly, and needs the progress word only for chunks that are never
  // written (skipped as dead: every jump publishes) and for its tag scan behind the band, so
  // in-band flushes publish every 8th chunk and skip the fence's round trip otherwise.
  auto flush = [&](int k, bool publish) {
    const long long tf0 = wa.prof ? clock64() : 0;
    const int col = (k << 5) + lane;
    __syncwarp();
    const double v = out_row[((k & 1) << 5) + lane];
    const bool valid = col < C;
    if (valid) st_relaxed_f64(out_bnd + col, v);
    wlo = min(wlo, k);
    whi = max(whi, k);
    const unsigned live = __ballot_sync(kFull, valid && !isd(v));
    out_row[((k & 1) << 5) + lane] = dv;
    __syncwarp();
    if (lane == 0) {
      if (live) {
        __stcg(out_tags + k, E);
        if (first_live_out == kNone) {
          first_live_out = (unsigned)k;
          out_prog->first_live = (unsigned)k;
          if (trace) trace[2] = global_ns();
        }
        out_prog->last_live = (unsigned)k;
      }
      if (publish) {
        __threadfence();
        st_release(&out_prog->word, ((unsigned long long)E << 32) | (unsigned)min((k + 1) << 5, C));
      }
    }
    if (wa.prof) {
      __syncwarp();
      if (lane == 0) {
        atomicAdd(&wa.prof[11], (unsigned long long)(clock64() - tf0));
        atomicAdd(&wa.prof[12], 1ull);
      }
    }
  };
  auto publish_cols = [&](int cols) {
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      st_release(&out_prog->word, ((unsigned long long)E << 32) | (unsigned)cols);
    }
  };
  auto wait_cols = [&](unsigned need, unsigned long long& w) -> int {
    const long long tw0 = wa.prof ? clock64() : 0;
    for (int it = 0;; ++it) {
      w = bcast(lane == 0 ? ld_acquire(&in_prog->word) : 0ull);
      if ((unsigned)(w >> 32) == E && (unsigned)(w & 0xffffffffu) >= need) {
        if (wa.prof && lane == 0) atomicAdd(&wa.prof[0], (unsigned long long)(clock64() - tw0));
        return 0;
      }
      const int r = wt.check(it);
      if (r) return r;
    }
  };

  // The row above the strip for the next chunk is loaded at the end of the current chunk.
  // The rows were filled with kBndEmpty before the launch and every word is written once, so
  // a chunk whose 32 words are all written is final and is used at once, without the
  // progress word or the tag; otherwise the flag protocol below decides.
  unsigned long long pre = kBndEmpty;
  int pre_c = -1;
  bool seen_live = false;  // has a live input chunk reached this strip yet
  auto prefetch = [&](int k) {
    pre_c = -1;
    if (!has_prod || (k << 5) >= C) return;
    const int col = (k << 5) + lane;
    pre = col < C ? ld_relaxed_u64(in_bnd + col) : __double_as_longlong(dv);
    pre_c = k;
  };

  int c = 0;
  while (!dead_tail && (c << 5) < nsteps) {
    if (has_cons)
      while (next_flush <= c - 2) {
        flush(next_flush, (next_flush & 7) == 7);
        ++next_flush;
      }
    double inreg = dv;
    if (inj && c == 0 && lane == 0) inreg = -1.0;  // column 0 of the mirror's first input row
    bool in_live = false;
    bool fast = false;
    if (has_prod && (c << 5) < C) {
      // Poll the chunk's words themselves (and, alongside, the progress word): a complete
      // chunk is used as soon as it lands.  A chunk the progress word calls final while
      // words are still missing was skipped (dead) or read early: the flag protocol below
      // settles it, as it does a dead strip or an expired wait.
      const int col = (c << 5) + lane;
      const unsigned need = (unsigned)min((c + 1) << 5, C);
      auto load = [&]() {
        return col < C ? ld_relaxed_u64(in_bnd + col) : __double_as_longlong(dv);
      };
      unsigned long long v = pre_c == c ? pre : load();
      unsigned long long w = 0ull;
      for (int it = 0;; ++it) {
        if (__all_sync(kFull, v != kBndEmpty)) {
          inreg = __longlong_as_double(v);
          in_live = __any_sync(kFull, col < C && !isd(inreg));
          fast = true;
          break;
        }
        if (it > 0 && (unsigned)(w >> 32) == E && (unsigned)(w & 0xffffffffu) >= need) break;
        if (wt.check(it)) break;
        if (lane == 0) w = ld_relaxed_u64(&in_prog->word);  // both loads in flight together
        if (v == kBndEmpty) v = load();
        w = bcast(w);
      }
    }
    if (!fast && (c << 5) < C) {
      if (has_prod) {
        unsigned long long w;
        const int r = wait_cols((unsigned)min((c + 1) << 5, C), w);
        if (r == 2) { status = 1; break; }
        if (r == 1) { dead_tail = true; break; }
        const unsigned tg = bcast(lane == 0 ? __ldcg(in_tags + c) : 0u);
        in_live = tg == E;
        if (in_live) {
          const int col = (c << 5) + lane;
          if (col < C) inreg = __ldcg(in_bnd + col);
        }
      } else {
        // (mirror: warp-uniform, only the decision's column 0 can be live here; otherwise
        // every lane's input is dead)
        if (MIR) in_live = __any_sync(kFull, !isd(inreg));
        else in_live = !isd(inreg);
      }
    }
    if (in_live && !seen_live) {
      seen_live = true;
      // the band reached this strip: a helper queues one more strip of the probe
      if (wa.dyn_items && lane == 0) *(volatile int*)&sh->push_req = 1;
      // Liveness enters a strip only through its input row, so no output chunk before c can
      // be live: publish c as a lower bound of the first live output chunk (the flush of the
      // actual one overwrites it), so the next strip moves to this strip's band and starts
      // its tile about two chunks before that flush.  Any value the consumer reads is a valid
      // lower bound, so no release is needed.
      if (has_cons && lane == 0 && first_live_out == kNone) out_prog->first_live = (unsigned)c;
    }
    if (trace && trace_step == 2) {
      trace_step = 3;
      if (lane == 0) trace[5] = global_ns();
    }
    if (trace && in_live && !traced_in) {
      traced_in = true;
      if (lane == 0) trace[1] = global_ns();
    }
    if (!dense && !in_live) {
      const bool ldead = (!rowv || isd(bot) || ((c << 5) - lane >= C)) &&
                         isd(carry);
      if (__all_sync(kFull, ldead)) {
        int nc = -1;
        if (has_prod && (c << 5) < C) {
          int pos = c + 1;
          const long long tj0 = wa.prof ? clock64() : 0;
          // the speculative tile in flight (chunk c) is not needed: the warp skips c
          if (!drop_pending()) { status = 1; break; }
          for (int it = 0;; ++it) {
            unsigned long long w = 0ull;
            unsigned fl = kNone, ll = 0u;
            if (lane == 0) {
              w = ld_acquire(&in_prog->word);
              fl = __ldcg(&in_prog->first_live);
              ll = __ldcg(&in_prog->last_live);
            }
            w = bcast(w);
            fl = bcast(fl);
            ll = bcast(ll);
            const bool ours = (unsigned)(w >> 32) == E;
            const unsigned cols = ours ? (unsigned)(w & 0xffffffffu) : 0u;
            const bool done = ours && cols >= (unsigned)C;
            if (!ours) fl = kNone;
            const int avail = done ? nout : (int)(cols >> 5);
            if (fl != kNone) {
              pos = max(pos, (int)fl);
              const int end = done ? min(nout, (int)ll + 1) : avail;
              while (pos < end && nc < 0) {
                const int k = pos + lane;
                const bool hit = k < end && __ldcg(in_tags + k) == E;
                const unsigned b = __ballot_sync(kFull, hit);
                if (b) nc = pos + __ffs(b) - 1;
                else pos = min(pos + 32, end);
              }
              // No chunk before the producer's first live chunk is live, and the producer
              // writes every chunk from there on: until this strip has seen live input, go
              // to the next candidate chunk now and wait for its words in the input path (a
              // chunk that turns out dead moves on by one).  After the band has passed, the
              // tag scan finds the next live chunk, 32 at a time.
              if (nc < 0 && !done && pos < nout && !seen_live) nc = pos;
              // The producer's first live chunk at or after pos is where this strip will
              // most likely resume: start its tile now so it is ready at the jump.
              if (nc < 0 && pos < nout && pending != pos) {
                if (!drop_pending()) { status = 1; break; }
                request(pos);
                pending = pos;
              }
            } else {
              pos = max(pos, avail);
            }
            if (nc >= 0 || done) break;
            const int r = wt.check(it);
            if (r == 2) { status = 1; break; }
            if (r == 1) break;
          }
          if (status) break;
          if (wa.prof && lane == 0) {
            atomicAdd(&wa.prof[1], (unsigned long long)(clock64() - tj0));
            atomicAdd(&wa.prof[6], 1ull);
          }
        }
        // (published below: by publish_cols at the jump, or at the end of the strip)
        if (has_cons)
          while (next_flush <= c - 1) {
            flush(next_flush, false);
            ++next_flush;
          }
        if (nc >= 0 && pending == nc) {
          // the speculative cold-start tile is the one we need: keep it
        } else if (!drop_pending()) {
          status = 1;
          break;
        }
        if (nc < 0) {
          dead_tail = true;
          break;
        }
        if (has_cons) {
          next_flush = nc - 1;
          publish_cols(min((nc - 1) << 5, C));
        }
        carry = dv;
        __syncwarp();
        out_row[lane] = dv;
        out_row[32 + lane] = dv;
        __syncwarp();
        c = nc;
        if (pending != c) {
          request(c);  // cold start of the live stretch
          pending = c;
        }
        continue;
      }
    }
    // ---- process step-chunk c from tile c
    if (pending != c) {
      if (!drop_pending()) { status = 1; break; }
      request(c);
      pending = c;
    }
    const int slot = take();
    if (slot < 0) { status = 1; break; }
    if (trace && traced_in && trace_step == 0) {
      trace_step = 1;
      if (lane == 0) trace[3] = global_ns();
    }
    pending = -1;
    if (((c + 1) << 5) < nsteps) {  // speculative: the next chunk is usually processed too
      request(c + 1);
      pending = c + 1;
    }
    const double2* T0 = tiles + (size_t)slot * TileT<KIND>::vals * 1024;
    const double2* T1 = T0 + 1024;
    const long long ts0 = wa.prof ? clock64() : 0;
    // 32 steps.  The step is issue-bound rather than latency-bound, so chunks whose every
    // cell lies inside the grid (all rows of the strip valid, columns 0 <= j < C - 1) take a
    // body without the activity selects and the last-cell bookkeeping; others take the full
    // one.  Both compute the same values.
    auto steps = [&](auto interior) {
      constexpr bool IN = decltype(interior)::value;
#pragma unroll
      for (int u = 0; u < 32; ++u) {
        // tile reads and the input broadcast do not depend on the previous step
        const double2 ta = T0[(u << 5) + lane];
        const double2 tb = KIND == K_DEC ? T1[(u << 5) + lane] : ta;
        const double lin = __shfl_sync(kFull, inreg, u);
        const double lup = __shfl_up_sync(kFull, carry, 1);
        const double left = lane == 0 ? lin : lup;
        const int j = (c << 5) + u - lane;
        const bool act = IN || (rowv && j >= 0 && j < C);
        double ncarry, nbot, nres;
        if (KIND == K_DEC) {
          // same propagation as the solo cell, written with selects (no divergence)
          const double rLB = ta.x, rUB = ta.y, tLB = tb.x, tUB = tb.y;
          const bool bdead = bot < dthr, ldead = left < dthr;
          const bool rinv = (left > rUB) || ldead;
          const bool tinv = (bot > tUB) || bdead;
          const double rm = dmax(rLB, left);
          const double tm = dmax(tLB, bot);
          ncarry = bdead ? (rinv ? dv : rm) : rLB;
          // the result is the last cell's right edge: on a transposed grid, its top edge
          nres = IN ? 0.0
                    : (tr ? (ldead ? (tinv ? -2.0 : tUB) : tUB)
                          : (bdead ? (rinv ? -2.0 : rUB) : rUB));
          nbot = ldead ? (tinv ? dv : tm) : tLB;
        } else {
          const double in = dmin(left, bot);
          const double top = dmax(ta.x, in);
          const double right = dmax(ta.y, in);
          ncarry = right;
          nbot = top;
          nres = IN ? 0.0 : dmin(top, right);
        }
        carry = act ? ncarry : carry;
        bot = act ? nbot : bot;
        if (!IN && act && last_row && j == C - 1) res = nres;
        // lane olane (31) produced column (c << 5) + u - olane of the strip's last row
        if (lane == olane) out_row[((c << 5) + u - olane) & 63] = carry;
      }
    };
    if (c >= 1 && (c << 5) + 33 <= C && (s + 1) * 32 <= R) steps(std::true_type{});
    else steps(std::false_type{});
    if (wa.prof && lane == 0) {
      atomicAdd(&wa.prof[3], (unsigned long long)(clock64() - ts0));
      atomicAdd(&wa.prof[5], 1ull);
    }
    if (trace && trace_step == 1) {
      trace_step = 2;
      if (lane == 0) trace[4] = global_ns();
    }
    // the next chunk's input words load while this chunk is flushed and the next one set up;
    // issued before the steps, the load slowed every step by about a third
    prefetch(c + 1);
    ++c;
  }
  if (status == 0 && !drop_pending()) status = 1;
  // tell the helpers this strip is over (also after an error: they must not wait forever)
  // and take their acknowledgement
  if (lane == 0) {
    const int slot = seqP & 1;
    *(volatile int*)&sh->req_chunk[slot] = kStop;
    mbar_arrive(&sh->req[slot]);
  }
  __syncwarp();
  ++seqP;
  if (take() < 0) status = 1;

  if (status == 0 && has_cons) {
    if (!dead_tail) {
      while (next_flush < nout) {
        flush(next_flush, true);
        ++next_flush;
      }
    } else {
      publish_cols(C);
    }
    if (!dense && lane == 0 && first_live_out == kNone) {
      atomicMin(&st->dead_from, s + 1);
      if (wa.dyn_items) *(volatile int*)&sh->push_req = 3;  // every later strip is dead too
    }
  }
  if (has_cons && lane == 0) {
    out_prog->wlo = wlo;
    out_prog->whi = whi;
  }
  if (s == S - 1 && last_row) st->result = res;
  if (wa.prof && lane == 0) atomicAdd(&wa.prof[4], (unsigned long long)(clock64() - t0));
  return status;
}

}  // namespace rfd
