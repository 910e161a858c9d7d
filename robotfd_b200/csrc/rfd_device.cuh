// Device side of the wavefront engine (sm_100a, FP64).
//
// One free-space DP (DFD, VE-FD or the reachability decision) of one curve pair is a grid
// of R rows (segments/points of curve 1) by C columns (of curve 2).  Rows are cut into
// strips of 32; one warp owns a strip, lane l owns row 32*s + l and the warp sweeps the
// columns skewed by lane (step t: lane l at column t - l), so the value passed from row
// i-1 to row i moves one lane down per step through a shuffle and the value passed along
// a row stays in a register.  Strip s hands its last row's outputs to strip s+1 through a
// per-pair boundary row in global memory (L2 resident) in chunks of 32 columns, each chunk
// published with a release store of a progress word tagged by the phase epoch.
//
// Work items are (pair, strip) tickets taken in order from one atomic counter per launch,
// so every strip a warp waits on was taken earlier by a running warp: no co-residency
// assumption and no cooperative launch are needed.  Every wait is bounded by a clock
// budget, after which the kernel raises an error word and all warps leave.
//
// Dead regions.  For the decision a boundary value is dead when it is negative
// (unreachable); for the min-max DPs when it exceeds the pruning bound U.  A cell whose
// two inputs are dead produces dead outputs whatever its geometry, so a warp whose whole
// state is dead skips straight to the next live input chunk, and a strip that publishes
// no live value ends every strip below it.  Live values are computed exactly as in the
// dense sweep; min and max are exact, so the results are bit-identical.
#pragma once

#include <cfloat>
#include <climits>
#include <cstdint>

#include "rfd_search.h"

namespace rfd {

constexpr double kFltMax = (double)FLT_MAX;  // "infinity" of the reference DPs
constexpr unsigned kNone = 0xffffffffu;
constexpr unsigned kFull = 0xffffffffu;

enum Kind : int { K_DFD = 0, K_VEFD = 1, K_DEC = 2 };
enum Phase : int {
  PH_DFD = 0,
  PH_VEFD = 1,
  PH_VEFD_DENSE = 2,
  PH_SEARCH = 3,
  PH_DONE = 4,
  PH_BRACKET = 5,  // waiting for the learned bracket
  PH_KWAIT = 6     // k-ary round: this decision is done, the round's others are not
};

// Progress record of a strip's output boundary.
struct Prog {
  unsigned long long word;  // (epoch << 32) | number of leading columns that are final
  unsigned int first_live;  // first chunk holding a live value (kNone while none)
  unsigned int last_live;   // last such chunk
  int wlo, whi;             // chunks of the strip's output row it wrote (wlo > whi: none)
};

// Boundary ring of the DFD strips.  The rows DFD strips hand to each other live in a ring of
// `ring` rows per pair, not one row per strip: strip s writes row s % ring, so their boundary
// memory is O(ring * columns), independent of the number of rows.  A count per strip,
// slots[s], says how many leading columns of its row have been cleared for it.  The reader of
// a row sets each chunk back to "not yet written" (kBndEmpty: a reader takes any other word as
// final) right after reading it and releases the count of the row's next writer every few
// chunks; a writer writes a column only once it is cleared, and its reader trusts a word only
// where its writer's count covers it.  The DFD's strips all run the full width at once, so a
// row is handed on column by column, not as a whole.  (VE-FD and decision strips keep one row
// per strip.)
constexpr unsigned kSlotAll = 0xffffffffu;  // cleared count: every column

struct PairDesc {
  const double* P;        // curve 1, [n1][d]
  const double* Q;        // curve 2, [n2][d]
  const double2* rowc;    // [n1-1]: (|p_{i+1}-p_i|^2, 0.5 / that)
  const double2* colrec;  // [n2-1][RECW(d)]: q_j, q_{j+1}, (|q_{j+1}-q_j|^2, 0.5 / that)
  double* bnd;            // boundary rows: [ring][cstride] (team strips and DFD)
  unsigned int* tags;     // [ring][tstride] epoch tag of every live chunk (team strips)
  Prog* prog;             // [S]
  unsigned long long* slots;  // [S] cleared count of every DFD strip (see Boundary ring)
  // rows of the boundary ring (>= 1; rows never wrap when >= S-1).  DFD strips: see Boundary
  // ring.  Team strips: S - 1 (one row each), or the rows of a launch window plus one.
  int ring;
  // tr: the team strips of a pair whose first curve is the longer run on the transposed
  // grid (rows = curve 2), whose free intervals are the same values (the interval of an edge
  // is the same function of its point and segment in either orientation) with the roles of
  // the right and top edges exchanged
  int n1, n2, d, tr;
  // Meet in the middle (team strips of one pair, run_batch): the forward sweep of a split pair
  // runs its first `split` strips only; the pair's mirror descriptor (split = -(p + 1) for
  // pair p) sweeps the rest of the grid from the far corner, its row r being row mrow - r of
  // the pair's grid (n1 then counts the mirror's rows + 1).  0 for every other descriptor.
  int split, mrow;
  long long cstride, tstride;
};

struct PairState {
  Search srch;
  double U;          // pruning bound of the running min-max DP (squared)
  double seed;       // VE-FD seed: endpoint bound squared
  double r2;         // radius^2 of the running decision
  double split;      // radius of the running decision
  double endpoint, dfd, vefd, result, distance;
  double blo, bhi;   // proposed bracket (NaN when none)
  unsigned long long cells_eval, cells_nominal, cells_fp64, cells_vefd;
  unsigned int epoch;
  int phase, active, quirks, dense, decide_only, flags;
  int dead_from, done_count;
  int use_model;
  int filter;  // 1: decision intervals through the FP32 filter (RFD_PREC_FP32_FILTER)
  int coarse;  // 1: the DFD phase computes the coarse upper bound (rfd_options.coarse_ub)
  int formula;  // decision intervals: 0 the fused path's, 1 the materialised path's (rfd.h)
  int pushed;      // continuous search: queue entries of the running probe so far (<= strips)
  int next_strip;  // continuous search: strips of the running probe taken so far
  unsigned long long t_done;  // %globaltimer (ns) when the pair's search ended (RFD_PROF report)
  // k-ary rounds of the continuous search (rfd_options.search_arity).  A pair with members
  // owns kary_cap extra decision workspaces, whose states are st[kary_base ..]; every state of
  // such a group (the pair's own included) has kary_real = the pair's index.
  int kary_real, kary_base, kary_cap;
  int kary_n;     // the pair: decisions of the running round (0: plain probe)
  int kary_left;  // the pair: decisions of the round still running
  int kary_in;    // this decision belongs to a round
  int kary_reach; // its outcome
  int corner;     // mirror decision: the far corner lies in the free space (see split_sync_kernel)
};

template <int D>
struct RecW {
  static constexpr int value = D == 2 ? 3 : 4;  // double2 per column record
};

struct WaveArgs {
  const PairDesc* pairs;
  PairState* st;
  const int2* items;
  int nitems;
  int phase;
  unsigned int* ticket;
  int* error;
  int* active_pairs;
  long long spin_cycles;
  unsigned long long* prof;  // RFD_PROF=1: cycle counters (see rfd_team.cuh), else null
  // Continuous search (team decision strips, null otherwise): tickets past nitems take the
  // queue entry in slot ticket - nitems: a pair, whose next strip the taker then runs.
  unsigned long long* dyn_items;  // pair index; all ones while not published
  unsigned int* dyn_tail;         // slots reserved so far
  long long dyn_cap;
  // A probe round launched ahead of the continuous search runs only while at least gate_min
  // pairs, or a single one, are active; its fill kernel decides once for the launch (1: run,
  // 2: skip).
  int* gate;
  int gate_min;
  int window;        // continuous search: strips a probe queues at its start, at least,
  int window_teams;  // ... and at least this over the active pairs (a lone pair: its teams)
  int kary_k;        // continuous search: radii per k-ary round (< 2: none)
  int kary_gate;     // ... run while at most this many pairs are active
};

// ------------------------------------------------------------------ memory helpers

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ int ld_volatile(const int* p) { return *(const volatile int*)p; }

// Boundary rows are filled with this pattern before every launch that hands rows between
// strips (a NaN that no DP value takes: arithmetic makes canonical NaNs), so a consumer can
// tell a value written in this launch from an old one without reading a flag first.
constexpr unsigned long long kBndEmpty = ~0ull;

// Relaxed (coherent, unordered) accesses of the handed-over rows.  No ordering with other
// memory accesses is needed, so there is no compiler memory barrier.
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const double* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ void st_relaxed_f64(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v));
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// ------------------------------------------------------------------ cell arithmetic
// Every operation is an explicit round-to-nearest intrinsic, so the result does not
// depend on the compiler's contraction choices; the CPU oracle performs the same ops.
// They restate the reference kernels as nvcc compiles them with its default contraction.

// Sum of squares of t[0..D): the reference's "s = 0.0; s += t*t" loops (DFD .cu:615-619,
// segment lengths .cu:1004-1007 and :1133-1137, VE-FD .cu:381-392) compile with the zero
// start folded away and the first square fused with the second one rounded,
// fma(t0, t0, t1*t1); each later square is fused into the running sum.  (The source-order
// chain fma(t1, t1, t0*t0) misses the reference's own 2D DFD output by one ulp.)
template <int D>
__device__ __forceinline__ double sq_sum(const double* t) {
  static_assert(D >= 2, "two or more coordinates");
  double s = __fma_rn(t[0], t[0], __dmul_rn(t[1], t[1]));
#pragma unroll
  for (int k = 2; k < D; ++k) s = __fma_rn(t[k], t[k], s);
  return s;
}

template <int D>
__device__ __forceinline__ double dist_sq(const double* a, const double* b) {
  double t[D];
#pragma unroll
  for (int k = 0; k < D; ++k) t[k] = __dsub_rn(a[k], b[k]);
  return sq_sum<D>(t);
}

// Squared distance from x to the segment a -> a + ab with ab2 = |ab|^2 (VE-FD weights,
// reference .cu:375-394; the top weight mirrors it with the README direction p_{i+1}-p_i).
template <int D>
__device__ __forceinline__ double pt_seg_sq(const double* x, const double* a, const double* ab,
                                            double ab2) {
  double apab = 0.0;
#pragma unroll
  for (int k = 0; k < D; ++k) apab = __fma_rn(__dsub_rn(x[k], a[k]), ab[k], apab);
  double t = __ddiv_rn(apab, ab2);
  t = fmin(1.0, fmax(0.0, t));
  double dd[D];
#pragma unroll
  for (int k = 0; k < D; ++k) dd[k] = __dsub_rn(x[k], __fma_rn(t, ab[k], a[k]));
  return sq_sum<D>(dd);
}

// Free interval on segment a -> a + di inside the ball of radius^2 r2 around x
// (reference .cu:1175-1230).  Empty: (-1, -2).  mat: the reference's materialised path
// (interval_calculation, .cu:730-742 and :765-776), which forms C as (sum of mi^2) - r2, one
// rounding more than the fused path's chain from -r2; everything else is the same.
template <int D>
__device__ __forceinline__ void free_interval(const double* x, const double* a, const double* di,
                                              double A, double inv2A, double r2, double& lo,
                                              double& hi, bool mat = false) {
  double B = 0.0, Cc = -r2, m[D];
#pragma unroll
  for (int k = 0; k < D; ++k) {
    m[k] = __dsub_rn(a[k], x[k]);
    B = __fma_rn(m[k], di[k], B);
    Cc = __fma_rn(m[k], m[k], Cc);
  }
  if (mat) Cc = __dsub_rn(sq_sum<D>(m), r2);
  B = __dmul_rn(B, 2.0);
  const double disc = __fma_rn(B, B, -__dmul_rn(__dmul_rn(4.0, A), Cc));
  lo = -1.0;
  hi = -2.0;
  if (disc >= 0.0) {
    const double s = __dsqrt_rn(disc);
    const double ta = __dmul_rn(__dsub_rn(-B, s), inv2A);
    const double tb = __dmul_rn(__dadd_rn(-B, s), inv2A);
    const bool invalid = (tb < 0.0) || (ta > 1.0);
    lo = invalid ? -1.0 : fmax(ta, 0.0);
    hi = invalid ? -2.0 : fmin(tb, 1.0);
  }
}

// Compare-and-select minimum / maximum, on the dependency chain of the sweeps in place of
// fmin / fmax (whose NaN handling costs several instructions of latency).  They agree with
// fmin / fmax whenever neither operand is NaN, which holds for every value the sweeps
// propagate from finite coordinates: DFD and VE-FD values are squared distances (a
// degenerate segment clamps its parameter with fmax / fmin, which drop the NaN), and free
// intervals are finished by fmax / fmin in free_interval.  Signs of zero may differ only
// in interval lower bounds, which enter comparisons alone (-0 == +0).
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }

// ------------------------------------------------------------------ per-kind policy

template <int KIND>
__device__ __forceinline__ bool is_dead(double v, double U) {
  if (KIND == K_DEC) return v < 0.0;
  return v > U;
}
template <int KIND>
__device__ __forceinline__ double dead_value() {
  return KIND == K_DEC ? -1.0 : kFltMax;
}

// Per-lane row data.
template <int KIND, int D>
struct RowData {
  double a[D];   // DFD: p_i ; segments: p_i
  double b[D];   // segments: p_{i+1}
  double ab[D];  // segments: p_{i+1} - p_i
  double A, inv2A;
  __device__ __forceinline__ void load(const PairDesc& pd, int i) {
#pragma unroll
    for (int k = 0; k < D; ++k) a[k] = __ldg(pd.P + (size_t)i * D + k);
    if (KIND != K_DFD) {
#pragma unroll
      for (int k = 0; k < D; ++k) {
        b[k] = __ldg(pd.P + (size_t)(i + 1) * D + k);
        ab[k] = __dsub_rn(b[k], a[k]);
      }
      const double2 rc = __ldg(pd.rowc + i);
      A = rc.x;
      inv2A = rc.y;
    }
  }
};

// Column data of one cell: DFD needs point q_j, the segment kinds q_j, q_{j+1} and the
// segment constants.  Loaded one step ahead of use (see run_strip) so that no global load
// sits on the dependent chain of a step.
template <int KIND, int D>
struct ColRec {
  double qa[D], qb[D];
  double A, inv2A;
};

template <int KIND, int D>
__device__ __forceinline__ void load_col(const PairDesc& pd, int j, ColRec<KIND, D>& c) {
  if (KIND == K_DFD) {
#pragma unroll
    for (int k = 0; k < D; ++k) c.qa[k] = __ldg(pd.Q + (size_t)j * D + k);
  } else {
    constexpr int W = RecW<D>::value;
    const double2* rec = pd.colrec + (size_t)j * W;
    if (D == 2) {
      const double2 r0 = __ldg(rec), r1 = __ldg(rec + 1), r2 = __ldg(rec + 2);
      c.qa[0] = r0.x; c.qa[1] = r0.y;
      c.qb[0] = r1.x; c.qb[1] = r1.y;
      c.A = r2.x; c.inv2A = r2.y;
    } else {
      const double2 r0 = __ldg(rec), r1 = __ldg(rec + 1), r2 = __ldg(rec + 2), r3 = __ldg(rec + 3);
      c.qa[0] = r0.x; c.qa[1] = r0.y; c.qa[2] = r1.x;
      c.qb[0] = r1.y; c.qb[1] = r2.x; c.qb[2] = r2.y;
      c.A = r3.x; c.inv2A = r3.y;
    }
  }
}

// One cell.  left: value from row i-1 (same column); bot: running value along row i.
// On return carry holds the value for row i+1 and bot the value for column j+1.
template <int KIND, int D>
__device__ __forceinline__ void cell(const RowData<KIND, D>& row, const ColRec<KIND, D>& col, int i,
                                     int j, double left, double& bot, double& carry, double r2,
                                     double& res, bool last, bool tr = false, bool mat = false) {
  if (KIND == K_DFD) {
    const double dist = dist_sq<D>(row.a, col.qa);
    if (i == 0) {
      if (j == 0) {
        bot = kFltMax;
        left = 0.0;
      } else {
        left = kFltMax;
      }
    } else if (j == 0) {
      bot = kFltMax;
    }
    const double in = fmin(left, bot);
    const double top = fmax(dist, in);
    carry = fmin(top, bot);
    bot = top;
    if (last) res = top;
  } else {
    double qd[D];
#pragma unroll
    for (int k = 0; k < D; ++k) qd[k] = __dsub_rn(col.qb[k], col.qa[k]);
    if (KIND == K_VEFD) {
      const double in = fmin(left, bot);
      const double wr = pt_seg_sq<D>(row.b, col.qa, qd, col.A);    // p_{i+1} vs q_j q_{j+1}
      const double wt = pt_seg_sq<D>(col.qb, row.a, row.ab, row.A); // q_{j+1} vs p_i p_{i+1}
      const double top = fmax(wt, in);
      const double right = fmax(wr, in);
      carry = right;
      bot = top;
      if (last) res = fmin(top, right);
    } else {
      double rLB, rUB, tLB, tUB;
      free_interval<D>(row.b, col.qa, qd, col.A, col.inv2A, r2, rLB, rUB, mat);  // right edge
      free_interval<D>(col.qb, row.a, row.ab, row.A, row.inv2A, r2, tLB, tUB, mat); // top edge
      const double leftLB = left, botLB = bot;
      if (botLB < 0.0) {
        const bool invalid = (leftLB > rUB) || (leftLB < 0.0);
        const double m = fmax(rLB, leftLB);
        rLB = invalid ? -1.0 : m;
        rUB = invalid ? -2.0 : rUB;
      }
      if (leftLB < 0.0) {
        const bool invalid = (botLB > tUB) || (botLB < 0.0);
        const double m = fmax(tLB, botLB);
        tLB = invalid ? -1.0 : m;
        tUB = invalid ? -2.0 : tUB;
      }
      bot = tLB;
      carry = rLB;
      if (last) res = tr ? tUB : rUB;  // transposed grid: the right edge is the top one
    }
  }
}

// ------------------------------------------------------------------ waits

// Self-check of the DFD boundary ring's indices: a failed check records its code in the error
// word (codes from kCheckBase; the call then fails with RFD_ERR_INTERNAL) and the strip does
// not touch the ring.
constexpr int kCheckBase = 16;
__device__ __forceinline__ bool ring_check(const WaveArgs& wa, bool ok, int code) {
  if (!ok) atomicCAS(wa.error, 0, kCheckBase + code);
  return ok;
}

// Broadcast lane 0's value: every value that steers control flow is read by lane 0 only
// and shared, so all 32 lanes always take the same branch around full-mask shuffles.
__device__ __forceinline__ int bcast(int v) { return __shfl_sync(kFull, v, 0); }
__device__ __forceinline__ unsigned bcast(unsigned v) { return __shfl_sync(kFull, v, 0); }
__device__ __forceinline__ unsigned long long bcast(unsigned long long v) {
  return __shfl_sync(kFull, v, 0);
}

struct Waiter {
  long long t0, budget;
  const int* error;
  const int* dead_from;
  int strip;
  __device__ __forceinline__ void start(const WaveArgs& wa, const PairState* st, int s) {
    t0 = clock64();
    budget = wa.spin_cycles;
    error = wa.error;
    dead_from = &st->dead_from;
    strip = s;
  }
  // Warp-uniform.  0: keep waiting, 1: strip known dead (stop), 2: error / timeout.
  __device__ __forceinline__ int check(int iter) {
    int r = 0;
    if ((iter & 15) == 15 && (threadIdx.x & 31) == 0) {
      if (ld_volatile(error)) r = 2;
      else if (ld_volatile(dead_from) <= strip) r = 1;
      else if (clock64() - t0 > budget) {
        atomicExch((int*)error, 1);
        r = 2;
      }
    }
    r = bcast(r);
    if (!r && iter > 64) __nanosleep(iter > 1024 ? 256 : 32);
    return r;
  }
};

// ------------------------------------------------------------------ one strip

struct StripOut {
  unsigned long long evaluated;
  int status;  // 0 ok, 1 error
};

template <int KIND, int D>
__device__ StripOut run_strip(const WaveArgs& wa, const PairDesc& pd, PairState* st, const int s) {
  const int lane = threadIdx.x & 31;
  const int R = KIND == K_DFD ? pd.n1 : pd.n1 - 1;
  const int C = KIND == K_DFD ? pd.n2 : pd.n2 - 1;
  const int S = (R + 31) >> 5;
  const unsigned E = st->epoch;
  const double U = st->U;
  const double r2 = st->r2;
  const bool mat = st->formula == 1;
  const bool dense = KIND == K_DFD || st->dense != 0;  // DFD runs unpruned (U = +inf)
  const bool has_prod = s > 0;
  const bool has_cons = s + 1 < S;

  Prog* in_prog = has_prod ? pd.prog + (s - 1) : nullptr;
  Prog* out_prog = has_cons ? pd.prog + s : nullptr;
  const double* in_bnd = has_prod ? pd.bnd + (size_t)(s - 1) * pd.cstride : nullptr;
  double* out_bnd = has_cons ? pd.bnd + (size_t)s * pd.cstride : nullptr;
  const unsigned* in_tags = has_prod ? pd.tags + (size_t)(s - 1) * pd.tstride : nullptr;
  unsigned* out_tags = has_cons ? pd.tags + (size_t)s * pd.tstride : nullptr;

  StripOut so{0ull, 0};
  Waiter wt;
  wt.start(wa, st, s);

  const int i = (s << 5) + lane;
  const bool rowv = i < R;
  const bool last_row = i == R - 1;
  const int nout = (C + 31) >> 5;  // output / input chunks
  const int nsteps = C + 31;
  double res = KIND == K_DEC ? -2.0 : kFltMax;

  // Known-dead strip: nothing to compute.
  bool dead_tail = !dense && bcast(lane == 0 ? ld_volatile(&st->dead_from) : 0) <= s;

  if (has_cons && lane == 0) {
    out_prog->first_live = kNone;
    out_prog->last_live = 0;
  }

  RowData<KIND, D> row;
  if (rowv) row.load(pd, i);
  double bot;
  if (KIND == K_DEC) bot = i == 0 ? 0.0 : -1.0;
  else if (KIND == K_VEFD) bot = i == 0 ? st->seed : kFltMax;
  else bot = kFltMax;
  double carry = dead_value<KIND>();
  double ob0 = dead_value<KIND>(), ob1 = dead_value<KIND>();
  unsigned first_live_out = kNone;
  int next_flush = 0;
  unsigned long long evaluated = 0;

  // Flush output chunk k (columns [32k, 32k+32)) and publish progress.
  auto flush = [&](int k) {
    const int col = (k << 5) + lane;
    double v = (k & 1) ? ob1 : ob0;
    const bool valid = col < C;
    if (valid) __stcg(out_bnd + col, v);
    const unsigned live = __ballot_sync(kFull, valid && !is_dead<KIND>(v, U));
    if (k & 1) ob1 = dead_value<KIND>();
    else ob0 = dead_value<KIND>();
    __syncwarp();
    if (lane == 0) {
      if (live) {
        __stcg(out_tags + k, E);
        if (first_live_out == kNone) {
          first_live_out = (unsigned)k;
          out_prog->first_live = (unsigned)k;
        }
        out_prog->last_live = (unsigned)k;
      }
      __threadfence();
      const unsigned cols = min((k + 1) << 5, C);
      st_release(&out_prog->word, ((unsigned long long)E << 32) | cols);
    }
  };
  auto publish_cols = [&](int cols) {
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      st_release(&out_prog->word, ((unsigned long long)E << 32) | (unsigned)cols);
    }
  };
  // Wait until the producer has published at least `need` columns; returns the word.
  // Lane 0 polls with acquire semantics and shares the word; the other lanes read the
  // boundary through L2 (ld.cg) after that warp-synchronising broadcast.
  auto wait_cols = [&](unsigned need, unsigned long long& w) -> int {
    for (int it = 0;; ++it) {
      w = bcast(lane == 0 ? ld_acquire(&in_prog->word) : 0ull);
      if ((unsigned)(w >> 32) == E && (unsigned)(w & 0xffffffffu) >= need) return 0;
      const int r = wt.check(it);
      if (r) return r;
    }
  };

  int c = 0;
  while (!dead_tail && (c << 5) < nsteps) {
    if (has_cons)
      while (next_flush <= c - 2) flush(next_flush++);
    // ---- input chunk c (values of row 32s-1 for columns [32c, 32c+32))
    double inreg = dead_value<KIND>();
    bool in_live = false;
    if ((c << 5) < C) {
      if (has_prod) {
        unsigned long long w;
        const int r = wait_cols((unsigned)min((c + 1) << 5, C), w);
        if (r == 2) { so.status = 1; break; }
        if (r == 1) { dead_tail = true; break; }
        const unsigned tg = bcast(lane == 0 ? __ldcg(in_tags + c) : 0u);
        in_live = tg == E;
        if (in_live) {
          const int col = (c << 5) + lane;
          if (col < C) inreg = __ldcg(in_bnd + col);
        }
      } else {
        // row -1: unreachable (decision, reference .cu:656) or FLT_MAX (DPs, .cu:196/:454)
        in_live = !is_dead<KIND>(inreg, U);
      }
    }
    // ---- dead-state skip
    if (!dense && !in_live) {
      const bool ldead = (!rowv || is_dead<KIND>(bot, U) || ((c << 5) - lane >= C)) &&
                         is_dead<KIND>(carry, U);
      if (__all_sync(kFull, ldead)) {
        // next live input chunk after c, or none
        int nc = -1;
        // Past the last input chunk only finishing rows remain: all dead means done.
        if (has_prod && (c << 5) < C) {
          int pos = c + 1;
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
              // scan [pos, end) 32 tags at a time; without a hit every chunk below `end`
              // has been seen, so the next round resumes exactly at `end`
              while (pos < end && nc < 0) {
                const int k = pos + lane;
                const bool hit = k < end && __ldcg(in_tags + k) == E;
                const unsigned b = __ballot_sync(kFull, hit);
                if (b) nc = pos + __ffs(b) - 1;
                else pos = min(pos + 32, end);
              }
            } else {
              pos = max(pos, avail);
            }
            if (nc >= 0 || done) break;
            const int r = wt.check(it);
            if (r == 2) { so.status = 1; break; }
            if (r == 1) break;  // strip known dead: nc stays -1
          }
          if (so.status) break;
        }
        if (has_cons)
          while (next_flush <= c - 1) flush(next_flush++);
        if (nc < 0) {
          dead_tail = true;
          break;
        }
        if (has_cons) {
          next_flush = nc - 1;
          publish_cols(min((nc - 1) << 5, C));
        }
        carry = dead_value<KIND>();
        ob0 = ob1 = dead_value<KIND>();
        c = nc;
        continue;
      }
    }
    // ---- 32 skewed steps; the column record of step t+1 is loaded during step t
    ColRec<KIND, D> cur, nxt;
    load_col<KIND, D>(pd, min(max((c << 5) - lane, 0), C - 1), cur);
#pragma unroll 1
    for (int u = 0; u < 32; ++u) {
      const int t = (c << 5) + u;
      const int j = t - lane;
      load_col<KIND, D>(pd, min(max(j + 1, 0), C - 1), nxt);
      const double lin = __shfl_sync(kFull, inreg, u);
      const double lup = __shfl_up_sync(kFull, carry, 1);
      const double left = lane == 0 ? lin : lup;
      const bool act = rowv && j >= 0 && j < C;
      bool need = act;
      if (!dense) need = act && !(is_dead<KIND>(left, U) && is_dead<KIND>(bot, U));
      if (__any_sync(kFull, need)) {
        if (act) {
          cell<KIND, D>(row, cur, i, j, left, bot, carry, r2, res, last_row && j == C - 1,
                        pd.tr != 0, mat);
          ++evaluated;
        }
      } else if (act) {
        carry = dead_value<KIND>();
        bot = dead_value<KIND>();
      }
      const double o = __shfl_sync(kFull, carry, 31);
      const int jo = t - 31;
      if (jo >= 0 && (jo & 31) == lane) {
        if (jo & 32) ob1 = o;
        else ob0 = o;
      }
      cur = nxt;
    }
    ++c;
  }

  if (so.status == 0 && has_cons) {
    if (!dead_tail) {
      while (next_flush < nout) flush(next_flush++);
    } else {
      publish_cols(C);
    }
    if (!dense && lane == 0 && first_live_out == kNone) atomicMin(&st->dead_from, s + 1);
  }
  if (s == S - 1 && last_row) st->result = res;
  // warp total of evaluated cells
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) evaluated += __shfl_xor_sync(kFull, evaluated, o);
  so.evaluated = evaluated;
  return so;
}

}  // namespace rfd
