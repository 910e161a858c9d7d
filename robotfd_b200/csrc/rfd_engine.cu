// Host orchestration and C ABI of the wavefront engine (librfd.so).
//
// One call solves a batch of pairs (a single pair is a batch of one) with a fixed launch
// sequence on one stream and no host synchronisation until the results are read:
//   prep  : per-segment constants, endpoint bound, state init
//   DFD   : dense min-max DP over the n1 x n2 points            -> ub (reference .cu:1268-1326)
//   VE-FD : min-max DP over the (n1-1) x (n2-1) cells, pruned
//           by DFD^2 (exact, see rfd_device.cuh)               -> lb (reference .cu:1328-1391)
//   VE-FD : dense recomputation for pairs whose pruned pass did not reach the last cell
//   probe : one reachability decision per active pair per launch; the warp that completes a
//           pair's probe applies the outcome and proposes the next radius on the device
//           (reference host loop src/frechet.cpp:36-63)
#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "rfd.h"
#include "rfd_device.cuh"
#include "rfd_dfd.cuh"
#include "rfd_filter.h"
#include "rfd_team.cuh"
#include "rfd_features.cuh"
#include "rfd_mlp.h"

using namespace rfd;

namespace {

constexpr int kBlock = 128;

// Boundary ring rows per pair of the DFD strips, which hand rows on column by column and
// need only a few strips' lag: kPublish chunks plus the publication's latency.
constexpr int kDfdRingRows = 32;
thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
}  // namespace

int rfd_mlp::set_error(int code, const char* msg) {
  g_last_error = msg;
  return code;
}

namespace {

#define RFD_CUDA(call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(e_ == cudaErrorMemoryAllocation ? RFD_ERR_NOMEM : RFD_ERR_CUDA,         \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                    \
  } while (0)

__device__ __forceinline__ void begin_search(PairState* st, int* active_pairs,
                                             bool threshold_first);
__device__ __forceinline__ void next_probe(PairState* st, int* active_pairs);

__device__ __forceinline__ void finish_pair(PairState* st, int* active_pairs) {
  st->t_done = global_ns();
  st->phase = PH_DONE;
  st->active = 0;
  st->distance = (st->srch.ub + st->srch.lb) / 2.0;
  atomicSub(active_pairs, 1);
}

__device__ __forceinline__ void next_probe(PairState* st, int* active_pairs) {
  double eps;
  if (search_next(st->srch, &eps)) {
    st->phase = PH_SEARCH;
    st->split = eps;
    st->r2 = __dmul_rn(eps, eps);  // radius * radius (host product in the reference, .cu:1440)
  } else {
    finish_pair(st, active_pairs);
  }
}

// threshold_first: the bracket comes from the learned network, which is trained on the
// pairs whose distance lies above the stop threshold over VE-FD (the others end at the
// threshold probe, which the search therefore always tries first).
__device__ __forceinline__ void begin_search(PairState* st, int* active_pairs,
                                             bool threshold_first) {
  if (st->vefd > st->dfd) st->flags |= RFD_FLAG_LB_GT_UB;
  search_begin(st->srch, st->vefd, st->dfd, st->blo, st->bhi, threshold_first);
  next_probe(st, active_pairs);
}

template <int KIND>
__device__ void finalize(PairState* st, const PairDesc& pd, int* active_pairs) {
  double r = *(volatile double*)&st->result;
  if (KIND == K_DFD) {
    if (st->coarse) {
      // coarse upper bound: the inflated DFD of the anchors, widened by a margin that covers
      // the roundings of its weights
      const double ub = __dmul_rn(__dsqrt_rn(r), 1.0 + 0x1p-40);
      r = __dmul_rn(ub, ub);
      st->flags |= RFD_FLAG_DFD_COARSE;
    }
    st->dfd = __dsqrt_rn(r);  // reference .cu:633
    if (pd.n1 < 2 || pd.n2 < 2) {
      // one-point curve: every coupling maps the other curve onto that point
      st->vefd = st->dfd;
      st->srch.lb = st->srch.ub = st->dfd;
      st->flags |= RFD_FLAG_DEGENERATE;
      finish_pair(st, active_pairs);
    } else {
      const int prod = (int)((unsigned)pd.n1 * (unsigned)pd.n2);  // int product, .cu:1343
      if (st->quirks && prod <= 10000) {
        st->vefd = st->endpoint;
        st->flags |= RFD_FLAG_VEFD_SKIPPED;
        if (st->use_model) st->phase = PH_BRACKET;
        else begin_search(st, active_pairs, false);
      } else {
        st->phase = PH_VEFD;
        // VE-FD <= CFD <= DFD; the margin absorbs rounding when they coincide.
        st->U = st->dense ? (double)INFINITY : __dmul_rn(r, 1.0 + 0x1p-30);
      }
    }
  } else if (KIND == K_VEFD) {
    if (!(r <= st->U)) {
      st->phase = PH_VEFD_DENSE;
      st->U = (double)INFINITY;
      st->flags |= RFD_FLAG_VEFD_DENSE;
    } else {
      st->vefd = __dsqrt_rn(r);  // reference .cu:427
      if (st->use_model) st->phase = PH_BRACKET;
      else begin_search(st, active_pairs, false);
    }
  } else {
    st->cells_nominal += (unsigned long long)(pd.n1 - 1) * (unsigned long long)(pd.n2 - 1);
    st->result = r;
    if (st->decide_only) {
      st->srch.probes += 1;
      st->phase = PH_DONE;
      st->active = 0;
      atomicSub(active_pairs, 1);
    } else if (st->kary_in) {
      // one decision of a k-ary round: its outcome waits for the round's others (kary_done)
      st->kary_reach = r == 1.0;
      st->kary_in = 0;
      st->phase = PH_KWAIT;
    } else {
      search_update(st->srch, st->split, r == 1.0);  // reference .cu:1592, frechet.cpp:80-85
      next_probe(st, active_pairs);
    }
  }
  st->epoch += 1;
  st->done_count = 0;
  st->dead_from = INT_MAX;
}

template <int KIND>
__global__ void __launch_bounds__(kBlock) wave_kernel(WaveArgs wa) {
  const int lane = threadIdx.x & 31;
  if (bcast(lane == 0 ? ld_volatile(wa.active_pairs) : 0) == 0) return;
  for (;;) {
    unsigned t = 0;
    int err = 0;
    if (lane == 0) {
      t = atomicAdd(wa.ticket, 1u);
      err = ld_volatile(wa.error);
    }
    t = bcast(t);
    if ((int)t >= wa.nitems || bcast(err)) return;
    const int2 it = wa.items[t];
    PairState* st = wa.st + it.x;
    const int ok = lane == 0 ? (ld_volatile(&st->phase) == wa.phase && ld_volatile(&st->active)) : 0;
    if (!bcast(ok)) continue;
    const PairDesc pd = wa.pairs[it.x];
    const int R = KIND == K_DFD ? pd.n1 : pd.n1 - 1;
    const int S = (R + 31) >> 5;
    if (it.y >= S) continue;
    const StripOut so =
        pd.d == 2 ? run_strip<KIND, 2>(wa, pd, st, it.y) : run_strip<KIND, 3>(wa, pd, st, it.y);
    if (so.status) return;
    __syncwarp();
    if (lane == 0) {
      if (KIND == K_DEC && so.evaluated) atomicAdd(&st->cells_eval, so.evaluated);
      if (KIND == K_VEFD && so.evaluated) atomicAdd(&st->cells_vefd, so.evaluated);
      __threadfence();
      const int n = atomicAdd(&st->done_count, 1);
      if (n == S - 1) {
        __threadfence();
        finalize<KIND>(st, pd, wa.active_pairs);
        __threadfence();
      }
    }
  }
}

// Coarse upper bound (rfd_options.coarse_ub = k), step 1: the anchors (every k-th point
// and the last) of both curves into the coarse pair's arrays, with an inflation as extra
// coordinate.  The interior points of the block between anchors lo and hi split at the
// middle index into a prefix, charged to lo, and a suffix, charged to hi; an anchor's
// inflation is the larger of the radius of the suffix before it (largest distance of a
// suffix point to the anchor) and of the prefix after it.  A monotone coupling of the anchors
// extends block by block to the full point sequences: on a step that advances one curve, its
// prefix points pair with the anchor that stays and its suffix points with the same anchor
// again, now coupled to the next anchor; on a diagonal step prefixes pair with prefixes, then
// suffixes with suffixes.  Every full pair then lies within |a - b| + inflation(a) +
// inflation(b) of a coupled anchor pair (a, b), so the DFD of the anchors with those cell
// weights, squared, is at least the DFD of the curves.  One block per pair (grid-stride);
// pairs with coarse = 0 keep the DFD.
__global__ void coarse_prep_kernel(const PairDesc* pairs, const PairDesc* coarse, PairState* st,
                                   int npairs, int k) {
  for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
    // a pair with a one-point curve (coarse = 0): every point, inflation 0, so the inflated
    // sweep computes its exact DFD
    const bool exact = !st[p].coarse;
    const PairDesc pd = pairs[p], cd = coarse[p];
    const int d = pd.d, ds = d + 1;
    for (int side = 0; side < 2; ++side) {
      const double* X = side ? pd.Q : pd.P;
      double* Y = const_cast<double*>(side ? cd.Q : cd.P);
      const long long n = side ? pd.n2 : pd.n1, cn = side ? cd.n2 : cd.n1;
      auto anchor = [&](long long a) { return exact ? a : (a == cn - 1 ? n - 1 : a * k); };
      // squared distance of point i to point j
      auto dist2 = [&](long long i, long long j) {
        double m = 0.0;
        for (int e = 0; e < d; ++e) {
          const double t = __dsub_rn(X[i * d + e], X[j * d + e]);
          m = __fma_rn(t, t, m);
        }
        return m;
      };
      // block b (anchors b, b+1): the radius of its prefix around its first anchor (head) or
      // of its suffix around its last anchor (tail)
      auto block_radius = [&](long long b, bool tail) {
        const long long lo = anchor(b), hi = anchor(b + 1), mid = lo + (hi - lo) / 2;
        double m = 0.0;
        if (tail) {
          for (long long i = mid + 1; i < hi; ++i) m = fmax(m, dist2(i, hi));
        } else {
          for (long long i = lo + 1; i <= mid && i < hi; ++i) m = fmax(m, dist2(i, lo));
        }
        return __dsqrt_rn(m);
      };
      // each anchor: its coordinates and its inflation (each block's radii are computed by
      // its own two anchors: no thread reads another's result)
      for (long long a = threadIdx.x; a < cn; a += blockDim.x) {
        const long long at = anchor(a);
        for (int e = 0; e < d; ++e) Y[a * ds + e] = X[at * d + e];
        const double before = !exact && a > 0 ? block_radius(a - 1, true) : 0.0;
        const double after = !exact && a + 1 < cn ? block_radius(a, false) : 0.0;
        Y[a * ds + d] = fmax(before, after);
      }
    }
  }
}

// drop_repeats on device-memory curves (rfd_options.drop_repeats): point k is kept unless
// every coordinate equals point k-1's, as same_point on the host.
struct SrcCurve {
  const double* src;  // the caller's curve
  double* dst;        // its kept points, in the workspace
  long long n;        // the caller's point count
  int d, pad;
};
__device__ __forceinline__ bool same_point_dev(const double* a, const double* b, int d) {
  for (int e = 0; e < d; ++e)
    if (!(a[e] == b[e])) return false;
  return true;
}

// Points kept per curve.  One block of 256 per curve (grid-stride).
__global__ void __launch_bounds__(256) count_kept_kernel(const SrcCurve* cs, int ncurves,
                                                         long long* kept) {
  __shared__ long long part[8];
  for (int c = blockIdx.x; c < ncurves; c += gridDim.x) {
    const SrcCurve sc = cs[c];
    long long m = 0;
    for (long long k = 1 + threadIdx.x; k < sc.n; k += blockDim.x)
      m += !same_point_dev(sc.src + (k - 1) * sc.d, sc.src + k * sc.d, sc.d);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m += __shfl_xor_sync(kFull, m, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      long long t = sc.n > 0 ? 1 : 0;
      for (int w = 0; w < 8; ++w) t += part[w];
      kept[c] = t;
    }
    __syncthreads();
  }
}

// The kept points, in order, into the workspace: tiles of 256 points, each point's place the
// tile's running count plus a block scan of the keep flags.  One block of 256 per curve.
__global__ void __launch_bounds__(256) compact_kept_kernel(const SrcCurve* cs, int ncurves) {
  __shared__ int warp_tot[8];
  __shared__ long long base;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = blockIdx.x; c < ncurves; c += gridDim.x) {
    const SrcCurve sc = cs[c];
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    for (long long t0 = 0; t0 < sc.n; t0 += 256) {
      const long long k = t0 + threadIdx.x;
      const bool keep =
          k < sc.n && (k == 0 || !same_point_dev(sc.src + (k - 1) * sc.d, sc.src + k * sc.d, sc.d));
      const unsigned b = __ballot_sync(kFull, keep);
      if (lane == 0) warp_tot[warp] = __popc(b);
      __syncthreads();
      int before = 0;
      for (int w = 0; w < warp; ++w) before += warp_tot[w];
      if (keep) {
        const long long at = base + before + __popc(b & ((1u << lane) - 1u));
        for (int e = 0; e < sc.d; ++e) sc.dst[at * sc.d + e] = sc.src[k * sc.d + e];
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < 8; ++w) tot += warp_tot[w];
        base += tot;
      }
      __syncthreads();
    }
  }
}

// Marks the rows the DFD strips of 32*K rows hand to each other as not yet written (the
// all-ones pattern, a NaN no DFD value takes).  Pairs are spread over grid rows (y) and
// each pair's rows over grid columns (x), so one large pair uses every SM.
__global__ void dfd_fill_kernel(const PairDesc* pairs, int npairs, int rows_per_strip) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (int p = blockIdx.y; p < npairs; p += gridDim.y) {
    const PairDesc pd = pairs[p];
    const long long S = (pd.n1 + rows_per_strip - 1) / rows_per_strip;
    if (S < 2) continue;
    const long long rows = min(S - 1, (long long)pd.ring);
    // cstride is a multiple of 32 doubles and bnd 256-byte aligned: 16-byte stores
    ulonglong2* b = reinterpret_cast<ulonglong2*>(pd.bnd);
    const long long n = rows * pd.cstride / 2;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride)
      b[k] = make_ulonglong2(kBndEmpty, kBndEmpty);
    // cleared counts: the first `ring` strips write fresh rows (every column cleared), the
    // others wait for their row's previous reader
    if (blockIdx.x == 0)
      for (long long k = threadIdx.x; k < S; k += blockDim.x)
        pd.slots[k] = k < pd.ring ? kSlotAll : 0ull;
  }
}

// Marks the boundary rows of the 32-row strips of every pair about to run `phase` as not
// yet written (VE-FD and decision launches; see kBndEmpty).  Grid as dfd_fill_kernel.
// A gated probe round (WaveArgs.gate): the first block to look decides for the whole launch
// whether enough pairs are still active (or a single one, which gains nothing from the
// queue); true to run.  A skipped round does no work, so the rounds after it skip too.
__device__ bool gate_open(int* gate, const int* active, int gate_min) {
  int d = ld_volatile(gate);
  if (d == 0) {
    const int a = ld_volatile(active);
    atomicCAS(gate, 0, (a >= gate_min || a == 1) ? 1 : 2);
    d = ld_volatile(gate);
  }
  return d == 1;
}

__global__ void bnd_fill_kernel(const PairDesc* pairs, const PairState* st, int npairs, int phase,
                                int* gate, const int* active, int gate_min) {
  if (gate) {
    __shared__ int open;
    if (threadIdx.x == 0) open = gate_open(gate, active, gate_min);
    __syncthreads();
    if (!open) return;
  }
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (int p = blockIdx.y; p < npairs; p += gridDim.y) {
    if (st[p].phase != phase || !st[p].active) continue;
    const PairDesc pd = pairs[p];
    const long long S = (pd.n1 - 1 + 31) / 32;
    // a split pair's forward and mirror sweeps: every row of the ring (the mirror's last
    // strip hands a row to the meet kernel)
    const bool meet = pd.split != 0;
    if (S < 2 && !meet) continue;
    ulonglong2* b = reinterpret_cast<ulonglong2*>(pd.bnd);
    const long long n = (meet ? (long long)pd.ring : S - 1) * pd.cstride / 2;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride)
      b[k] = make_ulonglong2(kBndEmpty, kBndEmpty);
  }
}

// The k-ary members' boundary rows (descriptors first .. first + count - 1) to the
// "not yet written" pattern, before the continuous search.
__global__ void member_fill_kernel(const PairDesc* pairs, int first, int count) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (int v = blockIdx.y; v < count; v += gridDim.y) {
    const PairDesc pd = pairs[first + v];
    const long long S = (pd.n1 - 1 + 31) / 32;
    if (S < 2) continue;
    unsigned long long* b = reinterpret_cast<unsigned long long*>(pd.bnd);
    const long long n = (S - 1) * pd.cstride;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride)
      b[k] = kBndEmpty;
  }
}

// Launch windows of the team strips (O(n+m) boundary memory): strips s0 .. s0+count-1 of
// every pair about to run `phase` write ring rows s % ring; those rows go back to "not yet
// written" and their tags to 0 (no epoch is 0) before the window's launch.  The ring has at
// least count + 1 rows, so the row the window's first strip reads - written by strip s0 - 1
// in the previous window, which has ended - is not among them.  Pairs over grid rows (y),
// each pair's rows over grid columns (x).
__global__ void team_window_fill_kernel(const PairDesc* pairs, const PairState* st, int npairs,
                                        int phase, int s0, int count) {
  for (int p = blockIdx.y; p < npairs; p += gridDim.y) {
    if (st[p].phase != phase || !st[p].active) continue;
    const PairDesc pd = pairs[p];
    const int S = (pd.n1 - 1 + 31) / 32;
    // strips with a consumer write a row: all S - 1 of them, a split pair's forward half all
    // its `split` strips, a mirror (split < 0) all S
    const int s1 = min(s0 + count, pd.split > 0 ? pd.split : (pd.split < 0 ? S : S - 1));
    for (int s = s0 + (int)blockIdx.x; s < s1; s += gridDim.x) {
      const long long r = s % pd.ring;
      // cstride is a multiple of 32 doubles and bnd 256-byte aligned: 16-byte stores
      ulonglong2* b = reinterpret_cast<ulonglong2*>(pd.bnd + r * pd.cstride);
      for (long long k = threadIdx.x; k < pd.cstride / 2; k += blockDim.x)
        b[k] = make_ulonglong2(kBndEmpty, kBndEmpty);
      unsigned* t = pd.tags + r * pd.tstride;
      for (long long k = threadIdx.x; k < pd.tstride; k += blockDim.x) t[k] = 0u;
    }
  }
}

// Dense DFD strips of 32*K rows (rfd_dfd.cuh), same in-order ticket scheme as wave_kernel
// over the (pair, 32-row strip) item list: item (p, s) is strip s of 32*K rows, items past
// the pair's last tall strip are skipped.
template <int K, bool SKEW, bool INFL = false>
__global__ void __launch_bounds__(kBlock) dfd_kernel(WaveArgs wa) {
  __shared__ double ring[kBlock / 32][(INFL ? 4 : 3) * DfdRing<K>::cols];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (bcast(lane == 0 ? ld_volatile(wa.active_pairs) : 0) == 0) return;
  for (;;) {
    unsigned t = 0;
    int err = 0;
    if (lane == 0) {
      t = atomicAdd(wa.ticket, 1u);
      err = ld_volatile(wa.error);
    }
    t = bcast(t);
    if ((int)t >= wa.nitems || bcast(err)) return;
    const int2 it = wa.items[t];
    PairState* st = wa.st + it.x;
    const int ok = lane == 0 ? (ld_volatile(&st->phase) == PH_DFD && ld_volatile(&st->active)) : 0;
    if (!bcast(ok)) continue;
    const PairDesc pd = wa.pairs[it.x];
    const int S = (pd.n1 + 32 * K - 1) / (32 * K);
    if (it.y >= S) continue;
    const int status = pd.d == 2 ? dfd_strip<2, K, SKEW, INFL>(wa, pd, st, it.y, ring[warp])
                                 : dfd_strip<3, K, SKEW, INFL>(wa, pd, st, it.y, ring[warp]);
    if (status) return;
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      const int n = atomicAdd(&st->done_count, 1);
      if (n == S - 1) {
        __threadfence();
        finalize<K_DFD>(st, pd, wa.active_pairs);
        __threadfence();
      }
    }
  }
}

// Continuous search: waits (bounded) for queue slot k to be published and returns its pair
// index; -1 when every pair is done, on an error, or when the wait runs out (which sets the
// error word).
__device__ int wait_dyn_item(const WaveArgs& wa, long long k) {
  const long long t0 = clock64();
  for (int it = 0;; ++it) {
    const unsigned long long v = ld_acquire(wa.dyn_items + k);
    if (v != ~0ull) return (int)(unsigned)v;
    if ((it & 15) == 15) {
      if (ld_volatile(wa.active_pairs) == 0 || ld_volatile(wa.error)) return -1;
      if (clock64() - t0 > wa.spin_cycles) {
        atomicExch(wa.error, 1);
        return -1;
      }
    }
    if (it > 64) __nanosleep(it > 1024 ? 256 : 32);
  }
}

// Continuous search: the probe's counters from zero, then its first strips: wa.window, or
// more while few pairs share the teams (a lone pair queues as many strips as there are
// teams, as a launch's item list would).
__device__ void start_probe(const WaveArgs& wa, PairState* st, int p, int S) {
  st->next_strip = 0;
  st->pushed = 0;
  __threadfence();
  queue_strips(wa, st, p, S,
               max(wa.window, wa.window_teams / max(1, ld_volatile(wa.active_pairs))));
}

// ---- k-ary rounds of the continuous search (rfd_options.search_arity)
//
// A pair with members (extra decision workspaces, st[kary_base ..]) decides, once few pairs
// remain and its search is plain bisection, n radii per round that split (lb, ub) into n + 1
// equal parts; the round's last decision to end combines the outcomes (kary_done): the
// smallest reachable radius is the new ub, the largest unreachable one below it the new lb.
// Every decision is the same function of its radius as a bisection probe's.
constexpr int kMaxArity = RFD_MAX_ARITY;

__device__ PairState* kary_member(const WaveArgs& wa, PairState* g, int m) {
  return m == 0 ? g : wa.st + g->kary_base + (m - 1);
}

// Sets up pair g's next probe (phase PH_SEARCH, split set by next_probe): a k-ary round's
// members get their radii and states; returns the decisions of the round (1: one decision at
// the split).  Queues nothing: a launch round takes the members' strips from its item list,
// the continuous search queues them (start_next).  One thread.
__device__ int kary_arm(const WaveArgs& wa, PairState* g) {
  int n = 1;
  if (g->kary_cap > 0 && wa.kary_k >= 2 && g->srch.mode == SM_BISECT &&
      ld_volatile(wa.active_pairs) <= wa.kary_gate) {
    // the widest round whose decisions still close the gap within the probe cap: halvings
    // left h (against the stop width at lb, which the final ub cannot undercut), rounds of n
    // radii take ceil(h / log2(n + 1)) of them
    const Search& q = g->srch;
    const double w = q.stop_mode == 0 ? q.tol : q.tol * q.lb;
    const double h = w > 0.0 ? ceil(log2(fmax((q.ub - q.lb) / w, 1.0))) : 64.0;
    const int budget = q.max_probes - q.probes;
    for (n = min(wa.kary_k, g->kary_cap + 1); n >= 2; --n)
      if (ceil(h / log2((double)(n + 1))) * n <= (double)budget) break;
    n = max(n, 1);
  }
  double r[kMaxArity];
  int m = 0;
  if (n >= 2) {
    // n radii strictly inside (lb, ub) and increasing (fewer where doubles run out)
    double prev = g->srch.lb;
    for (int i = 1; i <= n; ++i) {
      const double x = g->srch.lb + (g->srch.ub - g->srch.lb) * ((double)i / (double)(n + 1));
      if (x > prev && x < g->srch.ub) r[m++] = prev = x;
    }
  }
  if (m < 2) return 1;
  g->kary_n = m;
  g->kary_left = m;
  for (int k = 0; k < m; ++k) {
    PairState* ms = kary_member(wa, g, k);
    ms->split = r[k];
    ms->r2 = __dmul_rn(r[k], r[k]);
    ms->kary_in = 1;
    ms->phase = PH_SEARCH;
    ms->active = 1;
  }
  __threadfence();
  return m;
}

// Continuous search: queues the first strips of every decision of pair p's armed probe.
__device__ void start_armed(const WaveArgs& wa, PairState* g, int p, int S) {
  if (g->kary_n < 2) {
    start_probe(wa, g, p, S);
    return;
  }
  for (int k = 0; k < g->kary_n; ++k)
    start_probe(wa, kary_member(wa, g, k), k == 0 ? p : g->kary_base + (k - 1), S);
}

// Continuous search: arms and starts pair p's next probe.  One thread.
__device__ void start_next(const WaveArgs& wa, PairState* g, int p, int S) {
  kary_arm(wa, g);
  start_armed(wa, g, p, S);
}

// A decision of a k-ary round ended (in the continuous search, its boundary words are cleared);
// the round's last one combines the outcomes and arms the pair's next probe, and in the
// continuous search (queue) starts it.  One thread.
__device__ void kary_done(const WaveArgs& wa, PairState* ms, int S, bool queue) {
  const int p = ms->kary_real;
  PairState* g = wa.st + p;
  __threadfence();
  if (atomicSub(&g->kary_left, 1) != 1) return;
  __threadfence();
  const int n = g->kary_n;
  double ub = g->srch.ub, lb = g->srch.lb;
  for (int k = 0; k < n; ++k) {
    const PairState* m = kary_member(wa, g, k);
    if (ld_volatile(&m->kary_reach) && m->split < ub) ub = m->split;
  }
  for (int k = 0; k < n; ++k) {
    const PairState* m = kary_member(wa, g, k);
    if (!ld_volatile(&m->kary_reach) && m->split < ub && m->split > lb) lb = m->split;
  }
  for (int k = 1; k < n; ++k) {
    PairState* m = kary_member(wa, g, k);
    g->cells_eval += m->cells_eval;
    g->cells_fp64 += m->cells_fp64;
    g->cells_nominal += m->cells_nominal;
    m->cells_eval = m->cells_fp64 = m->cells_nominal = 0;
  }
  g->srch.lb = lb;
  g->srch.ub = ub;
  g->srch.probes += n;
  g->kary_n = 0;
  next_probe(g, wa.active_pairs);
  if (g->phase == PH_SEARCH && g->active) {
    if (queue) start_next(wa, g, p, S);
    else kary_arm(wa, g);
  }
}

// Continuous search: the first strips of every pair in the search phase.
__global__ void search_queue_init_kernel(const PairDesc* pairs, PairState* st, int npairs,
                                         WaveArgs wa) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npairs; p += gridDim.x * blockDim.x) {
    if (st[p].phase != PH_SEARCH || !st[p].active) continue;
    start_armed(wa, st + p, p, (pairs[p].n1 - 1 + 31) >> 5);
  }
}

// VE-FD and decision strips with the geometry computed off the dependency chain
// (rfd_team.cuh): one CTA per strip, warp 0 propagates, warps 1..7 fill tiles.
//
// Continuous search (wa.dyn_items set, decisions): one launch runs every probe of every pair.
// Strips come from a queue.  A probe starts with a few strips queued (start_probe), and
// each strip queues one more when the band reaches it (its first live input), or when it ends
// without live input (then every later strip is dead: it queues all of them).  A pair so keeps
// queued about the strips its wavefront is about to need, and waiting strips hold few
// teams.  The CTA whose strip ends a pair's probe clears the boundary words the probe's
// strips wrote (each strip records its written chunk range), then starts the next probe: a
// pair starts its next probe as soon as its last one ends, not after every pair's.
// MIR: the mirror halves of split pairs (meet in the middle), a kernel of their own so that
// the forward kernel's registers stay as they are; it runs beside the forward kernel, on
// another stream, each on half the teams.
template <int KIND, int NW = kTeamThreads / 32, bool MIR = false>
__global__ void __launch_bounds__(NW * 32, NW == 8 ? 2 : 1) team_kernel(WaveArgs wa) {
  constexpr int H = NW - 1;  // helper warps
  extern __shared__ __align__(128) unsigned char team_smem[];
  TeamShared* sh = (TeamShared*)team_smem;
  double2* tiles = (double2*)(team_smem + kTeamHeader);
  double* stage = (double*)(team_smem + kTeamHeader + 2 * TileT<KIND>::slot_bytes);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int k = 0; k < 2; ++k) {
      mbar_init(&sh->full[k], H);
      mbar_init(&sh->req[k], 1);
    }
    mbar_init(&sh->staged, H);
  }
  __syncthreads();
  unsigned seqP = 0, seqC = 0, seqH = 0, seqS = 0;
  for (;;) {
    if (threadIdx.x == 0) {
      int go = 0, quit = 0;
      if (ld_volatile(wa.active_pairs) == 0 || ld_volatile(wa.error) ||
          (wa.gate && ld_volatile(wa.gate) != 1)) {
        quit = 1;
      } else {
        const unsigned t = atomicAdd(wa.ticket, 1u);
        int2 it = make_int2(-1, -1);
        if ((int)t < wa.nitems) {
          it = wa.items[t];
        } else if (KIND == K_DEC && wa.dyn_items && (long long)t - wa.nitems < wa.dyn_cap) {
          it.x = wait_dyn_item(wa, (long long)t - wa.nitems);
          if (it.x >= 0) it.y = atomicAdd(&wa.st[it.x].next_strip, 1);
        }
        if (it.x < 0) {
          quit = 1;
        } else {
          PairState* st = wa.st + it.x;
          const int S = (wa.pairs[it.x].n1 - 1 + 31) >> 5;
          if (ld_volatile(&st->phase) == wa.phase && ld_volatile(&st->active) && it.y < S) {
            go = 1;
            sh->item_pair = it.x;
            sh->item_strip = it.y;
          }
        }
      }
      sh->go = go;
      sh->quit = quit;
      sh->push_req = 0;
      sh->evaluated = 0ull;
      sh->evaluated64 = 0ull;
      sh->status = 0;
    }
    __syncthreads();
    const int go = sh->go, quit = sh->quit, p = sh->item_pair, s = sh->item_strip;
    __syncthreads();
    if (quit) break;
    if (!go) continue;
    const PairDesc pd = wa.pairs[p];
    PairState* st = wa.st + p;
    if (warp == 0) {
      const int status =
          pd.d == 2 ? team_propagator<KIND, 2, MIR>(wa, pd, st, s, sh, tiles, seqP, seqC)
                    : team_propagator<KIND, 3, MIR>(wa, pd, st, s, sh, tiles, seqP, seqC);
      if (lane == 0) sh->status = status;
    } else {
      if (pd.d == 2) team_helpers<KIND, 2, H, MIR>(wa, pd, st, s, sh, tiles, stage, seqH, seqS, warp - 1);
      else team_helpers<KIND, 3, H, MIR>(wa, pd, st, s, sh, tiles, stage, seqH, seqS, warp - 1);
    }
    __syncthreads();
    const int S = (pd.n1 - 1 + 31) >> 5;
    const bool dyn = KIND == K_DEC && wa.dyn_items != nullptr;
    if (threadIdx.x == 0) {
      sh->push = 0;
      if (sh->status == 0) {
        const unsigned long long ev = sh->evaluated;
        if (ev) atomicAdd(KIND == K_DEC ? &st->cells_eval : &st->cells_vefd, ev);
        if (KIND == K_DEC && sh->evaluated64) atomicAdd(&st->cells_fp64, sh->evaluated64);
        // the strip's queue entry if its band start did not queue it (all the rest for a
        // strip without live input), before the strip counts as done: the probe's last
        // strip then finds every strip queued
        if (dyn && sh->push_req != 2) queue_strips(wa, st, p, S, sh->push_req == 3 ? S : 1);
        __threadfence();
        const int n = atomicAdd(&st->done_count, 1);
        // (the halves of a split pair, split != 0, end in split_meet_kernel instead; read
        // from the descriptor here, not kept in registers across the strip)
        if (n == S - 1 && !MIR && !ld_volatile(&wa.pairs[p].split)) {
          __threadfence();
          finalize<KIND>(st, pd, wa.active_pairs);
          __threadfence();
          if (dyn && st->phase == PH_SEARCH && st->active) sh->push = 1;
          else if (dyn && st->phase == PH_KWAIT) sh->push = 2;
          // launch rounds: the next launch runs what is armed here (its fill resets the rows)
          else if (KIND == K_DEC && !dyn && st->phase == PH_KWAIT) kary_done(wa, st, S, false);
          else if (KIND == K_DEC && !dyn && st->phase == PH_SEARCH && st->active &&
                   st->kary_cap > 0)
            kary_arm(wa, st);
        }
      }
    }
    __syncthreads();
    if (KIND == K_DEC && sh->push) {
      // the probe's written boundary words back to "not yet written", one strip per warp
      const long long C = pd.n2 - 1;
      for (int r = warp; r < S - 1; r += NW) {
        const int lo = pd.prog[r].wlo, hi = pd.prog[r].whi;
        double* row = pd.bnd + (size_t)r * pd.cstride;
        const long long end = min((long long)(hi + 1) << 5, C);
        for (long long w = ((long long)lo << 5) + lane; lo <= hi && w < end; w += 32)
          reinterpret_cast<unsigned long long*>(row)[w] = kBndEmpty;
      }
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) {
        if (sh->push == 1) start_next(wa, st, p, S);
        else kary_done(wa, st, S, true);
      }
    }
  }
}

// ---- meet in the middle (one pair's VE-FD and search decisions)
//
// A split pair's forward sweep runs its first k strips (grid rows 0 .. 32k - 1) and its mirror
// sweep (rfd_team.cuh, mirror_interval) the other rows from the far corner, both in the same
// launch, each a chain half as long.  Every monotone path crosses the boundary between rows
// 32k - 1 and 32k exactly once, through one edge b of it; the forward sweep's last strip hands
// over, for each b, the value entering the rows above and the mirror's last strip the value
// of the rest of the path through the same edge.  split_meet_kernel combines them:
//   VE-FD: min over b of max(forward, mirror) - the min-max over all paths, split at the
//          crossing (the same doubles, combined by exact min and max);
//   decision: reachable iff for some b the forward reachable part [F, ub] and the co-reachable
//          part [lb, -M] of edge b meet, F <= -M (exact comparisons of the same doubles).
// Both equal what the unsplit sweep computes.  The decision's right UB is not formed (the
// search needs only reachable or not), so rfd_decide never splits.

// The far corner of a split pair's mirror: VE-FD starts from min(w_top, w_right) of the last
// cell, which the forward sweep's last step adds; the decision from the last cell's right
// edge (top edge on a transposed grid) when its free interval reaches the corner (upper end
// 1.0), the condition under which the forward sweep reports reachable.  Same functions and
// operands as the forward sweep's tile of that cell.  One thread.
template <int D>
__device__ void split_corner(const PairDesc& pd, PairState* m, const PairState* g, bool dec) {
  const int R = pd.n1 - 1, C = pd.n2 - 1;
  RowData<K_DEC, D> row;
  row.load(pd, R - 1);
  ColRec<K_DEC, D> col;
  load_col<K_DEC, D>(pd, C - 1, col);
  double qd[D];
#pragma unroll
  for (int k = 0; k < D; ++k) qd[k] = __dsub_rn(col.qb[k], col.qa[k]);
  if (!dec) {
    const double wr = pt_seg_sq<D>(row.b, col.qa, qd, col.A);
    const double wt = pt_seg_sq<D>(col.qb, row.a, row.ab, row.A);
    m->seed = dmin(wt, wr);
  } else {
    double lo, hi;
    const bool mat = g->formula == 1;
    if (pd.tr) free_interval<D>(col.qb, row.a, row.ab, row.A, row.inv2A, g->r2, lo, hi, mat);
    else free_interval<D>(row.b, col.qa, qd, col.A, col.inv2A, g->r2, lo, hi, mat);
    m->corner = hi == 1.0;
  }
}

// Mirror m of pair p before a team launch: it follows the pair's running phase - radius,
// pruning bound, epoch, options - with fresh counters and its far corner set up; idle when
// the pair does not run the phase.
__device__ void split_sync_one(const PairDesc* pairs, PairState* sts, int p, int m, int phase) {
  const PairState* g = sts + p;
  PairState* ms = sts + m;
  const bool run = g->phase == phase && g->active;
  ms->active = run ? 1 : 0;
  ms->phase = run ? phase : PH_DONE;
  if (!run) return;
  ms->r2 = g->r2;
  ms->split = g->split;
  ms->U = g->U;
  ms->epoch = g->epoch;
  ms->dense = g->dense;
  ms->filter = g->filter;
  ms->formula = g->formula;
  ms->done_count = 0;
  ms->dead_from = INT_MAX;
  const PairDesc pd = pairs[p];
  const bool dec = phase == PH_SEARCH;
  if (pd.d == 2) split_corner<2>(pd, ms, g, dec);
  else split_corner<3>(pd, ms, g, dec);
  __threadfence();
}

// Before each team launch with split pairs: every mirror (descriptors mbase .. mbase + nm - 1,
// each naming its pair p by split = -(p + 1)) set up by split_sync_one.  One thread a mirror.
__global__ void split_sync_kernel(const PairDesc* pairs, PairState* sts, int mbase, int nm,
                                  int phase) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nm; v += gridDim.x * blockDim.x)
    split_sync_one(pairs, sts, -pairs[mbase + v].split - 1, mbase + v, phase);
}

// After each team launch with split pairs: for each (one CTA a mirror, mbase + blockIdx.x) the
// meet (see above) gives its pair's result for the phase, which then ends the phase as the
// unsplit sweep's last strip would (finalize).  Unwritten boundary words are NaN (all ones)
// and fail every comparison, i.e. count as dead.
template <int KIND>
__global__ void __launch_bounds__(1024) split_meet_kernel(const PairDesc* pairs, PairState* sts,
                                                          int mbase, int phase, const int* error,
                                                          int* active_pairs) {
  const int m = mbase + blockIdx.x;
  const int p = -pairs[m].split - 1;
  PairState* g = sts + p;
  PairState* ms = sts + m;
  if (ld_volatile(&g->phase) != phase || !ld_volatile(&g->active) || ld_volatile(error)) return;
  const PairDesc pd = pairs[p], md = pairs[m];
  const int C = pd.n2 - 1;
  const int Sm = (md.n1 - 1 + 31) >> 5;
  const double* F = pd.bnd + (size_t)((pd.split - 1) % pd.ring) * pd.cstride;
  const double* M = md.bnd + (size_t)((Sm - 1) % md.ring) * md.cstride;
  double r;
  if (KIND == K_DEC) {
    int found = 0;
    for (int b = threadIdx.x; b < C; b += blockDim.x) {
      const double f = __ldcg(F + b), mm = __ldcg(M + (C - 1 - b));
      found |= (f >= 0.0 && mm >= -1.5 && f <= -mm) ? 1 : 0;
    }
    r = __syncthreads_or(found) ? 1.0 : -2.0;
  } else {
    __shared__ double red[32];
    const double U = g->U;
    double v = kFltMax;
    for (int b = threadIdx.x; b < C; b += blockDim.x) {
      const double f = __ldcg(F + b), mm = __ldcg(M + (C - 1 - b));
      if (f <= U && mm <= U) v = dmin(v, dmax(f, mm));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(kFull, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
      v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : kFltMax;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(kFull, v, o));
    }
    r = v;
  }
  if (threadIdx.x == 0) {
    g->result = r;
    g->cells_eval += ms->cells_eval;
    g->cells_fp64 += ms->cells_fp64;
    g->cells_vefd += ms->cells_vefd;
    ms->cells_eval = ms->cells_fp64 = ms->cells_vefd = 0;
    __threadfence();
    finalize<KIND>(g, pd, active_pairs);
    __threadfence();
  }
}

// Learned bracket, step 1: features of every pair waiting in PH_BRACKET (one CTA each).
__global__ void __launch_bounds__(kFeatThreads) bracket_features_kernel(const PairDesc* pairs,
                                                                       const PairState* st,
                                                                       int npairs, float* feat) {
  __shared__ FeatScratch sh;
  for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
    float* out = feat + (size_t)p * rfd_mlp::kInputWidth;
    if (st[p].phase != PH_BRACKET) {
      for (int f = threadIdx.x; f < rfd_mlp::kInputWidth; f += blockDim.x) out[f] = 0.f;
      continue;
    }
    const PairDesc pd = pairs[p];
    pair_features(pd.P, pd.n1, pd.Q, pd.n2, pd.d, st[p].endpoint, st[p].vefd, sh, out);
  }
}

// Learned bracket, step 2: q = model quantiles of log10(FD/VEFD - 1 + 1e-13); bracket
// [VEFD (1 + 10^q05), VEFD (1 + 10^q95)], then the verified search starts.
__global__ void bracket_apply_kernel(PairState* st, int npairs, const float* y, int* active_pairs) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npairs; p += gridDim.x * blockDim.x) {
    PairState* s = st + p;
    if (s->phase != PH_BRACKET) continue;
    double qlo = fmin(1.0, fmax(-13.0, (double)y[2 * p]));
    double qhi = fmin(1.0, fmax(-13.0, (double)y[2 * p + 1]));
    if (qhi < qlo) {
      const double tq = qlo;
      qlo = qhi;
      qhi = tq;
    }
    s->blo = s->vefd * (1.0 + exp10(qlo));
    s->bhi = s->vefd * (1.0 + exp10(qhi));
    begin_search(s, active_pairs, true);
  }
}

__global__ void __launch_bounds__(kFeatThreads) features_kernel(const PairDesc* pairs, int npairs,
                                                               const double* endpoint,
                                                               const double* vefd, float* feat) {
  __shared__ FeatScratch sh;
  for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
    const PairDesc pd = pairs[p];
    pair_features(pd.P, pd.n1, pd.Q, pd.n2, pd.d, endpoint[p], vefd[p], sh,
                  feat + (size_t)p * rfd_mlp::kInputWidth);
  }
}

// Per-pair constants and state.  One block per pair (grid-stride).
__global__ void prep_kernel(const PairDesc* pairs, PairState* st, int npairs, int start_phase) {
  for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
    const PairDesc pd = pairs[p];
    const int d = pd.d;
    double2* rowc = const_cast<double2*>(pd.rowc);
    double2* colrec = const_cast<double2*>(pd.colrec);
    for (int i = threadIdx.x; i < pd.n1 - 1; i += blockDim.x) {
      double t[3] = {0.0, 0.0, 0.0};
      for (int k = 0; k < d; ++k)
        t[k] = __dsub_rn(pd.P[(size_t)(i + 1) * d + k], pd.P[(size_t)i * d + k]);
      const double A = d == 3 ? sq_sum<3>(t) : sq_sum<2>(t);
      rowc[i] = make_double2(A, __ddiv_rn(0.5, A));
    }
    for (int j = threadIdx.x; j < pd.n2 - 1; j += blockDim.x) {
      double q0[3] = {0, 0, 0}, q1[3] = {0, 0, 0}, t[3] = {0, 0, 0};
      for (int k = 0; k < d; ++k) {
        q0[k] = pd.Q[(size_t)j * d + k];
        q1[k] = pd.Q[(size_t)(j + 1) * d + k];
        t[k] = __dsub_rn(q0[k], q1[k]);  // reference stages q_j - q_{j+1} (.cu:1137)
      }
      const double A = d == 3 ? sq_sum<3>(t) : sq_sum<2>(t);
      const double inv = __ddiv_rn(0.5, A);
      if (d == 2) {
        double2* r = colrec + (size_t)j * 3;
        r[0] = make_double2(q0[0], q0[1]);
        r[1] = make_double2(q1[0], q1[1]);
        r[2] = make_double2(A, inv);
      } else {
        double2* r = colrec + (size_t)j * 4;
        r[0] = make_double2(q0[0], q0[1]);
        r[1] = make_double2(q0[2], q1[0]);
        r[2] = make_double2(q1[1], q1[2]);
        r[3] = make_double2(A, inv);
      }
    }
    if (threadIdx.x == 0) {
      PairState* s = st + p;
      // endpoint bound: host arithmetic in the reference, no fusion (src/frechet.cpp:30)
      double a = 0.0, b = 0.0;
      for (int k = 0; k < d; ++k) {
        const double t0 = __dsub_rn(pd.P[k], pd.Q[k]);
        a = __dadd_rn(a, __dmul_rn(t0, t0));
        const double t1 = __dsub_rn(pd.P[(size_t)(pd.n1 - 1) * d + k], pd.Q[(size_t)(pd.n2 - 1) * d + k]);
        b = __dadd_rn(b, __dmul_rn(t1, t1));
      }
      s->endpoint = __dsqrt_rn(a < b ? b : a);
      s->seed = __dmul_rn(s->endpoint, s->endpoint);  // init_value * init_value, .cu:259
      s->epoch = 1;
      s->done_count = 0;
      s->dead_from = INT_MAX;
      s->U = (double)INFINITY;
      s->active = 1;
      s->phase = start_phase;
    }
  }
}

// FP64 FMA throughput probe: 8 independent chains per thread, values kept finite.
__global__ void __launch_bounds__(256) fp64_fma_kernel(double* out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-3 + k;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = __fma_rn(x[k], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == 1234.5) out[0] = s;  // keeps the chains live without a store per thread
}

}  // namespace

// ============================================================================ context

struct rfd_context {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  // split pairs: the mirror kernel's stream, forked from and joined to `stream` by events
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  int num_sms = 0;
  int grid[3] = {0, 0, 0};
  int team_grid[3] = {0, 0, 0};     // teams of the chosen shape (team_warps)
  int team_grids[2][3] = {{0, 0, 0}, {0, 0, 0}};  // [teams of 4, of 8 warps][kind]
  int team_warps = 8;  // warps per team: 8 or 4 (RFD_TEAM_WARPS, rfd_autotune_search)
  int solo = 0;  // RFD_SOLO=1: VE-FD and decisions on the solo-warp strips (A/B checks)
  int lockstep = 0;  // RFD_LOCKSTEP=1: one launch per probe round instead of the continuous search
  int search_switch = 0;  // active pairs below which the continuous search takes over
  int search_window = 2;  // continuous search: strips a probe queues ahead of its band
  int dfd_rows = 8;    // rows per lane of the DFD strips (RFD_DFD_ROWS = 1, 2, 4 or 8)
  int dfd_skew = -1;   // RFD_DFD_SKEW: 1 skewed rows, 0 stacked, unset: chosen per call
  int dfd_grid[2] = {0, 0};  // [stacked, skewed] for dfd_rows
  int dfd_grid_all[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};  // for rows 1, 2, 4, 8
  int dfd_grid_infl[2] = {0, 0};  // inflated coarse sweep, 1 row per lane
  int prof = 0;  // RFD_PROF=1: team-strip cycle counters printed to stderr after each call
  // rows of the DFD strips' boundary ring per pair (RFD_DFD_RING_ROWS, at least 2; see
  // "Boundary ring" in rfd_device.cuh)
  int dfd_ring_rows = kDfdRingRows;
  // rows of the VE-FD and decision strips' boundary ring (RFD_TEAM_RING_ROWS, at least 2):
  // 0 keeps one row per strip unless a lone pair's rows do not fit (launch windows, run_batch)
  int team_ring_rows = 0;
  // meet in the middle for lone pairs of at least this many team strips (RFD_SPLIT; 0: off)
  int split_min = 64;
  void* dws = nullptr;
  size_t dws_size = 0;
  void* hws = nullptr;
  size_t hws_size = 0;
  long long spin_cycles = 0;   // budget of every bounded wait, in SM clock cycles
  long long spin_default = 0;  // about 20 s at the maximum SM clock
  // phase timing (rfd_context_phase_times)
  int timing = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  // rfd_options.graph: the last call's work as an instantiated CUDA graph, and the layout it
  // was captured for (a call with the same layout replays it)
  cudaGraphExec_t gexec = nullptr;
  uint64_t gkey = 0;
  int glaunches = 0;
};

namespace {

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// The team kernel of the context's shape (warps per team) on its grid (grid > 0: that many
// teams); MIR: the mirror kernel of split pairs.
template <int KIND, bool MIR = false>
void launch_team(const rfd_context* ctx, const WaveArgs& wa, cudaStream_t st, int grid = 0) {
  const int g = grid > 0 ? grid : ctx->team_grid[KIND];
  if (ctx->team_warps == 4)
    team_kernel<KIND, 4, MIR><<<g, 128, team_smem_bytes<KIND>(), st>>>(wa);
  else
    team_kernel<KIND, 8, MIR><<<g, 256, team_smem_bytes<KIND>(), st>>>(wa);
}

// Row of rfd_context::team_grids for a team shape.
int team_shape_index(int warps) { return warps == 4 ? 0 : 1; }

int ring_of(int64_t strips, int rows) {  // strips - 1 rows are handed over; at least 1
  return (int)std::max<int64_t>(1, std::min<int64_t>(strips - 1, rows));
}

int env_rows(const char* name, int dflt) {
  const char* e = getenv(name);
  if (!e || !*e) return dflt;
  char* end = nullptr;
  const long v = strtol(e, &end, 10);
  return (end && *end == 0 && v >= 2 && v <= (1 << 20)) ? (int)v : dflt;
}

// RFD_SPIN_CYCLES (a positive integer): the budget of every bounded wait, in SM clock
// cycles, in place of the default of about 20 s.  A small budget makes waits run out (the
// call then reports RFD_ERR_TIMEOUT), which is how the failure path is tested.
long long env_spin_cycles(long long dflt) {
  const char* e = getenv("RFD_SPIN_CYCLES");
  if (!e || !*e) return dflt;
  char* end = nullptr;
  const long long v = strtoll(e, &end, 10);
  return (end && *end == 0 && v > 0) ? v : dflt;
}

int ensure_device(rfd_context* ctx, size_t bytes) {
  if (bytes <= ctx->dws_size) return RFD_OK;
  if (ctx->dws) cudaFree(ctx->dws);
  ctx->dws = nullptr;
  ctx->dws_size = 0;
  size_t want = std::max(bytes, ctx->dws_size + ctx->dws_size / 4);
  cudaError_t e = cudaMalloc(&ctx->dws, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    e = cudaMalloc(&ctx->dws, bytes);
    want = bytes;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(RFD_ERR_NOMEM, "device workspace of " + std::to_string(bytes) + " bytes");
  }
  ctx->dws_size = want;
  return RFD_OK;
}

int ensure_host(rfd_context* ctx, size_t bytes) {
  if (bytes <= ctx->hws_size) return RFD_OK;
  if (ctx->hws) cudaFreeHost(ctx->hws);
  ctx->hws = nullptr;
  ctx->hws_size = 0;
  size_t want = std::max(bytes, ctx->hws_size + ctx->hws_size / 4);
  if (cudaMallocHost(&ctx->hws, want) != cudaSuccess) {
    cudaGetLastError();
    return fail(RFD_ERR_NOMEM, "pinned staging of " + std::to_string(want) + " bytes");
  }
  ctx->hws_size = want;
  return RFD_OK;
}

enum Mode { MODE_DISTANCE = 0, MODE_BOUNDS = 1, MODE_DECIDE = 2 };

struct Layout {
  // device offsets
  size_t descs, tdescs, states, items, titems, counters, error, active, zero_begin, zero_end,
      total;
  std::vector<size_t> P, Q, rowc, colrec, bnd, tags, prog, slots;
  std::vector<int> ring_d, ring_t, ring_c;  // ring rows: DFD, team strips, coarse DFD
  // host staging offsets
  size_t h_descs, h_tdescs, h_states, h_items, h_titems, h_misc, h_curves, h_total;
  std::vector<size_t> hP, hQ;
  int nitems, ntitems, nlaunch;
};

// Device workspace of one pair in a batch (an upper bound of what run_batch lays out for
// it): curves, segment records, boundary rows (the team strips' n1 n2 / 4 bytes dominate),
// tags, progress and slot words, items.
double pair_workspace_bytes(const rfd_context* ctx, int64_t n1, int64_t n2, int d, int ck) {
  const int64_t rows = std::min(n1, n2), cols = std::max(n1, n2);
  const int64_t St = (std::max<int64_t>(rows - 1, 0) + 31) / 32;
  const double rt = (double)std::max<int64_t>(St - 1, 1);  // team strips: a row per strip
  const double rd = (double)ring_of((n1 + 31) / 32, ctx->dfd_ring_rows);
  const double ring_words = std::max(rt * (double)(cols + 32), rd * (double)(n2 + 32));
  double b = 8.0 * (double)d * (double)(n1 + n2)         // curves
             + 16.0 * (double)rows + 64.0 * (double)cols  // segment records
             + 8.0 * ring_words                           // boundary ring
             + 4.0 * rt * (double)(cols / 32 + 64)        // tags
             + 40.0 * (double)(St + 1) + 16.0 * (double)(n1 / 32 + rows / 32 + 2)  // progress, items
             + 24.0 * (rt + rd) + 8192.0;                 // slot words, descriptors, state
  if (ck) b += 8.0 * (double)(d + 1) * (double)(n1 + n2) / ck + 16384.0;
  return b;
}

int check_pair(const double* c1, int64_t n1, const double* c2, int64_t n2, int32_t d) {
  if (!c1 || !c2) return fail(RFD_ERR_ARG, "null curve pointer");
  if (d != 2 && d != 3) return fail(RFD_ERR_ARG, "dims must be 2 or 3");
  if (n1 < 1 || n2 < 1) return fail(RFD_ERR_ARG, "empty curve");
  if (n1 > (1 << 30) || n2 > (1 << 30)) return fail(RFD_ERR_LIMIT, "curve longer than 2^30 points");
  return RFD_OK;
}

// Consecutive repeated points (rfd_options.drop_repeats): point k is kept unless every
// coordinate equals point k-1's.  A zero-length segment is exactly the case A = 0 of the
// free-interval quadratic, so the kept curve has none.
static bool same_point(const double* a, const double* b, int d) {
  for (int k = 0; k < d; ++k)
    if (!(a[k] == b[k])) return false;
  return true;
}

static int64_t kept_points(const double* c, int64_t n, int d) {
  int64_t m = n > 0 ? 1 : 0;
  for (int64_t k = 1; k < n; ++k) m += !same_point(c + (k - 1) * d, c + k * d, d);
  return m;
}

static void copy_kept(double* dst, const double* c, int64_t n, int d) {
  if (n < 1) return;
  memcpy(dst, c, sizeof(double) * d);
  double* last = dst;
  for (int64_t k = 1; k < n; ++k) {
    if (same_point(c + (k - 1) * d, c + k * d, d)) continue;
    last += d;
    memcpy(last, c + k * d, sizeof(double) * d);
  }
}

int run_batch(rfd_context* ctx, int64_t npairs, const double* const* c1s, const int64_t* n1s,
              const double* const* c2s, const int64_t* n2s, const int32_t* dims,
              const rfd_options* opt, rfd_result* out, int mode, double radius) {
  if (!ctx || npairs < 0 || (npairs > 0 && (!c1s || !n1s || !c2s || !n2s || !dims || !out)))
    return fail(RFD_ERR_ARG, "null argument");
  if (npairs == 0) return RFD_OK;
  if (npairs > (1 << 24)) return fail(RFD_ERR_LIMIT, "more than 2^24 pairs");
  rfd_options o;
  rfd_options_init(&o, 0);
  if (opt) o = *opt;
  if (o.max_probes < 0 || o.max_probes > RFD_MAX_PROBES) return fail(RFD_ERR_ARG, "max_probes");
  if (o.stop_mode != RFD_STOP_ABS && o.stop_mode != RFD_STOP_REL) return fail(RFD_ERR_ARG, "stop_mode");
  if (!(o.tol >= 0.0)) return fail(RFD_ERR_ARG, "tol");
  if (o.precision != RFD_PREC_FP64 && o.precision != RFD_PREC_FP32_FILTER)
    return fail(RFD_ERR_ARG, "precision");
  if (o.coarse_ub < 0 || o.coarse_ub == 1 || o.coarse_ub > 4096)
    return fail(RFD_ERR_ARG, "coarse_ub must be 0 or in [2, 4096]");
  if (o.coarse_ub && o.reference_quirks)
    return fail(RFD_ERR_ARG, "coarse_ub needs reference_quirks = 0 (the quirk reads the DFD sizes)");
  if (o.formula < RFD_FORMULA_FUSED || o.formula > RFD_FORMULA_REFERENCE)
    return fail(RFD_ERR_ARG, "formula");
  if (o.formula != RFD_FORMULA_FUSED && o.precision == RFD_PREC_FP32_FILTER)
    return fail(RFD_ERR_ARG, "the FP32 filter certifies the fused formula's intervals only");
  for (int64_t p = 0; p < npairs; ++p) {
    int rc = check_pair(c1s[p], n1s[p], c2s[p], n2s[p], dims[p]);
    if (rc) return rc;
    if (mode != MODE_DISTANCE && (n1s[p] < 2 || n2s[p] < 2))
      return fail(RFD_ERR_ARG, "bounds and decisions need curves of at least two points");
  }
  const bool on_device = o.memory == RFD_MEM_DEVICE;
  const int max_probes = mode == MODE_DISTANCE ? o.max_probes : 0;
  if (o.drop_repeats != 0 && o.drop_repeats != 1) return fail(RFD_ERR_ARG, "drop_repeats");
  // with drop_repeats the layout is sized by the kept points; the staging copy compacts
  const int64_t* const in_n1s = n1s;
  const int64_t* const in_n2s = n2s;
  std::vector<int64_t> kept1, kept2;
  const bool drop = mode == MODE_DISTANCE && o.drop_repeats;
  // device-memory curves with drop_repeats are compacted into the workspace on the device
  const bool dcompact = drop && on_device;
  if (drop) {
    kept1.resize(npairs);
    kept2.resize(npairs);
    if (on_device) {
      // the kept counts size the layout: counted on the device, read back before it
      const size_t nb = align_up(sizeof(SrcCurve) * 2 * npairs, 256);
      const size_t kb = sizeof(long long) * 2 * npairs;
      int rc0 = ensure_device(ctx, nb + kb);
      if (rc0) return rc0;
      rc0 = ensure_host(ctx, nb + kb);
      if (rc0) return rc0;
      SrcCurve* hsc = (SrcCurve*)ctx->hws;
      for (int64_t p = 0; p < npairs; ++p) {
        hsc[2 * p] = SrcCurve{c1s[p], nullptr, (long long)n1s[p], dims[p], 0};
        hsc[2 * p + 1] = SrcCurve{c2s[p], nullptr, (long long)n2s[p], dims[p], 0};
      }
      RFD_CUDA(cudaMemcpyAsync(ctx->dws, ctx->hws, sizeof(SrcCurve) * 2 * npairs,
                               cudaMemcpyHostToDevice, ctx->stream));
      count_kept_kernel<<<(int)std::min<int64_t>(2 * npairs, 8 * ctx->num_sms), 256, 0,
                          ctx->stream>>>((const SrcCurve*)ctx->dws, (int)(2 * npairs),
                                         (long long*)((char*)ctx->dws + nb));
      RFD_CUDA(cudaGetLastError());
      RFD_CUDA(cudaMemcpyAsync((char*)ctx->hws + nb, (char*)ctx->dws + nb, kb,
                               cudaMemcpyDeviceToHost, ctx->stream));
      RFD_CUDA(cudaStreamSynchronize(ctx->stream));
      const long long* kc = (const long long*)((char*)ctx->hws + nb);
      for (int64_t p = 0; p < npairs; ++p) {
        kept1[p] = kc[2 * p];
        kept2[p] = kc[2 * p + 1];
      }
    } else {
      for (int64_t p = 0; p < npairs; ++p) {
        kept1[p] = kept_points(c1s[p], n1s[p], dims[p]);
        kept2[p] = kept_points(c2s[p], n2s[p], dims[p]);
      }
    }
    n1s = kept1.data();
    n2s = kept2.data();
  }

  // decision formula per pair: RFD_FORMULA_REFERENCE takes the materialised path where the
  // reference would, i.e. where its interval arrays fit in this device's free memory
  // (src/intersection_algorithm_in_parallel.cu:87-97: maxThreadsPerBlock x SMs bytes plus
  // 4 arrays of (n1-1)(n2-2+n1-2)+n1 doubles)
  std::vector<int> formula((size_t)npairs, o.formula == RFD_FORMULA_MATERIALISED ? 1 : 0);
  if (o.formula == RFD_FORMULA_REFERENCE) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      fr = 0;
    }
    int mtpb = 1024;
    cudaDeviceGetAttribute(&mtpb, cudaDevAttrMaxThreadsPerBlock, ctx->device);
    for (int64_t p = 0; p < npairs; ++p) {
      const double a = (double)n1s[p];
      const double need = (double)ctx->num_sms * (double)mtpb +
                          ((a - 1.0) * ((double)n2s[p] - 2.0 + a - 2.0) + a) * 8.0 * 4.0;
      formula[p] = (double)fr >= need ? 1 : 0;
    }
  }

  // ---------------- layout
  Layout L;
  L.P.resize(npairs); L.Q.resize(npairs); L.rowc.resize(npairs); L.colrec.resize(npairs);
  L.bnd.resize(npairs); L.tags.resize(npairs); L.prog.resize(npairs);
  L.slots.resize(npairs);
  L.ring_d.resize(npairs); L.ring_t.resize(npairs); L.ring_c.resize(npairs);
  L.hP.resize(npairs); L.hQ.resize(npairs);
  const int ck = mode == MODE_DISTANCE ? o.coarse_ub : 0;  // coarse upper bound, every ck-th point
  auto coarse_n = [&](int64_t n) { return n < 2 ? n : (n - 2) / ck + 2; };  // anchors 0, ck, ..., n-1
  std::vector<size_t> cP(ck ? npairs : 0), cQ(ck ? npairs : 0);
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t r = off; off = align_up(off + bytes, 256); return r; };
  L.descs = take(sizeof(PairDesc) * npairs);
  const size_t cdescs = ck ? take(sizeof(PairDesc) * npairs) : 0;
  // VE-FD and decision strips run on the transposed grid when the first curve is the longer:
  // a strip costs its 32 rows' hand-over (~7 us on B200) and a 32-column chunk ~1.8 us, so
  // rows along the shorter curve shorten the chain of strips (50000 x 1039 points: 1563
  // strips, 11 ms a decision, against 33).  The DFD sweeps keep the given orientation.
  std::vector<unsigned char> trv(npairs, 0);
  for (int64_t p = 0; p < npairs; ++p)
    trv[p] = n1s[p] >= 2 && n2s[p] >= 2 && n1s[p] > n2s[p];
  auto trows = [&](int64_t p) { return trv[p] ? n2s[p] : n1s[p]; };
  auto tcols = [&](int64_t p) { return trv[p] ? n1s[p] : n2s[p]; };
  // items: interleave pairs by strip index so early strips of every pair go first
  std::vector<int> order(npairs);
  for (int64_t p = 0; p < npairs; ++p) order[p] = (int)p;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return (double)n1s[a] * (double)n2s[a] > (double)n1s[b] * (double)n2s[b];
  });
  int64_t maxS = 0, nitems = 0, maxSt = 0, ntitems = 0;
  for (int64_t p = 0; p < npairs; ++p) {
    int64_t S = (n1s[p] + 31) / 32;
    maxS = std::max(maxS, S);
    nitems += S;
    const int64_t St = (trows(p) + 31) / 32;
    maxSt = std::max(maxSt, St);
    ntitems += St;
  }
  if (nitems > INT32_MAX / 2) return fail(RFD_ERR_LIMIT, "too many strips");
  // Launch windows of the team strips (O(n+m) boundary memory).  One boundary row per 32-row
  // strip takes about n1 n2 / 4 bytes (250 GB for two curves of 10^6 points).  When a lone
  // pair's workspace does not fit in the memory this context may use (3/4 of what is free and
  // its own workspace, or RFD_BATCH_BUDGET bytes), or RFD_TEAM_RING_ROWS = R asks for it, the
  // VE-FD and decision strips run in launch windows of W consecutive strips: strip s writes
  // ring row s % (W + 1), a window's rows are reset right before its launch, and the next
  // window starts once it has ended.  The boundary then takes W + 1 rows whatever the curves'
  // lengths; W is the most the budget holds, at most 4096 strips (R - 1 when forced): a window
  // of 4096 strips keeps every team busy, and a window's end costs one strip's drain (tens of
  // microseconds in a pruned band).  Results are bit-identical:
  // the same strips compute the same values and hand over the same rows.  The continuous
  // search and the k-ary members, which keep every strip's row at once, are off (one launch
  // round per probe, one launch per window).
  int64_t twin = 0;  // team strips per launch window; 0: every strip in one launch
  if (!ctx->solo) {
    if (ctx->team_ring_rows >= 2) {
      twin = ctx->team_ring_rows - 1;
    } else if (npairs == 1 && n1s[0] >= 2 && n2s[0] >= 2) {
      const int64_t St = (trows(0) - 1 + 31) / 32;
      const double full = pair_workspace_bytes(ctx, n1s[0], n2s[0], dims[0], ck);
      double budget = 0.0;
      if (const char* e = getenv("RFD_BATCH_BUDGET")) budget = atof(e);
      if (!(budget > 0.0)) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
          cudaGetLastError();
          fr = 0;
        }
        budget = 0.75 * ((double)fr + (double)ctx->dws_size);
      }
      if (St > 2 && full > budget) {
        // a team row and its tags, as pair_workspace_bytes counts them
        const double row = 8.0 * (double)(tcols(0) + 32) + 4.0 * (double)(tcols(0) / 32 + 64);
        const double rows = std::floor((budget - (full - (double)(St - 1) * row)) / row);
        // fewer than 2 rows: not even a window of one strip fits (the allocation reports it)
        twin = rows >= 2.0 ? std::min<int64_t>({St - 2, (int64_t)rows - 1, (int64_t)4096}) : 0;
      }
    }
    if (twin >= maxSt) twin = 0;  // one window holds every strip: nothing to gain
  }
  int64_t nwin = twin ? (maxSt + twin - 1) / twin : 0;  // (recomputed for split pairs below)
  // Continuous search: a queue slot for every strip of every probe
  // (at most 512 MB; past that, and for the solo strips, one launch per probe round)
  int64_t dyn_cap = 0;
  if (mode == MODE_DISTANCE && max_probes > 1 && !ctx->solo && !ctx->lockstep && !twin) {
    for (int64_t p = 0; p < npairs; ++p)
      dyn_cap += (std::max<int64_t>(trows(p) - 1, 0) + 31) / 32 * max_probes;
    if (dyn_cap * (int64_t)sizeof(unsigned long long) > ((int64_t)512 << 20)) dyn_cap = 0;
  }
  const size_t dyn_off = dyn_cap ? take(sizeof(unsigned long long) * dyn_cap) : 0;
  // k-ary rounds (rfd_options.search_arity = K): the pairs whose probe chains are longest get
  // K - 1 member decisions each (descriptor, state and boundary rows of their own, after the
  // pairs' in the same arrays).  A decision's chain is about max(strips x 7 us, 32-column
  // chunks x 3 us) on a B200.  The members of all pairs together use at most a quarter of
  // the device memory that is free or already the context's; a pair whose members would
  // exceed what is left gets none.
  const int karity = (mode == MODE_DISTANCE && max_probes > 1 && !ctx->solo && !twin &&
                      o.search_arity >= 2) ? std::min<int>(o.search_arity, RFD_MAX_ARITY) : 0;
  std::vector<int64_t> kpairs;
  if (karity) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      cudaGetLastError();
      free_b = 0;
    }
    double room = 0.25 * ((double)free_b + (double)ctx->dws_size);
    std::vector<double> mbytes(npairs, 0.0);
    std::vector<std::pair<double, int64_t>> est;
    for (int64_t p = 0; p < npairs; ++p) {
      if (n1s[p] < 2 || n2s[p] < 2) continue;
      const int64_t St = (trows(p) - 1 + 31) / 32, C = tcols(p);
      const double bytes = 8.0 * (double)std::max<int64_t>(St - 1, 1) * (double)align_up((size_t)C, 32) +
                           4.0 * (double)std::max<int64_t>(St - 1, 1) * (double)(C / 32 + 64) +
                           (double)sizeof(Prog) * (double)St;
      mbytes[p] = bytes * (karity - 1);
      est.push_back({std::max(7.0 * (double)St, 3.0 * (double)((C + 31) / 32)), p});
    }
    std::stable_sort(est.begin(), est.end(), [](const std::pair<double, int64_t>& a,
                                                const std::pair<double, int64_t>& b) {
      return a.first > b.first;
    });
    for (size_t k = 0; k < est.size() && kpairs.size() < (size_t)RFD_ARITY_PAIRS; ++k) {
      if (mbytes[est[k].second] > room) continue;
      room -= mbytes[est[k].second];
      kpairs.push_back(est[k].second);
    }
  }
  const int64_t nmem = (int64_t)kpairs.size() * (karity > 1 ? karity - 1 : 0);
  // Meet in the middle (split_meet_kernel): in a call of at most kSplitPairs pairs, the chain
  // of a pair's team strips, which bounds a long pair's VE-FD and decisions, runs as two halves
  // at once.  Pairs of at least RFD_SPLIT strips (default 64; 0: never); not with k-ary
  // members, launch windows, the solo strips or rfd_decide (which reports the right UB, which
  // the meet does not form).  Results are bit-identical.  A split pair's boundary rows
  // k .. S - 1, which its forward half does not use, hold its mirror's rows (S rows in all,
  // one more than unsplit); the probe rounds run as launches.  Larger calls keep every team
  // busy with pairs already and keep the continuous search.
  constexpr int64_t kSplitPairs = 8;
  std::vector<int64_t> ksp(npairs, 0);  // forward strips of a split pair (0: not split)
  std::vector<int64_t> mirror_of(npairs, -1);  // its mirror's descriptor index
  int64_t nsplit = 0, nfwd = 0, nmir = 0;  // split pairs; forward and mirror team items
  if (npairs <= kSplitPairs && mode != MODE_DECIDE && !ctx->solo && nmem == 0 &&
      ctx->split_min > 0)
    for (int64_t p = 0; p < npairs; ++p) {
      const int64_t St = (std::max<int64_t>(trows(p) - 1, 0) + 31) / 32;
      if (n1s[p] >= 2 && n2s[p] >= 2 && St >= std::max(2, ctx->split_min)) {
        ksp[p] = St / 2;
        mirror_of[p] = npairs + nmem + nsplit++;
        nmir += St - ksp[p];
      }
    }
  if (nsplit) {
    dyn_cap = 0;
    for (int64_t p = 0; p < npairs; ++p) nfwd += ksp[p] ? ksp[p] : (trows(p) + 31) / 32;
    ntitems = nfwd + nmir;  // the forward kernel's list, then the mirror kernel's
  }
  if (nsplit && twin) {
    // launch windows of both halves: window g runs strips g W .. g W + W - 1 of every
    // forward half and of every mirror, each half through a ring of its own (W + 1 rows, or
    // its strips if fewer); with windows chosen by the budget, W is halved for the two rings
    if (ctx->team_ring_rows < 2) twin = std::max<int64_t>(1, (twin + 1) / 2 - 1);
    int64_t most = 0;
    for (int64_t p = 0; p < npairs; ++p) {
      const int64_t St = (std::max<int64_t>(trows(p) - 1, 0) + 31) / 32;
      most = std::max(most, ksp[p] ? std::max(ksp[p], St - ksp[p]) : (trows(p) + 31) / 32);
    }
    nwin = (most + twin - 1) / twin;
  }
  const int64_t mbase = npairs + nmem;  // the first mirror descriptor
  // descriptors and states: the pairs', then the members', then the split pairs' mirrors
  const int64_t nst = npairs + nmem + nsplit;
  auto mpair = [&](int64_t v) { return kpairs[v / (karity - 1)]; };
  // the members' strips join the team item list, interleaved with their pair's
  for (int64_t v = 0; v < nmem; ++v) ntitems += (trows(mpair(v)) + 31) / 32;
  if (ntitems > INT32_MAX / 2) return fail(RFD_ERR_LIMIT, "too many strips");
  L.nitems = (int)nitems;
  L.ntitems = (int)ntitems;
  L.items = take(sizeof(int2) * nitems);
  L.titems = take(sizeof(int2) * ntitems);
  L.tdescs = take(sizeof(PairDesc) * nst);
  L.states = take(sizeof(PairState) * nst);
  // ticket counters: DFD, two VE-FD, probe rounds (+1 for a decision), the continuous
  // search's ticket and queue tail; then a gate word per probe round
  L.nlaunch = 3 + max_probes + (mode == MODE_DECIDE ? 1 : 0) + 2;
  // launch windows: a ticket counter per window of every VE-FD phase and probe round
  const int64_t wbase = L.nlaunch + max_probes + 1;
  // (split pairs: one per VE-FD phase and probe round for the mirror kernel, or, with
  // windows, one per window for each half)
  const int64_t wtickets =
      (nsplit ? (twin ? 2 * nwin : 1) : nwin) * (2 + std::max(max_probes, 1));
  L.zero_begin = off;
  L.counters = take(sizeof(unsigned) * (wbase + wtickets));
  const size_t prof_off = take(sizeof(unsigned long long) * (kTraceBase + kTraceW * kTrace));
  L.error = take(sizeof(int));
  for (int64_t p = 0; p < npairs; ++p) {
    // boundary rows: team strips of 32 segment rows, one row each; the DFD ring for strips of
    // at least 32 point rows (the strip height the autotuner may pick); the coarse pair's DFD
    const int64_t St = (std::max<int64_t>(trows(p) - 1, 0) + 31) / 32;
    // team strips hand rows over through one row per strip (S - 1 rows)
    // (a split pair: its forward ring, then its mirror's - S rows, or two window rings)
    L.ring_t[p] = ksp[p] ? (int)(twin ? std::min(twin + 1, ksp[p]) + std::min(twin + 1, St - ksp[p])
                                      : St)
                         : ring_of(St, twin ? (int)(twin + 1) : INT32_MAX);
    L.ring_d[p] = ring_of((n1s[p] + 31) / 32, ctx->dfd_ring_rows);
    L.ring_c[p] = ck && n1s[p] >= 2 && n2s[p] >= 2
                      ? ring_of((coarse_n(n1s[p]) + 31) / 32, ctx->dfd_ring_rows) : 1;
    // progress words, tags (team strips) and the DFD ring's slot words: cleared every call
    const int64_t tstride = align_up((size_t)((tcols(p) + 31) / 32), 32);
    L.tags[p] = take(sizeof(unsigned) * L.ring_t[p] * tstride);
    L.prog[p] = take(sizeof(Prog) * std::max<int64_t>(St, (trows(p) + 31) / 32));
    L.slots[p] = take(sizeof(unsigned long long) * (n1s[p] + 31) / 32);  // a count per DFD strip
  }
  std::vector<size_t> mtags(nmem), mprog(nmem), mbnd(nmem);
  for (int64_t v = 0; v < nmem; ++v) {
    const int64_t p = mpair(v);
    const int64_t St = (std::max<int64_t>(trows(p) - 1, 0) + 31) / 32;
    const int64_t tstride = align_up((size_t)((tcols(p) + 31) / 32), 32);
    mtags[v] = take(sizeof(unsigned) * ring_of(St, INT32_MAX) * tstride);
    mprog[v] = take(sizeof(Prog) * std::max<int64_t>(St, 1));
  }
  L.zero_end = off;
  L.active = take(sizeof(int));
  const bool use_model = mode == MODE_DISTANCE && o.model && !o.bracket;
  const size_t feat_off = use_model ? take(sizeof(float) * rfd_mlp::kInputWidth * npairs) : 0;
  const size_t y_off = use_model ? take(sizeof(float) * rfd_mlp::kOutputs * npairs) : 0;
  // host curves: one contiguous region laid out exactly as the pinned staging area below
  // (same sizes, same 256-byte alignment), so a single copy moves every curve
  const size_t curves_begin = off;
  if (!on_device || dcompact)
    for (int64_t p = 0; p < npairs; ++p) {
      L.P[p] = take(sizeof(double) * n1s[p] * dims[p]);
      L.Q[p] = take(sizeof(double) * n2s[p] * dims[p]);
    }
  const size_t curves_end = off;
  const size_t src_off = dcompact ? take(sizeof(SrcCurve) * 2 * npairs) : 0;
  for (int64_t p = 0; p < npairs; ++p) {
    const int64_t n1 = n1s[p], n2 = n2s[p];
    const int d = dims[p];
    const int64_t cstride = align_up((size_t)n2, 32);
    // segment records in the team strips' orientation; the boundary ring, shared by the DFD
    // sweep (given orientation), the coarse DFD and the team strips, which run one after another
    const int64_t tcstride = align_up((size_t)tcols(p), 32);
    L.rowc[p] = take(sizeof(double2) * std::max<int64_t>(trows(p) - 1, 1));
    L.colrec[p] = take(sizeof(double2) * (d == 2 ? 3 : 4) * std::max<int64_t>(tcols(p) - 1, 1));
    const int64_t ccstride = ck ? align_up((size_t)coarse_n(n2), 32) : 0;
    L.bnd[p] = take(sizeof(double) * std::max(std::max((int64_t)L.ring_d[p] * cstride,
                                                       (int64_t)L.ring_t[p] * tcstride),
                                              (int64_t)L.ring_c[p] * ccstride));
    if (ck) {
      // anchors and their inflations; a pair with a one-point curve keeps every point, with
      // inflation 0 (its DFD is its exact, closed-form answer)
      const bool full = n1 < 2 || n2 < 2;
      cP[p] = take(sizeof(double) * (full ? n1 : coarse_n(n1)) * (d + 1));
      cQ[p] = take(sizeof(double) * (full ? n2 : coarse_n(n2)) * (d + 1));
    }
  }
  for (int64_t v = 0; v < nmem; ++v) {
    const int64_t p = mpair(v);
    const int64_t St = (std::max<int64_t>(trows(p) - 1, 0) + 31) / 32;
    mbnd[v] = take(sizeof(double) * ring_of(St, INT32_MAX) * align_up((size_t)tcols(p), 32));
  }
  L.total = off;

  size_t hoff = 0;
  auto htake = [&](size_t bytes) { size_t r = hoff; hoff = align_up(hoff + bytes, 256); return r; };
  L.h_descs = htake(sizeof(PairDesc) * npairs);
  const size_t h_cdescs = ck ? htake(sizeof(PairDesc) * npairs) : 0;
  L.h_tdescs = htake(sizeof(PairDesc) * nst);
  L.h_states = htake(sizeof(PairState) * nst);
  L.h_items = htake(sizeof(int2) * nitems);
  L.h_titems = htake(sizeof(int2) * ntitems);
  L.h_misc = htake(4 * sizeof(int));
  const size_t h_src = dcompact ? htake(sizeof(SrcCurve) * 2 * npairs) : 0;
  L.h_curves = hoff;
  if (!on_device) {
    for (int64_t p = 0; p < npairs; ++p) {
      L.hP[p] = htake(sizeof(double) * n1s[p] * dims[p]);
      L.hQ[p] = htake(sizeof(double) * n2s[p] * dims[p]);
    }
  }
  L.h_total = hoff;

  // RFD_GUARD=1 (debugging): a guard band after the workspace, filled with a pattern before the
  // call's launches and checked after them; a changed byte means a write past the workspace
  const size_t guard = getenv("RFD_GUARD") ? ((size_t)8 << 20) : 0;
  int rc = ensure_device(ctx, L.total + guard);
  if (rc) return rc;
  rc = ensure_host(ctx, L.h_total);
  if (rc) return rc;
  char* dbase = (char*)ctx->dws;
  char* hbase = (char*)ctx->hws;
  if (guard) {
    RFD_CUDA(cudaMemsetAsync(dbase + L.total, 0xA5, guard, ctx->stream));
  }

  // ---------------- host staging
  PairDesc* hd = (PairDesc*)(hbase + L.h_descs);
  PairState* hs = (PairState*)(hbase + L.h_states);
  int2* hi = (int2*)(hbase + L.h_items);
  for (int64_t p = 0; p < npairs; ++p) {
    const int64_t n1 = n1s[p], n2 = n2s[p];
    const int d = dims[p];
    PairDesc& D = hd[p];
    memset(&D, 0, sizeof(D));
    if (on_device && !dcompact) {
      D.P = c1s[p];
      D.Q = c2s[p];
    } else {  // staged below, or compacted on the device
      D.P = (const double*)(dbase + L.P[p]);
      D.Q = (const double*)(dbase + L.Q[p]);
    }
    if (dcompact) {
      SrcCurve* hsc = (SrcCurve*)(hbase + h_src);
      hsc[2 * p] = SrcCurve{c1s[p], (double*)(dbase + L.P[p]), (long long)in_n1s[p], d, 0};
      hsc[2 * p + 1] = SrcCurve{c2s[p], (double*)(dbase + L.Q[p]), (long long)in_n2s[p], d, 0};
    }
    D.rowc = (const double2*)(dbase + L.rowc[p]);
    D.colrec = (const double2*)(dbase + L.colrec[p]);
    D.bnd = (double*)(dbase + L.bnd[p]);
    D.tags = (unsigned*)(dbase + L.tags[p]);
    D.prog = (Prog*)(dbase + L.prog[p]);
    D.slots = (unsigned long long*)(dbase + L.slots[p]);
    D.ring = L.ring_d[p];
    D.n1 = (int)n1;
    D.n2 = (int)n2;
    D.d = d;
    D.cstride = (long long)align_up((size_t)n2, 32);
    D.tstride = (long long)align_up((size_t)((n2 + 31) / 32), 32);
    PairDesc& Dt = ((PairDesc*)(hbase + L.h_tdescs))[p];
    Dt = D;
    Dt.ring = L.ring_t[p];
    if (trv[p]) {
      Dt.P = D.Q;
      Dt.Q = D.P;
      Dt.n1 = (int)n2;
      Dt.n2 = (int)n1;
      Dt.tr = 1;
      Dt.cstride = (long long)align_up((size_t)n1, 32);
      Dt.tstride = (long long)align_up((size_t)((n1 + 31) / 32), 32);
    }
    if (ksp[p]) {
      // the mirror sweeps rows 32k .. R - 1 from the top; its rows, tags and progress words
      // are the pair's from strip k on; split = -(p + 1) names its pair
      const int64_t St = (trows(p) - 1 + 31) / 32, ksplit = ksp[p];
      // the halves' rings: every strip's row, or, in launch windows, W + 1 rows each
      const int64_t rf = twin ? std::min(twin + 1, ksplit) : ksplit;
      const int64_t rm = twin ? std::min(twin + 1, St - ksplit) : St - ksplit;
      Dt.split = (int)ksplit;
      Dt.ring = (int)rf;
      PairDesc& Dm = ((PairDesc*)(hbase + L.h_tdescs))[mirror_of[p]];
      Dm = Dt;
      Dm.split = -(int)(p + 1);
      Dm.mrow = Dt.n1 - 2;
      Dm.n1 = Dt.n1 - 32 * (int)ksplit;
      Dm.bnd = Dt.bnd + rf * Dt.cstride;
      Dm.tags = Dt.tags + rf * Dt.tstride;
      Dm.prog = Dt.prog + ksplit;
      Dm.ring = (int)rm;
    }
    if (ck) {
      // the coarse pair: anchors of both curves, handing rows over through the pair's own
      // boundary rows (fewer rows of fewer columns).  A one-point curve keeps the exact DFD,
      // which is its closed-form answer.
      PairDesc& Dc = ((PairDesc*)(hbase + h_cdescs))[p];
      Dc = D;
      Dc.P = (const double*)(dbase + cP[p]);
      Dc.Q = (const double*)(dbase + cQ[p]);
      if (n1 >= 2 && n2 >= 2) {
        Dc.n1 = (int)coarse_n(n1);
        Dc.n2 = (int)coarse_n(n2);
        Dc.cstride = (long long)align_up((size_t)Dc.n2, 32);
        Dc.ring = L.ring_c[p];
      }
    }
    PairState& s = hs[p];
    memset(&s, 0, sizeof(s));
    s.srch.tol = o.tol;
    s.srch.stop_mode = o.stop_mode;
    s.srch.max_probes = max_probes;
    s.quirks = o.reference_quirks;
    s.dense = o.dense;
    s.use_model = use_model ? 1 : 0;
    s.filter = o.precision == RFD_PREC_FP32_FILTER ? 1 : 0;
    s.blo = s.bhi = NAN;
    s.coarse = (ck && n1 >= 2 && n2 >= 2) ? 1 : 0;
    s.formula = formula[p];
    if (o.bracket && mode == MODE_DISTANCE) {
      s.blo = o.bracket[2 * p];
      s.bhi = o.bracket[2 * p + 1];
    }
    if (mode == MODE_DECIDE) {
      s.decide_only = 1;
      s.split = radius;
      s.r2 = radius * radius;
    }
  }
  // k-ary members: the pair's team descriptor with boundary rows, tags and progress words of
  // their own; states idle (PH_KWAIT) until a round starts them
  for (int64_t v = 0; v < nmem; ++v) {
    const int64_t p = mpair(v), idx = npairs + v;
    PairDesc* td = (PairDesc*)(hbase + L.h_tdescs);
    td[idx] = td[p];
    td[idx].bnd = (double*)(dbase + mbnd[v]);
    td[idx].tags = (unsigned*)(dbase + mtags[v]);
    td[idx].prog = (Prog*)(dbase + mprog[v]);
    PairState& m = hs[idx];
    memset(&m, 0, sizeof(m));
    m.quirks = hs[p].quirks;
    m.dense = hs[p].dense;
    m.filter = hs[p].filter;
    m.formula = hs[p].formula;
    m.use_model = hs[p].use_model;
    m.epoch = 1;
    m.dead_from = INT_MAX;
    m.U = (double)INFINITY;
    m.phase = PH_KWAIT;
    m.kary_real = (int)p;
    if (v % (karity - 1) == 0) {
      hs[p].kary_real = (int)p;
      hs[p].kary_base = (int)idx;
      hs[p].kary_cap = karity - 1;
    }
  }
  // launch windows: first team item of each (split pairs: forward windows, then the mirrors')
  std::vector<int> wstart(2 * (nwin + 1), 0);
  for (int64_t v = mbase; v < nst; ++v) {  // mirrors: idle until split_sync_kernel
    PairState& m = hs[v];
    memset(&m, 0, sizeof(m));
    m.epoch = 1;
    m.dead_from = INT_MAX;
    m.U = (double)INFINITY;
    m.phase = PH_DONE;
  }
  {
    int64_t k = 0;
    for (int64_t sidx = 0; sidx < maxS; ++sidx)
      for (int64_t q = 0; q < npairs; ++q) {
        const int p = order[q];
        if (sidx < (n1s[p] + 31) / 32) hi[k++] = make_int2(p, (int)sidx);
      }
    int2* ht = (int2*)(hbase + L.h_titems);
    k = 0;
    // with split pairs: the forward kernel's list (every pair, a split pair's strips 0 .. k-1),
    // then the mirror kernel's, each strip-major
    if (nsplit) {
      const int64_t lim = twin ? nwin * twin : maxSt;  // (windows cover every strip)
      for (int64_t sidx = 0; sidx < lim; ++sidx) {
        if (twin && sidx % twin == 0) wstart[sidx / twin] = (int)k;
        for (int64_t q = 0; q < npairs; ++q) {
          const int p = order[q];
          if (sidx < (ksp[p] ? ksp[p] : (trows(p) + 31) / 32)) ht[k++] = make_int2(p, (int)sidx);
        }
      }
      if (twin) wstart[nwin] = (int)k;
      for (int64_t sidx = 0; sidx < lim; ++sidx) {
        if (twin && sidx % twin == 0) wstart[nwin + 1 + sidx / twin] = (int)k;
        for (int64_t q = 0; q < npairs; ++q) {
          const int p = order[q];
          if (ksp[p] && sidx < (trows(p) - 1 + 31) / 32 - ksp[p])
            ht[k++] = make_int2((int)mirror_of[p], (int)sidx);
        }
      }
      if (twin) wstart[2 * nwin + 1] = (int)k;
    }
    for (int64_t sidx = 0; sidx < (nsplit ? 0 : maxSt); ++sidx) {
      if (twin && sidx % twin == 0) wstart[sidx / twin] = (int)k;  // strip-major: windows are ranges
      for (int64_t q = 0; q < npairs; ++q) {
        const int p = order[q];
        if (sidx < (trows(p) + 31) / 32) {
          ht[k++] = make_int2(p, (int)sidx);
          for (int m = 0; m < hs[p].kary_cap; ++m)
            ht[k++] = make_int2(hs[p].kary_base + m, (int)sidx);
        }
      }
    }
    if (twin && !nsplit) wstart[nwin] = (int)k;
  }

  if (!on_device) {
    // Copy every curve into the pinned staging area (compacting repeated points with
    // drop_repeats).  Large batches split the pairs over host threads by bytes: a single
    // thread copying pageable memory was a good part of a 4096-pair call.
    auto work = [&](int64_t p0, int64_t p1) {
      for (int64_t p = p0; p < p1; ++p) {
        const int d = dims[p];
        if (drop) {
          copy_kept((double*)(hbase + L.hP[p]), c1s[p], in_n1s[p], d);
          copy_kept((double*)(hbase + L.hQ[p]), c2s[p], in_n2s[p], d);
        } else {
          memcpy(hbase + L.hP[p], c1s[p], sizeof(double) * n1s[p] * d);
          memcpy(hbase + L.hQ[p], c2s[p], sizeof(double) * n2s[p] * d);
        }
      }
    };
    const size_t bytes = curves_end - curves_begin;
    const unsigned hw = std::thread::hardware_concurrency();
    const int nt = bytes >= ((size_t)32 << 20) ? (int)std::min(8u, std::max(1u, hw)) : 1;
    bool done = false;
    if (nt > 1) {
      std::vector<int64_t> cut(nt + 1, npairs);
      cut[0] = 0;
      size_t acc = 0;
      int k = 1;
      for (int64_t p = 0; p < npairs && k < nt; ++p) {
        acc += sizeof(double) * (size_t)(in_n1s[p] + in_n2s[p]) * dims[p];
        if (acc >= bytes / nt * k) cut[k++] = p + 1;
      }
      try {
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t) th.emplace_back(work, cut[t], cut[t + 1]);
        for (auto& t : th) t.join();
        done = true;
      } catch (...) {
        done = false;  // no thread could be started: copy on this one
      }
    }
    if (!done) work(0, npairs);
  }

  // ---------------- transfers
  cudaStream_t st = ctx->stream;
  size_t h2d_bytes = sizeof(PairDesc) * (npairs + nst) + sizeof(PairState) * nst +
                     sizeof(int2) * (nitems + ntitems) + sizeof(int);
  if (!on_device)
    for (int64_t p = 0; p < npairs; ++p) h2d_bytes += sizeof(double) * (n1s[p] + n2s[p]) * dims[p];
  // k-ary rounds run while at most kary_gate pairs are active (RFD_ARITY_GATE, read per call)
  int kary_gate = std::max(1, ctx->team_grid[K_DEC] / std::max(1, 2 * karity));
  if (const char* kg = getenv("RFD_ARITY_GATE"))
    if (atoi(kg) >= 1) kary_gate = atoi(kg);
  int* hmisc = (int*)(hbase + L.h_misc);  // [0] active pairs, [1] error word read back
  hmisc[0] = (int)npairs;
  hmisc[1] = 0;
  const rfd_model* gmodel = use_model ? o.model : nullptr;
  if (gmodel) {  // activation buffers allocated now: the launches below allocate nothing
    const int rc = rfd_mlp::reserve(const_cast<rfd_model*>(gmodel), (int)npairs);
    if (rc) return rc;
  }

  // Transfers, launches and the results' read-back.  With rfd_options.graph they are captured
  // as one CUDA graph; a later call with the same layout (sizes, options, workspace) replays it,
  // reading the new inputs from the same pinned staging area.
  int launches = 0;
  // Phase events.  Inside a stream capture a plain record only orders the capture; an
  // external record becomes a graph node, so the replayed graph records the events.
  auto record = [&](int k) {
    return cudaEventRecordWithFlags(ctx->ev[k], st,
                                    o.graph ? cudaEventRecordExternal : cudaEventRecordDefault);
  };
  auto issue = [&]() -> int {
    RFD_CUDA(cudaMemcpyAsync(dbase + L.descs, hbase + L.h_descs, sizeof(PairDesc) * npairs,
                             cudaMemcpyHostToDevice, st));
    if (ck) {
      RFD_CUDA(cudaMemcpyAsync(dbase + cdescs, hbase + h_cdescs, sizeof(PairDesc) * npairs,
                               cudaMemcpyHostToDevice, st));
      h2d_bytes += sizeof(PairDesc) * npairs;
    }
    RFD_CUDA(cudaMemcpyAsync(dbase + L.states, hbase + L.h_states, sizeof(PairState) * nst,
                             cudaMemcpyHostToDevice, st));
    RFD_CUDA(cudaMemcpyAsync(dbase + L.items, hbase + L.h_items, sizeof(int2) * nitems,
                             cudaMemcpyHostToDevice, st));
    RFD_CUDA(cudaMemcpyAsync(dbase + L.tdescs, hbase + L.h_tdescs, sizeof(PairDesc) * nst,
                             cudaMemcpyHostToDevice, st));
    RFD_CUDA(cudaMemcpyAsync(dbase + L.titems, hbase + L.h_titems, sizeof(int2) * ntitems,
                             cudaMemcpyHostToDevice, st));
    if (dcompact) {
      // the caller's curves (pointers refreshed every call) compacted into the workspace
      RFD_CUDA(cudaMemcpyAsync(dbase + src_off, hbase + h_src, sizeof(SrcCurve) * 2 * npairs,
                               cudaMemcpyHostToDevice, st));
      h2d_bytes += sizeof(SrcCurve) * 2 * npairs;
      compact_kept_kernel<<<(int)std::min<int64_t>(2 * npairs, 8 * ctx->num_sms), 256, 0, st>>>(
          (const SrcCurve*)(dbase + src_off), (int)(2 * npairs));
      RFD_CUDA(cudaGetLastError());
      ++launches;
    }
    if (!on_device && curves_end > curves_begin) {
      // the device curve region mirrors the staging area byte for byte: one copy
      RFD_CUDA(cudaMemcpyAsync(dbase + curves_begin, hbase + L.h_curves, curves_end - curves_begin,
                               cudaMemcpyHostToDevice, st));
    }
    RFD_CUDA(cudaMemsetAsync(dbase + L.zero_begin, 0, L.zero_end - L.zero_begin, st));
    RFD_CUDA(cudaMemcpyAsync(dbase + L.active, hmisc, sizeof(int), cudaMemcpyHostToDevice, st));

    // ---------------- launches
    const PairDesc* dd = (const PairDesc*)(dbase + L.descs);
    const PairDesc* dt = (const PairDesc*)(dbase + L.tdescs);  // team strips' orientation
    PairState* ds = (PairState*)(dbase + L.states);
    const int start_phase = mode == MODE_DECIDE ? PH_SEARCH : PH_DFD;
    if (ctx->timing) RFD_CUDA(record(0));
    launches = 1;
    prep_kernel<<<(int)std::min<int64_t>(npairs, 8 * ctx->num_sms), 256, 0, st>>>(dt, ds, (int)npairs,
                                                                                  start_phase);
    RFD_CUDA(cudaGetLastError());
    WaveArgs wa{};
    wa.pairs = dt;
    wa.st = ds;
    wa.items = (const int2*)(dbase + L.titems);
    wa.nitems = L.ntitems;
    wa.error = (int*)(dbase + L.error);
    wa.active_pairs = (int*)(dbase + L.active);
    wa.spin_cycles = ctx->spin_cycles;
    wa.prof = ctx->prof ? (unsigned long long*)(dbase + prof_off) : nullptr;
    unsigned* counters = (unsigned*)(dbase + L.counters);
    int li = 0;
    // boundary rows of the pairs about to run `ph` back to "not yet written" (team strips)
    // (at least 32 blocks per pair: late probe rounds leave a few large pairs active)
    const int fill_gy = (int)std::min<int64_t>(nst, 8 * ctx->num_sms);
    const int fill_gx = std::max(32, 8 * ctx->num_sms / fill_gy);
    auto fill = [&](int ph) {
      bnd_fill_kernel<<<dim3(fill_gx, fill_gy), 256, 0, st>>>(dt, ds, (int)nst, ph, wa.gate,
                                                               wa.active_pairs, wa.gate_min);
      ++launches;
    };
    // One VE-FD phase or probe round of the team strips: the rows reset and one launch, or
    // with launch windows a reset and a launch per window, in strip order (each window's
    // items are a range of the strip-major item list).
    unsigned* wtick = counters + wbase;
    auto team_round = [&](auto kind, int ph) -> int {
      constexpr int KIND = decltype(kind)::value;
      if (nsplit) {
        // the forward halves here (the first nfwd items), the mirror halves on the side stream
        // (the others, a ticket of their own), each on half the teams; then the meets
        split_sync_kernel<<<1, 32, 0, st>>>(dt, ds, (int)mbase, (int)nsplit, ph);
        const int half = std::max(1, ctx->team_grid[KIND] / 2);
        // one pass: the forward list here, the mirror list on the side stream, together
        auto both = [&](const WaveArgs& wf, const WaveArgs& wm) -> int {
          RFD_CUDA(cudaEventRecordWithFlags(ctx->fork_ev, st, cudaEventRecordDefault));
          RFD_CUDA(cudaStreamWaitEvent(ctx->side, ctx->fork_ev, 0));
          if (wm.nitems > 0) launch_team<KIND, true>(ctx, wm, ctx->side, half);
          RFD_CUDA(cudaGetLastError());
          RFD_CUDA(cudaEventRecordWithFlags(ctx->join_ev, ctx->side, cudaEventRecordDefault));
          if (wf.nitems > 0) launch_team<KIND>(ctx, wf, st, half);
          RFD_CUDA(cudaGetLastError());
          RFD_CUDA(cudaStreamWaitEvent(st, ctx->join_ev, 0));
          return RFD_OK;
        };
        if (!twin) {
          fill(ph);
          WaveArgs wf = wa, wm = wa;
          wf.nitems = (int)nfwd;
          wm.items = wa.items + nfwd;
          wm.nitems = (int)nmir;
          wm.ticket = wtick++;
          const int rc = both(wf, wm);
          if (rc) return rc;
        } else {
          // launch windows: window g of every half at once, its rows reset first
          const int2* items0 = (const int2*)(dbase + L.titems);
          for (int64_t g = 0; g < nwin; ++g) {
            team_window_fill_kernel<<<dim3(fill_gx, fill_gy), 256, 0, st>>>(
                dt, ds, (int)nst, ph, (int)(g * twin), (int)twin);
            WaveArgs wf = wa, wm = wa;
            wf.items = items0 + wstart[g];
            wf.nitems = wstart[g + 1] - wstart[g];
            wf.ticket = wtick++;
            wm.items = items0 + wstart[nwin + 1 + g];
            wm.nitems = wstart[nwin + 2 + g] - wstart[nwin + 1 + g];
            wm.ticket = wtick++;
            const int rc = both(wf, wm);
            if (rc) return rc;
          }
          launches += (int)(3 * nwin - 2);
        }
        split_meet_kernel<KIND><<<(int)nsplit, 1024, 0, st>>>(dt, ds, (int)mbase, ph, wa.error,
                                                              wa.active_pairs);
        launches += 3;
        return RFD_OK;
      }
      if (!twin) {
        fill(ph);
        launch_team<KIND>(ctx, wa, st);
        return RFD_OK;
      }
      WaveArgs w = wa;
      const int2* items0 = (const int2*)(dbase + L.titems);
      for (int64_t g = 0; g < nwin; ++g) {
        team_window_fill_kernel<<<dim3(fill_gx, fill_gy), 256, 0, st>>>(
            dt, ds, (int)nst, ph, (int)(g * twin), (int)twin);
        w.items = items0 + wstart[g];
        w.nitems = wstart[g + 1] - wstart[g];
        w.ticket = wtick++;
        launch_team<KIND>(ctx, w, st);
      }
      launches += (int)(2 * nwin - 1);  // the caller counts one team launch
      return RFD_OK;
    };
    if (mode != MODE_DECIDE) {
      wa.phase = PH_DFD;
      wa.ticket = counters + li++;
      // the DFD sweep runs on the coarse pairs when the coarse upper bound is asked for
      const PairDesc* ddfd = ck ? (const PairDesc*)(dbase + cdescs) : dd;
      if (ck) {
        coarse_prep_kernel<<<(int)std::min<int64_t>(npairs, 8 * ctx->num_sms), 256, 0, st>>>(
            dd, ddfd, ds, (int)npairs, ck);
        ++launches;
      }
      // The coarse pair has k times fewer points per curve: one row per lane gives its sweep
      // the most strips in flight (long pair, k = 6: 21 ms against 38 with four rows).
      const int rows = ck ? 1 : ctx->dfd_rows;
      {
        const int gy = (int)std::min<int64_t>(npairs, 8 * ctx->num_sms);
        const int gx = std::max(32, 8 * ctx->num_sms / gy);
        dfd_fill_kernel<<<dim3(gx, gy), 256, 0, st>>>(ddfd, (int)npairs, 32 * rows);
      }
      ++launches;
      wa.pairs = ddfd;  // the DFD sweep: given orientation, its own item list
      wa.items = (const int2*)(dbase + L.items);
      wa.nitems = L.nitems;
      {
        // skewed rows when the strips cannot fill the resident warps twice over (the sweep's
        // latency decides), stacked rows otherwise (instruction throughput decides)
        int64_t strips = 0;
        for (int64_t p = 0; p < npairs; ++p) {
          const int64_t n1 = ck && n1s[p] >= 2 && n2s[p] >= 2 ? coarse_n(n1s[p]) : n1s[p];
          strips += (n1 + 32 * rows - 1) / (32 * rows);
        }
        const int* grid = ck ? ctx->dfd_grid_infl : ctx->dfd_grid;
        const int sk = ctx->dfd_skew >= 0 ? ctx->dfd_skew
                                           : (strips < 2 * (int64_t)grid[1] * (kBlock / 32) ? 1 : 0);
        const int g = grid[sk];
        switch (ck ? 100 + sk : ctx->dfd_rows * 2 + sk) {
          case 100: dfd_kernel<1, false, true><<<g, kBlock, 0, st>>>(wa); break;
          case 101: dfd_kernel<1, true, true><<<g, kBlock, 0, st>>>(wa); break;
          case 2: dfd_kernel<1, false><<<g, kBlock, 0, st>>>(wa); break;
          case 3: dfd_kernel<1, true><<<g, kBlock, 0, st>>>(wa); break;
          case 4: dfd_kernel<2, false><<<g, kBlock, 0, st>>>(wa); break;
          case 5: dfd_kernel<2, true><<<g, kBlock, 0, st>>>(wa); break;
          case 8: dfd_kernel<4, false><<<g, kBlock, 0, st>>>(wa); break;
          case 9: dfd_kernel<4, true><<<g, kBlock, 0, st>>>(wa); break;
          case 16: dfd_kernel<8, false><<<g, kBlock, 0, st>>>(wa); break;
          default: dfd_kernel<8, true><<<g, kBlock, 0, st>>>(wa); break;
        }
      }
      wa.pairs = dt;
      wa.items = (const int2*)(dbase + L.titems);
      wa.nitems = L.ntitems;
      RFD_CUDA(cudaGetLastError());
      if (ctx->timing) RFD_CUDA(record(1));
      for (int ph : {PH_VEFD, PH_VEFD_DENSE}) {
        wa.phase = ph;
        wa.ticket = counters + li++;
        if (ctx->solo) {
          wave_kernel<K_VEFD><<<ctx->grid[K_VEFD], kBlock, 0, st>>>(wa);
        } else {
          const int rc = team_round(std::integral_constant<int, K_VEFD>{}, ph);
          if (rc) return rc;
        }
        RFD_CUDA(cudaGetLastError());
      }
      launches += 3;
      if (use_model) {
        rfd_model* md = const_cast<rfd_model*>(o.model);
        if (rfd_mlp::model_device(md) != ctx->device)
          return fail(RFD_ERR_ARG, "the model lives on another device");
        float* feat = (float*)(dbase + feat_off);
        float* yout = (float*)(dbase + y_off);
        bracket_features_kernel<<<(int)std::min<int64_t>(npairs, 16 * ctx->num_sms), kFeatThreads, 0,
                                  st>>>(dd, ds, (int)npairs, feat);
        RFD_CUDA(cudaGetLastError());
        int rc2 = rfd_mlp::infer(md, feat, (int)npairs, yout, st);
        if (rc2) return rc2;
        bracket_apply_kernel<<<(int)std::min<int64_t>((npairs + 255) / 256, 1024), 256, 0, st>>>(
            ds, (int)npairs, yout, wa.active_pairs);
        RFD_CUDA(cudaGetLastError());
        launches += 2 + 4;
      }
    }
    if (ctx->timing) RFD_CUDA(record(2));
    const int nprobe = mode == MODE_DECIDE ? 1 : max_probes;
    wa.kary_k = karity;
    wa.kary_gate = kary_gate;
    if (dyn_cap) {
      // Probe rounds as single launches while many pairs are active (the rounds then keep
      // every team busy, and a launch interleaves all pairs' strips), each skipped once
      // fewer than search_switch remain; the continuous search finishes the rest.
      for (int k = 0; k < nprobe; ++k) {
        wa.phase = PH_SEARCH;
        wa.ticket = counters + li++;
        wa.gate = (int*)(counters + L.nlaunch + k);
        wa.gate_min = ctx->search_switch;
        fill(PH_SEARCH);
        launch_team<K_DEC>(ctx, wa, st);
        RFD_CUDA(cudaGetLastError());
        ++launches;
      }
      wa.gate = nullptr;
      // every probe of every pair in one launch: the queue starts unpublished (all ones)
      RFD_CUDA(cudaMemsetAsync(dbase + dyn_off, 0xff, sizeof(unsigned long long) * dyn_cap, st));
      wa.phase = PH_SEARCH;
      wa.ticket = counters + (L.nlaunch - 2);
      wa.dyn_items = (unsigned long long*)(dbase + dyn_off);
      wa.dyn_tail = counters + (L.nlaunch - 1);
      wa.dyn_cap = dyn_cap;
      wa.window = ctx->search_window;
      wa.window_teams = ctx->team_grid[K_DEC];
      const int nstatic = wa.nitems;
      wa.nitems = 0;  // every strip comes from the queue
      fill(PH_SEARCH);
      if (nmem) {  // the members' boundary rows: not yet written
        member_fill_kernel<<<dim3(64, (unsigned)std::min<int64_t>(nmem, 1024)), 256, 0, st>>>(
            dt, (int)npairs, (int)nmem);
        RFD_CUDA(cudaGetLastError());
        ++launches;
      }
      search_queue_init_kernel<<<(int)std::min<int64_t>((npairs + 255) / 256, 1024), 256, 0, st>>>(
          dt, ds, (int)npairs, wa);
      launch_team<K_DEC>(ctx, wa, st);
      RFD_CUDA(cudaGetLastError());
      launches += 2;
      wa.nitems = nstatic;
      wa.dyn_items = nullptr;
      wa.dyn_tail = nullptr;
      wa.dyn_cap = 0;
    }
    for (int k = 0; k < (dyn_cap ? 0 : nprobe); ++k) {
      wa.phase = PH_SEARCH;
      wa.ticket = counters + li++;
      if (ctx->solo) {
        wave_kernel<K_DEC><<<ctx->grid[K_DEC], kBlock, 0, st>>>(wa);
      } else {
        const int rc = team_round(std::integral_constant<int, K_DEC>{}, PH_SEARCH);
        if (rc) return rc;
      }
      RFD_CUDA(cudaGetLastError());
      ++launches;
    }
    if (ctx->timing) RFD_CUDA(record(3));

    // ---------------- results
    RFD_CUDA(cudaMemcpyAsync(hs, ds, sizeof(PairState) * npairs, cudaMemcpyDeviceToHost, st));
    RFD_CUDA(cudaMemcpyAsync(hmisc + 1, wa.error, sizeof(int), cudaMemcpyDeviceToHost, st));
    return RFD_OK;
  };
  const bool use_graph = o.graph != 0;
  uint64_t key = 1469598103934665603ull;  // FNV-1a over everything the launches depend on
  auto mix = [&](const void* p, size_t n) {
    const unsigned char* b = (const unsigned char*)p;
    for (size_t i = 0; i < n; ++i) key = (key ^ b[i]) * 1099511628211ull;
  };
  if (use_graph) {
    const int flags[] = {mode, (int)on_device, (int)drop, ck, max_probes, o.stop_mode, o.reference_quirks,
                         o.dense, o.precision, o.bracket != nullptr, ctx->timing, ctx->prof,
                         ctx->solo, ctx->dfd_rows, ctx->dfd_skew, ctx->lockstep,
                         ctx->search_switch, ctx->search_window, ctx->team_warps,
                         (int)(ctx->spin_cycles >> 32),
                         (int)(ctx->spin_cycles & 0xffffffff), karity, kary_gate, (int)twin,
                         (int)nsplit, ctx->split_min};
    const void* ptrs[] = {dbase, hbase, gmodel, gmodel ? rfd_mlp::buffers_id(gmodel) : nullptr,
                          (const void*)st};
    mix(flags, sizeof(flags));
    mix(ptrs, sizeof(ptrs));
    mix(&o.tol, sizeof(o.tol));
    mix(&npairs, sizeof(npairs));
    mix(n1s, sizeof(int64_t) * npairs);
    mix(n2s, sizeof(int64_t) * npairs);
    mix(dims, sizeof(int32_t) * npairs);
    mix(formula.data(), sizeof(int) * formula.size());
    if (!kpairs.empty()) mix(kpairs.data(), sizeof(int64_t) * kpairs.size());
  }
  if (use_graph && ctx->gexec && ctx->gkey == key) {
    RFD_CUDA(cudaGraphLaunch(ctx->gexec, st));
    launches = ctx->glaunches;
  } else {
    if (use_graph) {
      if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
      ctx->gexec = nullptr;
      RFD_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    }
    const int rc = issue();
    if (use_graph) {
      cudaGraph_t g = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(st, &g);
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (ec != cudaSuccess) return fail(RFD_ERR_CUDA, std::string("cudaStreamEndCapture: ") +
                                                          cudaGetErrorString(ec));
      cudaGraphExec_t ex = nullptr;
      const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      if (ei != cudaSuccess) return fail(RFD_ERR_CUDA, std::string("cudaGraphInstantiate: ") +
                                                          cudaGetErrorString(ei));
      ctx->gexec = ex;
      ctx->gkey = key;
      ctx->glaunches = launches;
      RFD_CUDA(cudaGraphLaunch(ex, st));
    } else if (rc) {
      return rc;
    }
  }
  RFD_CUDA(cudaStreamSynchronize(st));
  if (guard) {
    std::vector<unsigned char> g(guard);
    RFD_CUDA(cudaMemcpy(g.data(), dbase + L.total, guard, cudaMemcpyDeviceToHost));
    size_t bad = 0, first = guard, last = 0;
    for (size_t k = 0; k < guard; ++k)
      if (g[k] != 0xA5) {
        ++bad;
        first = std::min(first, k);
        last = k;
      }
    if (bad)
      fprintf(stderr, "rfd guard: %zu bytes written past the workspace (offsets %zu..%zu of %zu)\n",
              bad, first, last, guard);
  }
  if (hmisc[1] >= kCheckBase)
    return fail(RFD_ERR_INTERNAL, "device self-check " + std::to_string(hmisc[1] - kCheckBase) +
                                      " failed (boundary ring index out of range)");
  if (hmisc[1]) return fail(RFD_ERR_TIMEOUT, "an inter-warp wait exceeded its budget");
  if (ctx->prof) {
    std::vector<unsigned long long> pc(kTraceBase + kTraceW * kTrace);
    RFD_CUDA(cudaMemcpy(pc.data(), dbase + prof_off, sizeof(unsigned long long) * pc.size(),
                        cudaMemcpyDeviceToHost));
    fprintf(stderr,
            "rfd prof (Mcycles): in_wait %.1f jump %.1f tile_wait %.1f steps %.1f strip_total %.1f |"
            " chunks %llu jumps %llu strips %llu | helpers: tile %.1f (staging %.1f) req_wait %.1f"
            " tiles %llu | flush %.1f flushes %llu\n",
            pc[0] / 1e6, pc[1] / 1e6, pc[2] / 1e6, pc[3] / 1e6, pc[4] / 1e6, pc[5], pc[6], pc[7],
            pc[8] / 1e6, pc[13] / 1e6, pc[9] / 1e6, pc[10], pc[11] / 1e6, pc[12]);
    // strip chain of the first pair: handoff = first live input of strip s after the first
    // live output of strip s-1; lag = first live output of strip s after its first live input
    // (lag split: input -> its tile taken -> its steps done -> the next chunk's input in hand
    // -> the first live output flushed)
    std::vector<double> hand, lag, adv, l1, l2, l3, l4;
    const unsigned long long* tr = pc.data() + kTraceBase;
    for (int s = 1; s < kTrace; ++s) {
      const unsigned long long* t = tr + kTraceW * s;
      const unsigned long long in = t[1], out = t[2], pout = tr[kTraceW * (s - 1) + 2];
      if (!in || !out || !pout) continue;
      hand.push_back((double)in - (double)pout);
      lag.push_back((double)out - (double)in);
      adv.push_back((double)out - (double)pout);
      if (t[3] && t[4] && t[5]) {
        l1.push_back((double)t[3] - (double)in);
        l2.push_back((double)t[4] - (double)t[3]);
        l3.push_back((double)t[5] - (double)t[4]);
        l4.push_back((double)out - (double)t[5]);
      }
    }
    auto med = [](std::vector<double> v) {
      if (v.empty()) return 0.0;
      std::sort(v.begin(), v.end());
      return v[v.size() / 2];
    };
    fprintf(stderr, "rfd trace (ns, median over %zu strips): handoff %.0f  lag %.0f  advance %.0f\n",
            hand.size(), med(hand), med(lag), med(adv));
    fprintf(stderr, "rfd trace lag split (ns, %zu strips): input->tile %.0f  tile->steps %.0f  "
            "steps->next input %.0f  next input->output %.0f\n",
            l1.size(), med(l1), med(l2), med(l3), med(l4));
    // batch: when pairs ended their searches (ms after the first), and the last ones
    if (npairs > 1) {
      std::vector<std::pair<unsigned long long, int64_t>> fin;
      for (int64_t p = 0; p < npairs; ++p)
        if (hs[p].t_done) fin.push_back({hs[p].t_done, p});
      std::sort(fin.begin(), fin.end());
      if (!fin.empty()) {
        const double t0 = (double)fin.front().first;
        auto at = [&](double q) {
          return ((double)fin[std::min(fin.size() - 1, (size_t)(q * fin.size()))].first - t0) / 1e6;
        };
        fprintf(stderr, "rfd search ends (ms after the first, %zu pairs): 50%% %.1f  90%% %.1f  "
                "97%% %.1f  99%% %.1f  last %.1f\n", fin.size(), at(0.5), at(0.9), at(0.97),
                at(0.99), ((double)fin.back().first - t0) / 1e6);
        for (size_t k = fin.size() > 12 ? fin.size() - 12 : 0; k < fin.size(); ++k) {
          const int64_t p = fin[k].second;
          const PairDesc& Dt = ((const PairDesc*)(hbase + L.h_tdescs))[p];
          fprintf(stderr, "  pair %lld: %d x %d (team strips %d%s), probes %d, ended %.1f ms\n",
                  (long long)p, hd[p].n1, hd[p].n2, (Dt.n1 - 1 + 31) / 32,
                  Dt.tr ? ", transposed" : "", hs[p].srch.probes,
                  ((double)fin[k].first - t0) / 1e6);
        }
      }
    }
  }
  if (ctx->timing) {
    float a = 0.f, b = 0.f, c = 0.f;
    if (mode != MODE_DECIDE) {
      RFD_CUDA(cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]));
      RFD_CUDA(cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[2]));
      RFD_CUDA(cudaEventElapsedTime(&c, ctx->ev[2], ctx->ev[3]));
    } else {
      RFD_CUDA(cudaEventElapsedTime(&c, ctx->ev[0], ctx->ev[3]));
    }
    ctx->acc[0] += a;
    ctx->acc[1] += b;
    ctx->acc[2] += c;
    ctx->acc[3] += 1;
    ctx->acc[4] += launches;
  }
  ctx->acc[5] += (double)h2d_bytes;
  ctx->acc[6] += (double)(sizeof(PairState) * npairs + sizeof(int));
  for (int64_t p = 0; p < npairs; ++p) {
    const PairState& s = hs[p];
    rfd_result& r = out[p];
    memset(&r, 0, sizeof(r));
    r.dfd = s.dfd;
    r.vefd = s.vefd;
    r.endpoint = s.endpoint;
    r.lb = s.srch.lb;
    r.ub = s.srch.ub;
    r.distance = s.distance;
    r.probes = s.srch.probes;
    r.flags = s.flags | s.srch.flags;
    r.cells_nominal = (int64_t)s.cells_nominal;
    r.cells_evaluated = (int64_t)s.cells_eval;
    r.cells_fp64 = (int64_t)(s.filter ? s.cells_fp64 : s.cells_eval);
    r.cells_vefd = (int64_t)s.cells_vefd;
    if (mode == MODE_DECIDE) r.distance = s.result;  // propagated right UB of the last cell
    if (mode == MODE_DISTANCE && s.phase != PH_DONE)
      return fail(RFD_ERR_INTERNAL, "pair " + std::to_string(p) + " did not finish");
  }
  return RFD_OK;
}

}  // namespace

// ============================================================================ C ABI

extern "C" {

int32_t rfd_abi_version(void) { return RFD_ABI_VERSION; }

const char* rfd_status_string(int32_t s) {
  switch (s) {
    case RFD_OK: return "ok";
    case RFD_ERR_ARG: return "invalid argument";
    case RFD_ERR_CUDA: return "CUDA error";
    case RFD_ERR_NOMEM: return "out of memory";
    case RFD_ERR_TIMEOUT: return "inter-warp wait timed out";
    case RFD_ERR_NODEV: return "no CUDA device";
    case RFD_ERR_INTERNAL: return "internal error";
    case RFD_ERR_LIMIT: return "size limit exceeded";
    default: return "unknown status";
  }
}

const char* rfd_last_error(void) { return g_last_error.c_str(); }

void rfd_options_init(rfd_options* o, int32_t precise) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  if (precise) {
    o->stop_mode = RFD_STOP_REL;
    o->tol = 0x1p-33;
    o->reference_quirks = 0;
  } else {
    o->stop_mode = RFD_STOP_ABS;
    o->tol = (double)FLT_EPSILON;
    o->reference_quirks = 1;
  }
  o->max_probes = 64;
  o->dense = 0;
  o->precision = RFD_PREC_FP64;
  o->memory = RFD_MEM_HOST;
  o->bracket = nullptr;
}

int32_t rfd_context_create(int32_t device, rfd_context** out) {
  if (!out) return fail(RFD_ERR_ARG, "null context pointer");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(RFD_ERR_NODEV, "no CUDA device");
  }
  if (device < 0 || device >= n) return fail(RFD_ERR_ARG, "device index");
  RFD_CUDA(cudaSetDevice(device));
  rfd_context* c = new rfd_context();
  c->device = device;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
    delete c;
    return fail(RFD_ERR_CUDA, "cudaGetDeviceProperties");
  }
  c->num_sms = prop.multiProcessorCount;
  int occ[3] = {0, 0, 0};
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], wave_kernel<K_VEFD>, kBlock, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[2], wave_kernel<K_DEC>, kBlock, 0);
  for (int k = 0; k < 3; ++k) c->grid[k] = std::max(1, occ[k]) * c->num_sms;
  {
    const size_t sm_ve = team_smem_bytes<K_VEFD>(), sm_dec = team_smem_bytes<K_DEC>();
    if (cudaFuncSetAttribute(team_kernel<K_VEFD, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm_ve) != cudaSuccess ||
        cudaFuncSetAttribute(team_kernel<K_DEC, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm_dec) != cudaSuccess ||
        cudaFuncSetAttribute(team_kernel<K_VEFD, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm_ve) != cudaSuccess ||
        cudaFuncSetAttribute(team_kernel<K_DEC, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm_dec) != cudaSuccess ||
        cudaFuncSetAttribute(team_kernel<K_VEFD, 8, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_ve) != cudaSuccess ||
        cudaFuncSetAttribute(team_kernel<K_DEC, 8, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_dec) != cudaSuccess ||
        cudaFuncSetAttribute(team_kernel<K_VEFD, 4, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_ve) != cudaSuccess ||
        cudaFuncSetAttribute(team_kernel<K_DEC, 4, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_dec) != cudaSuccess) {
      delete c;
      return fail(RFD_ERR_CUDA, "cudaFuncSetAttribute(team smem)");
    }
    int o[4] = {0, 0, 0, 0};
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[0], team_kernel<K_VEFD, 4>, 128, sm_ve);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[1], team_kernel<K_DEC, 4>, 128, sm_dec);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[2], team_kernel<K_VEFD, 8>, 256, sm_ve);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[3], team_kernel<K_DEC, 8>, 256, sm_dec);
    // RFD_TEAM_PER_SM (1 or more): caps the teams resident per SM (the grid is persistent)
    if (const char* tp = getenv("RFD_TEAM_PER_SM")) {
      const int cap = atoi(tp);
      if (cap >= 1)
        for (int k = 0; k < 4; ++k) o[k] = std::min(std::max(1, o[k]), cap);
    }
    c->team_grids[0][K_VEFD] = std::max(1, o[0]) * c->num_sms;
    c->team_grids[0][K_DEC] = std::max(1, o[1]) * c->num_sms;
    c->team_grids[1][K_VEFD] = std::max(1, o[2]) * c->num_sms;
    c->team_grids[1][K_DEC] = std::max(1, o[3]) * c->num_sms;
    const char* tw = getenv("RFD_TEAM_WARPS");
    c->team_warps = tw && strcmp(tw, "4") == 0 ? 4 : 8;
    for (int k = 0; k < 3; ++k) c->team_grid[k] = c->team_grids[team_shape_index(c->team_warps)][k];
    const char* e = getenv("RFD_SOLO");
    c->solo = e && e[0] == '1';
    const char* ls = getenv("RFD_LOCKSTEP");
    c->lockstep = ls && ls[0] == '1';
    c->search_switch = c->team_grid[K_DEC];  // fewer pairs than teams: rounds leave teams idle
    const char* sw = getenv("RFD_SEARCH_SWITCH");
    if (sw && atoi(sw) >= 0) c->search_switch = atoi(sw);
    const char* sn = getenv("RFD_SEARCH_WINDOW");
    if (sn && atoi(sn) >= 1) c->search_window = atoi(sn);
    const char* dr = getenv("RFD_DFD_ROWS");
    if (dr && (dr[0] == '1' || dr[0] == '2' || dr[0] == '4' || dr[0] == '8') && !dr[1])
      c->dfd_rows = dr[0] - '0';
    const char* dk = getenv("RFD_DFD_SKEW");
    if (dk && (dk[0] == '0' || dk[0] == '1') && !dk[1]) c->dfd_skew = dk[0] - '0';
    for (int ri = 0; ri < 4; ++ri)
      for (int sk = 0; sk < 2; ++sk) {
        int od = 0;
        switch ((1 << ri) * 2 + sk) {
          case 2: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&od, dfd_kernel<1, false>, kBlock, 0); break;
          case 3: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&od, dfd_kernel<1, true>, kBlock, 0); break;
          case 4: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&od, dfd_kernel<2, false>, kBlock, 0); break;
          case 5: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&od, dfd_kernel<2, true>, kBlock, 0); break;
          case 8: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&od, dfd_kernel<4, false>, kBlock, 0); break;
          case 9: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&od, dfd_kernel<4, true>, kBlock, 0); break;
          case 16: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&od, dfd_kernel<8, false>, kBlock, 0); break;
          default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&od, dfd_kernel<8, true>, kBlock, 0); break;
        }
        c->dfd_grid_all[ri][sk] = std::max(1, od) * c->num_sms;
      }
    for (int sk = 0; sk < 2; ++sk) {
      c->dfd_grid[sk] = c->dfd_grid_all[c->dfd_rows == 1 ? 0 : c->dfd_rows == 2 ? 1 : c->dfd_rows == 4 ? 2 : 3][sk];
      int od = 0;
      if (sk) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&od, dfd_kernel<1, true, true>, kBlock, 0);
      else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&od, dfd_kernel<1, false, true>, kBlock, 0);
      c->dfd_grid_infl[sk] = std::max(1, od) * c->num_sms;
    }
    const char* pe = getenv("RFD_PROF");
    c->prof = pe && pe[0] == '1';
    c->dfd_ring_rows = env_rows("RFD_DFD_RING_ROWS", kDfdRingRows);
    c->team_ring_rows = env_rows("RFD_TEAM_RING_ROWS", 0);
    if (const char* e = getenv("RFD_SPLIT"))
      if (*e) c->split_min = std::max(0, atoi(e));
  }
  // wait budget: about 20 s at the maximum SM clock, or RFD_SPIN_CYCLES
  c->spin_default = (long long)prop.clockRate * 1000LL * 20LL;
  c->spin_cycles = env_spin_cycles(c->spin_default);
  if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming) != cudaSuccess) {
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->fork_ev) cudaEventDestroy(c->fork_ev);
    if (c->join_ev) cudaEventDestroy(c->join_ev);
    delete c;
    return fail(RFD_ERR_CUDA, "cudaStreamCreate / cudaEventCreate");
  }
  c->stream = c->own_stream;
  *out = c;
  return RFD_OK;
}

int32_t rfd_context_destroy(rfd_context* ctx) {
  if (!ctx) return RFD_OK;
  cudaSetDevice(ctx->device);
  if (ctx->dws) cudaFree(ctx->dws);
  if (ctx->hws) cudaFreeHost(ctx->hws);
  for (int k = 0; k < 4; ++k)
    if (ctx->ev[k]) cudaEventDestroy(ctx->ev[k]);
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  if (ctx->side) cudaStreamDestroy(ctx->side);
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  if (ctx->join_ev) cudaEventDestroy(ctx->join_ev);
  delete ctx;
  return RFD_OK;
}

int32_t rfd_context_phase_times(rfd_context* ctx, int32_t enable, double* out) {
  if (!ctx) return fail(RFD_ERR_ARG, "null context");
  RFD_CUDA(cudaSetDevice(ctx->device));
  if (enable > 0 && !ctx->ev[0])
    for (int k = 0; k < 4; ++k) RFD_CUDA(cudaEventCreate(&ctx->ev[k]));
  if (enable >= 0) ctx->timing = enable > 0;
  if (out) {
    for (int k = 0; k < 7; ++k) {
      out[k] = ctx->acc[k];
      ctx->acc[k] = 0;
    }
  }
  return RFD_OK;
}

int32_t rfd_fp64_peak(rfd_context* ctx, double* tflops) {
  if (!ctx || !tflops) return fail(RFD_ERR_ARG, "null argument");
  RFD_CUDA(cudaSetDevice(ctx->device));
  int per_sm = 0;
  RFD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fp64_fma_kernel, 256, 0));
  const int blocks = std::max(1, per_sm) * ctx->num_sms;
  const int iters = 1 << 14;
  double* scratch = nullptr;
  RFD_CUDA(cudaMalloc(&scratch, sizeof(double)));
  cudaEvent_t e0, e1;
  RFD_CUDA(cudaEventCreate(&e0));
  RFD_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(e0, ctx->stream);
    fp64_fma_kernel<<<blocks, 256, 0, ctx->stream>>>(scratch, iters, 0.999999, 1e-7);
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0) best = std::min(best, ms);
  }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(scratch);
  if (e != cudaSuccess) return fail(RFD_ERR_CUDA, cudaGetErrorString(e));
  const double flops = 2.0 * 8.0 * (double)iters * (double)blocks * 256.0;
  *tflops = flops / (best * 1e-3) / 1e12;
  return RFD_OK;
}

int32_t rfd_context_set_wait_budget(rfd_context* ctx, int64_t cycles) {
  if (!ctx) return fail(RFD_ERR_ARG, "null context");
  ctx->spin_cycles = cycles > 0 ? (long long)cycles : ctx->spin_default;
  return RFD_OK;
}

int32_t rfd_context_set_stream(rfd_context* ctx, void* stream) {
  if (!ctx) return fail(RFD_ERR_ARG, "null context");
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return RFD_OK;
}

int32_t rfd_distance(rfd_context* ctx, const double* c1, int64_t n1, const double* c2, int64_t n2,
                     int32_t dims, const rfd_options* opt, rfd_result* out) {
  if (!ctx) return fail(RFD_ERR_ARG, "null context");
  RFD_CUDA(cudaSetDevice(ctx->device));
  return run_batch(ctx, 1, &c1, &n1, &c2, &n2, &dims, opt, out, MODE_DISTANCE, 0.0);
}

int32_t rfd_distance_batch(rfd_context* ctx, int64_t npairs, const double* const* c1s,
                           const int64_t* n1s, const double* const* c2s, const int64_t* n2s,
                           const int32_t* dims, const rfd_options* opt, rfd_result* out) {
  if (!ctx) return fail(RFD_ERR_ARG, "null context");
  RFD_CUDA(cudaSetDevice(ctx->device));
  if (npairs <= 1 || !c1s || !n1s || !c2s || !n2s || !dims || !out)
    return run_batch(ctx, npairs, c1s, n1s, c2s, n2s, dims, opt, out, MODE_DISTANCE, 0.0);
  // Pairs go in chunks whose device workspace stays within the budget: RFD_BATCH_BUDGET
  // bytes, else 3/4 of the device memory this context may use (its workspace and what is
  // free).  A call that fits runs whole (and may be a CUDA graph); chunks run one after
  // another without one.  Results do not depend on the chunking.
  double budget = 0.0;
  if (const char* e = getenv("RFD_BATCH_BUDGET")) budget = atof(e);
  if (!(budget > 0.0)) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      fr = 0;
    }
    budget = 0.75 * ((double)fr + (double)ctx->dws_size);
  }
  const int ck = opt ? opt->coarse_ub : 0;
  std::vector<double> bytes((size_t)npairs);
  double total = 0.0;
  for (int64_t p = 0; p < npairs; ++p) {
    if (n1s[p] < 1 || n2s[p] < 1 || (dims[p] != 2 && dims[p] != 3))
      return run_batch(ctx, npairs, c1s, n1s, c2s, n2s, dims, opt, out, MODE_DISTANCE, 0.0);
    bytes[p] = pair_workspace_bytes(ctx, n1s[p], n2s[p], dims[p], ck);
    total += bytes[p];
  }
  if (total <= budget)
    return run_batch(ctx, npairs, c1s, n1s, c2s, n2s, dims, opt, out, MODE_DISTANCE, 0.0);
  rfd_options o;
  rfd_options_init(&o, 0);
  if (opt) o = *opt;
  o.graph = 0;
  int64_t p0 = 0;
  while (p0 < npairs) {
    int64_t p1 = p0 + 1;
    double acc = bytes[p0];
    while (p1 < npairs && acc + bytes[p1] <= budget) acc += bytes[p1++];
    rfd_options oc = o;
    if (o.bracket) oc.bracket = o.bracket + 2 * p0;  // per-pair bracket: this chunk's slice
    const int rc = run_batch(ctx, p1 - p0, c1s + p0, n1s + p0, c2s + p0, n2s + p0, dims + p0, &oc,
                             out + p0, MODE_DISTANCE, 0.0);
    if (rc) return rc;
    p0 = p1;
  }
  return RFD_OK;
}

// Autotuner of the DFD sweep's tile shape: rows per lane (the strip height, 32 x 1, 2, 4 or 8)
// and the layout of a lane's rows (stacked: fewer instructions per cell; skewed: independent
// cells per step).  Each candidate sweeps the caller's pairs `reps` times (CUDA-event phase
// times of rfd_bounds-style calls); the fastest is kept in the context for later calls, which
// otherwise use 8 rows and choose the layout by strip count.
int32_t rfd_autotune(rfd_context* ctx, int64_t npairs, const double* const* c1s, const int64_t* n1s,
                     const double* const* c2s, const int64_t* n2s, const int32_t* dims,
                     const rfd_options* opt, int32_t reps, double* ms_out, int32_t* best_out) {
  if (!ctx || npairs < 1 || reps < 1 || reps > 100) return fail(RFD_ERR_ARG, "autotune arguments");
  RFD_CUDA(cudaSetDevice(ctx->device));
  if (!ctx->ev[0])
    for (int k = 0; k < 4; ++k) RFD_CUDA(cudaEventCreate(&ctx->ev[k]));
  rfd_options o;
  rfd_options_init(&o, 1);
  if (opt) o = *opt;
  o.graph = 0;
  const int rows[4] = {1, 2, 4, 8};
  const int keep_rows = ctx->dfd_rows, keep_skew = ctx->dfd_skew, keep_timing = ctx->timing;
  double keep_acc[7];
  memcpy(keep_acc, ctx->acc, sizeof(keep_acc));
  std::vector<rfd_result> res((size_t)npairs);
  double best = 1e300;
  int best_r = keep_rows, best_s = keep_skew;
  int rc = RFD_OK;
  for (int ri = 0; ri < 4 && rc == RFD_OK; ++ri)
    for (int sk = 0; sk < 2 && rc == RFD_OK; ++sk) {
      ctx->dfd_rows = rows[ri];
      ctx->dfd_skew = sk;
      ctx->dfd_grid[0] = ctx->dfd_grid_all[ri][0];
      ctx->dfd_grid[1] = ctx->dfd_grid_all[ri][1];
      ctx->timing = 1;
      for (int k = 0; k < 7; ++k) ctx->acc[k] = 0;
      // one untimed call (first use of the code path), then the timed ones
      rc = run_batch(ctx, npairs, c1s, n1s, c2s, n2s, dims, &o, res.data(), MODE_BOUNDS, 0.0);
      for (int k = 0; k < 7; ++k) ctx->acc[k] = 0;
      for (int r = 0; r < reps && rc == RFD_OK; ++r)
        rc = run_batch(ctx, npairs, c1s, n1s, c2s, n2s, dims, &o, res.data(), MODE_BOUNDS, 0.0);
      const double ms = rc == RFD_OK ? ctx->acc[0] / reps : -1.0;
      if (ms_out) ms_out[ri * 2 + sk] = ms;
      if (rc == RFD_OK && ms < best) {
        best = ms;
        best_r = rows[ri];
        best_s = sk;
      }
    }
  ctx->dfd_rows = rc == RFD_OK ? best_r : keep_rows;
  ctx->dfd_skew = rc == RFD_OK ? best_s : keep_skew;
  const int bi = ctx->dfd_rows == 1 ? 0 : ctx->dfd_rows == 2 ? 1 : ctx->dfd_rows == 4 ? 2 : 3;
  ctx->dfd_grid[0] = ctx->dfd_grid_all[bi][0];
  ctx->dfd_grid[1] = ctx->dfd_grid_all[bi][1];
  ctx->timing = keep_timing;
  memcpy(ctx->acc, keep_acc, sizeof(keep_acc));
  if (best_out) {
    best_out[0] = ctx->dfd_rows;
    best_out[1] = ctx->dfd_skew;
  }
  return rc;
}

// Autotuner of the team strips' shape and of the search's split between probe rounds run as
// launches and the continuous queue: warps per team (4: 3 helpers, twice the teams; 8: 7
// helpers), the switch point (active pairs below which the continuous search takes over: a
// quarter of the team count, the team count, or every pair from the first probe) and the start window (strips a probe queues ahead: 1, 2,
// 4).  Each candidate solves the caller's pairs once untimed and `reps` times timed (CUDA-event
// phase times of whole solves with the caller's options); the fastest is kept in the context.
int32_t rfd_autotune_search(rfd_context* ctx, int64_t npairs, const double* const* c1s,
                            const int64_t* n1s, const double* const* c2s, const int64_t* n2s,
                            const int32_t* dims, const rfd_options* opt, int32_t reps,
                            double* ms_out, int32_t* best_out) {
  if (!ctx || npairs < 1 || reps < 1 || reps > 100) return fail(RFD_ERR_ARG, "autotune arguments");
  RFD_CUDA(cudaSetDevice(ctx->device));
  if (!ctx->ev[0])
    for (int k = 0; k < 4; ++k) RFD_CUDA(cudaEventCreate(&ctx->ev[k]));
  rfd_options o;
  rfd_options_init(&o, 1);
  if (opt) o = *opt;
  o.graph = 0;
  const int keep_w = ctx->team_warps, keep_sw = ctx->search_switch, keep_win = ctx->search_window,
            keep_timing = ctx->timing;
  double keep_acc[7];
  memcpy(keep_acc, ctx->acc, sizeof(keep_acc));
  std::vector<rfd_result> res((size_t)npairs);
  const int warps[2] = {4, 8}, windows[3] = {1, 2, 4};
  double best = 1e300;
  int bw = keep_w, bs = keep_sw, bn = keep_win, rc = RFD_OK;
  for (int wi = 0; wi < 2 && rc == RFD_OK; ++wi)
    for (int si = 0; si < 3 && rc == RFD_OK; ++si)
      for (int ni = 0; ni < 3 && rc == RFD_OK; ++ni) {
        ctx->team_warps = warps[wi];
        for (int k = 0; k < 3; ++k) ctx->team_grid[k] = ctx->team_grids[wi][k];
        ctx->search_switch = si == 0 ? ctx->team_grid[K_DEC] / 4
                             : si == 1 ? ctx->team_grid[K_DEC] : INT32_MAX;
        ctx->search_window = windows[ni];
        ctx->timing = 1;
        rc = run_batch(ctx, npairs, c1s, n1s, c2s, n2s, dims, &o, res.data(), MODE_DISTANCE, 0.0);
        for (int k = 0; k < 7; ++k) ctx->acc[k] = 0;
        for (int r = 0; r < reps && rc == RFD_OK; ++r)
          rc = run_batch(ctx, npairs, c1s, n1s, c2s, n2s, dims, &o, res.data(), MODE_DISTANCE, 0.0);
        const double ms = rc == RFD_OK ? (ctx->acc[0] + ctx->acc[1] + ctx->acc[2]) / reps : -1.0;
        if (ms_out) ms_out[(wi * 3 + si) * 3 + ni] = ms;
        if (rc == RFD_OK && ms < best) {
          best = ms;
          bw = warps[wi];
          bs = ctx->search_switch;
          bn = windows[ni];
        }
      }
  ctx->team_warps = rc == RFD_OK ? bw : keep_w;
  for (int k = 0; k < 3; ++k) ctx->team_grid[k] = ctx->team_grids[team_shape_index(ctx->team_warps)][k];
  ctx->search_switch = rc == RFD_OK ? bs : keep_sw;
  ctx->search_window = rc == RFD_OK ? bn : keep_win;
  ctx->timing = keep_timing;
  memcpy(ctx->acc, keep_acc, sizeof(keep_acc));
  if (best_out) {
    best_out[0] = ctx->team_warps;
    best_out[1] = ctx->search_switch;
    best_out[2] = ctx->search_window;
  }
  return rc;
}

int32_t rfd_distance_matrix(rfd_context* ctx, int64_t ncurves, const double* const* curves,
                            const int64_t* ns, const int32_t* dims, const rfd_options* opt,
                            double budget_bytes, double* out, rfd_result* results) {
  if (!ctx || !curves || !ns || !dims || !out || ncurves < 1)
    return fail(RFD_ERR_ARG, "distance_matrix arguments");
  if (ncurves > (1 << 20)) return fail(RFD_ERR_LIMIT, "more than 2^20 curves");
  if (opt && opt->bracket) return fail(RFD_ERR_ARG, "distance_matrix takes no per-pair bracket");
  RFD_CUDA(cudaSetDevice(ctx->device));
  // pairs (i, j), i < j, go to the batch engine in chunks whose workspace (the boundary ring,
  // O(ring rows x columns) a pair, is the bulk of it) stays within the budget
  const double budget = budget_bytes > 0.0 ? budget_bytes : 8e9;
  const int64_t N = ncurves;
  std::vector<const double*> c1, c2;
  std::vector<int64_t> n1, n2, where;
  std::vector<int32_t> dm;
  std::vector<rfd_result> res;
  double acc = 0.0;
  auto flush = [&]() -> int {
    if (where.empty()) return RFD_OK;
    res.resize(where.size());
    const int rc = run_batch(ctx, (int64_t)where.size(), c1.data(), n1.data(), c2.data(), n2.data(),
                             dm.data(), opt, res.data(), MODE_DISTANCE, 0.0);
    if (rc) return rc;
    for (size_t k = 0; k < where.size(); ++k) {
      const int64_t i = where[k] / N, j = where[k] % N;
      out[i * N + j] = out[j * N + i] = res[k].distance;
      if (results) results[i * N - i * (i + 1) / 2 + (j - i - 1)] = res[k];
    }
    c1.clear(); c2.clear(); n1.clear(); n2.clear(); dm.clear(); where.clear();
    acc = 0.0;
    return RFD_OK;
  };
  for (int64_t i = 0; i < N; ++i) out[i * N + i] = 0.0;
  for (int64_t i = 0; i < N; ++i)
    for (int64_t j = i + 1; j < N; ++j) {
      if (dims[i] != dims[j]) return fail(RFD_ERR_ARG, "curves of a pair differ in dimension");
      const double bytes =
          pair_workspace_bytes(ctx, ns[i], ns[j], dims[i], opt ? opt->coarse_ub : 0);
      if (acc + bytes > budget && !where.empty()) {
        const int rc = flush();
        if (rc) return rc;
      }
      c1.push_back(curves[i]);
      c2.push_back(curves[j]);
      n1.push_back(ns[i]);
      n2.push_back(ns[j]);
      dm.push_back(dims[i]);
      where.push_back(i * N + j);
      acc += bytes;
    }
  return flush();
}

int32_t rfd_bounds(rfd_context* ctx, const double* c1, int64_t n1, const double* c2, int64_t n2,
                   int32_t dims, int32_t reference_quirks, int32_t dense, double* dfd, double* vefd) {
  if (!ctx || !dfd || !vefd) return fail(RFD_ERR_ARG, "null argument");
  RFD_CUDA(cudaSetDevice(ctx->device));
  rfd_options o;
  rfd_options_init(&o, 0);
  o.reference_quirks = reference_quirks;
  o.dense = dense;
  rfd_result r;
  int rc = run_batch(ctx, 1, &c1, &n1, &c2, &n2, &dims, &o, &r, MODE_BOUNDS, 0.0);
  if (rc) return rc;
  *dfd = r.dfd;
  if (!(r.flags & RFD_FLAG_VEFD_SKIPPED)) *vefd = r.vefd;
  return RFD_OK;
}

int32_t rfd_decide(rfd_context* ctx, const double* c1, int64_t n1, const double* c2, int64_t n2,
                   int32_t dims, double radius, int32_t dense, int32_t* reachable, double* right_ub) {
  return rfd_decide_formula(ctx, c1, n1, c2, n2, dims, radius, dense, RFD_FORMULA_FUSED, reachable,
                            right_ub);
}

int32_t rfd_decide_formula(rfd_context* ctx, const double* c1, int64_t n1, const double* c2,
                           int64_t n2, int32_t dims, double radius, int32_t dense, int32_t formula,
                           int32_t* reachable, double* right_ub) {
  if (!ctx || !reachable) return fail(RFD_ERR_ARG, "null argument");
  if (!(radius >= 0.0)) return fail(RFD_ERR_ARG, "radius");
  RFD_CUDA(cudaSetDevice(ctx->device));
  rfd_options o;
  rfd_options_init(&o, 0);
  o.dense = dense;
  o.formula = formula;
  rfd_result r;
  int rc = run_batch(ctx, 1, &c1, &n1, &c2, &n2, &dims, &o, &r, MODE_DECIDE, radius);
  if (rc) return rc;
  *reachable = r.distance == 1.0;
  if (right_ub) *right_ub = r.distance;
  return RFD_OK;
}

int32_t rfd_features(rfd_context* ctx, int64_t npairs, const double* const* c1s, const int64_t* n1s,
                     const double* const* c2s, const int64_t* n2s, const int32_t* dims,
                     const double* endpoint, const double* vefd, float* out) {
  if (!ctx || npairs < 0 || !c1s || !n1s || !c2s || !n2s || !dims || !endpoint || !vefd || !out)
    return fail(RFD_ERR_ARG, "null argument");
  if (npairs == 0) return RFD_OK;
  RFD_CUDA(cudaSetDevice(ctx->device));
  size_t bytes = 0;
  std::vector<size_t> o1(npairs), o2(npairs);
  for (int64_t p = 0; p < npairs; ++p) {
    int rc = check_pair(c1s[p], n1s[p], c2s[p], n2s[p], dims[p]);
    if (rc) return rc;
    if (n1s[p] < 2 || n2s[p] < 2) return fail(RFD_ERR_ARG, "features need curves of two points");
    o1[p] = bytes;
    bytes = align_up(bytes + sizeof(double) * n1s[p] * dims[p], 256);
    o2[p] = bytes;
    bytes = align_up(bytes + sizeof(double) * n2s[p] * dims[p], 256);
  }
  const size_t o_desc = bytes;
  bytes = align_up(bytes + sizeof(PairDesc) * npairs, 256);
  const size_t o_ep = bytes;
  bytes = align_up(bytes + sizeof(double) * npairs, 256);
  const size_t o_ve = bytes;
  bytes = align_up(bytes + sizeof(double) * npairs, 256);
  const size_t o_feat = bytes;
  bytes = align_up(bytes + sizeof(float) * rfd_mlp::kInputWidth * npairs, 256);
  int rc = ensure_device(ctx, bytes);
  if (rc) return rc;
  char* base = (char*)ctx->dws;
  std::vector<PairDesc> hd(npairs);
  cudaStream_t st = ctx->stream;
  for (int64_t p = 0; p < npairs; ++p) {
    memset(&hd[p], 0, sizeof(PairDesc));
    hd[p].P = (const double*)(base + o1[p]);
    hd[p].Q = (const double*)(base + o2[p]);
    hd[p].n1 = (int)n1s[p];
    hd[p].n2 = (int)n2s[p];
    hd[p].d = dims[p];
    RFD_CUDA(cudaMemcpyAsync(base + o1[p], c1s[p], sizeof(double) * n1s[p] * dims[p],
                             cudaMemcpyHostToDevice, st));
    RFD_CUDA(cudaMemcpyAsync(base + o2[p], c2s[p], sizeof(double) * n2s[p] * dims[p],
                             cudaMemcpyHostToDevice, st));
  }
  RFD_CUDA(cudaMemcpyAsync(base + o_desc, hd.data(), sizeof(PairDesc) * npairs, cudaMemcpyHostToDevice, st));
  RFD_CUDA(cudaMemcpyAsync(base + o_ep, endpoint, sizeof(double) * npairs, cudaMemcpyHostToDevice, st));
  RFD_CUDA(cudaMemcpyAsync(base + o_ve, vefd, sizeof(double) * npairs, cudaMemcpyHostToDevice, st));
  features_kernel<<<(int)std::min<int64_t>(npairs, 16 * ctx->num_sms), kFeatThreads, 0, st>>>(
      (const PairDesc*)(base + o_desc), (int)npairs, (const double*)(base + o_ep),
      (const double*)(base + o_ve), (float*)(base + o_feat));
  RFD_CUDA(cudaGetLastError());
  RFD_CUDA(cudaMemcpyAsync(out, base + o_feat, sizeof(float) * rfd_mlp::kInputWidth * npairs,
                           cudaMemcpyDeviceToHost, st));
  RFD_CUDA(cudaStreamSynchronize(st));
  return RFD_OK;
}

int32_t rfd_interval_class(int64_t n, const double* x, const double* a, const double* b,
                           const double* A, double r2, int32_t dims, int32_t* cls) {
  if (n < 0 || !x || !a || !b || !A || !cls || (dims != 2 && dims != 3))
    return fail(RFD_ERR_ARG, "interval_class arguments");
  for (int64_t e = 0; e < n; ++e) {
    double di[3];
    for (int k = 0; k < dims; ++k) di[k] = b[e * dims + k] - a[e * dims + k];
    cls[e] = dims == 2 ? interval_class32<2>(x + e * dims, a + e * dims, di, A[e], r2)
                       : interval_class32<3>(x + e * dims, a + e * dims, di, A[e], r2);
  }
  return RFD_OK;
}

int32_t rfd_search_step(double* state, int32_t* istate, int32_t stop_mode, int32_t have_outcome,
                        double eps, int32_t reachable, double* next_eps) {
  if (!state || !istate || !next_eps) return fail(RFD_ERR_ARG, "null argument");
  Search s;
  s.lb = state[0];
  s.ub = state[1];
  s.lo = state[2];
  s.hi = state[3];
  s.tol = state[4];
  s.mode = istate[0];
  s.probes = istate[1];
  s.max_probes = istate[2];
  s.flags = istate[3];
  s.t = state[5];
  s.stop_mode = stop_mode;
  // the first call starts the search as the device does (bracket checks, threshold probe)
  if (!have_outcome && s.probes == 0) search_begin(s, s.lb, s.ub, s.lo, s.hi);
  if (have_outcome) search_update(s, eps, reachable != 0);
  double e = 0.0;
  const int more = search_next(s, &e) ? 1 : 0;
  state[0] = s.lb;
  state[1] = s.ub;
  state[2] = s.lo;
  state[3] = s.hi;
  state[5] = s.t;
  istate[0] = s.mode;
  istate[1] = s.probes;
  istate[3] = s.flags;
  *next_eps = e;
  return more;
}

}  // extern "C"

// ============================================================================ no-allocation decision
//
// rfd_decide_noalloc: one reachability decision for callers that cannot allocate device
// memory at call time - a robot's control loop that must not allocate once it runs (an
// allocation can stall for an unbounded time or fail when the GPU is full), or a process
// that shares the GPU under a fixed memory budget reserved at start-up.  Everything the
// decision needs beyond the caller's inputs and output lives in one file-scope device
// array of kNoAllocBytes, which every GPU that loads this library holds until the process
// exits.  Calls share that array: a call clears what must start at zero, and two calls
// whose work overlaps on the GPU (different streams, or different host threads) race on it.

namespace {

constexpr size_t kNoAllocBytes = (size_t)64 << 20;  // 64 MiB
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

struct NoAllocDevice {
  int ready;
  unsigned char* scratch;  // device address of g_noalloc_scratch on this device
  int team_grid;
  long long spin_cycles;
};
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc[64];

__global__ void noalloc_setup_kernel(PairDesc* desc, PairState* st, int2* items, int nitems,
                                     int* active, PairDesc d, double radius, double r2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    *desc = d;
    PairState s;
    memset(&s, 0, sizeof(s));
    s.srch.tol = 0.0;
    s.srch.stop_mode = RFD_STOP_ABS;
    s.decide_only = 1;
    s.split = radius;
    s.r2 = r2;
    s.blo = s.bhi = CUDART_NAN;
    *st = s;
    *active = 1;
  }
  for (int k = t; k < nitems; k += gridDim.x * blockDim.x) items[k] = make_int2(0, k);
}

__global__ void noalloc_emit_kernel(const PairState* st, const int* error, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) out[0] = *error ? CUDART_NAN : st->result;
}

}  // namespace

extern "C" int32_t rfd_decide_noalloc(const double* c1, int64_t n1, const double* c2, int64_t n2,
                                      int32_t dims, double radius, void* stream,
                                      double* right_ub) {
  if (!c1 || !c2 || !right_ub) return fail(RFD_ERR_ARG, "null pointer");
  if (dims != 2 && dims != 3) return fail(RFD_ERR_ARG, "dims must be 2 or 3");
  if (n1 < 2 || n2 < 2) return fail(RFD_ERR_ARG, "decisions need curves of at least two points");
  if (!(radius >= 0.0)) return fail(RFD_ERR_ARG, "radius");
  // the layout below is computed in size_t from these counts: bound them first (the
  // engine's own per-curve limit), so no product can wrap past the array-size check
  if (n1 > (1 << 30) || n2 > (1 << 30))
    return fail(RFD_ERR_LIMIT, "rfd_decide_noalloc: curve longer than 2^30 points");
  int dev = 0;
  RFD_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(RFD_ERR_ARG, "device index above 63");
  {
    // once per device, with that device current: the array's device address and the
    // launch attributes of the decision kernel
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoAllocDevice& nd = g_noalloc[dev];
    if (!nd.ready) {
      void* p = nullptr;
      RFD_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
      const size_t sm_dec = team_smem_bytes<K_DEC>();
      RFD_CUDA(cudaFuncSetAttribute(team_kernel<K_DEC, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sm_dec));
      int occ = 0, nsm = 0, clk = 0;
      RFD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, team_kernel<K_DEC, 8>, kTeamThreads,
                                                             sm_dec));
      RFD_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
      RFD_CUDA(cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, dev));
      nd.scratch = (unsigned char*)p;
      nd.team_grid = std::max(1, occ) * nsm;
      nd.spin_cycles = (long long)clk * 1000LL * 20LL;
      nd.ready = 1;
    }
  }
  const NoAllocDevice nd = g_noalloc[dev];
  // layout inside the array (same records as the allocating path: one boundary row per strip)
  const int64_t S = (n1 - 1 + 31) / 32;  // 32-row strips over the n1 - 1 segment rows
  const int ring = ring_of(S, INT32_MAX);
  const int64_t cstride = (int64_t)align_up((size_t)n2, 32);
  const int64_t tstride = (int64_t)align_up((size_t)((n2 + 31) / 32), 32);
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t r = off; off = align_up(off + bytes, 256); return r; };
  const size_t o_desc = take(sizeof(PairDesc));
  const size_t o_state = take(sizeof(PairState));
  const size_t o_items = take(sizeof(int2) * S);
  const size_t o_zero = off;
  const size_t o_ticket = take(sizeof(unsigned));
  const size_t o_error = take(sizeof(int));
  const size_t o_tags = take(sizeof(unsigned) * (size_t)ring * tstride);
  const size_t o_prog = take(sizeof(Prog) * S);
  const size_t zero_end = off;
  const size_t o_active = take(sizeof(int));
  const size_t o_rowc = take(sizeof(double2) * (size_t)(n1 - 1));
  const size_t o_colrec = take(sizeof(double2) * (dims == 2 ? 3 : 4) * (size_t)(n2 - 1));
  const size_t o_bnd = take(sizeof(double) * (size_t)ring * cstride);
  if (off > kNoAllocBytes)
    return fail(RFD_ERR_LIMIT, "rfd_decide_noalloc: the pair needs " + std::to_string(off) +
                                   " bytes of scratch, the fixed array holds " +
                                   std::to_string(kNoAllocBytes));
  unsigned char* base = nd.scratch;
  PairDesc d;
  memset(&d, 0, sizeof(d));
  d.P = c1;
  d.Q = c2;
  d.rowc = (const double2*)(base + o_rowc);
  d.colrec = (const double2*)(base + o_colrec);
  d.bnd = (double*)(base + o_bnd);
  d.tags = (unsigned*)(base + o_tags);
  d.prog = (Prog*)(base + o_prog);
  d.ring = ring;
  d.n1 = (int)n1;
  d.n2 = (int)n2;
  d.d = dims;
  d.cstride = cstride;
  d.tstride = tstride;
  cudaStream_t st = (cudaStream_t)stream;
  PairDesc* ddesc = (PairDesc*)(base + o_desc);
  PairState* dstate = (PairState*)(base + o_state);
  RFD_CUDA(cudaMemsetAsync(base + o_zero, 0, zero_end - o_zero, st));
  noalloc_setup_kernel<<<(int)std::min<int64_t>((S + 255) / 256, 64) + 1, 256, 0, st>>>(
      ddesc, dstate, (int2*)(base + o_items), (int)S, (int*)(base + o_active), d, radius,
      radius * radius);
  RFD_CUDA(cudaGetLastError());
  prep_kernel<<<1, 256, 0, st>>>(ddesc, dstate, 1, PH_SEARCH);
  RFD_CUDA(cudaGetLastError());
  bnd_fill_kernel<<<dim3(256, 1), 256, 0, st>>>(ddesc, dstate, 1, PH_SEARCH, nullptr, nullptr, 0);
  RFD_CUDA(cudaGetLastError());
  WaveArgs wa{};
  wa.pairs = ddesc;
  wa.st = dstate;
  wa.items = (const int2*)(base + o_items);
  wa.nitems = (int)S;
  wa.phase = PH_SEARCH;
  wa.ticket = (unsigned*)(base + o_ticket);
  wa.error = (int*)(base + o_error);
  wa.active_pairs = (int*)(base + o_active);
  wa.spin_cycles = env_spin_cycles(nd.spin_cycles);
  wa.prof = nullptr;
  team_kernel<K_DEC, 8><<<nd.team_grid, kTeamThreads, team_smem_bytes<K_DEC>(), st>>>(wa);
  RFD_CUDA(cudaGetLastError());
  noalloc_emit_kernel<<<1, 32, 0, st>>>(dstate, wa.error, right_ub);
  RFD_CUDA(cudaGetLastError());
  return RFD_OK;
}
