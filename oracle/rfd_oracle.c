/*
 * rfd_oracle.c - CPU restatement of the reference's continuous Frechet distance path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load this library, and only as the checker or the timed CPU
 * baseline; the product (robotfd_b200/) never calls it.
 *
 * What it restates (paths relative to the reference project):
 *   - endpoint bound              src/frechet.cpp:30, Point::dist_sqr include/geometry_basics.hpp:72-81
 *   - DFD cell + boundary rules   src/intersection_algorithm_in_parallel.cu:608-637 (init :435-456)
 *   - VE-FD cell (T/R recurrence) src/intersection_algorithm_in_parallel.cu:361-430, seed :259,
 *                                 w_top as specified by README.md:79 (the kernel reads an
 *                                 uninitialised direction at .cu:397; the README formula uses
 *                                 p_{i+1} - p_i, written here mirroring w_right .cu:375-394)
 *   - fused decision cell         src/intersection_algorithm_in_parallel.cu:1173-1253,
 *                                 boundaries .cu:1026-1027 (start) and .cu:656 (left edge -1)
 *   - epsilon search              src/frechet.cpp:36-63, eps = FLT_EPSILON
 *                                 (src/compute_distance_wrapper.cpp:6); VE-FD launch rule .cu:1343
 *   - and, with no reference counterpart, the CUDA engine's meet in the middle
 *     (rfd_oracle_split), to check on the CPU that it gives the unsplit DPs' results
 *
 * Arithmetic contract (shared bit for bit with the CUDA kernels): FP64, compiled with
 * -ffp-contract=off, restating the reference kernels as nvcc compiles them (default
 * contraction): a sum of squares from 0.0 is sq_sum() (the zero start folds away and the
 * first square is fused with the second); every other "acc += x*y" is fma(x, y, acc)
 * starting from acc = 0.0 (or -r^2); "b*b - 4*A*C" is fma(b, b, -((4*A)*C)); q = t*ab + a
 * is fma(t, ab, a); sqrt and '/' are IEEE correctly rounded on both sides.  The endpoint
 * bound and the bisection midpoint are host arithmetic in the reference (g++, no FMA) and
 * are restated without fusion.
 *
 * Parity pin: the reference has no tests or golden data.  The search driver, stop rule,
 * endpoint bound and loaders are pinned by the reference's own host code run on the same
 * inputs (tests/golden/reference_host.json, made through oracle/refharness/); the DFD,
 * VE-FD and decision cells by the reference's own GPU kernels run once on a B200 on four
 * seeded pairs (tests/golden/reference_gpu.json: bounds, every probe and its decision),
 * by mathematical known-answer tests and by independent brute-force definitions
 * (tests/test_oracle.py).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORA_FLTMAX ((double)FLT_MAX)

enum { K_DFD = 0, K_VEFD = 1, K_DEC = 2 };

/* CUDA fmax/fmin semantics: a NaN operand yields the other operand. */
static inline double cmax(double a, double b) {
  if (a != a) return b;
  if (b != b) return a;
  return a > b ? a : b;
}
static inline double cmin(double a, double b) {
  if (a != a) return b;
  if (b != b) return a;
  return a < b ? a : b;
}

typedef struct {
  int kind, d;
  const double *P, *Q;
  int64_t R, C;          /* DP rows / columns */
  double *rowA, *rowInv; /* per row (segment of P): |p_{i+1}-p_i|^2, 0.5/that */
  double *colA, *colInv; /* per column (segment of Q) */
  double r2, seed;
  double *down;          /* [C] value passed from row i-1 to row i per column */
  double *bot;           /* [R] running value along each row */
  double last_ub;        /* decision: propagated right UB of the last cell */
  double last_val;       /* DP: value at the last cell */
  int mat;               /* decision: the materialised path's rounding of C (see free_interval) */
} ora_t;

/* Sum of squares t_0^2 + ... + t_{d-1}^2 as nvcc compiles the reference's
   "s = 0.0; for k: s += t_k * t_k" loops (DFD .cu:615-619, segment lengths .cu:1004-1007 and
   :1133-1137, VE-FD .cu:381-392): the zero start folds away (a square is never -0), the
   first product is fused with the second one rounded, fma(t0, t0, t1*t1), and each later
   square is fused into the running sum, fma(t2, t2, s).  Pinned by the reference's own
   GPU output (tests/golden/reference_gpu.json: a 2D DFD that the source-order chain
   fma(t1, t1, t0*t0) misses by one ulp). */
static inline double sq_sum(const double* t, int d) {
  if (d == 1) return t[0] * t[0];
  double s = t[1] * t[1];
  s = fma(t[0], t[0], s);
  for (int k = 2; k < d; ++k) s = fma(t[k], t[k], s);
  return s;
}

/* |a-b|^2 (DFD .cu:615-619). */
static inline double dist_sq_fma(const double* a, const double* b, int d) {
  double t[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < d; ++k) t[k] = a[k] - b[k];
  return sq_sum(t, d);
}

/* |a-b|^2 without fusion (host Point::dist_sqr). */
static inline double dist_sq_plain(const double* a, const double* b, int d) {
  double s = 0.0;
  for (int k = 0; k < d; ++k) {
    double t = a[k] - b[k];
    double m = t * t;
    s = s + m;
  }
  return s;
}

/* Point-to-segment squared distance of VE-FD (.cu:375-394): point x, segment a -> b,
   ab2 = |b-a|^2 (fma chain). */
static inline double pt_seg_sq(const double* x, const double* a, const double* b, double ab2, int d) {
  double apab = 0.0;
  for (int k = 0; k < d; ++k) {
    double ab = b[k] - a[k];
    double ap = x[k] - a[k];
    apab = fma(ap, ab, apab);
  }
  double t = apab / ab2;
  t = cmin(1.0, cmax(0.0, t));
  double dd[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < d; ++k) {
    double q = fma(t, b[k] - a[k], a[k]);
    dd[k] = x[k] - q;
  }
  return sq_sum(dd, d);
}

/* Free interval of segment a -> b inside the ball of radius^2 r2 around x (.cu:1175-1199):
   di = b - a, mi = a - x, B = 2*sum(mi*di), Cc = -r2 + sum(mi^2), disc = B^2 - 4*A*Cc.
   mat: the materialised path's C (interval_calculation, .cu:730-742 and :765-776): the sum
   of mi^2 from 0, then minus r2 (mm - radius2), one rounding more than the fused chain. */
static inline void free_interval(const double* x, const double* a, const double* b, double A,
                                 double inv2A, double r2, int d, int mat, double* lo, double* hi) {
  double B = 0.0, Cc = -r2, m[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < d; ++k) {
    double di = b[k] - a[k];
    m[k] = a[k] - x[k];
    B = fma(m[k], di, B);
    Cc = fma(m[k], m[k], Cc);
  }
  if (mat) Cc = sq_sum(m, d) - r2;
  B = B * 2.0;
  double disc = fma(B, B, -((4.0 * A) * Cc));
  *lo = -1.0;
  *hi = -2.0;
  if (disc >= 0.0) {
    double s = sqrt(disc);
    double ta = (-B - s) * inv2A;
    double tb = (-B + s) * inv2A;
    int invalid = (tb < 0.0) || (ta > 1.0);
    *lo = invalid ? -1.0 : cmax(ta, 0.0);
    *hi = invalid ? -2.0 : cmin(tb, 1.0);
  }
}

static void tile(ora_t* o, int64_t i0, int64_t i1, int64_t j0, int64_t j1) {
  const int d = o->d;
  for (int64_t i = i0; i < i1; ++i) {
    double b = o->bot[i];
    if (o->kind == K_DFD) {
      const double* pa = o->P + i * d;
      for (int64_t j = j0; j < j1; ++j) {
        double left = o->down[j];
        double dist = dist_sq_fma(pa, o->Q + j * d, d);
        if (i == 0 && j == 0) {
          b = ORA_FLTMAX;
          left = 0.0;
        } else if (i == 0) {
          left = ORA_FLTMAX;
        } else if (j == 0) {
          b = ORA_FLTMAX;
        }
        double in = cmin(left, b);
        double top = cmax(dist, in);
        double right = cmin(top, b);
        o->down[j] = right;
        b = top;
        if (i == o->R - 1 && j == o->C - 1) o->last_val = top;
      }
    } else if (o->kind == K_VEFD) {
      const double* pa1 = o->P + i * d;
      const double* pa2 = o->P + (i + 1) * d;
      const double Aa = o->rowA[i];
      for (int64_t j = j0; j < j1; ++j) {
        const double* qb1 = o->Q + j * d;
        const double* qb2 = o->Q + (j + 1) * d;
        double left = o->down[j];
        double in = cmin(left, b);
        double wr = pt_seg_sq(pa2, qb1, qb2, o->colA[j], d); /* right edge: p_{i+1} vs q_j q_{j+1} */
        double wt = pt_seg_sq(qb2, pa1, pa2, Aa, d);         /* top edge: q_{j+1} vs p_i p_{i+1} */
        double top = cmax(wt, in);
        double right = cmax(wr, in);
        o->down[j] = right;
        b = top;
        if (i == o->R - 1 && j == o->C - 1) o->last_val = cmin(top, right);
      }
    } else {
      const double* pa1 = o->P + i * d;
      const double* pa2 = o->P + (i + 1) * d;
      const double Aa = o->rowA[i], inv2Aa = o->rowInv[i];
      for (int64_t j = j0; j < j1; ++j) {
        const double* qb1 = o->Q + j * d;
        const double* qb2 = o->Q + (j + 1) * d;
        double leftLB = o->down[j];
        double rLB, rUB, tLB, tUB;
        /* right edge: ball around p_{i+1}, segment q_j -> q_{j+1} */
        free_interval(pa2, qb1, qb2, o->colA[j], o->colInv[j], o->r2, d, o->mat, &rLB, &rUB);
        /* top edge: ball around q_{j+1}, segment p_i -> p_{i+1} */
        free_interval(qb2, pa1, pa2, Aa, inv2Aa, o->r2, d, o->mat, &tLB, &tUB);
        if (b < 0.0) {
          int invalid = (leftLB > rUB) || (leftLB < 0.0);
          double m = cmax(rLB, leftLB);
          rLB = invalid ? -1.0 : m;
          rUB = invalid ? -2.0 : rUB;
        }
        if (leftLB < 0.0) {
          int invalid = (b > tUB) || (b < 0.0);
          double m = cmax(tLB, b);
          tLB = invalid ? -1.0 : m;
          tUB = invalid ? -2.0 : tUB;
        }
        b = tLB;
        o->down[j] = rLB;
        if (i == o->R - 1 && j == o->C - 1) o->last_ub = rUB;
      }
    }
    o->bot[i] = b;
  }
}

/* Anti-diagonal wavefront over TR x TC tiles; tiles of one anti-diagonal touch disjoint
   rows and columns, so they run in parallel. */
static void sweep(ora_t* o, int threads) {
  const int64_t TR = 64, TC = 1024;
  const int64_t nr = (o->R + TR - 1) / TR, nc = (o->C + TC - 1) / TC;
  if (threads <= 1 || nr * nc < 4) {
    tile(o, 0, o->R, 0, o->C);
    return;
  }
  for (int64_t k = 0; k < nr + nc - 1; ++k) {
    int64_t a0 = k - (nc - 1) > 0 ? k - (nc - 1) : 0;
    int64_t a1 = k < nr - 1 ? k : nr - 1;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
    for (int64_t a = a0; a <= a1; ++a) {
      int64_t bcol = k - a;
      int64_t i0 = a * TR, i1 = i0 + TR < o->R ? i0 + TR : o->R;
      int64_t j0 = bcol * TC, j1 = j0 + TC < o->C ? j0 + TC : o->C;
      tile(o, i0, i1, j0, j1);
    }
  }
}

static int prep_segments(const double* X, int64_t n, int d, double** A, double** inv) {
  int64_t m = n - 1;
  *A = (double*)malloc(sizeof(double) * (m > 0 ? m : 1));
  *inv = (double*)malloc(sizeof(double) * (m > 0 ? m : 1));
  if (!*A || !*inv) return -1;
  for (int64_t i = 0; i < m; ++i) {
    double t[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < d; ++k) t[k] = X[(i + 1) * d + k] - X[i * d + k];
    double s = sq_sum(t, d);
    (*A)[i] = s;
    (*inv)[i] = 0.5 / s;
  }
  return 0;
}

static int run_mat(int kind, const double* P, int64_t n1, const double* Q, int64_t n2, int d,
                   double r2, double seed, int mat, int threads, double* out_ub, double* out_val) {
  ora_t o;
  memset(&o, 0, sizeof(o));
  o.kind = kind;
  o.mat = mat;  o.d = d;
  o.P = P;
  o.Q = Q;
  o.r2 = r2;
  o.seed = seed;
  o.R = kind == K_DFD ? n1 : n1 - 1;
  o.C = kind == K_DFD ? n2 : n2 - 1;
  if (o.R < 1 || o.C < 1 || d < 1 || d > 3) return -1;
  if (kind != K_DFD) {
    if (prep_segments(P, n1, d, &o.rowA, &o.rowInv) || prep_segments(Q, n2, d, &o.colA, &o.colInv))
      return -2;
  }
  o.down = (double*)malloc(sizeof(double) * o.C);
  o.bot = (double*)malloc(sizeof(double) * o.R);
  if (!o.down || !o.bot) return -2;
  for (int64_t j = 0; j < o.C; ++j) o.down[j] = kind == K_DEC ? -1.0 : ORA_FLTMAX;
  for (int64_t i = 0; i < o.R; ++i) {
    if (kind == K_DEC) o.bot[i] = i == 0 ? 0.0 : -1.0;
    else if (kind == K_VEFD) o.bot[i] = i == 0 ? seed : ORA_FLTMAX;
    else o.bot[i] = ORA_FLTMAX;
  }
  o.last_ub = -2.0;
  o.last_val = ORA_FLTMAX;
  sweep(&o, threads);
  if (out_ub) *out_ub = o.last_ub;
  if (out_val) *out_val = o.last_val;
  free(o.down);
  free(o.bot);
  free(o.rowA);
  free(o.rowInv);
  free(o.colA);
  free(o.colInv);
  return 0;
}


static int run(int kind, const double* P, int64_t n1, const double* Q, int64_t n2, int d,
               double r2, double seed, int threads, double* out_ub, double* out_val) {
  return run_mat(kind, P, n1, Q, n2, d, r2, seed, 0, threads, out_ub, out_val);
}

/* ------------------------------------------------------------------ exports */

double rfd_oracle_endpoint(const double* P, int64_t n1, const double* Q, int64_t n2, int d) {
  double a = dist_sq_plain(P, Q, d);
  double b = dist_sq_plain(P + (n1 - 1) * d, Q + (n2 - 1) * d, d);
  return sqrt(a < b ? b : a); /* std::max(a, b) */
}

/* Squared DFD (value at the last cell); the reference reports sqrt of it (.cu:633). */
int rfd_oracle_dfd_sq(const double* P, int64_t n1, const double* Q, int64_t n2, int d, int threads,
                      double* out) {
  return run(K_DFD, P, n1, Q, n2, d, 0.0, 0.0, threads, NULL, out);
}

/* Squared VE-FD with seed = lb*lb (.cu:259); the reference reports sqrt(min(T,R)) (.cu:427). */
int rfd_oracle_vefd_sq(const double* P, int64_t n1, const double* Q, int64_t n2, int d, double lb,
                       int threads, double* out) {
  return run(K_VEFD, P, n1, Q, n2, d, 0.0, lb * lb, threads, NULL, out);
}

/* Decision at radius: *right_ub = propagated right UB of the last cell, reachable iff == 1.0
   (.cu:1251, :1592).  r2 = radius*radius as the host computes it (.cu:1440). */
int rfd_oracle_decide(const double* P, int64_t n1, const double* Q, int64_t n2, int d, double radius,
                      int threads, double* right_ub) {
  double r2 = radius * radius;
  return run(K_DEC, P, n1, Q, n2, d, r2, 0.0, threads, right_ub, NULL);
}

/* The same with the free intervals of either reference path: formula 0 the fused kernel
   reachable<d> (.cu:1173-1244, taken with forceOversize or when memory is short), 1 the
   materialised interval_calculation<d> (.cu:725-789), whose propagation (reachability,
   .cu:907-934) is the fused one. */
int rfd_oracle_decide_formula(const double* P, int64_t n1, const double* Q, int64_t n2, int d,
                              double radius, int formula, int threads, double* right_ub) {
  double r2 = radius * radius;
  return run_mat(K_DEC, P, n1, Q, n2, d, r2, 0.0, formula == 1, threads, right_ub, NULL);
}

/* Full search.  stop_mode 0: while (ub-lb > tol) (reference); 1: while (ub-lb > tol*ub).
   quirks: skip VE-FD when (int)(n1*n2) <= 10000.  Optional logs of every probe. */
int rfd_oracle_distance_formula(const double* P, int64_t n1, const double* Q, int64_t n2, int d,
                                int stop_mode, double tol, int quirks, int max_probes, int threads,
                                int formula, double* out, int* out_probes, double* log_eps,
                                int* log_dec);

int rfd_oracle_distance(const double* P, int64_t n1, const double* Q, int64_t n2, int d,
                        int stop_mode, double tol, int quirks, int max_probes, int threads,
                        double* out /* [distance, dfd, vefd, endpoint, lb, ub] */,
                        int* out_probes, double* log_eps, int* log_dec) {
  return rfd_oracle_distance_formula(P, n1, Q, n2, d, stop_mode, tol, quirks, max_probes, threads,
                                     0, out, out_probes, log_eps, log_dec);
}

/* Full search with the decisions of either reference path (rfd_oracle_decide_formula). */
int rfd_oracle_distance_formula(const double* P, int64_t n1, const double* Q, int64_t n2, int d,
                                int stop_mode, double tol, int quirks, int max_probes, int threads,
                                int formula, double* out, int* out_probes, double* log_eps,
                                int* log_dec) {
  double endpoint = rfd_oracle_endpoint(P, n1, Q, n2, d);
  double dsq, vsq, ub, lb = endpoint;
  if (n1 < 2 || n2 < 2) return -1;
  if (rfd_oracle_dfd_sq(P, n1, Q, n2, d, threads, &dsq)) return -2;
  ub = sqrt(dsq);
  int32_t prod = (int32_t)((uint32_t)n1 * (uint32_t)n2);
  if (!quirks || prod > 10000) {
    if (rfd_oracle_vefd_sq(P, n1, Q, n2, d, lb, threads, &vsq)) return -2;
    lb = sqrt(vsq);
  }
  double vefd = lb;
  int probes = 0;
  for (;;) {
    double gap = ub - lb;
    int open = stop_mode == 0 ? (gap > tol) : (gap > tol * ub);
    if (!open || probes >= max_probes) break;
    double split = (ub + lb) / 2.0;
    if (!(split > lb && split < ub)) break;
    double rub;
    if (rfd_oracle_decide_formula(P, n1, Q, n2, d, split, formula, threads, &rub)) return -2;
    int reach = rub == 1.0;
    if (log_eps) log_eps[probes] = split;
    if (log_dec) log_dec[probes] = reach;
    ++probes;
    if (reach) ub = split;
    else lb = split;
  }
  out[0] = (ub + lb) / 2.0;
  out[1] = sqrt(dsq);
  out[2] = vefd;
  out[3] = endpoint;
  out[4] = lb;
  out[5] = ub;
  *out_probes = probes;
  return 0;
}

/* Bisection from a given bracket [lb, ub] (src/frechet.cpp:36-63 with the reference's own
   bounds), so a recorded reference search can be replayed decision by decision. */
int rfd_oracle_search(const double* P, int64_t n1, const double* Q, int64_t n2, int d, double lb,
                      double ub, int stop_mode, double tol, int max_probes, int threads,
                      double* out /* [distance, lb, ub] */, int* out_probes) {
  int probes = 0;
  for (;;) {
    double gap = ub - lb;
    int open = stop_mode == 0 ? (gap > tol) : (gap > tol * ub);
    if (!open || probes >= max_probes) break;
    double split = (ub + lb) / 2.0;
    if (!(split > lb && split < ub)) break;
    double rub;
    if (rfd_oracle_decide(P, n1, Q, n2, d, split, threads, &rub)) return -2;
    ++probes;
    if (rub == 1.0) ub = split;
    else lb = split;
  }
  out[0] = (ub + lb) / 2.0;
  out[1] = lb;
  out[2] = ub;
  *out_probes = probes;
  return 0;
}

/* Free intervals of n edges (test entry): edge e is the segment a_e -> b_e against the ball
   of radius^2 r2 around x_e, with A_e = |b_e - a_e|^2 and inv2A_e = 0.5 / A_e as given. */
int rfd_oracle_free_intervals_formula(int64_t n, const double* x, const double* a,
                                      const double* b, const double* A, const double* inv2A,
                                      double r2, int d, int formula, double* lo, double* hi) {
  if (n < 0 || (d != 2 && d != 3)) return 1;
  for (int64_t e = 0; e < n; ++e)
    free_interval(x + e * d, a + e * d, b + e * d, A[e], inv2A[e], r2, d, formula == 1, lo + e,
                  hi + e);
  return 0;
}

int rfd_oracle_free_intervals(int64_t n, const double* x, const double* a, const double* b,
                              const double* A, const double* inv2A, double r2, int d, double* lo,
                              double* hi) {
  return rfd_oracle_free_intervals_formula(n, x, a, b, A, inv2A, r2, d, 0, lo, hi);
}

/* Meet in the middle, restated (the CUDA engine's split pairs: split_meet_kernel and the
   mirror instantiation of the team strips, robotfd_b200/csrc/).  The decision or VE-FD DP of
   rows 0 .. h-1 runs forward from the start as above; rows h .. R-1 run from the far corner
   over the mirrored grid, whose cell (i, j) is cell (a, b) = (R-1-i, C-1-j) carrying that
   cell's entry edges - the right edge of cell (a-1, b) (p_a against q_b q_{b+1}) and the top
   edge of cell (a, b-1) (q_b against p_a p_{a+1}) - with the same propagation rule: VE-FD
   weights as they are, starting from min(w_top, w_right) of the last cell; free intervals
   [lo, hi] as [-hi, -lo] (empty (-3, -4), dead below -1.5), starting from the last cell's
   right edge when its interval reaches the corner (upper end 1.0).  The two rows handed
   across the boundary between rows h-1 and h then combine:
     K_VEFD: *out = min over b of max(forward(b), mirror(C-1-b)), the squared VE-FD;
     K_DEC:  *out = 1.0 if some b has forward(b) >= 0, mirror(C-1-b) >= -1.5 and
             forward(b) <= -mirror(C-1-b), else -2.0.
   Sequential; checks on real geometry that the split equals the unsplit DP (VE-FD bit for
   bit, reachable iff the unsplit right UB is 1.0).  x is the radius (K_DEC) or the lower
   bound seeding VE-FD (K_VEFD); 1 <= h <= R-1. */
static void mirror_iv(double* lo, double* hi) {
  if (*lo < 0.0) {
    *lo = -3.0;
    *hi = -4.0;
  } else {
    double l = *lo;
    *lo = -*hi;
    *hi = -l;
  }
}

int rfd_oracle_split(int kind, const double* P, int64_t n1, const double* Q, int64_t n2, int d,
                     double x, int64_t h, double* out) {
  if (kind != K_VEFD && kind != K_DEC) return -1;
  const int64_t R = n1 - 1, C = n2 - 1;
  if (R < 2 || C < 1 || d < 1 || d > 3 || h < 1 || h > R - 1) return -1;
  ora_t o;
  memset(&o, 0, sizeof(o));
  o.kind = kind;
  o.d = d;
  o.P = P;
  o.Q = Q;
  o.r2 = kind == K_DEC ? x * x : 0.0;
  o.seed = kind == K_VEFD ? x * x : 0.0;
  o.R = h; /* the forward half: rows 0 .. h-1 */
  o.C = C;
  if (prep_segments(P, n1, d, &o.rowA, &o.rowInv) || prep_segments(Q, n2, d, &o.colA, &o.colInv))
    return -2;
  o.down = (double*)malloc(sizeof(double) * C);
  o.bot = (double*)malloc(sizeof(double) * h);
  double* M = (double*)malloc(sizeof(double) * C);
  if (!o.down || !o.bot || !M) return -2;
  for (int64_t j = 0; j < C; ++j) o.down[j] = kind == K_DEC ? -1.0 : ORA_FLTMAX;
  for (int64_t i = 0; i < h; ++i) {
    if (kind == K_DEC) o.bot[i] = i == 0 ? 0.0 : -1.0;
    else o.bot[i] = i == 0 ? o.seed : ORA_FLTMAX;
  }
  tile(&o, 0, h, 0, C); /* o.down: the values handed from row h-1 to row h */
  const double* Pl = P + R * d;        /* p_R, the last point */
  const double* Ql = Q + C * d;        /* q_C */
  /* the far corner */
  double bm0;
  if (kind == K_VEFD) {
    const double wr = pt_seg_sq(Pl, Q + (C - 1) * d, Ql, o.colA[C - 1], d);
    const double wt = pt_seg_sq(Ql, P + (R - 1) * d, Pl, o.rowA[R - 1], d);
    bm0 = cmin(wt, wr);
    for (int64_t j = 0; j < C; ++j) M[j] = ORA_FLTMAX;
  } else {
    double lo, hi;
    free_interval(Pl, Q + (C - 1) * d, Ql, o.colA[C - 1], o.colInv[C - 1], o.r2, d, 0, &lo, &hi);
    for (int64_t j = 0; j < C; ++j) M[j] = -3.0;
    if (hi == 1.0) M[0] = -1.0;
    bm0 = -3.0;
  }
  for (int64_t i = 0; i < R - h; ++i) {
    const int64_t a = R - 1 - i;
    const double* pa = P + a * d;
    const double* pa1 = P + (a + 1) * d;
    double bm = i == 0 ? bm0 : (kind == K_DEC ? -3.0 : ORA_FLTMAX);
    for (int64_t jm = 0; jm < C; ++jm) {
      const int64_t b = C - 1 - jm;
      const double* qb = Q + b * d;
      const double* qb1 = Q + (b + 1) * d;
      if (kind == K_VEFD) {
        const double in = cmin(M[jm], bm);
        const double wr = pt_seg_sq(pa, qb, qb1, o.colA[b], d);      /* p_a vs q_b q_{b+1} */
        const double wt = pt_seg_sq(qb, pa, pa1, o.rowA[a], d);      /* q_b vs p_a p_{a+1} */
        const double top = cmax(wt, in), right = cmax(wr, in);
        M[jm] = right;
        bm = top;
      } else {
        double rLB, rUB, tLB, tUB;
        free_interval(pa, qb, qb1, o.colA[b], o.colInv[b], o.r2, d, 0, &rLB, &rUB);
        free_interval(qb, pa, pa1, o.rowA[a], o.rowInv[a], o.r2, d, 0, &tLB, &tUB);
        mirror_iv(&rLB, &rUB);
        mirror_iv(&tLB, &tUB);
        const double left = M[jm];
        if (bm < -1.5) {
          const int invalid = (left > rUB) || (left < -1.5);
          const double m = cmax(rLB, left);
          rLB = invalid ? -3.0 : m;
        }
        if (left < -1.5) {
          const int invalid = (bm > tUB) || (bm < -1.5);
          const double m = cmax(tLB, bm);
          tLB = invalid ? -3.0 : m;
        }
        bm = tLB;
        M[jm] = rLB;
      }
    }
  }
  if (kind == K_VEFD) {
    double v = ORA_FLTMAX;
    for (int64_t b = 0; b < C; ++b) v = cmin(v, cmax(o.down[b], M[C - 1 - b]));
    *out = v;
  } else {
    int found = 0;
    for (int64_t b = 0; b < C && !found; ++b) {
      const double f = o.down[b], m = M[C - 1 - b];
      found = f >= 0.0 && m >= -1.5 && f <= -m;
    }
    *out = found ? 1.0 : -2.0;
  }
  free(M);
  free(o.down);
  free(o.bot);
  free(o.rowA);
  free(o.rowInv);
  free(o.colA);
  free(o.colInv);
  return 0;
}

int rfd_oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
