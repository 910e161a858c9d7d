/* Robust decision verifier (TEST INFRASTRUCTURE ONLY: not linked into the engine).
 *
 * Decides whether the free space of two polylines at radius r is traversable in EXACT real
 * arithmetic on the given doubles, or says it cannot tell.  It follows the idea of the
 * reference's IntersectionAlgorithm::intersection_interval (include/geometry_basics.hpp:
 * 161-298: an interval whose end points are checked by point-distance tests), in both
 * directions:
 *   - a point of an edge is "certainly inside" (or outside) the ball when its squared
 *     distance, computed in long double, clears r^2 by a bound on the rounding error;
 *   - the inner interval of an edge is spanned by certainly-inside points (found by
 *     bisection towards the near-closest point), so it lies inside the true free interval
 *     (the free set of a segment is convex);
 *   - the outer interval ends at certainly-outside points (or at the edge's ends), so it
 *     contains the true free interval; it is empty only when a tangent lower bound of the
 *     convex squared distance at the near-closest point certainly exceeds r^2;
 *   - reachability is monotone in the free space: reachable with inner intervals means
 *     reachable, unreachable with outer intervals means unreachable.
 * The propagation is the standard free-space reachability (Alt and Godau), in exact
 * comparisons of the interval end points.
 *
 * rfd_verify_decision returns +1 (certainly reachable), -1 (certainly not), 0 (cannot tell).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

typedef long double ld;

typedef struct {
  double lo, hi; /* empty when lo > hi */
} ivl;

static const ivl kEmpty = {2.0, -1.0};

/* +1 certainly inside, -1 certainly outside, 0 cannot tell: the point s + t (e - s) against
   the ball of radius^2 r2 (|r2 - true r^2| <= er2) around x */
static int where(const double* x, const double* s, const double* e, double t, ld r2, ld er2,
                 int d) {
  ld sum = 0.0L, mag = 0.0L;
  for (int k = 0; k < d; ++k) {
    const ld v = (ld)e[k] - (ld)s[k];
    const ld w = (ld)s[k] - (ld)x[k];
    const ld u = w + (ld)t * v;
    sum += u * u;
    const ld m = fabsl(w) + fabsl((ld)t * v) + fabsl(v);
    mag += m * m;
  }
  const ld err = 64.0L * LDBL_EPSILON * mag + er2;
  if (sum + err < r2) return 1;
  if (sum - err > r2) return -1;
  return 0;
}

/* +1 certainly increasing, -1 certainly decreasing, 0 cannot tell: f(t) = |s + t (e - s) - x|^2
   at t (f'(t) = 2 (w + t v) . v) */
static int slope(const double* x, const double* s, const double* e, double t, int d) {
  ld g = 0.0L, mag = 0.0L;
  for (int k = 0; k < d; ++k) {
    const ld v = (ld)e[k] - (ld)s[k];
    const ld w = (ld)s[k] - (ld)x[k];
    g += (w + (ld)t * v) * v;
    mag += (fabsl(w) + fabsl((ld)t * v) + fabsl(v)) * fabsl(v);
  }
  const ld err = 64.0L * LDBL_EPSILON * mag;
  if (g > err) return 1;
  if (g < -err) return -1;
  return 0;
}

/* bisection on [a, b] for the boundary of a predicate that holds at `a` (want_at_a) and is
   not known to hold at `b`; returns the last point at which it was seen to hold (on the side
   of `a`) -- every returned point was tested, so soundness does not rest on monotonicity */
static double bisect(const double* x, const double* s, const double* e, double a, double b,
                     int want, ld r2, ld er2, int d) {
  for (int it = 0; it < 80; ++it) {
    const double m = 0.5 * (a + b);
    if (!(m > fmin(a, b) && m < fmax(a, b))) break;
    if (where(x, s, e, m, r2, er2, d) == want) a = m;
    else b = m;
  }
  return a;
}

/* the free interval {t in [0, 1] : |s + t (e - s) - x| <= r} of segment s -> e against the
   ball around x, bounded from inside (`inner`, a subset) and outside (`outer`, a superset) */
static void free_bounds(const double* x, const double* s, const double* e, double r, int d,
                        ivl* inner, ivl* outer) {
  const ld r2 = (ld)r * (ld)r;
  const ld er2 = 2.0L * LDBL_EPSILON * r2;
  /* near-closest parameter */
  ld vv = 0.0L, wv = 0.0L;
  for (int k = 0; k < d; ++k) {
    const ld v = (ld)e[k] - (ld)s[k];
    vv += v * v;
    wv += ((ld)x[k] - (ld)s[k]) * v;
  }
  double ts = vv > 0.0L ? (double)(wv / vv) : 0.0;
  if (!(ts >= 0.0)) ts = 0.0;
  if (ts > 1.0) ts = 1.0;
  const int w0 = where(x, s, e, 0.0, r2, er2, d);
  const int w1 = where(x, s, e, 1.0, r2, er2, d);
  const int wt = where(x, s, e, ts, r2, er2, d);
  /* a certainly-inside point, if one of 0, ts, 1 is */
  const int have = wt == 1 || w0 == 1 || w1 == 1;
  const double anchor = wt == 1 ? ts : (w0 == 1 ? 0.0 : 1.0);
  if (!have) {
    *inner = kEmpty;
    /* certify emptiness: f is convex, so f(t) >= f(ts) + f'(ts) (t - ts), whose minimum on
       [0, 1] is at t = 0 or t = 1 (ts may sit at a clamped end, where f' is not small) */
    ld f = 0.0L, g = 0.0L, mag = 0.0L, gmag = 0.0L;
    for (int k = 0; k < d; ++k) {
      const ld v = (ld)e[k] - (ld)s[k];
      const ld w = (ld)s[k] - (ld)x[k];
      const ld u = w + (ld)ts * v;
      f += u * u;
      g += 2.0L * u * v;
      const ld m = fabsl(w) + fabsl(v);
      mag += m * m;
      gmag += 2.0L * m * fabsl(v);
    }
    const ld down = fminl(-g * (ld)ts, g * (1.0L - (ld)ts));
    const ld low = f + down - 64.0L * LDBL_EPSILON * (mag + gmag);
    if (low - er2 > r2) {
      *outer = kEmpty;
      return;
    }
  } else {
    /* the free set is an interval containing `anchor`: points between two certainly-inside
       points are inside */
    inner->lo = w0 == 1 ? 0.0 : bisect(x, s, e, anchor, 0.0, 1, r2, er2, d);
    inner->hi = w1 == 1 ? 1.0 : bisect(x, s, e, anchor, 1.0, 1, r2, er2, d);
  }
  /* outer ends: a certainly-outside point bounds the free interval on its side when the free
     interval is known to lie beyond it -- it contains `anchor`, or f certainly decreases
     (increases) there, so the convex f stays above r^2 towards the edge's end */
  const double mid = have ? anchor : ts;
  outer->lo = 0.0;
  if (w0 == -1) {
    const double a = bisect(x, s, e, 0.0, mid, -1, r2, er2, d);
    if (have || slope(x, s, e, a, d) == -1) outer->lo = a;
  }
  outer->hi = 1.0;
  if (w1 == -1) {
    const double b = bisect(x, s, e, 1.0, mid, -1, r2, er2, d);
    if (have || slope(x, s, e, b, d) == 1) outer->hi = b;
  }
}

/* Alt-Godau reachability over given edge intervals.
   V(i, j): edge of points (p_i.., q_j) with p on segment i (rows), q fixed at vertex j;
   H(i, j): edge of points (p_i, q on segment j).  Cell (i, j) has left edge V(i, j), bottom
   edge H(i, j), right edge V(i, j+1), top edge H(i+1, j). */
static int reachable(int64_t n1, int64_t n2, const ivl* V, const ivl* H, int start_free,
                     int end_free) {
  if (!start_free || !end_free) return 0;
  const int64_t R = n1 - 1, C = n2 - 1;
  if (R == 0 && C == 0) return 1;
  /* reachable parts: RV(i, j) on V edges, RH(i, j) on H edges */
  ivl* RV = (ivl*)malloc(sizeof(ivl) * (size_t)(R > 0 ? R : 1) * (size_t)n2);
  ivl* RH = (ivl*)malloc(sizeof(ivl) * (size_t)n1 * (size_t)(C > 0 ? C : 1));
  if (!RV || !RH) {
    free(RV);
    free(RH);
    return 0;
  }
#define V_(i, j) V[(i) * n2 + (j)]
#define H_(i, j) H[(i) * (C > 0 ? C : 1) + (j)]
#define RV_(i, j) RV[(i) * n2 + (j)]
#define RH_(i, j) RH[(i) * (C > 0 ? C : 1) + (j)]
  /* left boundary (column 0): reachable from the start going up while free from 0 */
  int cont = 1;
  for (int64_t i = 0; i < R; ++i) {
    const ivl f = V_(i, 0);
    if (cont && f.lo <= f.hi && f.lo == 0.0) {
      RV_(i, 0) = f;
      cont = f.hi == 1.0;
    } else {
      RV_(i, 0) = kEmpty;
      cont = 0;
    }
  }
  cont = 1;
  for (int64_t j = 0; j < C; ++j) {
    const ivl f = H_(0, j);
    if (cont && f.lo <= f.hi && f.lo == 0.0) {
      RH_(0, j) = f;
      cont = f.hi == 1.0;
    } else {
      RH_(0, j) = kEmpty;
      cont = 0;
    }
  }
  for (int64_t i = 0; i < R; ++i)
    for (int64_t j = 0; j < C; ++j) {
      const ivl left = RV_(i, j), bot = RH_(i, j);
      const int lv = left.lo <= left.hi, bv = bot.lo <= bot.hi;
      const ivl fr = V_(i, j + 1), ft = H_(i + 1, j);
      ivl r = kEmpty, t = kEmpty;
      if (fr.lo <= fr.hi) {
        if (bv) r = fr;
        else if (lv && left.lo <= fr.hi) r = (ivl){left.lo > fr.lo ? left.lo : fr.lo, fr.hi};
      }
      if (ft.lo <= ft.hi) {
        if (lv) t = ft;
        else if (bv && bot.lo <= ft.hi) t = (ivl){bot.lo > ft.lo ? bot.lo : ft.lo, ft.hi};
      }
      RV_(i, j + 1) = r;
      RH_(i + 1, j) = t;
    }
  int ok;
  if (R == 0) ok = RH_(0, C - 1).lo <= RH_(0, C - 1).hi && RH_(0, C - 1).hi == 1.0;
  else if (C == 0) ok = RV_(R - 1, 0).lo <= RV_(R - 1, 0).hi && RV_(R - 1, 0).hi == 1.0;
  else {
    const ivl a = RV_(R - 1, C), b = RH_(R, C - 1);
    ok = (a.lo <= a.hi && a.hi == 1.0) || (b.lo <= b.hi && b.hi == 1.0);
  }
#undef V_
#undef H_
#undef RV_
#undef RH_
  free(RV);
  free(RH);
  return ok;
}

int rfd_verify_decision(const double* P, int64_t n1, const double* Q, int64_t n2, int d,
                        double r) {
  if (n1 < 1 || n2 < 1 || (d != 2 && d != 3) || !(r >= 0.0)) return 0;
  const int64_t R = n1 - 1, C = n2 - 1;
  const size_t nv = (size_t)(R > 0 ? R : 1) * (size_t)n2, nh = (size_t)n1 * (size_t)(C > 0 ? C : 1);
  ivl *Vi = malloc(sizeof(ivl) * nv), *Vo = malloc(sizeof(ivl) * nv);
  ivl *Hi = malloc(sizeof(ivl) * nh), *Ho = malloc(sizeof(ivl) * nh);
  if (!Vi || !Vo || !Hi || !Ho) {
    free(Vi); free(Vo); free(Hi); free(Ho);
    return 0;
  }
  for (int64_t i = 0; i < R; ++i)
    for (int64_t j = 0; j < n2; ++j)
      free_bounds(Q + j * d, P + i * d, P + (i + 1) * d, r, d, &Vi[i * n2 + j], &Vo[i * n2 + j]);
  for (int64_t i = 0; i < n1; ++i)
    for (int64_t j = 0; j < C; ++j)
      free_bounds(P + i * d, Q + j * d, Q + (j + 1) * d, r, d, &Hi[i * C + j], &Ho[i * C + j]);
  const ld r2 = (ld)r * (ld)r, er2 = 2.0L * LDBL_EPSILON * r2;
  /* the start and end points, as degenerate edges */
  const int s = where(Q, P, P, 0.0, r2, er2, d);
  const int e = where(Q + (n2 - 1) * d, P + (n1 - 1) * d, P + (n1 - 1) * d, 0.0, r2, er2, d);
  int result = 0;
  if (reachable(n1, n2, Vi, Hi, s == 1, e == 1)) result = 1;
  else if (!reachable(n1, n2, Vo, Ho, s != -1, e != -1)) result = -1;
  free(Vi); free(Vo); free(Hi); free(Ho);
  return result;
}

/* the inner and outer bounds of one edge's free interval: out = {in_lo, in_hi, out_lo, out_hi}
   (an empty interval has lo > hi) */
void rfd_verify_free_bounds(const double* x, const double* s, const double* e, double r, int d,
                            double* out) {
  ivl in, ou;
  free_bounds(x, s, e, r, d, &in, &ou);
  out[0] = in.lo;
  out[1] = in.hi;
  out[2] = ou.lo;
  out[3] = ou.hi;
}
