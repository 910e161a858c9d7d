// Epsilon search state machine, compiled for host and device.
//
// The plain rule is the reference's bisection (src/frechet.cpp:36-63): while the gap is
// open, probe split = (ub + lb) / 2, a reachable probe becomes the new ub, an unreachable
// one the new lb, and the answer is (ub + lb) / 2.  Two additions change only the probe
// sequence, never what a probe decides:
//   - a proposed bracket [lo, hi] is verified before bisecting.  The search starts at a
//     proven lower bound lb (the VE-FD bound), so a reachable probe at the stop threshold
//     t above lb (0.999 of the tolerance, clear of rounding) ends the search at once.  When
//     the bracket reaches below t, t is probed first; then hi, then lo, each only while it
//     lies strictly inside (lb, ub).  A failed hi or lo check still tightens [lb, ub] and
//     moves the window geometrically (width x2 each time); once the window leaves
//     [lb, ub] the search is plain bisection of the bounds.
//   - a probe whose midpoint equals lb or ub in doubles stops the search (the reference
//     would loop forever there).
#pragma once

#if defined(__CUDACC__)
#define RFD_HD __host__ __device__ __forceinline__
#else
#define RFD_HD inline
#endif

namespace rfd {

enum SearchFlag {
  SF_MAX_PROBES = 4,
  SF_STALLED = 8,
  SF_BRACKET_USED = 32,
  SF_BRACKET_WIDENED = 64,
};

enum SearchMode { SM_BISECT = 0, SM_CHECK_HI = 1, SM_CHECK_LO = 2, SM_CHECK_T = 3 };

struct Search {
  double lb, ub;   // lb: known unreachable (or a proven lower bound), ub: known reachable
  double lo, hi;   // bracket window being verified
  double tol;
  double t;        // stop threshold above the starting lb (bracketed searches)
  int mode, probes, max_probes, flags;
  int stop_mode;   // 0: ub - lb > tol ; 1: ub - lb > tol * ub
};

RFD_HD bool search_gap_open(const Search& s) {
  const double g = s.ub - s.lb;
  return s.stop_mode == 0 ? (g > s.tol) : (g > s.tol * s.ub);
}

// The largest probe that closes the gap when it is reachable, for the current lb.
RFD_HD double search_threshold(const Search& s) {
  return s.stop_mode == 0 ? s.lb + 0.999 * s.tol : s.lb * (1.0 + 0.999 * s.tol);
}

// Proposes the next probe; false when the search is over.
RFD_HD bool search_next(Search& s, double* eps) {
  for (;;) {
    if (!search_gap_open(s)) return false;
    if (s.probes >= s.max_probes) {
      s.flags |= SF_MAX_PROBES;
      return false;
    }
    if (s.mode == SM_CHECK_T) {
      if (s.t > s.lb && s.t < s.ub) {
        *eps = s.t;
        return true;
      }
      s.mode = SM_CHECK_HI;
      continue;
    }
    if (s.mode == SM_CHECK_HI) {
      if (s.hi > s.lb && s.hi < s.ub) {
        *eps = s.hi;
        return true;
      }
      s.mode = SM_CHECK_LO;
      continue;
    }
    if (s.mode == SM_CHECK_LO) {
      if (s.lo > s.lb && s.lo < s.ub) {
        *eps = s.lo;
        return true;
      }
      s.mode = SM_BISECT;
      continue;
    }
    const double split = (s.ub + s.lb) / 2.0;
    if (!(split > s.lb && split < s.ub)) {
      s.flags |= SF_STALLED;
      return false;
    }
    *eps = split;
    return true;
  }
}

// Applies the outcome of a probe at eps.
RFD_HD void search_update(Search& s, double eps, bool reachable) {
  s.probes += 1;
  if (reachable) s.ub = eps;
  else s.lb = eps;
  if (s.mode == SM_CHECK_T) {
    // reachable: the gap is closed.  Unreachable: the bracket is checked next, and what
    // of it lies at or below t is skipped.
    s.mode = SM_CHECK_HI;
  } else if (s.mode == SM_CHECK_HI) {
    if (reachable) {
      s.mode = SM_CHECK_LO;
    } else {
      const double w = s.hi - s.lo;
      s.lo = s.hi;
      s.hi = s.hi + 2.0 * w;
      s.flags |= SF_BRACKET_WIDENED;
    }
  } else if (s.mode == SM_CHECK_LO) {
    if (!reachable) {
      s.mode = SM_BISECT;
    } else {
      const double w = s.hi - s.lo;
      s.hi = s.lo;
      s.lo = s.lo - 2.0 * w;
      s.flags |= SF_BRACKET_WIDENED;
    }
  }
}

// Starts a search on [lb, ub]; a finite bracket with lo < hi enables the check modes,
// beginning with the threshold probe when the bracket reaches below it or when
// threshold_first is set (a bracket that only describes distances above the threshold).
RFD_HD void search_begin(Search& s, double lb, double ub, double lo, double hi,
                         bool threshold_first = false) {
  s.lb = lb;
  s.ub = ub;
  s.probes = 0;
  s.mode = SM_BISECT;
  s.t = search_threshold(s);
  if (lo == lo && hi == hi && lo < hi) {
    s.lo = lo;
    s.hi = hi;
    s.mode = (threshold_first || lo < s.t) ? SM_CHECK_T : SM_CHECK_HI;
    s.flags |= SF_BRACKET_USED;
  }
}

}  // namespace rfd
