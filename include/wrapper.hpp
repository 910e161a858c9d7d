// Public entry point (drop-in for the reference's include/wrapper.hpp:1-4): the continuous
// Frechet distance of two curves, stop rule ub - lb <= FLT_EPSILON as in
// src/compute_distance_wrapper.cpp:6.  forceOversize chooses between the reference's two
// decision paths as the reference does: forced, or when the reference's materialised interval
// arrays would not fit in free device memory, the fused kernel's free intervals; otherwise the
// materialised path's (they differ in one rounding, rfd.h enum rfd_formula).  Device memory is
// the same either way: O(n1 + n2) for the curves, records and the DFD's boundary ring; the
// VE-FD and decision strips keep a boundary row per 32 rows (about n1 * n2 / 4 bytes) when that
// fits, and otherwise run in launch windows whose ring of at most 4097 rows is O(n1 + n2), so
// any pair whose points fit is solved, as by the reference's oversize path.
#pragma once

#include "curve.hpp"
#include "frechet.hpp"

double compute_distance_parallel(const Curve& curve1, const Curve& curve2, bool forceOversize = false);

// All pairwise distances of a Curves collection (no counterpart in the reference), row-major
// n x n, symmetric with a zero diagonal; precise selects the 2^-33 relative stop rule instead
// of the reference's FLT_EPSILON absolute one.
#include <vector>
std::vector<double> compute_distance_matrix(const Curves& curves, bool precise = false);
