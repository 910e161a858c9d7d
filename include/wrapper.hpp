// Public entry point (drop-in for the reference's include/wrapper.hpp:1-4): the continuous
// Frechet distance of two curves, stop rule ub - lb <= FLT_EPSILON as in
// src/compute_distance_wrapper.cpp:6.  forceOversize is accepted for source compatibility;
// this engine always runs the O(n+m)-memory fused decision.
#pragma once

#include "curve.hpp"
#include "frechet.hpp"

double compute_distance_parallel(const Curve& curve1, const Curve& curve2, bool forceOversize = false);
