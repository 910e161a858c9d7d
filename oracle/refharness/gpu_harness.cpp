// Runs the reference's own GPU path (TEST INFRASTRUCTURE ONLY): its Cuda_intersection class
// and kernels (src/intersection_algorithm_in_parallel.cu, built for sm_100a from the source
// in place by oracle/refharness/Makefile) driven by the steps of its search driver
// (src/frechet.cpp:26-63: endpoint bound, Bound_call_gpu, bisection while ub - lb > eps,
// midpoint), with every bound, probe and outcome recorded in full precision (the stock
// driver prints them with 14 digits).  Only the fused decision kernel is used
// (forceOversize = true, .cu:92-97): its materialised path asserts that the last cell is
// reachable (.cu:794), which fails below the endpoint bound.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "curve.hpp"
#include "intersection_algorithm_in_parallel.hpp"

extern "C" int ref_gpu_solve(const double* P, long n1, const double* Q, long n2, int d,
                             double eps, double* out /* endpoint, dfd, vefd, distance, lb, ub */,
                             int* nprobes, double* eps_log, int* dec_log, int max_log) {
  if (n1 < 2 || n2 < 2 || (d != 2 && d != 3)) return 1;
  Points a, b;
  for (long i = 0; i < n1; ++i) a.push_back(Point(std::vector<double>(P + i * d, P + (i + 1) * d)));
  for (long i = 0; i < n2; ++i) b.push_back(Point(std::vector<double>(Q + i * d, Q + (i + 1) * d)));
  Curve c1(a, d), c2(b, d);
  bool force = true;
  Cuda_intersection cuda(c1, c2, &force);
  cuda.data_move();
  double lb = std::sqrt(std::max(c1.front().dist_sqr(c2.front()), c1.back().dist_sqr(c2.back())));
  double ub = 0.0;
  out[0] = lb;
  cuda.Bound_call_gpu(&ub, &lb);
  out[1] = ub;
  out[2] = lb;
  int it = 0;
  while (ub - lb > eps && it < max_log) {
    const double split = (ub + lb) / 2.0;
    const bool r = cuda.intersection_interval_call_gpu(split);
    eps_log[it] = split;
    dec_log[it] = r ? 1 : 0;
    ++it;
    if (r) ub = split;
    else lb = split;
  }
  out[3] = (ub + lb) / 2.0;
  out[4] = lb;
  out[5] = ub;
  *nprobes = it;
  cuda.free_memory();
  return 0;
}
