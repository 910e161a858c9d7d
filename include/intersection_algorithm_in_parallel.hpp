// GPU host class of the public C++ API (drop-in for the reference's
// include/intersection_algorithm_in_parallel.hpp:11-61).  It keeps the reference's
// methods; each call runs on librfd.so (include/rfd.h):
//   Bound_call_gpu(&ub, &lb)            -> rfd_bounds   (lb in: endpoint bound, out: VE-FD)
//   intersection_interval_call_gpu(r)   -> rfd_decide_formula (the constructor's path choice:
//                                          *forceOversize in/out, as in the reference)
// The device buffers live in the library's context, so data_move and free_memory only
// manage the host copies.
#pragma once

#include "curve.hpp"
#include "geometry_basics.hpp"

struct rfd_context;

class Cuda_intersection {
 public:
  double intervalTime;
  double reachTime;
  Cuda_intersection(const Curve& curve1, const Curve& curve2, bool* forceOversize);
  ~Cuda_intersection();
  Cuda_intersection(const Cuda_intersection&) = delete;
  Cuda_intersection& operator=(const Cuda_intersection&) = delete;
  bool intersection_interval_call_gpu(double radius);
  void Bound_call_gpu(double* dfd, double* vefd);
  void data_move();
  void free_memory();

 private:
  int curve1_size;
  int curve2_size;
  bool oversize;
  unsigned int point_dimensions;
  double* points_curve1_p;
  double* points_curve2_p;
  rfd_context* ctx;
};
