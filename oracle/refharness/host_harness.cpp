// Runs the reference's host code on the CPU (TEST INFRASTRUCTURE ONLY).
//
// oracle/refharness/Makefile compiles the reference's own host sources in place -
// src/frechet.cpp (Frechet::Continuous::distance_cuda: endpoint bound, bisection, stop
// rule, midpoint), src/compute_distance_wrapper.cpp (eps = FLT_EPSILON), src/curve.cpp,
// include/geometry_basics.hpp (Point::dist_sqr) and include/txtReader.hpp (txtLoader2/3) -
// and links them with this file, which supplies the GPU class Cuda_intersection
// (include/intersection_algorithm_in_parallel.hpp:11-61) backed by the CPU oracle
// (oracle/rfd_oracle.c).  The reference's GPU kernels themselves are not run.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "intersection_algorithm_in_parallel.hpp"
#include "txtReader.hpp"
#include "wrapper.hpp"

extern "C" {
int rfd_oracle_dfd_sq(const double*, long, const double*, long, int, int, double*);
int rfd_oracle_vefd_sq(const double*, long, const double*, long, int, double, int, double*);
int rfd_oracle_decide(const double*, long, const double*, long, int, double, int, double*);
}

// Flattening and sizes as the reference constructor does (.cu:23-51).
Cuda_intersection::Cuda_intersection(const Curve& curve1, const Curve& curve2, bool* forceOversize) {
  point_dimensions = curve1[0].coordinates.size();
  curve1_size = curve1.size();
  curve2_size = curve2.size();
  points_curve1_p = (double*)malloc(sizeof(double) * point_dimensions * curve1.size());
  points_curve2_p = (double*)malloc(sizeof(double) * point_dimensions * curve2.size());
  for (unsigned i = 0; i < curve1.size(); i++)
    for (unsigned j = 0; j < point_dimensions; j++)
      points_curve1_p[i * point_dimensions + j] = curve1[i].coordinates[j];
  for (unsigned i = 0; i < curve2.size(); i++)
    for (unsigned j = 0; j < point_dimensions; j++)
      points_curve2_p[i * point_dimensions + j] = curve2[i].coordinates[j];
  intervalTime = 0.0;
  reachTime = 0.0;
  oversize = true;
  (void)forceOversize;
}

void Cuda_intersection::data_move() {}

void Cuda_intersection::free_memory() {
  free(points_curve1_p);
  free(points_curve2_p);
}

// DFD always; VE-FD only under the reference's launch rule (.cu:1343), seeded with *vefd.
void Cuda_intersection::Bound_call_gpu(double* dfd, double* vefd) {
  double d = 0.0;
  rfd_oracle_dfd_sq(points_curve1_p, curve1_size, points_curve2_p, curve2_size, point_dimensions, 1, &d);
  *dfd = std::sqrt(d);
  if ((int)((unsigned)curve1_size * (unsigned)curve2_size) > 10000) {
    double v = 0.0;
    rfd_oracle_vefd_sq(points_curve1_p, curve1_size, points_curve2_p, curve2_size, point_dimensions,
                       *vefd, 1, &v);
    *vefd = std::sqrt(v);
  }
}

bool Cuda_intersection::intersection_interval_call_gpu(double radius) {
  double rub = -2.0;
  rfd_oracle_decide(points_curve1_p, curve1_size, points_curve2_p, curve2_size, point_dimensions,
                    radius, 1, &rub);
  return rub == 1.0;
}

namespace {
Curve make_curve(const double* X, long n, int d) {
  Points pts;
  for (long i = 0; i < n; ++i) pts.push_back(Point(std::vector<double>(X + i * d, X + (i + 1) * d)));
  return Curve(pts, (unsigned)d);
}
}  // namespace

extern "C" {

// compute_distance_parallel of the reference (src/compute_distance_wrapper.cpp:8).
double refhost_distance(const double* P, long n1, const double* Q, long n2, int d) {
  return compute_distance_parallel(make_curve(P, n1, d), make_curve(Q, n2, d));
}

// The reference's endpoint bound expression (src/frechet.cpp:30).
double refhost_endpoint(const double* P, long n1, const double* Q, long n2, int d) {
  Curve a = make_curve(P, n1, d), b = make_curve(Q, n2, d);
  return std::sqrt(std::max(a.front().dist_sqr(b.front()), a.back().dist_sqr(b.back())));
}

// txtLoader2 / txtLoader3 of the reference; writes up to cap points, returns the count and
// each point's coordinate count (a line may carry more or fewer than dims).
long refhost_load(const char* path, int dims, int start, int limit, double* out, int* ncoord, long cap) {
  Points pts = dims == 2 ? txtLoader2(path, start, limit) : txtLoader3(path, start, limit);
  long n = (long)pts.size();
  for (long i = 0; i < n && i < cap; ++i) {
    ncoord[i] = (int)pts[i].coordinates.size();
    for (int k = 0; k < dims; ++k)
      out[i * dims + k] = k < (int)pts[i].coordinates.size() ? pts[i].coordinates[k] : 0.0;
  }
  return n;
}

}  // extern "C"
