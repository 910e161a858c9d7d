// Search driver entry point of the public C++ API (drop-in for the reference's
// include/frechet.hpp:9-18).  distance_cuda runs the whole solve on the GPU through
// rfd_distance (include/rfd.h) with the reference's absolute stop rule at `eps`.
#pragma once

#include "curve.hpp"
#include "geometry_basics.hpp"
#include "intersection_algorithm_in_parallel.hpp"

namespace Frechet {
namespace Continuous {
double distance_cuda(const Curve& curve1, const Curve& curve2, const double eps, bool forceOversize);
}  // namespace Continuous
}  // namespace Frechet
