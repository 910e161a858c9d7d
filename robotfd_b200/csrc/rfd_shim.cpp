// C++ drop-in API over the C ABI: compute_distance_parallel, Frechet::Continuous::
// distance_cuda, Cuda_intersection, plus the C loader rfd_load_txt.
//
// Output and conventions follow the reference: distance_cuda prints the same lines
// (src/frechet.cpp:21-71), the stop rule is ub - lb <= eps, curve 1 is taken as given.
// Errors are printed to stderr, as the reference does, and the returned distance is NaN
// (the reference would return an unrelated value after a failed launch).
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cerrno>
#include <thread>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "frechet.hpp"
#include "intersection_algorithm_in_parallel.hpp"
#include "rfd.h"
#include "rfd_txt_parse.hpp"
#include "wrapper.hpp"

namespace {

std::mutex g_ctx_mu;
rfd_context* g_ctx = nullptr;

// Process-wide context on device 0 (the reference hard-codes device 0, .cu:33/:52).
rfd_context* shared_context() {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (!g_ctx) {
    int rc = rfd_context_create(0, &g_ctx);
    if (rc) {
      std::fprintf(stderr, "rfd: context creation failed: %s (%s)\n", rfd_status_string(rc),
                   rfd_last_error());
      g_ctx = nullptr;
    }
  }
  return g_ctx;
}

std::vector<double> flatten(const Curve& c, unsigned d) {
  std::vector<double> v(c.size() * d);
  for (std::size_t i = 0; i < c.size(); ++i)
    for (unsigned k = 0; k < d; ++k) v[i * d + k] = c[i].coordinates[k];
  return v;
}

unsigned curve_dims(const Curve& c) {
  if (c.empty()) return 0;
  return (unsigned)c[0].coordinates.size();
}

}  // namespace

namespace Frechet {
namespace Continuous {

double distance_cuda(const Curve& curve1, const Curve& curve2, const double eps, bool forceOversize) {
  std::printf("%ld, %ld\n", (long)curve1.size(), (long)curve2.size());
  const unsigned d = curve_dims(curve1);
  if (curve1.empty() || curve2.empty() || (d != 2 && d != 3) || curve_dims(curve2) != d) {
    std::fprintf(stderr, "Invalid dimension.\n");
    return NAN;
  }
  rfd_context* ctx = shared_context();
  if (!ctx) return NAN;
  auto t0 = std::chrono::high_resolution_clock::now();
  std::vector<double> a = flatten(curve1, d), b = flatten(curve2, d);
  rfd_options o;
  rfd_options_init(&o, 0);
  o.tol = eps;
  // the reference's path choice: the fused kernel when forced, else by free device memory
  o.formula = forceOversize ? RFD_FORMULA_FUSED : RFD_FORMULA_REFERENCE;
  rfd_result r;
  int rc = rfd_distance(ctx, a.data(), (int64_t)curve1.size(), b.data(), (int64_t)curve2.size(),
                        (int32_t)d, &o, &r);
  auto t1 = std::chrono::high_resolution_clock::now();
  if (rc) {
    std::fprintf(stderr, "rfd_distance failed: %s (%s)\n", rfd_status_string(rc), rfd_last_error());
    return NAN;
  }
  const double total = std::chrono::duration_cast<std::chrono::microseconds>(t1 - t0).count() / 1000.0;
  std::printf("Naive LB: %.14f\n", r.endpoint);
  std::printf("LB: %.14f\nUB: %.14f\n", r.vefd, r.dfd);
  std::printf("Iteration: %d\n", r.probes);
  std::printf("Result: %.7f\n", r.distance);
  // The whole solve is one device-side launch sequence; its parts are not timed apart.
  std::printf("To GPU Time: %f ms\n", 0.0);
  std::printf("Pre Time: %f ms\n", 0.0);
  std::printf("Interval Time: %f ms\n", 0.0);
  std::printf("Reachability Time: %f ms\n", 0.0);
  std::printf("Total Time: %f ms\n", total);
  return r.distance;
}

}  // namespace Continuous
}  // namespace Frechet

double compute_distance_parallel(const Curve& curve1, const Curve& curve2, bool forceOversize) {
  return Frechet::Continuous::distance_cuda(curve1, curve2, (double)FLT_EPSILON, forceOversize);
}

// All pairwise distances of a Curves collection (no reference counterpart), row-major
// n x n; precise = false keeps the reference's FLT_EPSILON absolute stop rule.  On an error
// the message goes to stderr and every entry is NaN.
std::vector<double> compute_distance_matrix(const Curves& curves, bool precise) {
  const std::size_t n = curves.size();
  std::vector<double> out(n * n, std::nan(""));
  if (n == 0) return out;
  std::vector<std::vector<double>> flat(n);
  std::vector<const double*> ptr(n);
  std::vector<int64_t> ns(n);
  std::vector<int32_t> dims(n);
  for (std::size_t i = 0; i < n; ++i) {
    dims[i] = (int32_t)curve_dims(curves[i]);
    flat[i] = flatten(curves[i], (unsigned)dims[i]);
    ptr[i] = flat[i].data();
    ns[i] = (int64_t)curves[i].size();
  }
  rfd_context* ctx = shared_context();
  rfd_options o;
  rfd_options_init(&o, precise ? 1 : 0);
  const int rc = ctx ? rfd_distance_matrix(ctx, (int64_t)n, ptr.data(), ns.data(), dims.data(), &o,
                                           0.0, out.data(), nullptr)
                     : RFD_ERR_NODEV;
  if (rc != RFD_OK) {
    std::fprintf(stderr, "compute_distance_matrix: %s: %s\n", rfd_status_string(rc), rfd_last_error());
    std::fill(out.begin(), out.end(), std::nan(""));
  }
  return out;
}

// ------------------------------------------------------------------ Cuda_intersection

Cuda_intersection::Cuda_intersection(const Curve& curve1, const Curve& curve2, bool* forceOversize)
    : intervalTime(0.0), reachTime(0.0), curve1_size((int)curve1.size()),
      curve2_size((int)curve2.size()), oversize(true), point_dimensions(curve_dims(curve1)),
      points_curve1_p(nullptr), points_curve2_p(nullptr), ctx(nullptr) {
  // The reference's choice of decision path (src/intersection_algorithm_in_parallel.cu:87-97):
  // fused ("oversize") when forced or when its materialised interval arrays would not fit in
  // free device memory, reported back through *forceOversize.  Here only the rounding of the
  // free intervals follows the choice; the decision's memory is O(n+m) either way.
  oversize = forceOversize ? *forceOversize : false;
  if (!oversize) {
    size_t fr = 0, tot = 0;
    int dev = 0, sms = 0, mtpb = 1024;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaMemGetInfo(&fr, &tot) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&mtpb, cudaDevAttrMaxThreadsPerBlock, dev) != cudaSuccess) {
      cudaGetLastError();
      fr = 0;
    }
    const double a = (double)curve1_size;
    const double need = (double)sms * (double)mtpb +
                        ((a - 1.0) * ((double)curve2_size - 2.0 + a - 2.0) + a) * 8.0 * 4.0;
    oversize = !((double)fr >= need);
  }
  if (forceOversize) *forceOversize = oversize;
  std::vector<double> a = flatten(curve1, point_dimensions), b = flatten(curve2, point_dimensions);
  points_curve1_p = (double*)std::malloc(sizeof(double) * (a.size() ? a.size() : 1));
  points_curve2_p = (double*)std::malloc(sizeof(double) * (b.size() ? b.size() : 1));
  if (points_curve1_p && !a.empty()) std::memcpy(points_curve1_p, a.data(), sizeof(double) * a.size());
  if (points_curve2_p && !b.empty()) std::memcpy(points_curve2_p, b.data(), sizeof(double) * b.size());
  ctx = shared_context();
}

Cuda_intersection::~Cuda_intersection() { free_memory(); }

void Cuda_intersection::data_move() {}

void Cuda_intersection::free_memory() {
  std::free(points_curve1_p);
  std::free(points_curve2_p);
  points_curve1_p = points_curve2_p = nullptr;
}

void Cuda_intersection::Bound_call_gpu(double* dfd, double* vefd) {
  if (!ctx || !points_curve1_p || !points_curve2_p) return;
  auto t0 = std::chrono::high_resolution_clock::now();
  int rc = rfd_bounds(ctx, points_curve1_p, curve1_size, points_curve2_p, curve2_size,
                      (int32_t)point_dimensions, 1, 0, dfd, vefd);
  if (rc)
    std::fprintf(stderr, "Bound_call_gpu failed: %s (%s)\n", rfd_status_string(rc), rfd_last_error());
  auto t1 = std::chrono::high_resolution_clock::now();
  (void)t0;
  (void)t1;
}

bool Cuda_intersection::intersection_interval_call_gpu(double radius) {
  if (!ctx || !points_curve1_p || !points_curve2_p) return false;
  auto t0 = std::chrono::high_resolution_clock::now();
  int32_t reach = 0;
  int rc = rfd_decide_formula(ctx, points_curve1_p, curve1_size, points_curve2_p, curve2_size,
                              (int32_t)point_dimensions, radius, 0,
                              oversize ? RFD_FORMULA_FUSED : RFD_FORMULA_MATERIALISED, &reach,
                              nullptr);
  auto t1 = std::chrono::high_resolution_clock::now();
  reachTime += std::chrono::duration_cast<std::chrono::microseconds>(t1 - t0).count() / 1000.0;
  if (rc) {
    std::fprintf(stderr, "intersection_interval_call_gpu failed: %s (%s)\n", rfd_status_string(rc),
                 rfd_last_error());
    return false;
  }
  return reach != 0;
}

// ------------------------------------------------------------------ C loader

extern "C" {

int32_t rfd_load_txt(const char* path, int32_t dims, int32_t start, int32_t limit, double** out,
                     int64_t* n) {
  if (!path || !out || !n || (dims != 2 && dims != 3)) return RFD_ERR_ARG;
  *out = nullptr;
  *n = 0;
  std::vector<double> flat;
  bool bad_dim = false;
  rfd_txt::ParseStats st = rfd_txt::parse_file(
      path, dims, start, limit,
      [&](const std::vector<double>& c) {
        if ((int)c.size() != dims) bad_dim = true;
        for (int k = 0; k < dims; ++k) flat.push_back(k < (int)c.size() ? c[k] : 0.0);
      },
      [&](const std::string&) {});
  if (!st.opened) return RFD_ERR_ARG;
  if (bad_dim) return RFD_ERR_ARG;
  const int64_t np = (int64_t)(flat.size() / dims);
  double* buf = (double*)std::malloc(sizeof(double) * (flat.empty() ? 1 : flat.size()));
  if (!buf) return RFD_ERR_NOMEM;
  if (!flat.empty()) std::memcpy(buf, flat.data(), sizeof(double) * flat.size());
  *out = buf;
  *n = np;
  return RFD_OK;
}

// ------------------------------------------------------------------ fast loader
// rfd_load_txt's rules (rfd_txt_parse.hpp), with the parsing spread over threads: the file
// is read whole, cut into line ranges of about equal bytes, every token is NUL-terminated in
// place and converted with strtod under std::stod's acceptance rule (something converted,
// no ERANGE); the point counter, START, LIMIT and the duplicate rule then run in one pass
// over the lines in order.

namespace {

struct LineResult {
  bool nonempty = false;
  std::vector<double> coords;
};

// std::getline(ss, token, ',') over one line: tokens between commas, no empty token after a
// trailing comma, one empty token for a line that is a single comma.
void parse_line(char* b, char* e, LineResult& r) {
  r.coords.clear();
  if (b == e) return;
  char* t = b;
  for (;;) {
    char* c = t;
    while (c < e && *c != ',') ++c;
    const bool last = c >= e;
    *c = '\0';  // the line's end or the comma
    errno = 0;
    char* end = nullptr;
    const double v = std::strtod(t, &end);
    if (end != t && errno != ERANGE) r.coords.push_back(v);
    if (last) break;
    t = c + 1;
    if (t >= e) break;  // a trailing comma ends the line without an empty token
  }
  r.nonempty = !r.coords.empty();
}

}  // namespace

int32_t rfd_load_txt_fast(const char* path, int32_t dims, int32_t start, int32_t limit,
                          int32_t threads, double** out, int64_t* n) {
  if (!path || !out || !n || (dims != 2 && dims != 3)) return RFD_ERR_ARG;
  *out = nullptr;
  *n = 0;
  FILE* f = std::fopen(path, "rb");
  if (!f) return RFD_ERR_ARG;
  std::vector<char> buf;
  {
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (size > 0) {
      buf.resize((size_t)size);
      buf.resize(std::fread(buf.data(), 1, (size_t)size, f));
    }
    char tmp[1 << 16];  // anything past the size seen (a growing file, a pipe)
    size_t got;
    while ((got = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + got);
    std::fclose(f);
  }
  buf.push_back('\n');  // every line, the last one included, ends with a newline
  // line starts
  std::vector<size_t> ls;
  ls.reserve(buf.size() / 16 + 2);
  ls.push_back(0);
  for (const char* q = buf.data(); ; ) {
    const char* e = (const char*)std::memchr(q, '\n', buf.data() + buf.size() - 1 - q);
    if (!e) break;
    ls.push_back((size_t)(e - buf.data()) + 1);
    q = e + 1;
  }
  const size_t nl = ls.size();  // the extra newline makes the last start the end of data
  std::vector<LineResult> res(nl - 1);
  int T = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
  T = std::max(1, std::min<int>(T, 64));
  auto work = [&](size_t l0, size_t l1) {
    for (size_t l = l0; l < l1; ++l) {
      char* b = buf.data() + ls[l];
      char* e = buf.data() + ls[l + 1] - 1;  // the newline
      parse_line(b, e, res[l]);
    }
  };
  if (T == 1 || nl < 4096) {
    work(0, nl - 1);
  } else {
    std::vector<std::thread> pool;
    const size_t per = (nl - 1 + T - 1) / T;
    for (int t = 0; t < T; ++t) {
      const size_t l0 = std::min(nl - 1, t * per), l1 = std::min(nl - 1, (t + 1) * per);
      if (l0 < l1) pool.emplace_back(work, l0, l1);
    }
    for (auto& th : pool) th.join();
  }
  std::vector<double> flat;
  bool bad_dim = false, have_last = false;
  std::vector<double> last;
  int count = 0;
  for (size_t l = 0; l + 1 < nl; ++l) {
    if (count >= limit) break;
    const LineResult& r = res[l];
    if (!r.nonempty) continue;
    ++count;
    if (count < start) continue;
    bool keep = !have_last;
    if (have_last)
      for (int k = 0; k < dims; ++k) {
        const double a = k < (int)last.size() ? last[k] : 0.0;
        const double b = k < (int)r.coords.size() ? r.coords[k] : 0.0;
        if (a != b) keep = true;
      }
    if (!keep) continue;
    last = r.coords;
    have_last = true;
    if ((int)r.coords.size() != dims) bad_dim = true;
    for (int k = 0; k < dims; ++k) flat.push_back(k < (int)r.coords.size() ? r.coords[k] : 0.0);
  }
  if (bad_dim) return RFD_ERR_ARG;
  double* o = (double*)std::malloc(sizeof(double) * (flat.empty() ? 1 : flat.size()));
  if (!o) return RFD_ERR_NOMEM;
  if (!flat.empty()) std::memcpy(o, flat.data(), sizeof(double) * flat.size());
  *out = o;
  *n = (int64_t)(flat.size() / dims);
  return RFD_OK;
}

// Binary trajectory file: "RFDB", uint32 version 1, int32 dims, int32 0, int64 n, then
// n * dims little-endian doubles (the interleaved [n][dims] layout).
int32_t rfd_save_bin(const char* path, const double* pts, int64_t n, int32_t dims) {
  if (!path || (!pts && n) || n < 0 || dims < 1 || dims > 3) return RFD_ERR_ARG;
  FILE* f = std::fopen(path, "wb");
  if (!f) return RFD_ERR_ARG;
  const uint32_t version = 1;
  const int32_t zero = 0;
  bool ok = std::fwrite("RFDB", 1, 4, f) == 4 && std::fwrite(&version, 4, 1, f) == 1 &&
            std::fwrite(&dims, 4, 1, f) == 1 && std::fwrite(&zero, 4, 1, f) == 1 &&
            std::fwrite(&n, 8, 1, f) == 1 &&
            (n == 0 || std::fwrite(pts, sizeof(double) * dims, (size_t)n, f) == (size_t)n);
  ok = (std::fclose(f) == 0) && ok;
  return ok ? RFD_OK : RFD_ERR_ARG;
}

int32_t rfd_load_bin(const char* path, double** out, int64_t* n, int32_t* dims) {
  if (!path || !out || !n || !dims) return RFD_ERR_ARG;
  *out = nullptr;
  *n = 0;
  *dims = 0;
  FILE* f = std::fopen(path, "rb");
  if (!f) return RFD_ERR_ARG;
  char magic[4];
  uint32_t version = 0;
  int32_t d = 0, zero = 0;
  int64_t cnt = 0;
  bool ok = std::fread(magic, 1, 4, f) == 4 && std::memcmp(magic, "RFDB", 4) == 0 &&
            std::fread(&version, 4, 1, f) == 1 && version == 1 && std::fread(&d, 4, 1, f) == 1 &&
            std::fread(&zero, 4, 1, f) == 1 && std::fread(&cnt, 8, 1, f) == 1 && d >= 1 &&
            d <= 3 && cnt >= 0 && cnt < ((int64_t)1 << 40);
  double* o = nullptr;
  if (ok) {
    o = (double*)std::malloc(sizeof(double) * (cnt ? cnt * d : 1));
    ok = o && (cnt == 0 || std::fread(o, sizeof(double) * d, (size_t)cnt, f) == (size_t)cnt);
  }
  std::fclose(f);
  if (!ok) {
    std::free(o);
    return RFD_ERR_ARG;
  }
  *out = o;
  *n = cnt;
  *dims = d;
  return RFD_OK;
}

void rfd_free(void* p) { std::free(p); }

}  // extern "C"
