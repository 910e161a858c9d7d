// FP32 filter of the free-interval computation, compiled for host and device.
//
// The FP64 free interval of an edge (rfd_device.cuh free_interval, reference
// .cu:1175-1230) has three kinds of outcome: empty, written (-1, -2); the whole edge,
// written (0, 1) exactly; and a partial edge, whose end points need the FP64 arithmetic.
// interval_class32 evaluates the same quadratic in FP32 together with a bound on the
// distance between each FP32 quantity and the one the FP64 code computes, and returns
//   1 when the FP64 code certainly yields empty,
//   2 when it certainly yields (0, 1),
//   0 otherwise (the caller computes the interval in FP64).
// A certain answer is exactly what the FP64 code writes, so decisions are unchanged.
//
// Error bounds (u = 2^-24; the FP64 code's own rounding, at 2^-53, is covered by the same
// margins).  With m_k = fl32(a_k - x_k) (the FP64 difference the FP64 code also uses) and
// d_k = fl32(di_k):
//   B = 2 sum m d:            |B32 - B64| <= 6u SB,   SB = 2 sum |m||d|      (bound used: 16u SB)
//   C = sum m^2 - r2:         |C32 - C64| <= 7u SC,   SC = sum m^2 + r2
//   disc = B^2 - 4 A C:       |disc32 - disc64| <= 23u Md,  Md = SB^2 + 4 A SC  (used: 64u Md)
//   s = sqrt(max(disc, 0)):   |s32 - s64| <= sqrt(|disc32 - disc64|) + 4u s
// and with P = -B, the end points are ta = (P - s) / 2A and tb = (P + s) / 2A, so
//   empty  <=> disc < 0, or P + s < 0 (tb < 0), or P - s > 2A (ta > 1);
//   (0, 1) <=> disc >= 0 and P - s < 0 (ta < 0) and P + s > 2A (tb > 1);
// each tested with the margin EB + Es + 16u (|P| + s + 2A).  Degenerate edges (A = 0, which
// the FP64 code turns into NaN end points), non-finite or underflowing magnitudes all
// return 0.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define RFD_FHD __host__ __device__ __forceinline__
#else
#define RFD_FHD inline
#endif

namespace rfd {

template <int D>
RFD_FHD int interval_class32(const double* x, const double* a, const double* di, double A,
                             double r2) {
  const float u = 5.9604644775390625e-08f;  // 2^-24
  float B = 0.f, SB = 0.f, S2 = 0.f;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    const float m = (float)(a[k] - x[k]);
    const float d = (float)di[k];
    B = fmaf(m, d, B);
    SB = fmaf(fabsf(m), fabsf(d), SB);
    S2 = fmaf(m, m, S2);
  }
  B *= 2.f;
  SB *= 2.f;
  const float Af = (float)A, r2f = (float)r2;
  const float C = S2 - r2f;
  const float SC = S2 + r2f;
  const float disc = fmaf(B, B, -4.f * Af * C);
  const float Md = fmaf(SB, SB, 4.f * Af * SC);
  // degenerate, non-finite or underflowing magnitudes: leave it to FP64
  if (!(Af > 1e-30f) || !(Md > 1e-30f) || !(Md < 1e30f) || !(SB < 1e15f)) return 0;
  const float Ed = 64.f * u * Md;
  const float EB = 16.f * u * SB;
  if (disc < -Ed) return 1;
  const float P = -B;
  const float s = sqrtf(fmaxf(disc, 0.f));
  const float Es = sqrtf(Ed) + 4.f * u * s;
  const float twoA = 2.f * Af;
  const float Mt = EB + Es + 16.f * u * (fabsf(P) + s + twoA);
  if (P + s < -Mt) return 1;         // tb < 0
  if (P - s > twoA + Mt) return 1;   // ta > 1
  if (disc > Ed && P - s < -Mt && P + s > twoA + Mt) return 2;
  return 0;
}

}  // namespace rfd
