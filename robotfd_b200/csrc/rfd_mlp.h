// Learned-bracket network: shared constants and the host entry used by the solver.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

struct rfd_model;

namespace rfd_mlp {
constexpr int kFeatures = 386;   // 2 curves x 64 points x 3 coords + log endpoint + log VE-FD
constexpr int kInputWidth = 400; // padded to a multiple of the 16-wide MMA k step
constexpr int kHidden = 256;
constexpr int kOutputs = 2;      // quantiles of y = log10(FD / VEFD - 1 + 1e-13)
constexpr int kPoints = 64;
constexpr float kTauLo = 0.05f, kTauHi = 0.95f;
constexpr long long kNumParams = 400LL * 256 + 256 + 256LL * 256 + 256 + 256LL * 256 + 256 + 256LL * 2 + 2;
constexpr double kYFloor = 1e-13;

int infer(rfd_model* md, const float* X, int B, float* Yout, cudaStream_t s);
// Activation buffers for B rows, allocated ahead of a stream capture (infer then allocates
// nothing); and an identity of those buffers (changes when they are reallocated).
int reserve(rfd_model* md, int B);
const void* buffers_id(const rfd_model* md);
int model_device(const rfd_model* md);
// records the message returned by rfd_last_error and returns code
int set_error(int code, const char* msg);
}  // namespace rfd_mlp
