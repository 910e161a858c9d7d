// Learned bracket network: a BF16 MLP (FP32 accumulation) on the tensor cores.
//
//   x[400] (386 features + zero padding) -> 256 -> 256 -> 256 (GELU, tanh form) -> 2
//
// The two outputs are the 5% and 95% quantiles of y = log10(FD/VEFD - 1 + 1e-13), trained
// with the pinball loss on FD values the plain method produced; the solver turns them into
// the bracket [VEFD (1 + 10^q05), VEFD (1 + 10^q95)] and verifies it with two decisions.
//
// Every matrix product (forward, input gradients, weight gradients) runs through one
// mma.sync.m16n8k16 BF16 GEMM kernel with per-use element loaders and fused epilogues
// (bias, GELU, GELU derivative).  Layer widths are 400/256/256/256/2 and batches a few
// thousand rows, so a call is a few GFLOP: latency-bound, which is why the kernel stays a
// plain 64x64 tile without TMA or TMEM staging.  Master weights and Adam moments are FP32.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "rfd.h"
#include "rfd_mlp.h"

namespace rfd_mlp {

// ------------------------------------------------------------------ parameters

constexpr int kLayers = 4;
constexpr int kIn[kLayers] = {kInputWidth, kHidden, kHidden, kHidden};
constexpr int kOut[kLayers] = {kHidden, kHidden, kHidden, kOutputs};

constexpr size_t w_off(int l) {
  return l == 0 ? 0
                : w_off(l - 1) + (size_t)kIn[l - 1] * kOut[l - 1] + (size_t)kOut[l - 1];
}
constexpr size_t b_off(int l) { return w_off(l) + (size_t)kIn[l] * kOut[l]; }
constexpr size_t kParams = w_off(kLayers);
static_assert(kParams == kNumParams, "parameter count");

// ------------------------------------------------------------------ GEMM

__device__ __forceinline__ float gelu(float z) {
  const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
  return 0.5f * z * (1.0f + tanhf(u));
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
  const float th = tanhf(u);
  return 0.5f * (1.0f + th) +
         0.5f * z * (1.0f - th * th) * 0.7978845608028654f * (1.0f + 3.0f * 0.044715f * z * z);
}

__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

constexpr int BM = 64, BN = 64, BK = 32, PAD = 8;

// Operand element (r, c) = ptr[r * sr + c * sc], read as FP32 or BF16.
struct Operand {
  const void* ptr;
  long long sr, sc;
  int bf16;
  __device__ __forceinline__ float at(long long r, long long c) const {
    const long long i = r * sr + c * sc;
    return bf16 ? __bfloat162float(((const __nv_bfloat16*)ptr)[i]) : ((const float*)ptr)[i];
  }
};

enum Epi {
  EPI_STORE_F32 = 0,       // outf[m][n] = acc (+ bias)
  EPI_BIAS_GELU = 1,       // z = acc + bias -> outf (pre-activation), outh = bf16(gelu(z))
  EPI_GELU_GRAD = 2,       // outf[m][n] = acc * gelu'(aux[m][n])
};

struct EpiArgs {
  int kind;
  const float* bias;  // [N] or null
  float* outf;        // FP32 [M][N] (ld = N)
  __nv_bfloat16* outh;  // BF16 [M][N]
  const float* aux;   // FP32 [M][N] pre-activations for EPI_GELU_GRAD
};

// C[M][N] = A[M][K] * B[K][N], A(m,k) and B(k,n) through Operand strides.
__global__ void __launch_bounds__(128) gemm_kernel(int M, int N, int K, Operand A, Operand B,
                                                   EpiArgs ep) {
  __shared__ __align__(16) __nv_bfloat16 As[BM][BK + PAD];
  __shared__ __align__(16) __nv_bfloat16 Bs[BN][BK + PAD];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;
  for (int k0 = 0; k0 < K; k0 += BK) {
    for (int e = tid; e < BM * BK; e += 128) {
      const int r = e / BK, k = e % BK;
      const int gm = m0 + r, gk = k0 + k;
      As[r][k] = __float2bfloat16(gm < M && gk < K ? A.at(gm, gk) : 0.f);
    }
    for (int e = tid; e < BN * BK; e += 128) {
      const int n = e / BK, k = e % BK;
      const int gn = n0 + n, gk = k0 + k;
      Bs[n][k] = __float2bfloat16(gn < N && gk < K ? B.at(gk, gn) : 0.f);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      uint32_t af[2][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + i * 16 + g;
        af[i][0] = *(const uint32_t*)&As[r][kk + 2 * t];
        af[i][1] = *(const uint32_t*)&As[r + 8][kk + 2 * t];
        af[i][2] = *(const uint32_t*)&As[r][kk + 2 * t + 8];
        af[i][3] = *(const uint32_t*)&As[r + 8][kk + 2 * t + 8];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int n = wn + j * 8 + g;
        bfr[j][0] = *(const uint32_t*)&Bs[n][kk + 2 * t];
        bfr[j][1] = *(const uint32_t*)&Bs[n][kk + 2 * t + 8];
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma16816(acc[i][j], af[i], bfr[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int m = m0 + wm + i * 16 + g + (q >= 2 ? 8 : 0);
        const int n = n0 + wn + j * 8 + 2 * t + (q & 1);
        if (m >= M || n >= N) continue;
        float v = acc[i][j][q];
        const size_t o = (size_t)m * N + n;
        if (ep.kind == EPI_STORE_F32) {
          if (ep.bias) v += ep.bias[n];
          ep.outf[o] = v;
        } else if (ep.kind == EPI_BIAS_GELU) {
          v += ep.bias[n];
          if (ep.outf) ep.outf[o] = v;
          ep.outh[o] = __float2bfloat16(gelu(v));
        } else {
          ep.outf[o] = v * gelu_grad(ep.aux[o]);
        }
      }
}

void gemm(cudaStream_t s, int M, int N, int K, Operand A, Operand B, EpiArgs ep) {
  dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
  gemm_kernel<<<grid, 128, 0, s>>>(M, N, K, A, B, ep);
}

// ------------------------------------------------------------------ small kernels

__global__ void to_bf16_kernel(const float* in, __nv_bfloat16* out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16(in[i]);
}

// Pinball loss of the two quantile outputs; dY = dLoss/dY (mean over the batch).
__global__ void pinball_kernel(const float* Y, const float* target, int B, float* dY, float* loss) {
  __shared__ float red[256];
  float l = 0.f;
  const float tau[2] = {kTauLo, kTauHi};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B; i += gridDim.x * blockDim.x) {
    for (int k = 0; k < 2; ++k) {
      const float u = target[i] - Y[(size_t)i * 2 + k];
      const float ind = u < 0.f ? 1.f : 0.f;
      l += u * (tau[k] - ind);
      dY[(size_t)i * 2 + k] = -(tau[k] - ind) / (float)B;
    }
  }
  red[threadIdx.x] = l;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] / (float)B);
}

// db[n] = sum_m dZ[m][n]
__global__ void colsum_kernel(const float* dZ, int M, int N, float* db) {
  const int n = blockIdx.x;
  float s = 0.f;
  for (int m = threadIdx.x; m < M; m += blockDim.x) s += dZ[(size_t)m * N + n];
  __shared__ float red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[n] = red[0];
}

__global__ void adam_kernel(float* w, const float* g, float* m, float* v, size_t n, float lr,
                            float b1, float b2, float eps, float c1, float c2, __nv_bfloat16* wh) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wh[i] = __float2bfloat16(wi);
  }
}

}  // namespace rfd_mlp

using namespace rfd_mlp;

// ------------------------------------------------------------------ model object

struct rfd_model {
  int device = 0;
  cudaStream_t stream = nullptr;
  float* w = nullptr;       // FP32 master parameters [kParams]
  __nv_bfloat16* wh = nullptr;  // BF16 copies used by the GEMMs
  float* g = nullptr;       // gradients
  float* m = nullptr;       // Adam moments
  float* v = nullptr;
  long long step = 0;
  // activation scratch for a batch of up to cap rows
  int cap = 0;
  float* Z[3] = {nullptr, nullptr, nullptr};  // pre-activations
  __nv_bfloat16* H[3] = {nullptr, nullptr, nullptr};
  float* Y = nullptr;
  float* dY = nullptr;
  float* dZa = nullptr;
  float* dZb = nullptr;
  float* loss = nullptr;
};

namespace {

int mfail(int code, const std::string& m) { return rfd_mlp::set_error(code, m.c_str()); }
#define MLP_CUDA(call)                                                                        \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return mfail(RFD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int ensure_cap(rfd_model* md, int B) {
  if (B <= md->cap) return RFD_OK;
  for (int l = 0; l < 3; ++l) {
    cudaFree(md->Z[l]);
    cudaFree(md->H[l]);
  }
  cudaFree(md->Y);
  cudaFree(md->dY);
  cudaFree(md->dZa);
  cudaFree(md->dZb);
  const int cap = std::max(B, 4096);
  for (int l = 0; l < 3; ++l) {
    MLP_CUDA(cudaMalloc(&md->Z[l], sizeof(float) * (size_t)cap * kHidden));
    MLP_CUDA(cudaMalloc(&md->H[l], sizeof(__nv_bfloat16) * (size_t)cap * kHidden));
  }
  MLP_CUDA(cudaMalloc(&md->Y, sizeof(float) * (size_t)cap * kOutputs));
  MLP_CUDA(cudaMalloc(&md->dY, sizeof(float) * (size_t)cap * kOutputs));
  MLP_CUDA(cudaMalloc(&md->dZa, sizeof(float) * (size_t)cap * kHidden));
  MLP_CUDA(cudaMalloc(&md->dZb, sizeof(float) * (size_t)cap * kHidden));
  md->cap = cap;
  return RFD_OK;
}

Operand weight_T(const rfd_model* md, int l) {
  // B(k, n) = W_l[n][k]
  return Operand{md->wh + w_off(l), 1, (long long)kIn[l], 1};
}

// Forward pass for B rows of X (FP32 [B][400], device); fills Z, H, Y.
int forward(rfd_model* md, const float* X, int B, cudaStream_t s) {
  int rc = ensure_cap(md, B);
  if (rc) return rc;
  Operand in{X, kInputWidth, 1, 0};
  for (int l = 0; l < 3; ++l) {
    EpiArgs ep{EPI_BIAS_GELU, md->w + b_off(l), md->Z[l], md->H[l], nullptr};
    gemm(s, B, kHidden, kIn[l], in, weight_T(md, l), ep);
    in = Operand{md->H[l], kHidden, 1, 1};
  }
  EpiArgs ep{EPI_STORE_F32, md->w + b_off(3), md->Y, nullptr, nullptr};
  gemm(s, B, kOutputs, kHidden, in, weight_T(md, 3), ep);
  MLP_CUDA(cudaGetLastError());
  return RFD_OK;
}

// Loss and gradients (md->g) for B rows with targets T (device).
int backward(rfd_model* md, const float* X, const float* T, int B, cudaStream_t s) {
  int rc = forward(md, X, B, s);
  if (rc) return rc;
  MLP_CUDA(cudaMemsetAsync(md->loss, 0, sizeof(float), s));
  pinball_kernel<<<std::min(64, (B + 255) / 256), 256, 0, s>>>(md->Y, T, B, md->dY, md->loss);
  // layer 4: dW4[n][k] = sum_m dY[m][n] H3[m][k]; db4; dZ3 = (dY W4) * gelu'(Z3)
  const float* dcur = md->dY;
  int Ncur = kOutputs;
  float* dnext[2] = {md->dZa, md->dZb};
  for (int l = 3; l >= 0; --l) {
    const Operand dZT{dcur, 1, Ncur, 0};  // A(n, m) = dZ[m][n]
    const Operand Xin = l == 0 ? Operand{X, kInputWidth, 1, 0}
                               : Operand{md->H[l - 1], kHidden, 1, 1};  // B(m, k)
    EpiArgs ew{EPI_STORE_F32, nullptr, md->g + w_off(l), nullptr, nullptr};
    gemm(s, Ncur, kIn[l], B, dZT, Xin, ew);
    colsum_kernel<<<Ncur, 256, 0, s>>>(dcur, B, Ncur, md->g + b_off(l));
    if (l > 0) {
      // dH[m][k] = sum_n dZ[m][n] W_l[n][k]; times gelu'(Z_{l-1})
      float* out = dnext[l & 1];
      const Operand dZ{dcur, Ncur, 1, 0};
      const Operand W{md->wh + w_off(l), (long long)kIn[l], 1, 1};  // B(n, k) = W[n][k]
      EpiArgs ed{EPI_GELU_GRAD, nullptr, out, nullptr, md->Z[l - 1]};
      gemm(s, B, kIn[l], Ncur, dZ, W, ed);
      dcur = out;
      Ncur = kIn[l];
    }
  }
  MLP_CUDA(cudaGetLastError());
  return RFD_OK;
}

}  // namespace

namespace rfd_mlp {
int model_device(const rfd_model* md) { return md->device; }
// Inference for the solver: X FP32 [B][400] (device) -> Y FP32 [B][2] (device, ld 2).
int reserve(rfd_model* md, int B) { return ensure_cap(md, B); }
const void* buffers_id(const rfd_model* md) { return md->Y; }

int infer(rfd_model* md, const float* X, int B, float* Yout, cudaStream_t s) {
  int rc = forward(md, X, B, s);
  if (rc) return rc;
  MLP_CUDA(cudaMemcpyAsync(Yout, md->Y, sizeof(float) * (size_t)B * kOutputs,
                           cudaMemcpyDeviceToDevice, s));
  return RFD_OK;
}
}  // namespace rfd_mlp

extern "C" {

int64_t rfd_model_num_params(void) { return (int64_t)kParams; }

int32_t rfd_gemm_bf16(int32_t M, int32_t N, int32_t K, const float* A, int64_t a_sr, int64_t a_sc,
                      const float* B, int64_t b_sr, int64_t b_sc, float* C) {
  if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0) return mfail(RFD_ERR_ARG, "gemm args");
  EpiArgs ep{EPI_STORE_F32, nullptr, C, nullptr, nullptr};
  gemm(0, M, N, K, Operand{A, a_sr, a_sc, 0}, Operand{B, b_sr, b_sc, 0}, ep);
  MLP_CUDA(cudaGetLastError());
  MLP_CUDA(cudaDeviceSynchronize());
  return RFD_OK;
}

int32_t rfd_model_create(int32_t device, uint64_t seed, rfd_model** out) {
  if (!out) return RFD_ERR_ARG;
  *out = nullptr;
  MLP_CUDA(cudaSetDevice(device));
  rfd_model* md = new rfd_model();
  md->device = device;
  if (cudaStreamCreateWithFlags(&md->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&md->w, sizeof(float) * kParams) != cudaSuccess ||
      cudaMalloc(&md->wh, sizeof(__nv_bfloat16) * kParams) != cudaSuccess ||
      cudaMalloc(&md->g, sizeof(float) * kParams) != cudaSuccess ||
      cudaMalloc(&md->m, sizeof(float) * kParams) != cudaSuccess ||
      cudaMalloc(&md->v, sizeof(float) * kParams) != cudaSuccess ||
      cudaMalloc(&md->loss, sizeof(float)) != cudaSuccess) {
    rfd_model_destroy(md);
    return mfail(RFD_ERR_NOMEM, "model allocation");
  }
  // He-style init from a seeded stream: w ~ U(-a, a), a = sqrt(6 / fan_in); biases 0
  std::vector<float> h(kParams, 0.f);
  uint64_t st = seed * 0x9E3779B97F4A7C15ULL + 1;
  auto nxt = [&]() {
    uint64_t z = (st += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return (double)((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
  };
  for (int l = 0; l < kLayers; ++l) {
    const double a = std::sqrt(6.0 / kIn[l]) * (l == kLayers - 1 ? 0.1 : 1.0);
    for (size_t i = 0; i < (size_t)kIn[l] * kOut[l]; ++i) h[w_off(l) + i] = (float)((2 * nxt() - 1) * a);
  }
  int rc = rfd_model_set_params(md, h.data(), (int64_t)kParams);
  if (rc) {
    rfd_model_destroy(md);
    return rc;
  }
  *out = md;
  return RFD_OK;
}

int32_t rfd_model_destroy(rfd_model* md) {
  if (!md) return RFD_OK;
  cudaSetDevice(md->device);
  cudaFree(md->w);
  cudaFree(md->wh);
  cudaFree(md->g);
  cudaFree(md->m);
  cudaFree(md->v);
  cudaFree(md->loss);
  for (int l = 0; l < 3; ++l) {
    cudaFree(md->Z[l]);
    cudaFree(md->H[l]);
  }
  cudaFree(md->Y);
  cudaFree(md->dY);
  cudaFree(md->dZa);
  cudaFree(md->dZb);
  if (md->stream) cudaStreamDestroy(md->stream);
  delete md;
  return RFD_OK;
}

int32_t rfd_model_set_params(rfd_model* md, const float* params, int64_t n) {
  if (!md || !params || n != (int64_t)kParams) return mfail(RFD_ERR_ARG, "parameter count");
  MLP_CUDA(cudaSetDevice(md->device));
  // On the model's stream, ahead of the BF16 conversion: a plain cudaMemcpy from pageable
  // memory may return before its DMA lands, and the model's stream (non-blocking) does not
  // wait for it, so the conversion could read stale parameters.
  MLP_CUDA(cudaMemcpyAsync(md->w, params, sizeof(float) * kParams, cudaMemcpyHostToDevice,
                           md->stream));
  to_bf16_kernel<<<256, 256, 0, md->stream>>>(md->w, md->wh, kParams);
  MLP_CUDA(cudaMemsetAsync(md->m, 0, sizeof(float) * kParams, md->stream));
  MLP_CUDA(cudaMemsetAsync(md->v, 0, sizeof(float) * kParams, md->stream));
  MLP_CUDA(cudaStreamSynchronize(md->stream));
  md->step = 0;
  return RFD_OK;
}

int32_t rfd_model_get_params(rfd_model* md, float* params, int64_t n) {
  if (!md || !params || n != (int64_t)kParams) return mfail(RFD_ERR_ARG, "parameter count");
  MLP_CUDA(cudaSetDevice(md->device));
  MLP_CUDA(cudaMemcpyAsync(params, md->w, sizeof(float) * kParams, cudaMemcpyDeviceToHost,
                           md->stream));
  MLP_CUDA(cudaStreamSynchronize(md->stream));
  return RFD_OK;
}

int32_t rfd_model_forward(rfd_model* md, const float* x_dev, int64_t B, float* y_dev) {
  if (!md || !x_dev || !y_dev || B <= 0 || B > (1 << 24)) return mfail(RFD_ERR_ARG, "forward args");
  MLP_CUDA(cudaSetDevice(md->device));
  int rc = infer(md, x_dev, (int)B, y_dev, md->stream);
  if (rc) return rc;
  MLP_CUDA(cudaStreamSynchronize(md->stream));
  return RFD_OK;
}

int32_t rfd_model_gradients(rfd_model* md, const float* x_dev, const float* t_dev, int64_t B,
                            float* grads, float* loss) {
  if (!md || !x_dev || !t_dev || B <= 0 || B > (1 << 24)) return mfail(RFD_ERR_ARG, "gradient args");
  MLP_CUDA(cudaSetDevice(md->device));
  int rc = backward(md, x_dev, t_dev, (int)B, md->stream);
  if (rc) return rc;
  if (grads) MLP_CUDA(cudaMemcpyAsync(grads, md->g, sizeof(float) * kParams, cudaMemcpyDeviceToHost, md->stream));
  if (loss) MLP_CUDA(cudaMemcpyAsync(loss, md->loss, sizeof(float), cudaMemcpyDeviceToHost, md->stream));
  MLP_CUDA(cudaStreamSynchronize(md->stream));
  return RFD_OK;
}

int32_t rfd_model_train_step(rfd_model* md, const float* x_dev, const float* t_dev, int64_t B,
                             float lr, float* loss) {
  if (!md || !x_dev || !t_dev || B <= 0 || B > (1 << 24)) return mfail(RFD_ERR_ARG, "train args");
  MLP_CUDA(cudaSetDevice(md->device));
  int rc = backward(md, x_dev, t_dev, (int)B, md->stream);
  if (rc) return rc;
  md->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)md->step), c2 = 1.f - powf(b2, (float)md->step);
  adam_kernel<<<512, 256, 0, md->stream>>>(md->w, md->g, md->m, md->v, kParams, lr, b1, b2, 1e-8f,
                                           c1, c2, md->wh);
  MLP_CUDA(cudaGetLastError());
  if (loss) MLP_CUDA(cudaMemcpyAsync(loss, md->loss, sizeof(float), cudaMemcpyDeviceToHost, md->stream));
  MLP_CUDA(cudaStreamSynchronize(md->stream));
  return RFD_OK;
}

}  // extern "C"
