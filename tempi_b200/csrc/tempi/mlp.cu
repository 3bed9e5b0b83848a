// The learned cost model's network: a 12 -> 64 -> 64 -> 23 FP32 perceptron
// with ReLU hidden layers, trained and run by these kernels.  It replaces the
// reference's measured-parameter tables (src/internal/measure_system.cpp,
// interp_2d :223-299) as the predictor of pack and transfer times.
//
// Layout of one member's parameters (floats, row-major [out][in]):
//   W1[64][12] b1[64] W2[64][64] b2[64] W3[19][64] b3[19]   (6227 floats)
// An ensemble is `members` such blocks back to back.
//
// Training: one CTA per member, the whole optimisation in one launch.  The
// member's parameters, its gradient and its Adam moments live in shared
// memory (4 x 6227 floats), as do the activations of one mini-batch, so
// the only global traffic is the mini-batch rows.  Loss: squared error on
// the observed outputs only (a mask marks them), averaged over them.

#include "internal.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace tempi {

constexpr int kIn = TEMPI_MLP_IN;
constexpr int kHid = TEMPI_MLP_HIDDEN;
constexpr int kOut = TEMPI_MLP_OUT;
constexpr int kP = TEMPI_MLP_PARAMS;
constexpr int kMaxBatch = 64;
constexpr int kThreads = 256;

// offsets in a member's parameter block
constexpr int oW1 = 0, oB1 = oW1 + kHid * kIn, oW2 = oB1 + kHid,
              oB2 = oW2 + kHid * kHid, oW3 = oB2 + kHid,
              oB3 = oW3 + kOut * kHid;
static_assert(oB3 + kOut == kP, "parameter layout");

struct Act {
  float x[kMaxBatch][kIn];
  float y[kMaxBatch][kOut];
  float m[kMaxBatch][kOut];
  float h1[kMaxBatch][kHid];
  float h2[kMaxBatch][kHid];
  float o[kMaxBatch][kOut]; // output, then its gradient
  float d2[kMaxBatch][kHid];
  float d1[kMaxBatch][kHid];
  float red[kThreads / 32];
};

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  // SplitMix64 finaliser (Steele, Lea, Flood, "Fast splittable
  // pseudorandom number generators", OOPSLA 2014)
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__device__ void forward(const float *p, Act &a, int nb) {
  for (int t = threadIdx.x; t < nb * kHid; t += blockDim.x) {
    const int b = t / kHid, j = t % kHid;
    float s = p[oB1 + j];
#pragma unroll
    for (int k = 0; k < kIn; ++k)
      s = fmaf(p[oW1 + j * kIn + k], a.x[b][k], s);
    a.h1[b][j] = fmaxf(s, 0.f);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nb * kHid; t += blockDim.x) {
    const int b = t / kHid, j = t % kHid;
    float s = p[oB2 + j];
#pragma unroll 8
    for (int k = 0; k < kHid; ++k)
      s = fmaf(p[oW2 + j * kHid + k], a.h1[b][k], s);
    a.h2[b][j] = fmaxf(s, 0.f);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nb * kOut; t += blockDim.x) {
    const int b = t / kOut, j = t % kOut;
    float s = p[oB3 + j];
#pragma unroll 8
    for (int k = 0; k < kHid; ++k)
      s = fmaf(p[oW3 + j * kHid + k], a.h2[b][k], s);
    a.o[b][j] = s;
  }
  __syncthreads();
}

__device__ float block_sum(float v, float *red) {
  for (int off = 16; off > 0; off >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0)
    red[threadIdx.x >> 5] = v;
  __syncthreads();
  float s = 0.f;
  if (threadIdx.x < 32) {
    s = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.f;
    for (int off = 16; off > 0; off >>= 1)
      s += __shfl_down_sync(0xffffffffu, s, off);
    if (threadIdx.x == 0)
      red[0] = s;
  }
  __syncthreads();
  s = red[0];
  __syncthreads();
  return s;
}

// gradient of the masked mean squared error into g; returns the loss
__device__ float backward(const float *p, float *g, Act &a, int nb) {
  float cnt = 0.f, se = 0.f;
  for (int t = threadIdx.x; t < nb * kOut; t += blockDim.x) {
    const int b = t / kOut, j = t % kOut;
    const float d = a.o[b][j] - a.y[b][j];
    cnt += a.m[b][j];
    se += a.m[b][j] * d * d;
  }
  cnt = block_sum(cnt, a.red);
  se = block_sum(se, a.red);
  const float inv = cnt > 0.f ? 1.f / cnt : 0.f;
  for (int t = threadIdx.x; t < nb * kOut; t += blockDim.x) {
    const int b = t / kOut, j = t % kOut;
    a.o[b][j] = 2.f * a.m[b][j] * (a.o[b][j] - a.y[b][j]) * inv; // dL/do
  }
  __syncthreads();
  // layer 3
  for (int t = threadIdx.x; t < kOut * kHid; t += blockDim.x) {
    const int j = t / kHid, k = t % kHid;
    float s = 0.f;
    for (int b = 0; b < nb; ++b)
      s = fmaf(a.o[b][j], a.h2[b][k], s);
    g[oW3 + t] = s;
  }
  for (int j = threadIdx.x; j < kOut; j += blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < nb; ++b)
      s += a.o[b][j];
    g[oB3 + j] = s;
  }
  for (int t = threadIdx.x; t < nb * kHid; t += blockDim.x) {
    const int b = t / kHid, k = t % kHid;
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < kOut; ++j)
      s = fmaf(p[oW3 + j * kHid + k], a.o[b][j], s);
    a.d2[b][k] = a.h2[b][k] > 0.f ? s : 0.f;
  }
  __syncthreads();
  // layer 2
  for (int t = threadIdx.x; t < kHid * kHid; t += blockDim.x) {
    const int j = t / kHid, k = t % kHid;
    float s = 0.f;
    for (int b = 0; b < nb; ++b)
      s = fmaf(a.d2[b][j], a.h1[b][k], s);
    g[oW2 + t] = s;
  }
  for (int j = threadIdx.x; j < kHid; j += blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < nb; ++b)
      s += a.d2[b][j];
    g[oB2 + j] = s;
  }
  for (int t = threadIdx.x; t < nb * kHid; t += blockDim.x) {
    const int b = t / kHid, k = t % kHid;
    float s = 0.f;
#pragma unroll 8
    for (int j = 0; j < kHid; ++j)
      s = fmaf(p[oW2 + j * kHid + k], a.d2[b][j], s);
    a.d1[b][k] = a.h1[b][k] > 0.f ? s : 0.f;
  }
  __syncthreads();
  // layer 1
  for (int t = threadIdx.x; t < kHid * kIn; t += blockDim.x) {
    const int j = t / kIn, k = t % kIn;
    float s = 0.f;
    for (int b = 0; b < nb; ++b)
      s = fmaf(a.d1[b][j], a.x[b][k], s);
    g[oW1 + t] = s;
  }
  for (int j = threadIdx.x; j < kHid; j += blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < nb; ++b)
      s += a.d1[b][j];
    g[oB1 + j] = s;
  }
  __syncthreads();
  return se * inv;
}

__device__ void load_rows(Act &a, const float *x, const float *y,
                          const float *m, const int *rows, int nb) {
  for (int t = threadIdx.x; t < nb * kIn; t += blockDim.x)
    a.x[t / kIn][t % kIn] = x[int64_t(rows[t / kIn]) * kIn + t % kIn];
  for (int t = threadIdx.x; t < nb * kOut; t += blockDim.x) {
    const int64_t r = rows[t / kOut];
    a.y[t / kOut][t % kOut] = y[r * kOut + t % kOut];
    a.m[t / kOut][t % kOut] = m ? m[r * kOut + t % kOut] : 1.f;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kThreads)
    k_mlp_train(float *params, const float *__restrict__ x,
                const float *__restrict__ y, const float *__restrict__ m,
                int n, int epochs, int batch, float lr, uint64_t seed,
                float *loss_out) {
  extern __shared__ float smem[];
  float *p = smem, *g = p + kP, *mo = g + kP, *ve = mo + kP;
  Act &a = *reinterpret_cast<Act *>(ve + kP);
  __shared__ int rows[kMaxBatch];
  float *gp = params + int64_t(blockIdx.x) * kP;
  for (int i = threadIdx.x; i < kP; i += blockDim.x) {
    p[i] = gp[i];
    mo[i] = 0.f;
    ve[i] = 0.f;
  }
  __syncthreads();
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float pw1 = 1.f, pw2 = 1.f;
  const int steps_per_epoch = (n + batch - 1) / batch;
  for (int e = 0; e < epochs; ++e) {
    float acc = 0.f;
    for (int s = 0; s < steps_per_epoch; ++s) {
      if (threadIdx.x < batch) {
        const uint64_t h = mix64(seed ^ (uint64_t(blockIdx.x) << 48) ^
                                 (uint64_t(e) << 32) ^
                                 (uint64_t(s) * kMaxBatch + threadIdx.x));
        rows[threadIdx.x] = int(h % uint64_t(n));
      }
      __syncthreads();
      load_rows(a, x, y, m, rows, batch);
      forward(p, a, batch);
      acc += backward(p, g, a, batch);
      pw1 *= b1;
      pw2 *= b2;
      const float c1 = 1.f / (1.f - pw1), c2 = 1.f / (1.f - pw2);
      for (int i = threadIdx.x; i < kP; i += blockDim.x) {
        const float gi = g[i];
        mo[i] = b1 * mo[i] + (1.f - b1) * gi;
        ve[i] = b2 * ve[i] + (1.f - b2) * gi * gi;
        p[i] -= lr * (mo[i] * c1) / (sqrtf(ve[i] * c2) + eps);
      }
      __syncthreads();
    }
    if (loss_out && threadIdx.x == 0)
      loss_out[int64_t(blockIdx.x) * epochs + e] = acc / steps_per_epoch;
  }
  for (int i = threadIdx.x; i < kP; i += blockDim.x)
    gp[i] = p[i];
}

// gradient of one member on rows [0, n) (n <= 64): the check against the
// CPU oracle
__global__ void __launch_bounds__(kThreads)
    k_mlp_grad(const float *params, const float *__restrict__ x,
               const float *__restrict__ y, const float *__restrict__ m, int n,
               float *grad, float *loss) {
  extern __shared__ float smem[];
  float *p = smem, *g = p + kP;
  Act &a = *reinterpret_cast<Act *>(g + kP);
  __shared__ int rows[kMaxBatch];
  for (int i = threadIdx.x; i < kP; i += blockDim.x)
    p[i] = params[i];
  if (threadIdx.x < n)
    rows[threadIdx.x] = threadIdx.x;
  __syncthreads();
  load_rows(a, x, y, m, rows, n);
  forward(p, a, n);
  const float l = backward(p, g, a, n);
  for (int i = threadIdx.x; i < kP; i += blockDim.x)
    grad[i] = g[i];
  if (threadIdx.x == 0 && loss)
    *loss = l;
}

// Batched inference: blockIdx.y picks the member, whose parameters are
// staged in shared memory; each thread evaluates one row.
__global__ void __launch_bounds__(128)
    k_mlp_predict(const float *__restrict__ params, const float *__restrict__ x,
                  int n, float *__restrict__ out) {
  __shared__ float p[kP];
  const float *gp = params + int64_t(blockIdx.y) * kP;
  for (int i = threadIdx.x; i < kP; i += blockDim.x)
    p[i] = gp[i];
  __syncthreads();
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += gridDim.x * blockDim.x) {
    float xi[kIn], h1[kHid], h2[kHid];
#pragma unroll
    for (int k = 0; k < kIn; ++k)
      xi[k] = x[int64_t(r) * kIn + k];
#pragma unroll 4
    for (int j = 0; j < kHid; ++j) {
      float s = p[oB1 + j];
#pragma unroll
      for (int k = 0; k < kIn; ++k)
        s = fmaf(p[oW1 + j * kIn + k], xi[k], s);
      h1[j] = fmaxf(s, 0.f);
    }
#pragma unroll 4
    for (int j = 0; j < kHid; ++j) {
      float s = p[oB2 + j];
#pragma unroll
      for (int k = 0; k < kHid; ++k)
        s = fmaf(p[oW2 + j * kHid + k], h1[k], s);
      h2[j] = fmaxf(s, 0.f);
    }
    float *o = out + (int64_t(blockIdx.y) * n + r) * kOut;
#pragma unroll
    for (int j = 0; j < kOut; ++j) {
      float s = p[oB3 + j];
#pragma unroll
      for (int k = 0; k < kHid; ++k)
        s = fmaf(p[oW3 + j * kHid + k], h2[k], s);
      o[j] = s;
    }
  }
}

static size_t train_smem() { return 4 * kP * sizeof(float) + sizeof(Act); }
static size_t grad_smem() { return 2 * kP * sizeof(float) + sizeof(Act); }

} // namespace tempi

using namespace tempi;

extern "C" int tempi_mlp_init(float *params, int members, uint64_t seed) {
  if (!params || members <= 0)
    return set_error(TEMPI_ERR_ARG, "bad arguments");
  // Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases, drawn
  // on the host from SplitMix64 and uploaded once.
  std::vector<float> h(size_t(members) * kP, 0.f);
  uint64_t st = seed;
  auto next = [&]() {
    uint64_t z = (st += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    return double(z >> 11) / double(1ull << 53);
  };
  for (int mbr = 0; mbr < members; ++mbr) {
    float *q = h.data() + size_t(mbr) * kP;
    auto fill = [&](int off, int nout, int nin) {
      const double r = 1.0 / std::sqrt(double(nin));
      for (int i = 0; i < nout * nin; ++i)
        q[off + i] = float((2.0 * next() - 1.0) * r);
    };
    fill(oW1, kHid, kIn);
    fill(oW2, kHid, kHid);
    fill(oW3, kOut, kHid);
  }
  cudaError_t e = copy_complete(params, h.data(), h.size() * sizeof(float));
  return e == cudaSuccess ? TEMPI_OK : cuda_error(e, "mlp init upload");
}

extern "C" int tempi_mlp_train(float *params, int members, const float *x,
                               const float *y, const float *mask, int n,
                               int epochs, int batch, float lr, uint64_t seed,
                               float *loss_out, void *stream) {
  if (!params || !x || !y || members <= 0 || n <= 0 || epochs <= 0 ||
      batch <= 0 || batch > kMaxBatch)
    return set_error(TEMPI_ERR_ARG, "bad training arguments");
  const size_t sm = train_smem();
  cudaError_t e = cudaFuncSetAttribute(
      k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
  if (e != cudaSuccess)
    return cuda_error(e, "mlp shared memory");
  k_mlp_train<<<members, kThreads, sm, static_cast<cudaStream_t>(stream)>>>(
      params, x, y, mask, n, epochs, batch, lr, seed, loss_out);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return cuda_error(e, "mlp train launch");
  counters().kernel_launches++;
  return TEMPI_OK;
}

extern "C" int tempi_mlp_grad(const float *params, const float *x,
                              const float *y, const float *mask, int n,
                              float *grad, float *loss, void *stream) {
  if (!params || !x || !y || !grad || n <= 0 || n > kMaxBatch)
    return set_error(TEMPI_ERR_ARG, "bad gradient arguments");
  const size_t sm = grad_smem();
  cudaError_t e = cudaFuncSetAttribute(
      k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
  if (e != cudaSuccess)
    return cuda_error(e, "mlp shared memory");
  k_mlp_grad<<<1, kThreads, sm, static_cast<cudaStream_t>(stream)>>>(
      params, x, y, mask, n, grad, loss);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return cuda_error(e, "mlp grad launch");
  counters().kernel_launches++;
  return TEMPI_OK;
}

extern "C" int tempi_mlp_predict(const float *params, int members,
                                 const float *x, int n, float *out,
                                 void *stream) {
  if (!params || !x || !out || members <= 0 || n < 0)
    return set_error(TEMPI_ERR_ARG, "bad inference arguments");
  if (n == 0)
    return TEMPI_OK;
  const int threads = 128;
  const int gx = std::min((n + threads - 1) / threads, 4 * num_sms());
  k_mlp_predict<<<dim3(gx, members), threads, 0,
                  static_cast<cudaStream_t>(stream)>>>(params, x, n, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return cuda_error(e, "mlp predict launch");
  counters().kernel_launches++;
  return TEMPI_OK;
}
