// nn_kernels.cu -- the small multilayer perceptron of the learned
// steady-state initial guess: forward, backward, loss and Adam, hand-written.
//
// Layer l: Z = X W^T + b, Y = tanh(Z) for hidden layers, Y = Z for the output
// layer.  X is B x in (row-major, FP32), W is out x in (row-major, BF16 for
// the forward / backward products, with an FP32 master copy updated by
// Adam), b is FP32.  Every product accumulates in FP32.  Sizes are small
// (B <= a few thousand, widths <= 256): one thread per output element, the
// reduction dimension in a loop; the weight-gradient reduction over the
// batch is a fixed-order loop, so training is deterministic.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/phi_b200.h"

namespace {

constexpr int kThreads = 256;

__global__ void linear_fwd_kernel(const float *__restrict__ X, const __nv_bfloat16 *__restrict__ W,
                                  const float *__restrict__ b, float *__restrict__ Y, int B, int in, int out,
                                  int act) {
  const long long idx = (long long)blockIdx.x * kThreads + threadIdx.x;
  if (idx >= (long long)B * out) return;
  const int r = (int)(idx / out), o = (int)(idx - (long long)r * out);
  const float *x = X + (long long)r * in;
  const __nv_bfloat16 *w = W + (long long)o * in;
  float z = b[o];
  for (int k = 0; k < in; ++k) z = fmaf(x[k], __bfloat162float(w[k]), z);
  Y[idx] = act ? tanhf(z) : z;
}

// dZ = dY * act'(Y) (tanh' = 1 - Y^2), written in place over dY.
__global__ void act_bwd_kernel(float *__restrict__ dY, const float *__restrict__ Y, long long n, int act) {
  const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
  if (i >= n || !act) return;
  const float y = Y[i];
  dY[i] *= 1.0f - y * y;
}

// dW[o, k] = sum_r dZ[r, o] X[r, k]; db[o] = sum_r dZ[r, o].
__global__ void linear_wgrad_kernel(const float *__restrict__ dZ, const float *__restrict__ X,
                                    float *__restrict__ dW, float *__restrict__ db, int B, int in, int out) {
  const long long idx = (long long)blockIdx.x * kThreads + threadIdx.x;
  const long long nw = (long long)out * in;
  if (idx < nw) {
    const int o = (int)(idx / in), k = (int)(idx - (long long)o * in);
    float s = 0.f;
    for (int r = 0; r < B; ++r) s = fmaf(dZ[(long long)r * out + o], X[(long long)r * in + k], s);
    dW[idx] = s;
  } else if (idx < nw + out) {
    const int o = (int)(idx - nw);
    float s = 0.f;
    for (int r = 0; r < B; ++r) s += dZ[(long long)r * out + o];
    db[o] = s;
  }
}

// dX[r, k] = sum_o dZ[r, o] W[o, k].
__global__ void linear_dgrad_kernel(const float *__restrict__ dZ, const __nv_bfloat16 *__restrict__ W,
                                    float *__restrict__ dX, int B, int in, int out) {
  const long long idx = (long long)blockIdx.x * kThreads + threadIdx.x;
  if (idx >= (long long)B * in) return;
  const int r = (int)(idx / in), k = (int)(idx - (long long)r * in);
  float s = 0.f;
  for (int o = 0; o < out; ++o) s = fmaf(dZ[(long long)r * out + o], __bfloat162float(W[(long long)o * in + k]), s);
  dX[idx] = s;
}

// loss = sum (P - T)^2 / B (one block, fixed-order reduction);
// dP = 2 (P - T) / B.
__global__ void mse_kernel(const float *__restrict__ P, const float *__restrict__ T, float *__restrict__ dP,
                           float *__restrict__ loss, long long n, int B) {
  __shared__ float sh[kThreads];
  float s = 0.f;
  const float inv = 1.0f / (float)B;
  for (long long i = threadIdx.x; i < n; i += kThreads) {
    const float d = P[i] - T[i];
    s = fmaf(d, d, s);
    dP[i] = 2.0f * d * inv;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = sh[0] * inv;
}

// Adam on the FP32 master weights; refreshes the BF16 copy.
__global__ void adam_kernel(float *__restrict__ w, __nv_bfloat16 *__restrict__ w16, const float *__restrict__ g,
                            float *__restrict__ m, float *__restrict__ v, long long n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (w16) w16[i] = __float2bfloat16_rn(wi);
}

__global__ void to_bf16_kernel(const float *__restrict__ a, __nv_bfloat16 *__restrict__ b, long long n) {
  const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
  if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}

unsigned blocks(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

int status(cudaError_t e) { return e == cudaSuccess ? PHI_OK : PHI_E_CUDA; }

bool bad_dims(int B, int in, int out) { return B <= 0 || in <= 0 || out <= 0; }

}  // namespace

extern "C" int phi_nn_linear_forward(const float *X, const void *W_bf16, const float *b, float *Y, int32_t B,
                                     int32_t in, int32_t out, int32_t act, void *stream) {
  if (!X || !W_bf16 || !b || !Y || bad_dims(B, in, out)) return PHI_E_INVALID;
  linear_fwd_kernel<<<blocks((long long)B * out), kThreads, 0, (cudaStream_t)stream>>>(
      X, static_cast<const __nv_bfloat16 *>(W_bf16), b, Y, B, in, out, act);
  return status(cudaGetLastError());
}

extern "C" int phi_nn_linear_backward(float *dY, const float *Y, const float *X, const void *W_bf16, float *dX,
                                      float *dW, float *db, int32_t B, int32_t in, int32_t out, int32_t act,
                                      void *stream) {
  if (!dY || !Y || !X || !W_bf16 || !dW || !db || bad_dims(B, in, out)) return PHI_E_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  act_bwd_kernel<<<blocks((long long)B * out), kThreads, 0, s>>>(dY, Y, (long long)B * out, act);
  linear_wgrad_kernel<<<blocks((long long)out * in + out), kThreads, 0, s>>>(dY, X, dW, db, B, in, out);
  if (dX)
    linear_dgrad_kernel<<<blocks((long long)B * in), kThreads, 0, s>>>(
        dY, static_cast<const __nv_bfloat16 *>(W_bf16), dX, B, in, out);
  return status(cudaGetLastError());
}

extern "C" int phi_nn_mse(const float *P, const float *T, float *dP, float *loss, int64_t n, int32_t B,
                          void *stream) {
  if (!P || !T || !dP || !loss || n <= 0 || B <= 0) return PHI_E_INVALID;
  mse_kernel<<<1, kThreads, 0, (cudaStream_t)stream>>>(P, T, dP, loss, n, B);
  return status(cudaGetLastError());
}

extern "C" int phi_nn_adam(float *w, void *w_bf16, const float *g, float *m, float *v, int64_t n, float lr,
                           float beta1, float beta2, float eps, int32_t step, void *stream) {
  if (!w || !g || !m || !v || n <= 0 || step < 1) return PHI_E_INVALID;
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  adam_kernel<<<blocks(n), kThreads, 0, (cudaStream_t)stream>>>(w, static_cast<__nv_bfloat16 *>(w_bf16), g, m, v,
                                                               n, lr, beta1, beta2, eps, c1, c2);
  return status(cudaGetLastError());
}

extern "C" int phi_nn_to_bf16(const float *a, void *b, int64_t n, void *stream) {
  if (!a || !b || n <= 0) return PHI_E_INVALID;
  to_bf16_kernel<<<blocks(n), kThreads, 0, (cudaStream_t)stream>>>(a, static_cast<__nv_bfloat16 *>(b), n);
  return status(cudaGetLastError());
}
