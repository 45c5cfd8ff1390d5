// Learned Davidson preconditioner: a 3-layer MLP (BF16 weights, FP32 accumulation)
// with hand-written forward, backward and Adam kernels, plus the kernels that
// build its per-block input features and apply its output to a residual.
//
// There is no counterpart in the reference: it replaces the diagonal (Jacobi)
// preconditioner of pdvdson (source/tools/pdvdson.py:275-278,
// r / (|diag - e| + 1e-4)) by  c_i = r_i * alpha_b / (|diag_i - e| + sigma_b),
// where (log alpha_b, log sigma_b) are the network's outputs for the symmetry
// block b that element i belongs to.  With alpha_b = 1, sigma_b = 1e-4 it is
// exactly the reference's preconditioner (the fallback).
//
// Network: h1 = relu(W1 x + b1), h2 = relu(W2 h1 + b2), y = W3 h2 + b3,
// x in R^F (F <= 32), hidden width H = 256, y in R^2.  One thread block per
// 32 rows; weights are read as BF16 and every product is accumulated in FP32.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdio>
#include "qc_types.h"

namespace {

constexpr int H = 256;
constexpr int ROWS = 32;     // rows (blocks) per CTA, forward
constexpr int ROWS_B = 16;   // rows per CTA, backward (two [rows x H] tiles in shared memory)
constexpr int MAXF = 32;

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

// Forward: X [B, F] -> Y [B, 2]; saves H1, H2 (post-activation) for the backward pass.
__global__ void __launch_bounds__(H) k_mlp_fwd(int B, int F, const float *__restrict__ X,
                                               const __nv_bfloat16 *__restrict__ W1, const float *__restrict__ b1,
                                               const __nv_bfloat16 *__restrict__ W2, const float *__restrict__ b2,
                                               const __nv_bfloat16 *__restrict__ W3, const float *__restrict__ b3,
                                               float *__restrict__ H1, float *__restrict__ H2, float *__restrict__ Y) {
  __shared__ float xs[ROWS][MAXF];
  __shared__ float hs[ROWS][H + 1];
  const int r0 = blockIdx.x * ROWS;
  const int j = threadIdx.x;                       // hidden unit
  for (int i = j; i < ROWS * F; i += H) {
    const int r = i / F, f = i % F;
    xs[r][f] = (r0 + r < B) ? X[(long long)(r0 + r) * F + f] : 0.f;
  }
  __syncthreads();
  // layer 1: W1 is [H, F]
  float w[MAXF];
  for (int f = 0; f < F; ++f) w[f] = bf(W1[j * F + f]);
  for (int r = 0; r < ROWS; ++r) {
    float a = b1[j];
    for (int f = 0; f < F; ++f) a = fmaf(w[f], xs[r][f], a);
    a = fmaxf(a, 0.f);
    hs[r][j] = a;
    if (r0 + r < B) H1[(long long)(r0 + r) * H + j] = a;
  }
  __syncthreads();
  // layer 2: W2 is [H, H]
  float acc[ROWS];
  for (int r = 0; r < ROWS; ++r) acc[r] = b2[j];
  for (int k = 0; k < H; ++k) {
    const float wk = bf(W2[j * H + k]);
#pragma unroll
    for (int r = 0; r < ROWS; ++r) acc[r] = fmaf(wk, hs[r][k], acc[r]);
  }
  __syncthreads();
  for (int r = 0; r < ROWS; ++r) {
    const float a = fmaxf(acc[r], 0.f);
    hs[r][j] = a;
    if (r0 + r < B) H2[(long long)(r0 + r) * H + j] = a;
  }
  __syncthreads();
  // layer 3: W3 is [2, H]; warp w < 2 reduces output w for all rows
  const int warp = j >> 5, lane = j & 31;
  if (warp < 2) {
    for (int r = 0; r < ROWS; ++r) {
      float a = 0.f;
      for (int k = lane; k < H; k += 32) a = fmaf(bf(W3[warp * H + k]), hs[r][k], a);
      for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
      if (lane == 0 && r0 + r < B) Y[(long long)(r0 + r) * 2 + warp] = a + b3[warp];
    }
  }
}

// Backward: given dY [B, 2] accumulate dW1 [H,F], db1, dW2 [H,H], db2, dW3 [2,H], db3 (FP32, atomics per CTA).
__global__ void __launch_bounds__(H) k_mlp_bwd(int B, int F, const float *__restrict__ X,
                                               const __nv_bfloat16 *__restrict__ W2,
                                               const __nv_bfloat16 *__restrict__ W3,
                                               const float *__restrict__ H1, const float *__restrict__ H2,
                                               const float *__restrict__ dY, float *__restrict__ dW1,
                                               float *__restrict__ db1, float *__restrict__ dW2,
                                               float *__restrict__ db2, float *__restrict__ dW3,
                                               float *__restrict__ db3) {
  constexpr int ROWS = ROWS_B;
  __shared__ float g2[ROWS][H + 1];   // dL/d(pre-activation of layer 2)
  __shared__ float h1s[ROWS][H + 1];
  __shared__ float dys[ROWS][2];
  const int r0 = blockIdx.x * ROWS;
  const int j = threadIdx.x;
  const int nr = min(ROWS, B - r0);
  for (int r = 0; r < ROWS; ++r) {
    const bool ok = r < nr;
    if (j < 2) dys[r][j] = ok ? dY[(long long)(r0 + r) * 2 + j] : 0.f;
    h1s[r][j] = ok ? H1[(long long)(r0 + r) * H + j] : 0.f;
  }
  __syncthreads();
  // layer 3 grads and g2 = (W3^T dy) * relu'(h2)
  float dw3a = 0.f, dw3b = 0.f;
  const float w3a = bf(W3[j]), w3b = bf(W3[H + j]);
  for (int r = 0; r < nr; ++r) {
    const float h2 = H2[(long long)(r0 + r) * H + j];
    dw3a = fmaf(dys[r][0], h2, dw3a);
    dw3b = fmaf(dys[r][1], h2, dw3b);
    const float g = (h2 > 0.f) ? (w3a * dys[r][0] + w3b * dys[r][1]) : 0.f;
    g2[r][j] = g;
  }
  for (int r = nr; r < ROWS; ++r) g2[r][j] = 0.f;
  atomicAdd(&dW3[j], dw3a);
  atomicAdd(&dW3[H + j], dw3b);
  if (j < 2) {
    float s = 0.f;
    for (int r = 0; r < nr; ++r) s += dys[r][j];
    atomicAdd(&db3[j], s);
  }
  __syncthreads();
  // layer 2 grads: dW2[j, k] += sum_r g2[r][j] * h1[r][k]; db2[j] += sum_r g2[r][j]
  {
    float s = 0.f;
    for (int r = 0; r < nr; ++r) s += g2[r][j];
    atomicAdd(&db2[j], s);
  }
  for (int k = 0; k < H; ++k) {
    float s = 0.f;
    for (int r = 0; r < nr; ++r) s = fmaf(g2[r][j], h1s[r][k], s);
    atomicAdd(&dW2[j * H + k], s);
  }
  // g1 = (W2^T g2) * relu'(h1): unit j of layer 1 sums over the layer-2 units
  float g1[ROWS];
  for (int r = 0; r < ROWS; ++r) g1[r] = 0.f;
  for (int k = 0; k < H; ++k) {
    const float wkj = bf(W2[k * H + j]);
#pragma unroll
    for (int r = 0; r < ROWS; ++r) g1[r] = fmaf(wkj, g2[r][k], g1[r]);
  }
  float sb1 = 0.f;
  for (int r = 0; r < nr; ++r) {
    if (h1s[r][j] <= 0.f) g1[r] = 0.f;
    sb1 += g1[r];
  }
  atomicAdd(&db1[j], sb1);
  for (int f = 0; f < F; ++f) {
    float s = 0.f;
    for (int r = 0; r < nr; ++r) s = fmaf(g1[r], X[(long long)(r0 + r) * F + f], s);
    atomicAdd(&dW1[j * F + f], s);
  }
}

// Adam step on FP32 master weights; the BF16 copy used by the kernels is refreshed.
__global__ void k_adam(int n, float *__restrict__ w, __nv_bfloat16 *__restrict__ wb, const float *__restrict__ g,
                       float *__restrict__ m, float *__restrict__ v, float lr, float b1, float b2, float eps,
                       float c1, float c2, float scale) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i] * scale;
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
  }
}

// Apply: c_i = r_i * alpha_b / (|d_i - e| + sigma_b),  (log alpha_b, log sigma_b) = Y[b].
__global__ void k_precond_apply(long long n, const double *__restrict__ r, const double *__restrict__ d, double e,
                                const int *__restrict__ blk, const float *__restrict__ Y, double *__restrict__ c) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int b = blk[i];
    // log alpha and log sigma are clamped to [-30, 30] (the range the training uses)
    const double alpha = exp(fmin(fmax((double)Y[2 * b], -30.0), 30.0));
    const double sigma = exp(fmin(fmax((double)Y[2 * b + 1], -30.0), 30.0));
    c[i] = r[i] * alpha / (fabs(d[i] - e) + sigma);
  }
}

}  // namespace

static int fail(const char *w) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return QC_OK;
  fprintf(stderr, "[qcgpu] %s: %s\n", w, cudaGetErrorString(e));
  return QC_ERR_CUDA;
}

extern "C" int qc_mlp_forward(int B, int F, const float *X, const void *W1, const float *b1, const void *W2,
                              const float *b2, const void *W3, const float *b3, float *H1, float *H2, float *Y,
                              void *stream) {
  if (B <= 0) return QC_OK;
  if (F < 1 || F > MAXF) return QC_ERR_ARG;
  k_mlp_fwd<<<(B + ROWS - 1) / ROWS, H, 0, (cudaStream_t)stream>>>(
      B, F, X, (const __nv_bfloat16 *)W1, b1, (const __nv_bfloat16 *)W2, b2, (const __nv_bfloat16 *)W3, b3, H1, H2,
      Y);
  return fail("qc_mlp_forward");
}

extern "C" int qc_mlp_backward(int B, int F, const float *X, const void *W2, const void *W3, const float *H1,
                               const float *H2, const float *dY, float *dW1, float *db1, float *dW2, float *db2,
                               float *dW3, float *db3, void *stream) {
  if (B <= 0) return QC_OK;
  if (F < 1 || F > MAXF) return QC_ERR_ARG;
  k_mlp_bwd<<<(B + ROWS_B - 1) / ROWS_B, H, 0, (cudaStream_t)stream>>>(
      B, F, X, (const __nv_bfloat16 *)W2, (const __nv_bfloat16 *)W3, H1, H2, dY, dW1, db1, dW2, db2, dW3, db3);
  return fail("qc_mlp_backward");
}

extern "C" int qc_adam_step(int n, float *w, void *wbf16, const float *g, float *m, float *v, float lr, float beta1,
                            float beta2, float eps, int step, float grad_scale, void *stream) {
  if (n <= 0) return QC_OK;
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  k_adam<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, w, (__nv_bfloat16 *)wbf16, g, m, v, lr, beta1, beta2,
                                                            1e-8f, c1, c2, grad_scale);
  return fail("qc_adam_step");
}

extern "C" int qc_precond_apply(long long n, const double *r, const double *d, double e, const int *blk,
                                const float *Y, double *c, void *stream) {
  if (n <= 0) return QC_OK;
  long long g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  k_precond_apply<<<(unsigned)g, 256, 0, (cudaStream_t)stream>>>(n, r, d, e, blk, Y, c);
  return fail("qc_precond_apply");
}
