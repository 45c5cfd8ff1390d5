// Dense panel GEMM (FP64 DFMA / FP32 FFMA) for contractions laid out as panels.
//
// The L.psi contraction of HVecQt (source/mpo_dmrg_kernelQt.py:301, top1 =
// tensordot(L, psi, axes=([2],[0]))) pairs every L block (a, l, l') with every
// psi block (l', n1, n2, r) of the same sector l'.  With the L blocks of one
// sector stacked into a row-major panel [M x K] (a per-dot permutation), each
// psi block is the row-major [K x N] operand of one dense GEMM whose [M x N]
// result is a run of T1 blocks.  No index maps are needed: the kernel is a plain
// tiled GEMM with a register-prefetch software pipeline (the next K-slice is
// loaded from global memory while the current one is multiplied out of shared
// memory) and one barrier per K-slice.
#include <cuda_runtime.h>
#include <cstdio>
#include "qc_types.h"

namespace {

template <typename T, int TM, int TN, int TK, int RM, int RN, int NT>
__global__ void __launch_bounds__(NT, 2)
k_pgemm(const qc_ptask *__restrict__ tasks, const qc_op *__restrict__ ops, const long long *__restrict__ crow,
        const T *__restrict__ A, const T *__restrict__ B, T *__restrict__ C) {
  constexpr int TX = TN / RN, TY = TM / RM;
  static_assert(TX * TY == NT, "thread tile");
  constexpr int LA = (TM * TK + NT - 1) / NT;       // A elements per thread per K-slice
  constexpr int LB = (TK * TN + NT - 1) / NT;
  __shared__ T As[2][TK][TM + 1];
  __shared__ T Bs[2][TK][TN + 1];

  const qc_ptask t = tasks[blockIdx.x];
  const int op = t.op_b + (int)blockIdx.y;
  if (op >= t.op_e) return;
  const qc_op o = ops[op];
  const T *Ab = A + o.a_base + t.a_off;
  const T *Bb = B + o.b_base + t.b_off;
  const T alpha = T(o.alpha);
  const int tid = threadIdx.x;
  const int tx = tid % TX, ty = tid / TX;
  const int M = t.M, N = t.N, K = t.K;
  const long long lda = t.lda > 0 ? t.lda : K;

  T ra[LA], rb[LB];
  auto load = [&](int k0) {
#pragma unroll
    for (int e = 0; e < LA; ++e) {       // A: TK consecutive k of one row per TK threads
      const int idx = tid + e * NT;
      const int kk = idx % TK, i = idx / TK;
      const int m = t.m0 + i, k = k0 + kk;
      ra[e] = (idx < TM * TK && m < M && k < K) ? Ab[(long long)m * lda + k] : T(0);
    }
#pragma unroll
    for (int e = 0; e < LB; ++e) {       // B: consecutive n of one k row
      const int idx = tid + e * NT;
      const int j = idx % TN, kk = idx / TN;
      const int n = t.n0 + j, k = k0 + kk;
      rb[e] = (idx < TK * TN && n < N && k < K) ? Bb[(long long)k * N + n] : T(0);
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int e = 0; e < LA; ++e) {
      const int idx = tid + e * NT;
      if (idx < TM * TK) As[buf][idx % TK][idx / TK] = ra[e];
    }
#pragma unroll
    for (int e = 0; e < LB; ++e) {
      const int idx = tid + e * NT;
      if (idx < TK * TN) Bs[buf][idx / TN][idx % TN] = rb[e];
    }
  };

  T acc[RM][RN];
#pragma unroll
  for (int i = 0; i < RM; ++i)
#pragma unroll
    for (int j = 0; j < RN; ++j) acc[i][j] = T(0);

  const int nsteps = (K + TK - 1) / TK;
  load(0);
  for (int s = 0; s < nsteps; ++s) {
    const int buf = s & 1;
    store(buf);
    __syncthreads();
    if (s + 1 < nsteps) load((s + 1) * TK);
#pragma unroll
    for (int kk = 0; kk < TK; ++kk) {
      T av[RM], bv[RN];
#pragma unroll
      for (int i = 0; i < RM; ++i) av[i] = As[buf][kk][ty + i * TY];
#pragma unroll
      for (int j = 0; j < RN; ++j) bv[j] = Bs[buf][kk][tx + j * TX];
#pragma unroll
      for (int i = 0; i < RM; ++i)
#pragma unroll
        for (int j = 0; j < RN; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
  }
  T *Cb = C + o.c_base;
#pragma unroll
  for (int i = 0; i < RM; ++i) {
    const int m = t.m0 + ty + i * TY;
    if (m >= M) continue;
    const long long row = (t.crow >= 0) ? crow[t.crow + m] : t.c_off + (long long)m * N;
#pragma unroll
    for (int j = 0; j < RN; ++j) {
      const int n = t.n0 + tx + j * TX;
      if (n < N) Cb[row + n] = alpha * acc[i][j];
    }
  }
}

template <typename T>
int launch_pgemm(const void *tasks, long long ntasks, int opspan, const void *ops, const long long *crow, const T *A,
                 const T *B, T *C, int cfg, cudaStream_t s) {
  if (ntasks <= 0) return QC_OK;
  if (ntasks > 0x7fffffffLL || opspan < 1 || opspan > 65535) return QC_ERR_ARG;
  dim3 grid((unsigned)ntasks, (unsigned)opspan);
  const qc_ptask *tk = (const qc_ptask *)tasks;
  const qc_op *op = (const qc_op *)ops;
  constexpr int KT = (sizeof(T) == 8) ? 8 : 16;
  switch (cfg) {
    case 0: k_pgemm<T, 128, 64, KT, 8, 4, 256><<<grid, 256, 0, s>>>(tk, op, crow, A, B, C); break;   // N > 32
    case 1: k_pgemm<T, 128, 32, KT, 8, 2, 256><<<grid, 256, 0, s>>>(tk, op, crow, A, B, C); break;   // 16 < N <= 32
    case 2: k_pgemm<T, 128, 16, KT, 4, 2, 256><<<grid, 256, 0, s>>>(tk, op, crow, A, B, C); break;   // N <= 16
    default: return QC_ERR_ARG;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "[qcgpu] qc_pgemm: %s\n", cudaGetErrorString(e));
    return QC_ERR_CUDA;
  }
  return QC_OK;
}

}  // namespace

extern "C" int qc_pgemm_f64(const void *tasks, long long ntasks, int opspan, const void *ops, const long long *crow,
                            const double *A, const double *B, double *C, int cfg, void *stream) {
  return launch_pgemm<double>(tasks, ntasks, opspan, ops, crow, A, B, C, cfg, (cudaStream_t)stream);
}

extern "C" int qc_pgemm_f32(const void *tasks, long long ntasks, int opspan, const void *ops, const long long *crow,
                            const float *A, const float *B, float *C, int cfg, void *stream) {
  return launch_pgemm<float>(tasks, ntasks, opspan, ops, crow, A, B, C, cfg, (cudaStream_t)stream);
}
