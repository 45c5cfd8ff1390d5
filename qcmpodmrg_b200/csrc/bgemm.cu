// Grouped block GEMM over block-pair work lists (FP64 / FP32, CUDA cores), the
// GPU integer block-mask kernel, and small gather/scatter/convert kernels.
//
// One CTA owns one output tile (qc_task) and accumulates, in registers, every
// block-pair product (qc_contrib) that lands on its output block; the tile is
// written once.  This executes one whole stage of the reference's operator
// loop -- tensordotCAL (source/qtensor/qtensor.py:642-659) for every operator
// and every symmetry block pair -- in a single launch with no atomics, so the
// summation order is fixed and runs are bitwise reproducible.
#include <cuda_runtime.h>
#include <cstdio>
#include <string>
#include "qc_types.h"

extern "C" const char *qc_last_error(void);
static thread_local std::string g_cuerr;
static int cuda_fail(const char *where) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return QC_OK;
  g_cuerr = std::string(where) + ": " + cudaGetErrorString(e);
  fprintf(stderr, "[qcgpu] %s\n", g_cuerr.c_str());
  return QC_ERR_CUDA;
}
extern "C" const char *qc_last_cuda_error(void) { return g_cuerr.c_str(); }

namespace {

// SUMMED = false: the task computes one tile for each operator in [t.op_b, t.op_e)
//                 of the operator table (same block structure, own base offsets).
// SUMMED = true:  the task computes one tile; every contribution accumulates the
//                 products of the operators in [c.op_b, c.op_e) (sum over p).
template <typename T, int TM, int TN, int TK, int RM, int RN, bool SUMMED, int kThreads>
__global__ void __launch_bounds__(kThreads)
k_bgemm(const qc_task *__restrict__ tasks, const qc_contrib *__restrict__ contribs,
        const qc_op *__restrict__ ops, const T *__restrict__ A, const T *__restrict__ B, T *__restrict__ C) {
  constexpr int TX = TN / RN;
  constexpr int TY = TM / RM;
  static_assert(TX * TY == kThreads, "thread tile");
  __shared__ T As[TK][TM + 1];
  __shared__ T Bs[TK][TN + 1];
  __shared__ int arow[TM];
  __shared__ int bcol[TN];
  __shared__ int akoff[TK];
  __shared__ int bkoff[TK];

  const qc_task t = tasks[blockIdx.x];
  // per-operator mode: blockIdx.y selects the operator of the task's range
  if (!SUMMED && t.op_b + (int)blockIdx.y >= t.op_e) return;
  const int tid = threadIdx.x;
  const int tx = tid % TX, ty = tid / TX;
  {
    const int oi = SUMMED ? 0 : (int)blockIdx.y;
    T acc[RM][RN];
#pragma unroll
    for (int i = 0; i < RM; ++i)
#pragma unroll
      for (int j = 0; j < RN; ++j) acc[i][j] = T(0);

    for (int ci = t.cb; ci < t.ce; ++ci) {
      const qc_contrib c = contribs[ci];
      __syncthreads();
      for (int i = tid; i < TM; i += kThreads) {
        const int m = t.m0 + i;
        arow[i] = (m < t.M) ? (m / t.mlo) * c.a_mh + (m % t.mlo) * c.a_ml : -1;
      }
      for (int j = tid; j < TN; j += kThreads) {
        const int n = t.n0 + j;
        bcol[j] = (n < t.N) ? (n / t.nlo) * c.b_nh + (n % t.nlo) * c.b_nl : -1;
      }
      const bool a_kfast = (c.a_kl == 1);
      const bool b_nfast = (c.b_nl == 1);
      const int opb = SUMMED ? c.op_b : t.op_b + oi;
      const int ope = SUMMED ? c.op_e : opb + 1;
      for (int op = opb; op < ope; ++op) {
        const qc_op o = ops[op];
        const T alpha = T(o.alpha * c.alpha);
        const T *Ab = A + o.a_base + c.a_off;
        const T *Bb = B + o.b_base + c.b_off;
        for (int k0 = 0; k0 < c.K; k0 += TK) {
          __syncthreads();
          if (tid < TK) {
            const int k = k0 + tid;
            akoff[tid] = (k < c.K) ? (k / c.klo) * c.a_kh + (k % c.klo) * c.a_kl : -1;
            bkoff[tid] = (k < c.K) ? (k / c.klo) * c.b_kh + (k % c.klo) * c.b_kl : -1;
          }
          __syncthreads();
          for (int idx = tid; idx < TM * TK; idx += kThreads) {
            int i, kk;
            if (a_kfast) { kk = idx % TK; i = idx / TK; } else { i = idx % TM; kk = idx / TM; }
            const int ro = arow[i], ko = akoff[kk];
            As[kk][i] = (ro >= 0 && ko >= 0) ? Ab[ro + ko] * alpha : T(0);
          }
          for (int idx = tid; idx < TK * TN; idx += kThreads) {
            int j, kk;
            if (b_nfast) { j = idx % TN; kk = idx / TN; } else { kk = idx % TK; j = idx / TK; }
            const int co = bcol[j], ko = bkoff[kk];
            Bs[kk][j] = (co >= 0 && ko >= 0) ? Bb[ko + co] : T(0);
          }
          __syncthreads();
#pragma unroll
          for (int kk = 0; kk < TK; ++kk) {
            T a[RM], b[RN];
#pragma unroll
            for (int i = 0; i < RM; ++i) a[i] = As[kk][ty + i * TY];
#pragma unroll
            for (int j = 0; j < RN; ++j) b[j] = Bs[kk][tx + j * TX];
#pragma unroll
            for (int i = 0; i < RM; ++i)
#pragma unroll
              for (int j = 0; j < RN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
          }
        }
      }
    }
    T *Cb = C + t.c_off + (SUMMED ? 0 : ops[t.op_b + oi].c_base);
#pragma unroll
    for (int i = 0; i < RM; ++i) {
      const int m = t.m0 + ty + i * TY;
      if (m >= t.M) continue;
      const long long rowoff = (long long)(m / t.mlo) * t.c_mh + (long long)(m % t.mlo) * t.c_ml;
#pragma unroll
      for (int j = 0; j < RN; ++j) {
        const int n = t.n0 + tx + j * TX;
        if (n >= t.N) continue;
        Cb[rowoff + (long long)(n / t.nlo) * t.c_nh + (long long)(n % t.nlo) * t.c_nl] = acc[i][j];
      }
    }
  }
}

template <typename T, bool S>
int launch_mode(const qc_task *tk, long long ntasks, int opspan, const qc_contrib *cb, const qc_op *ops,
                const T *A, const T *B, T *C, int cfg, cudaStream_t s) {
  dim3 grid((unsigned)ntasks, S ? 1u : (unsigned)opspan);
  switch (cfg) {
    case 0: k_bgemm<T, 64, 64, 16, 4, 4, S, 256><<<grid, 256, 0, s>>>(tk, cb, ops, A, B, C); break;
    case 1: k_bgemm<T, 128, 32, 16, 4, 4, S, 256><<<grid, 256, 0, s>>>(tk, cb, ops, A, B, C); break;
    case 2: k_bgemm<T, 256, 16, 16, 4, 4, S, 256><<<grid, 256, 0, s>>>(tk, cb, ops, A, B, C); break;
    case 3: k_bgemm<T, 32, 32, 16, 4, 4, S, 64><<<grid, 64, 0, s>>>(tk, cb, ops, A, B, C); break;
    case 4: k_bgemm<T, 64, 16, 16, 4, 4, S, 64><<<grid, 64, 0, s>>>(tk, cb, ops, A, B, C); break;
    case 5: k_bgemm<T, 128, 64, 16, 8, 4, S, 256><<<grid, 256, 0, s>>>(tk, cb, ops, A, B, C); break;
    default: return QC_ERR_ARG;
  }
  return cuda_fail("qc_bgemm");
}

template <typename T>
int launch_bgemm(const void *tasks, long long ntasks, int opspan, const void *contribs, const void *ops,
                 int summed, const T *A, const T *B, T *C, int cfg, cudaStream_t s) {
  if (ntasks <= 0) return QC_OK;
  if (ntasks > 0x7fffffffLL || opspan < 1 || opspan > 65535) return QC_ERR_ARG;
  const qc_task *tk = (const qc_task *)tasks;
  const qc_contrib *cb = (const qc_contrib *)contribs;
  const qc_op *op = (const qc_op *)ops;
  return summed ? launch_mode<T, true>(tk, ntasks, 1, cb, op, A, B, C, cfg, s)
                : launch_mode<T, false>(tk, ntasks, opspan, cb, op, A, B, C, cfg, s);
}

struct SymArgs {
  int rank, nqnum;
  int nsyms[8];
  int status[8];
  int first[9];
  long long nblks;
};

__global__ void k_sym_allowed(SymArgs a, const int *__restrict__ q2, int *__restrict__ allowed) {
  const long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (b >= a.nblks) return;
  long long rem = b;
  int acc[4] = {0, 0, 0, 0};
  for (int r = a.rank - 1; r >= 0; --r) {
    const int i = (int)(rem % a.nsyms[r]);
    rem /= a.nsyms[r];
    const int *q = q2 + (long long)(a.first[r] + i) * a.nqnum;
    const int s = a.status[r] ? -1 : 1;
    for (int k = 0; k < a.nqnum; ++k) acc[k] += s * q[k];
  }
  int ok = 1;
  for (int k = 0; k < a.nqnum; ++k) ok &= (acc[k] == 0);
  allowed[b] = ok;
}

__global__ void k_gather_f64(const double *__restrict__ src, const long long *__restrict__ idx,
                             double *__restrict__ dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = src[idx[i]];
}
__global__ void k_scatter_f64(const double *__restrict__ src, const long long *__restrict__ idx,
                              double *__restrict__ dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[idx[i]] = src[i];
}
__global__ void k_f64_to_f32(const double *__restrict__ s, float *__restrict__ d, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    d[i] = (float)s[i];
}
__global__ void k_f32_to_f64(const float *__restrict__ s, double *__restrict__ d, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    d[i] = (double)s[i];
}

template <typename T>
__global__ void k_reduce_ops(const T *__restrict__ part, int nops, long long n, T *__restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    T acc = T(0);
    for (int o = 0; o < nops; ++o) acc += part[(long long)o * n + i];   // fixed order: reproducible
    out[i] = acc;
  }
}

inline unsigned grid_for(long long n) {
  long long g = (n + 255) / 256;
  if (g > 148LL * 32) g = 148LL * 32;   // a multiple of the 148 SMs
  return (unsigned)(g < 1 ? 1 : g);
}

}  // namespace

// Internal launchers shared with sigma_noalloc.cu (not part of the C ABI).
__attribute__((visibility("hidden"))) int qc_internal_bgemm_f64(const void *tasks, long long ntasks, int opspan,
                                                                const void *contribs, const void *ops, int summed,
                                                                const double *A, const double *B, double *C,
                                                                int cfg, cudaStream_t s) {
  return launch_bgemm<double>(tasks, ntasks, opspan, contribs, ops, summed, A, B, C, cfg, s);
}

__attribute__((visibility("hidden"))) int qc_internal_reduce_f64(const double *part, int nops, long long n,
                                                                 double *out, cudaStream_t s) {
  if (n <= 0) return QC_OK;
  k_reduce_ops<double><<<grid_for(n), 256, 0, s>>>(part, nops, n, out);
  return cuda_fail("qc_internal_reduce_f64");
}

extern "C" int qc_bgemm_f64(const void *tasks, long long ntasks, int opspan, const void *contribs, const void *ops,
                            int summed, const double *A, const double *B, double *C, int cfg, void *stream) {
  return launch_bgemm<double>(tasks, ntasks, opspan, contribs, ops, summed, A, B, C, cfg, (cudaStream_t)stream);
}

extern "C" int qc_bgemm_f32(const void *tasks, long long ntasks, int opspan, const void *contribs, const void *ops,
                            int summed, const float *A, const float *B, float *C, int cfg, void *stream) {
  return launch_bgemm<float>(tasks, ntasks, opspan, contribs, ops, summed, A, B, C, cfg, (cudaStream_t)stream);
}

extern "C" int qc_sym_allowed_gpu(int rank, int nqnum, const int *nsyms, const int *status, const int *q2,
                                  int *allowed, void *stream) {
  if (rank < 1 || rank > 8 || nqnum < 1 || nqnum > 4) return QC_ERR_ARG;
  SymArgs a;
  a.rank = rank;
  a.nqnum = nqnum;
  a.first[0] = 0;
  a.nblks = 1;
  for (int r = 0; r < rank; ++r) {
    if (nsyms[r] <= 0) return QC_ERR_ARG;
    a.nsyms[r] = nsyms[r];
    a.status[r] = status[r] ? 1 : 0;
    a.first[r + 1] = a.first[r] + nsyms[r];
    a.nblks *= nsyms[r];
  }
  const long long g = (a.nblks + 255) / 256;
  k_sym_allowed<<<(unsigned)g, 256, 0, (cudaStream_t)stream>>>(a, q2, allowed);
  return cuda_fail("qc_sym_allowed_gpu");
}

extern "C" int qc_gather_f64(const double *src, const long long *idx, double *dst, long long n, void *stream) {
  if (n <= 0) return QC_OK;
  k_gather_f64<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(src, idx, dst, n);
  return cuda_fail("qc_gather_f64");
}

extern "C" int qc_scatter_f64(const double *src, const long long *idx, double *dst, long long n, long long ndst,
                              void *stream) {
  if (ndst > 0) cudaMemsetAsync(dst, 0, sizeof(double) * ndst, (cudaStream_t)stream);
  if (n <= 0) return cuda_fail("qc_scatter_f64");
  k_scatter_f64<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(src, idx, dst, n);
  return cuda_fail("qc_scatter_f64");
}

extern "C" int qc_reduce_ops_f64(const double *part, int nops, long long n, double *out, void *stream) {
  if (n <= 0) return QC_OK;
  k_reduce_ops<double><<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(part, nops, n, out);
  return cuda_fail("qc_reduce_ops_f64");
}

extern "C" int qc_reduce_ops_f32(const float *part, int nops, long long n, float *out, void *stream) {
  if (n <= 0) return QC_OK;
  k_reduce_ops<float><<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(part, nops, n, out);
  return cuda_fail("qc_reduce_ops_f32");
}

extern "C" int qc_convert_f64_to_f32(const double *s, float *d, long long n, void *stream) {
  if (n <= 0) return QC_OK;
  k_f64_to_f32<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(s, d, n);
  return cuda_fail("qc_convert_f64_to_f32");
}

extern "C" int qc_convert_f32_to_f64(const float *s, double *d, long long n, void *stream) {
  if (n <= 0) return QC_OK;
  k_f32_to_f64<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(s, d, n);
  return cuda_fail("qc_convert_f32_to_f64");
}
