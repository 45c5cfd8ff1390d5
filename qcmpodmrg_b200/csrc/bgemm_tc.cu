// Grouped block GEMM on the 5th-generation tensor cores (tcgen05.mma kind::tf32).
//
// Same work items as k_bgemm (qc_task / qc_contrib / qc_op, per-operator mode):
// one CTA = one 128 x 64 output tile of one operator.  For every block pair of
// the tile and every 32-wide slice of its contraction, the 128 threads gather
// the A (128 x 32) and B (32 x 64) slices from the packed blocks (two-level
// index maps, alpha folded into A), round them to TF32 and store them in shared
// memory in the canonical K-major, no-swizzle UMMA layout (8-row x 16-byte core
// matrices).  One thread issues four tcgen05.mma (K = 8 each) that accumulate
// into a 128 x 64 FP32 tile in tensor memory, and commits them to an mbarrier.
// The epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM lanes
// 32w..32w+31) and writes the output block.
//
// Operands cannot be fetched with TMA: each block pair has its own strides and
// two-level index maps (the reference's tensordot axis permutations), so the
// gather is done by the threads.  Every wait is bounded; on expiry the kernel
// raises *err, stops issuing work and still frees its tensor memory.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include "qc_types.h"

namespace {

constexpr int TC_M = 128;
constexpr int TC_N = 64;
constexpr int TC_K = 32;           // per shared-memory stage: 4 MMAs of K = 8 (TF32)
constexpr int TC_THREADS = 128;
constexpr uint32_t TC_TMEM_COLS = 64;
constexpr long long TC_SPIN_LIMIT = 1LL << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor, K-major, no swizzle (layout type 0), version 1.
// lbo: byte distance between the two 16-byte K halves of a core-matrix pair;
// sbo: byte distance between consecutive 8-row core-matrix groups.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;          // descriptor version for sm_100
  return d;                        // base offset 0, legacy LBO mode, layout type 0
}

// Instruction descriptor: D = F32, A = B = TF32, both K-major, N = TC_N, M = TC_M.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                            ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
  for (long long it = 0; it < TC_SPIN_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
}

// Offset (in floats) of element (row, k) in a canonical K-major slice with `rows` rows.
__device__ __forceinline__ int canon(int row, int k, int rows) {
  return (((k >> 2) * (rows >> 3) + (row >> 3)) << 5) + ((row & 7) << 2) + (k & 3);
}

__device__ __forceinline__ void issue_mma(uint32_t tmem, uint32_t a0, uint32_t b0, bool accumulate) {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
  for (int s = 0; s < TC_K / 8; ++s) {
    const uint64_t da = umma_desc(a0 + s * 2 * (TC_M / 8) * 128, (TC_M / 8) * 128, 128);
    const uint64_t db = umma_desc(b0 + s * 2 * (TC_N / 8) * 128, (TC_N / 8) * 128, 128);
    const uint32_t en = (accumulate || s > 0) ? 1u : 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        :
        : "r"(tmem), "l"(da), "l"(db), "r"(kIdesc), "r"(en));
  }
}

// Two shared-memory stages: while the tensor core multiplies K-slice s (stage
// s&1), the threads load K-slice s+1 from global memory into registers; stage
// s&1 is refilled only after the MMAs that read it (committed to mbar[s&1])
// have completed.
// SPLIT: each FP32 operand x is staged as hi = tf32(x) and lo = tf32(x - hi) and the
// product accumulates hi*hi + hi*lo + lo*hi (three MMAs per K-step): FP32-level
// accuracy (relative error ~2^-21) on the tensor cores.
template <bool SPLIT>
__global__ void __launch_bounds__(TC_THREADS)
k_bgemm_tc(const qc_task *__restrict__ tasks, const qc_contrib *__restrict__ contribs,
           const qc_op *__restrict__ ops, const float *__restrict__ A, const float *__restrict__ B,
           float *__restrict__ C, int *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  constexpr int NP = SPLIT ? 2 : 1;                                 // hi (and lo) planes
  float *As = reinterpret_cast<float *>(tc_smem);                 // [2][NP][TC_M * TC_K]
  float *Bs = As + 2 * NP * TC_M * TC_K;                            // [2][NP][TC_N * TC_K]
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  __shared__ int arow[TC_M];
  __shared__ int bcol[TC_N];
  __shared__ int abort_flag;
  constexpr int LA = TC_M * TC_K / TC_THREADS;
  constexpr int LB = TC_N * TC_K / TC_THREADS;

  const qc_task t = tasks[blockIdx.x];
  if (t.op_b + (int)blockIdx.y >= t.op_e) return;
  const int op = t.op_b + (int)blockIdx.y;
  const qc_op o = ops[op];
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    abort_flag = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  uint32_t ph[2] = {0u, 0u};           // parity of the next completion of mbar[0], mbar[1] (thread 0)
  int g = 0;                           // K-slices issued so far (all contributions)
  bool accumulate = false;

  for (int ci = t.cb; ci < t.ce && !abort_flag; ++ci) {
    const qc_contrib c = contribs[ci];
    __syncthreads();
    for (int i = tid; i < TC_M; i += TC_THREADS) {
      const int m = t.m0 + i;
      arow[i] = (m < t.M) ? (m / t.mlo) * c.a_mh + (m % t.mlo) * c.a_ml : -1;
    }
    for (int j = tid; j < TC_N; j += TC_THREADS) {
      const int n = t.n0 + j;
      bcol[j] = (n < t.N) ? (n / t.nlo) * c.b_nh + (n % t.nlo) * c.b_nl : -1;
    }
    __syncthreads();
    const float alpha = (float)(o.alpha * c.alpha);
    const float *Ab = A + o.a_base + c.a_off;
    const float *Bb = B + o.b_base + c.b_off;
    const bool a_kfast = (c.a_kl == 1);
    const bool b_nfast = (c.b_nl == 1);
    const bool k1 = (c.klo >= c.K);
    const int nsteps = (c.K + TC_K - 1) / TC_K;
    float ra[LA], rb[LB];
    auto load = [&](int k0) {
#pragma unroll
      for (int e = 0; e < LA; ++e) {
        const int idx = tid + e * TC_THREADS;
        int i, kk;
        if (a_kfast) { kk = idx % TC_K; i = idx / TC_K; } else { i = idx % TC_M; kk = idx / TC_M; }
        const int k = k0 + kk, ro = arow[i];
        float v = 0.f;
        if (ro >= 0 && k < c.K) {
          const int ko = k1 ? k * c.a_kl : (k / c.klo) * c.a_kh + (k % c.klo) * c.a_kl;
          v = Ab[ro + ko] * alpha;
        }
        ra[e] = v;
      }
#pragma unroll
      for (int e = 0; e < LB; ++e) {
        const int idx = tid + e * TC_THREADS;
        int j, kk;
        if (b_nfast) { j = idx % TC_N; kk = idx / TC_N; } else { kk = idx % TC_K; j = idx / TC_K; }
        const int k = k0 + kk, co = bcol[j];
        float v = 0.f;
        if (co >= 0 && k < c.K) {
          const int ko = k1 ? k * c.b_kl : (k / c.klo) * c.b_kh + (k % c.klo) * c.b_kl;
          v = Bb[ko + co];
        }
        rb[e] = v;
      }
    };
    load(0);
    for (int s = 0; s < nsteps; ++s) {
      const int buf = g & 1;
      if (tid == 0 && g >= 2) {          // stage buf last read by the MMAs of slice g-2
        if (!mbar_wait(smem_u32(&mbar[buf]), ph[buf])) {
          abort_flag = 1;
          if (err) atomicExch(err, 1);
        }
        ph[buf] ^= 1u;
      }
      __syncthreads();
      if (abort_flag) break;
      float *as = As + buf * NP * TC_M * TC_K;
      float *bs = Bs + buf * NP * TC_N * TC_K;
#pragma unroll
      for (int e = 0; e < LA; ++e) {
        const int idx = tid + e * TC_THREADS;
        int i, kk;
        if (a_kfast) { kk = idx % TC_K; i = idx / TC_K; } else { i = idx % TC_M; kk = idx / TC_M; }
        const float hi = to_tf32(ra[e]);
        as[canon(i, kk, TC_M)] = hi;
        if (SPLIT) as[TC_M * TC_K + canon(i, kk, TC_M)] = to_tf32(ra[e] - hi);
      }
#pragma unroll
      for (int e = 0; e < LB; ++e) {
        const int idx = tid + e * TC_THREADS;
        int j, kk;
        if (b_nfast) { j = idx % TC_N; kk = idx / TC_N; } else { kk = idx % TC_K; j = idx / TC_K; }
        const float hi = to_tf32(rb[e]);
        bs[canon(j, kk, TC_N)] = hi;
        if (SPLIT) bs[TC_N * TC_K + canon(j, kk, TC_N)] = to_tf32(rb[e] - hi);
      }
      // make the generic-proxy shared-memory stores visible to the tensor core
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        const uint32_t a_hi = smem_u32(as), b_hi = smem_u32(bs);
        if (SPLIT) {                     // small terms first, then hi*hi
          issue_mma(tmem, a_hi, b_hi + TC_N * TC_K * 4, accumulate);
          issue_mma(tmem, a_hi + TC_M * TC_K * 4, b_hi, true);
          issue_mma(tmem, a_hi, b_hi, true);
        } else {
          issue_mma(tmem, a_hi, b_hi, accumulate);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     ::"r"(smem_u32(&mbar[buf])) : "memory");
      }
      accumulate = true;
      ++g;
      if (s + 1 < nsteps) load((s + 1) * TC_K);   // global loads overlap the MMAs just issued
    }
  }
  // drain: the last commit covers every MMA issued before it
  if (tid == 0 && g >= 1) {
    const int lb = (g - 1) & 1;
    if (!mbar_wait(smem_u32(&mbar[lb]), ph[lb])) {
      mbar_wait(smem_u32(&mbar[lb]), ph[lb]);     // one more bounded chance before TMEM is released
      abort_flag = 1;
      if (err) atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!abort_flag) {
    float *Cb = C + o.c_base + t.c_off;
    const int m = t.m0 + warp * 32 + lane;
    long long rowoff = 0;
    if (m < t.M) rowoff = (long long)(m / t.mlo) * t.c_mh + (long long)(m % t.mlo) * t.c_ml;
#pragma unroll
    for (int c8 = 0; c8 < TC_N; c8 += 8) {
      uint32_t r[8];
      if (accumulate) {
        const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c8;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
            : "r"(addr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) r[q] = 0u;
      }
      if (m < t.M) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int n = t.n0 + c8 + q;
          if (n < t.N)
            Cb[rowoff + (long long)(n / t.nlo) * t.c_nh + (long long)(n % t.nlo) * t.c_nl] = __uint_as_float(r[q]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
  }
}

constexpr size_t tc_dsmem(bool split) { return (size_t)2 * (split ? 2 : 1) * (TC_M + TC_N) * TC_K * sizeof(float); }

int *g_tc_err = nullptr;   // device error flag (allocated once, host-visible through qc_tc_status)

}  // namespace

static thread_local std::string g_tcerr;

template <bool SPLIT>
static int launch_tc(const void *tasks, long long ntasks, int opspan, const void *contribs, const void *ops,
                     int summed, const float *A, const float *B, float *C, int cfg, cudaStream_t stream) {
  if (ntasks <= 0) return QC_OK;
  if (summed || cfg != 5 || ntasks > 0x7fffffffLL || opspan < 1 || opspan > 65535) return QC_ERR_ARG;
  if (!g_tc_err) {
    if (cudaMalloc(&g_tc_err, sizeof(int)) != cudaSuccess) return QC_ERR_CUDA;
    cudaMemset(g_tc_err, 0, sizeof(int));
  }
  static bool attr_set = false;
  if (!attr_set) {
    if (cudaFuncSetAttribute(k_bgemm_tc<SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_dsmem(SPLIT)) !=
        cudaSuccess)
      return QC_ERR_CUDA;
    attr_set = true;
  }
  dim3 grid((unsigned)ntasks, (unsigned)opspan);
  k_bgemm_tc<SPLIT><<<grid, TC_THREADS, tc_dsmem(SPLIT), stream>>>(
      (const qc_task *)tasks, (const qc_contrib *)contribs, (const qc_op *)ops, A, B, C, g_tc_err);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_tcerr = cudaGetErrorString(e);
    fprintf(stderr, "[qcgpu] qc_bgemm_tf32: %s\n", g_tcerr.c_str());
    return QC_ERR_CUDA;
  }
  return QC_OK;
}

extern "C" int qc_bgemm_tf32(const void *tasks, long long ntasks, int opspan, const void *contribs, const void *ops,
                             int summed, const float *A, const float *B, float *C, int cfg, void *stream) {
  return launch_tc<false>(tasks, ntasks, opspan, contribs, ops, summed, A, B, C, cfg, (cudaStream_t)stream);
}

extern "C" int qc_bgemm_tf32x3(const void *tasks, long long ntasks, int opspan, const void *contribs, const void *ops,
                               int summed, const float *A, const float *B, float *C, int cfg, void *stream) {
  return launch_tc<true>(tasks, ntasks, opspan, contribs, ops, summed, A, B, C, cfg, (cudaStream_t)stream);
}

extern "C" int qc_tc_status(void) {
  if (!g_tc_err) return 0;
  int h = 0;
  if (cudaMemcpy(&h, g_tc_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return QC_ERR_CUDA;
  return h;
}
