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

__global__ void __launch_bounds__(TC_THREADS)
k_bgemm_tc(const qc_task *__restrict__ tasks, const qc_contrib *__restrict__ contribs,
           const qc_op *__restrict__ ops, const float *__restrict__ A, const float *__restrict__ B,
           float *__restrict__ C, int *__restrict__ err) {
  __shared__ __align__(1024) float As[TC_M * TC_K];
  __shared__ __align__(1024) float Bs[TC_N * TC_K];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  __shared__ int arow[TC_M];
  __shared__ int bcol[TC_N];
  __shared__ int akoff[TC_K];
  __shared__ int bkoff[TC_K];
  __shared__ int abort_flag;

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
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t bar = smem_u32(&mbar);
  uint32_t phase = 0;
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
    const float alpha = (float)(o.alpha * c.alpha);
    const float *Ab = A + o.a_base + c.a_off;
    const float *Bb = B + o.b_base + c.b_off;
    const bool a_kfast = (c.a_kl == 1);
    const bool b_nfast = (c.b_nl == 1);
    for (int k0 = 0; k0 < c.K && !abort_flag; k0 += TC_K) {
      __syncthreads();
      if (tid < TC_K) {
        const int k = k0 + tid;
        akoff[tid] = (k < c.K) ? (k / c.klo) * c.a_kh + (k % c.klo) * c.a_kl : -1;
        bkoff[tid] = (k < c.K) ? (k / c.klo) * c.b_kh + (k % c.klo) * c.b_kl : -1;
      }
      __syncthreads();
      for (int idx = tid; idx < TC_M * TC_K; idx += TC_THREADS) {
        int i, kk;
        if (a_kfast) { kk = idx % TC_K; i = idx / TC_K; } else { i = idx % TC_M; kk = idx / TC_M; }
        const int ro = arow[i], ko = akoff[kk];
        As[canon(i, kk, TC_M)] = to_tf32((ro >= 0 && ko >= 0) ? Ab[ro + ko] * alpha : 0.f);
      }
      for (int idx = tid; idx < TC_N * TC_K; idx += TC_THREADS) {
        int j, kk;
        if (b_nfast) { j = idx % TC_N; kk = idx / TC_N; } else { kk = idx % TC_K; j = idx / TC_K; }
        const int co = bcol[j], ko = bkoff[kk];
        Bs[canon(j, kk, TC_N)] = to_tf32((co >= 0 && ko >= 0) ? Bb[ko + co] : 0.f);
      }
      // make the generic-proxy shared-memory stores visible to the tensor core
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_u32(As), b0 = smem_u32(Bs);
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
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                     : "memory");
        // only this thread waits; the barrier below publishes the outcome to the CTA
        if (!mbar_wait(bar, phase)) {
          // give the in-flight MMAs one more bounded chance before tensor memory is released
          mbar_wait(bar, phase);
          abort_flag = 1;
          if (err) atomicExch(err, 1);
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      }
      accumulate = true;
      phase ^= 1u;
      __syncthreads();
    }
  }
  __syncthreads();
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

int *g_tc_err = nullptr;   // device error flag (allocated once, host-visible through qc_tc_status)

}  // namespace

static thread_local std::string g_tcerr;

extern "C" int qc_bgemm_tf32(const void *tasks, long long ntasks, int opspan, const void *contribs, const void *ops,
                             int summed, const float *A, const float *B, float *C, int cfg, void *stream) {
  if (ntasks <= 0) return QC_OK;
  if (summed || cfg != 5 || ntasks > 0x7fffffffLL || opspan < 1 || opspan > 65535) return QC_ERR_ARG;
  if (!g_tc_err) {
    if (cudaMalloc(&g_tc_err, sizeof(int)) != cudaSuccess) return QC_ERR_CUDA;
    cudaMemset(g_tc_err, 0, sizeof(int));
  }
  dim3 grid((unsigned)ntasks, (unsigned)opspan);
  k_bgemm_tc<<<grid, TC_THREADS, 0, (cudaStream_t)stream>>>((const qc_task *)tasks, (const qc_contrib *)contribs,
                                                            (const qc_op *)ops, A, B, C, g_tc_err);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_tcerr = cudaGetErrorString(e);
    fprintf(stderr, "[qcgpu] qc_bgemm_tf32: %s\n", g_tcerr.c_str());
    return QC_ERR_CUDA;
  }
  return QC_OK;
}

extern "C" int qc_tc_status(void) {
  if (!g_tc_err) return 0;
  int h = 0;
  if (cudaMemcpy(&h, g_tc_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return QC_ERR_CUDA;
  return h;
}
