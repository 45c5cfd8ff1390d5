// Panel GEMM on the 5th-generation tensor cores, fed by TMA: the .R contraction of
// HVecQt (top4 = top3 . R, source/mpo_dmrg_kernelQt.py:302-306) in FP32-level
// precision from split TF32 products.
//
// For one output sector r' of one operator, sigma rows (the T3 panel [M x K], row
// stride Kp, written by the fiber kernel) times the R panel of r' (stored transposed,
// [N x K] with k contiguous, pre-split into TF32 hi and lo planes once per dot) give
// the sigma rows of that sector; the K extent (sum over MPO sectors c of D_c * D_r)
// is long, the N extent (D_r') short.
//
// Persistent, warp-specialised CTA (10 warps):
//   warp 0     one thread issues the TMA loads (cp.async.bulk.tensor, 128-byte swizzle)
//              of every 32-wide K stage into a ring of S shared-memory stages;
//   warp 1     owns the tensor memory (2 x BN columns: two accumulators) and one thread
//              issues tcgen05.mma kind::tf32, 12 per stage: a_lo.b_hi + a_hi.b_lo +
//              a_hi.b_hi for each 8-wide K step, committed to the stage's "empty"
//              barrier and, after a unit's last stage, to the accumulator's "full" one;
//   warps 2-9  split each raw FP32 A stage in place into hi = tf32(x) and a lo plane
//              tf32(x - hi) (A_SPLIT); every 2 K stages add the TMEM accumulator into FP32
//              registers (tcgen05.ld: warp w owns TMEM lanes 32*(w%4) .. and one half of the
//              columns), and store the finished tile (rows through the row table, or
//              column segments staged in shared memory); the other TMEM accumulator
//              meanwhile takes the next chunk.
// No cluster, no multicast: every CTA loads its own tiles of this GPU's own memory.
// Every wait is bounded: on expiry the CTA raises *err, stops issuing work, waits
// (bounded) for its loads and products in flight and still frees its tensor memory.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include "qc_types.h"

namespace {

constexpr int TP_BM = 128;
constexpr int TP_BK = 32;                  // 32 FP32 = 128 bytes: one swizzle row
constexpr int TP_THREADS = 320;             // producer warp, MMA warp, 8 helper warps
constexpr int TP_HELPERS = 8;
constexpr long long TP_SPIN = 1LL << 26;   // polls before a wait gives up (~seconds)
constexpr int TP_CHUNK = 2;                 // K stages accumulated in TMEM before promotion to FP32 registers

__device__ __forceinline__ uint32_t su32(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ bool wait_parity(uint32_t bar, uint32_t parity) {
  for (long long it = 0; it < TP_SPIN; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 256) __nanosleep(32);
  }
  return false;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load3(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

__device__ __forceinline__ void tma_load4(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
      "[%2];" ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
      : "memory");
}

// Tensor maps live in global memory (written from the host before the launch).
__device__ __forceinline__ void tmap_acquire(const CUtensorMap *map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
               : "memory");
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle (layout type 2), 8-row
// groups 1024 bytes apart (SBO); the leading offset is unused for this layout.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// Instruction descriptor: D = F32, A = B = TF32, both K-major, M = 128, N = n.
__device__ __forceinline__ uint32_t idesc_tf32(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TP_BM >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

template <int BN>
__host__ __device__ constexpr int stage_bytes() { return 2 * TP_BM * TP_BK * 4 + 2 * BN * TP_BK * 4; }

constexpr int EPI_ROWS = 0;       // rows through a row table, stored from registers
constexpr int EPI_SEGMENTS = 1;   // column segments, staged in shared memory, coalesced stores

template <bool A_SPLIT, int BN, int S, int EPI>
__global__ void __launch_bounds__(TP_THREADS, 1)
k_tcpanel(const qc_tcunit *__restrict__ units, int nunits, const CUtensorMap *__restrict__ maps,
          const qc_op *__restrict__ ops, const long long *__restrict__ crow, const qc_tcseg *__restrict__ segs,
          float *__restrict__ C, int *__restrict__ err) {
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "UMMA N");
  extern __shared__ unsigned char tp_smem_raw[];
  // stage s: [A0 (raw / hi) | A1 (lo) | B0 (hi) | B1 (lo)], each 1024-byte aligned
  unsigned char *smem = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(tp_smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  constexpr int A_BYTES = TP_BM * TP_BK * 4;
  constexpr int B_BYTES = BN * TP_BK * 4;
  constexpr int ST_BYTES = stage_bytes<BN>();
  __shared__ __align__(8) uint64_t full[S], empty[S], split[S], accf[2], acce[2], fin;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base)),
                 "r"(2 * BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int s = 0; s < S; ++s) {
      mbar_init(su32(&full[s]), 1);
      mbar_init(su32(&empty[s]), 1);
      mbar_init(su32(&split[s]), TP_HELPERS);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(su32(&accf[b]), 1);
      mbar_init(su32(&acce[b]), TP_HELPERS);
    }
    mbar_init(su32(&fin), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;

  auto fail = [&]() {
    abort_flag = 1;
    if (err) atomicExch(err, 1);
  };

  if (warp == 0) {
    // ------------------------------------------------------------ TMA producer
    if (lane == 0) {
      int it = 0;
      int issued[S];
      for (int s = 0; s < S; ++s) issued[s] = -1;
      for (int u = blockIdx.x; u < nunits && !abort_flag; u += gridDim.x) {
        const qc_tcunit t = units[u];
        const CUtensorMap *am = maps + t.a_map;
        const CUtensorMap *bm = maps + t.b_map;
        tmap_acquire(am);
        tmap_acquire(bm);
        for (int k = 0; k < t.nk; ++k, ++it) {
          const int s = it % S;
          const uint32_t ph = (uint32_t)((it / S) & 1);
          if (!wait_parity(su32(&empty[s]), ph ^ 1u)) {
            fail();
            break;
          }
          unsigned char *st = smem + s * ST_BYTES;
          mbar_arrive_tx(su32(&full[s]), (A_SPLIT ? A_BYTES : 2 * A_BYTES) + 2 * B_BYTES);
          if (A_SPLIT)
            tma_load3(su32(st), am, k * TP_BK, t.a_c1, t.a_c2, su32(&full[s]));
          else
            tma_load4(su32(st), am, k * TP_BK, t.a_c1, t.a_c2, 0, su32(&full[s]));
          tma_load4(su32(st + 2 * A_BYTES), bm, k * TP_BK, t.b_c1, t.b_c2, 0, su32(&full[s]));
          issued[s] = (int)ph;
        }
      }
      // loads still in flight land before the CTA leaves (bounded)
      for (int s = 0; s < S; ++s)
        if (issued[s] >= 0) wait_parity(su32(&full[s]), (uint32_t)issued[s]);
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    // A unit's K stages go in chunks of TP_CHUNK stages; chunk g (counted over all units of
    // this CTA) accumulates in TMEM buffer g & 1 from zero, and the helpers add it to FP32
    // registers: the tensor core's accumulation only ever spans TP_CHUNK * 32 products.
    if (lane == 0) {
      int it = 0, g = 0;
      bool any = false;
      for (int u = blockIdx.x; u < nunits && !abort_flag; u += gridDim.x) {
        const qc_tcunit t = units[u];
        const int nmma = ((t.n_valid + 15) / 16) * 16;
        const uint32_t idesc = idesc_tf32(nmma > BN ? BN : nmma);
        bool ok = true;
        for (int k0 = 0; k0 < t.nk && ok; k0 += TP_CHUNK, ++g) {
          const int buf = g & 1;
          if (!wait_parity(su32(&acce[buf]), (uint32_t)(((g >> 1) & 1) ^ 1))) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t d = tmem + (uint32_t)(buf * BN);
          const int k1 = (k0 + TP_CHUNK < t.nk) ? k0 + TP_CHUNK : t.nk;
          for (int k = k0; k < k1; ++k, ++it) {
            const int s = it % S;
            const uint32_t ph = (uint32_t)((it / S) & 1);
            if (!wait_parity(su32(A_SPLIT ? &split[s] : &full[s]), ph)) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st = su32(smem + s * ST_BYTES);
            const uint32_t a_hi = st, a_lo = st + A_BYTES, b_hi = st + 2 * A_BYTES, b_lo = b_hi + B_BYTES;
#pragma unroll
            for (int kk = 0; kk < TP_BK / 8; ++kk) {
              const uint32_t off = kk * 32;            // 8 TF32 = 32 bytes along the swizzled row
              const uint32_t first = (k == k0 && kk == 0) ? 0u : 1u;
              mma_tf32(d, desc_sw128(a_lo + off), desc_sw128(b_hi + off), idesc, first);
              mma_tf32(d, desc_sw128(a_hi + off), desc_sw128(b_lo + off), idesc, 1u);
              mma_tf32(d, desc_sw128(a_hi + off), desc_sw128(b_hi + off), idesc, 1u);
            }
            mma_commit(su32(&empty[s]));
            any = true;
          }
          if (!ok) break;
          mma_commit(su32(&accf[buf]));
        }
        if (!ok) {
          fail();
          break;
        }
      }
      // every product issued has finished before the tensor memory is released (bounded)
      if (any) {
        mma_commit(su32(&fin));
        if (!wait_parity(su32(&fin), 0u)) fail();
      }
    }
  } else {
    // ------------------------------------------------------------ split + promotion + epilogue (warps 2-9)
    // two warpgroups: warp w reads TMEM lanes 32*(w%4) .. (its quarter of the rows) and the
    // accumulator columns of its group, [BN/2 * gw, BN/2 * (gw + 1))
    constexpr int HALF = BN / 2;
    const int hid = threadIdx.x - 64;          // 0 .. 255
    const int q = warp & 3;                    // TMEM lane quarter of this warp
    const int gw = (warp - 2) >> 2;            // column half of this warp's group
    const int row = q * 32 + lane;
    float acc[HALF];
    int it = 0;                                // stages split so far
    // the chunk stream (unit, first stage) in the order the MMA issuer takes it; the next
    // chunk's stages are split before the current chunk is drained, so the tensor core
    // never waits for a drain
    int su = blockIdx.x, sk = 0;               // next chunk to split
    auto split_chunk = [&]() -> bool {
      if (su >= nunits) return true;
      const int nk = units[su].nk;
      const int k1 = (sk + TP_CHUNK < nk) ? sk + TP_CHUNK : nk;
      if (A_SPLIT) {
        for (int k = sk; k < k1; ++k, ++it) {
          const int s = it % S;
          const uint32_t ph = (uint32_t)((it / S) & 1);
          if (!wait_parity(su32(&full[s]), ph)) return false;
          float4 *a0 = reinterpret_cast<float4 *>(smem + s * ST_BYTES);
          float4 *a1 = reinterpret_cast<float4 *>(smem + s * ST_BYTES + A_BYTES);
#pragma unroll
          for (int j = 0; j < A_BYTES / 16 / (32 * TP_HELPERS); ++j) {
            const int i = hid + j * 32 * TP_HELPERS;
            const float4 x = a0[i];
            float4 h, l;
            h.x = tf32_rna(x.x); l.x = tf32_rna(x.x - h.x);
            h.y = tf32_rna(x.y); l.y = tf32_rna(x.y - h.y);
            h.z = tf32_rna(x.z); l.z = tf32_rna(x.z - h.z);
            h.w = tf32_rna(x.w); l.w = tf32_rna(x.w - h.w);
            a0[i] = h;
            a1[i] = l;
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (lane == 0) mbar_arrive(su32(&split[s]));
        }
      }
      sk = k1;
      if (sk >= nk) {
        su += gridDim.x;
        sk = 0;
      }
      return true;
    };
    bool ok = split_chunk();
    int g = 0;
    for (int u = blockIdx.x; u < nunits && ok && !abort_flag; u += gridDim.x) {
      const qc_tcunit t = units[u];
      const int ncol = t.n_valid < BN ? t.n_valid : BN;
      for (int k0 = 0; k0 < t.nk; k0 += TP_CHUNK, ++g) {
        ok = split_chunk();
        if (!ok) break;
        const int buf = g & 1;
        if (!wait_parity(su32(&accf[buf]), (uint32_t)((g >> 1) & 1))) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * BN + gw * HALF);
#pragma unroll
        for (int c0 = 0; c0 < HALF; c0 += 16) {
          if (gw * HALF + c0 < ncol) {
            uint32_t r[16];
            tmem_ld16(taddr + (uint32_t)c0, r);
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[c0 + j] = (k0 == 0) ? __uint_as_float(r[j]) : acc[c0 + j] + __uint_as_float(r[j]);
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(su32(&acce[buf]));
      }
      if (!ok) break;
      // ---- epilogue of unit u from the FP32 registers
      const qc_op o = ops[t.op];
      const float alpha = (float)o.alpha;
      if (EPI == EPI_ROWS) {
        if (row < t.m_valid) {
          float *dst = C + o.c_base + crow[t.c_off + row] + t.b_c1 + gw * HALF;
#pragma unroll
          for (int c = 0; c < HALF; ++c)
            if (gw * HALF + c < ncol) dst[c] = alpha * acc[c];
        }
      } else {
        // the whole tile staged in shared memory (row stride BN + 1: no bank conflicts), then
        // each warp copies whole rows of every segment, lanes on consecutive columns
        // (coalesced: a segment row is contiguous in memory)
        float *stg = reinterpret_cast<float *>(smem + S * ST_BYTES);
        float *Cb = C + o.c_base;
#pragma unroll
        for (int c = 0; c < HALF; ++c) stg[row * (BN + 1) + gw * HALF + c] = alpha * acc[c];
        asm volatile("bar.sync 1, %0;" ::"n"(32 * TP_HELPERS) : "memory");
        for (int si = 0; si < t.nseg; ++si) {
          const qc_tcseg sg = segs[t.c_off + si];
          const int w = sg.ncol;
          float *db = Cb + sg.off + (long long)t.a_c1 * sg.ldc;
          const float *sb = stg + sg.col0;
          for (int m = warp - 2; m < t.m_valid; m += TP_HELPERS)
            for (int c = lane; c < w; c += 32) db[(long long)m * sg.ldc + c] = sb[m * (BN + 1) + c];
        }
        asm volatile("bar.sync 1, %0;" ::"n"(32 * TP_HELPERS) : "memory");
      }
    }
    if (!ok) fail();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN));
  }
}

// hi = tf32(x), lo = tf32(x - hi), in place into hi (n values)
__global__ void k_tf32_split(float *__restrict__ hi, float *__restrict__ lo, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float x = hi[i];
    const float h = tf32_rna(x);
    hi[i] = h;
    lo[i] = tf32_rna(x - h);
  }
}

// hi[i] = tf32(x[idx[i]]), lo[i] = tf32(x[idx[i]] - hi[i]) (FP64 source; idx < 0: zero)
__global__ void k_gather_split(const double *__restrict__ x, const long long *__restrict__ idx, long long n,
                               float *__restrict__ hi, float *__restrict__ lo) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long j = idx[i];
    const float v = j >= 0 ? (float)x[j] : 0.f;
    const float h = tf32_rna(v);
    hi[i] = h;
    lo[i] = tf32_rna(v - h);
  }
}

int *g_tp_err = nullptr;
int g_nsm = 0;
std::mutex g_tp_mu;
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

constexpr int TP_BN = 128;
constexpr int TP_S = 3;
constexpr int tp_stages(int epi) { return epi == EPI_SEGMENTS ? 2 : TP_S; }
constexpr size_t tp_dsmem(int epi) {
  return (size_t)tp_stages(epi) * stage_bytes<TP_BN>() + 1024 + (epi == EPI_SEGMENTS ? TP_BM * (TP_BN + 1) * 4 : 0);
}
bool g_attr[2] = {false, false};

template <bool A_SPLIT, int EPI>
int launch_tcpanel(const void *units, long long nunits, const void *maps, const void *ops, const long long *crow,
                   const void *segs, float *C, cudaStream_t s) {
  if (nunits <= 0) return QC_OK;
  if (nunits > 0x7fffffffLL || !units || !maps || !ops || !C) return QC_ERR_ARG;
  if ((EPI == EPI_ROWS && !crow) || (EPI == EPI_SEGMENTS && !segs)) return QC_ERR_ARG;
  {
    std::lock_guard<std::mutex> lock(g_tp_mu);
    if (!g_tp_err) {
      if (cudaMalloc(&g_tp_err, sizeof(int)) != cudaSuccess) return QC_ERR_CUDA;
      if (cudaMemset(g_tp_err, 0, sizeof(int)) != cudaSuccess) return QC_ERR_CUDA;
      int dev = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&g_nsm, cudaDevAttrMultiProcessorCount, dev);
    }
    if (!g_attr[EPI]) {
      if (cudaFuncSetAttribute(k_tcpanel<A_SPLIT, TP_BN, tp_stages(EPI), EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)tp_dsmem(EPI)) != cudaSuccess)
        return QC_ERR_CUDA;
      g_attr[EPI] = true;
    }
  }
  const int grid = (int)(nunits < (long long)g_nsm ? nunits : (long long)g_nsm);
  k_tcpanel<A_SPLIT, TP_BN, tp_stages(EPI), EPI><<<grid, TP_THREADS, tp_dsmem(EPI), s>>>(
      (const qc_tcunit *)units, (int)nunits, (const CUtensorMap *)maps, (const qc_op *)ops, crow,
      (const qc_tcseg *)segs, C, g_tp_err);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "[qcgpu] qc_tcpanel: %s\n", cudaGetErrorString(e));
    return QC_ERR_CUDA;
  }
  return QC_OK;
}

}  // namespace

static thread_local std::string g_tperr;

extern "C" int qc_tmap_encode(int n, const void *descs, void *out_maps) {
  if (n < 0 || (n > 0 && (!descs || !out_maps))) return QC_ERR_ARG;
  {
    std::lock_guard<std::mutex> lock(g_tp_mu);
    if (!g_encode) {
      cudaDriverEntryPointQueryResult q;
      void *fn = nullptr;
      if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
          q != cudaDriverEntryPointSuccess || !fn) {
        fprintf(stderr, "[qcgpu] qc_tmap_encode: cuTensorMapEncodeTiled not available\n");
        return QC_ERR_CUDA;
      }
      g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
  }
  const qc_tmdesc *d = (const qc_tmdesc *)descs;
  CUtensorMap *m = (CUtensorMap *)out_maps;
  for (int i = 0; i < n; ++i) {
    const qc_tmdesc &x = d[i];
    if (x.rank < 2 || x.rank > 5 || (x.addr & 15)) return QC_ERR_ARG;
    cuuint64_t dims[5], strides[4];
    cuuint32_t box[5], es[5];
    for (int r = 0; r < x.rank; ++r) {
      if (x.dims[r] < 1 || x.box[r] < 1 || x.box[r] > 256) return QC_ERR_ARG;
      dims[r] = (cuuint64_t)x.dims[r];
      box[r] = (cuuint32_t)x.box[r];
      es[r] = 1;
      if (r > 0) {
        if (x.strides[r - 1] <= 0 || (x.strides[r - 1] & 15)) return QC_ERR_ARG;
        strides[r - 1] = (cuuint64_t)x.strides[r - 1];
      }
    }
    if (x.swizzle == 3 && box[0] * 4 > 128) return QC_ERR_ARG;
    CUresult rc = g_encode(&m[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (cuuint32_t)x.rank, (void *)x.addr, dims, strides,
                           box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, (CUtensorMapSwizzle)x.swizzle,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (rc != CUDA_SUCCESS) {
      fprintf(stderr, "[qcgpu] qc_tmap_encode: map %d rejected (CUresult %d)\n", i, (int)rc);
      return QC_ERR_ARG;
    }
  }
  return QC_OK;
}

// C rows (through the row table) = A . B^T on the tensor cores, A split into TF32 hi/lo
// in the kernel, B given as pre-split hi/lo planes (maps of rank 4, plane dimension last).
extern "C" int qc_tcpanel_f32(const void *units, long long nunits, const void *maps, const void *ops,
                              const long long *crow, float *C, void *stream) {
  return launch_tcpanel<true, EPI_ROWS>(units, nunits, maps, ops, crow, nullptr, C, (cudaStream_t)stream);
}

// Column segments of C = A . B^T on the tensor cores, both operands pre-split hi/lo planes.
extern "C" int qc_tcpanel_seg_f32(const void *units, long long nunits, const void *maps, const void *ops,
                                  const void *segs, float *C, void *stream) {
  return launch_tcpanel<false, EPI_SEGMENTS>(units, nunits, maps, ops, nullptr, segs, C, (cudaStream_t)stream);
}

extern "C" int qc_tf32_split(float *hi, float *lo, long long n, void *stream) {
  if (n <= 0) return QC_OK;
  if (!hi || !lo) return QC_ERR_ARG;
  long long blocks = (n + 255) / 256;
  if (blocks > 65535) blocks = 65535;
  k_tf32_split<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(hi, lo, n);
  return cudaGetLastError() == cudaSuccess ? QC_OK : QC_ERR_CUDA;
}

extern "C" int qc_gather_split_f32(const double *x, const long long *idx, long long n, float *hi, float *lo,
                                   void *stream) {
  if (n <= 0) return QC_OK;
  if (!x || !idx || !hi || !lo) return QC_ERR_ARG;
  long long blocks = (n + 255) / 256;
  if (blocks > 65535) blocks = 65535;
  k_gather_split<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(x, idx, n, hi, lo);
  return cudaGetLastError() == cudaSuccess ? QC_OK : QC_ERR_CUDA;
}

// Error flag of the tensor-core panel kernel (1 after a wait gave up); reset with clear != 0.
extern "C" int qc_tcpanel_status(int clear) {
  if (!g_tp_err) return 0;
  int h = 0;
  if (cudaMemcpy(&h, g_tp_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return QC_ERR_CUDA;
  if (clear && cudaMemset(g_tp_err, 0, sizeof(int)) != cudaSuccess) return QC_ERR_CUDA;
  return h;
}
