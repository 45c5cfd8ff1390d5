// Fiber-group kernel for the two W contractions of sigma (the .W_i and .W_{i+1}
// stages of HVecQt, source/mpo_dmrg_kernelQt.py:301-306).
//
// In those contractions every output block (fiber index f = (l, r), column index
// c from the MPO bond and a physical index) is a sum over a handful of input
// blocks times small W blocks (MPO-sector x MPO-sector).  The generic grouped
// GEMM reads each input block once per output block that uses it; here one CTA
// owns a tile of FT fibers of one group, stages every input row of the group for
// those fibers in shared memory once (coalesced along the storage order of each
// block), then writes every output block of the group for those fibers.  HBM
// traffic is the algorithmic one: inputs read once, outputs written once.
#include <cuda_runtime.h>
#include <cstdio>
#include "qc_types.h"

namespace {

constexpr int FT_THREADS = 256;
constexpr int CB = 8;           // output columns per warp work item (register accumulators)

// One CTA = one tile of FT = 32*FPL fibers of one fiber group, for one operator
// (grid.y).  Phase 1 stages every input row of the group for those fibers in
// shared memory.  Phase 2: each warp takes (output block, 8-column block)
// items; lane l owns fibers l, l+32, ... (FPL of them) with 8 accumulators each;
// W elements are warp-uniform (broadcast) loads, so every W value read serves
// 32*FPL fibers and every staged input value 8 columns.
template <typename T, int FPL>
__global__ void __launch_bounds__(FT_THREADS)
k_fiber(const qc_ftask *__restrict__ tasks, const qc_fin *__restrict__ fin, const qc_fout *__restrict__ fout,
        const qc_fpair *__restrict__ fpair, const qc_op *__restrict__ ops, const T *__restrict__ A,
        const T *__restrict__ W, T *__restrict__ C) {
  constexpr int FT = 32 * FPL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *As = reinterpret_cast<T *>(smem_raw);
  const qc_ftask t = tasks[blockIdx.x];
  const int op = t.op_b + (int)blockIdx.y;
  if (op >= t.op_e) return;
  const qc_op o = ops[op];
  const int tid = threadIdx.x;
  const int nf = min(FT, t.F - t.f0);
  const T *Ab = A + o.a_base;
  for (int i = t.in_b; i < t.in_e; ++i) {
    const qc_fin b = fin[i];
    const T *src = Ab + b.a_off;
    const int n = b.rows * FT;
    // unrolled so that several independent loads are in flight per thread
    if (!b.fiber_major) {             // [rows][F]: consecutive threads -> consecutive fibers
#pragma unroll 4
      for (int idx = tid; idx < n; idx += FT_THREADS) {
        const int r = idx / FT, f = idx % FT;
        As[(b.srow + r) * FT + f] = (f < nf) ? src[(long long)r * t.F + t.f0 + f] : T(0);
      }
    } else {                          // [F][rows]: consecutive threads -> consecutive rows
#pragma unroll 4
      for (int idx = tid; idx < n; idx += FT_THREADS) {
        const int f = idx / b.rows, r = idx % b.rows;
        As[(b.srow + r) * FT + f] = (f < nf) ? src[(long long)(t.f0 + f) * b.rows + r] : T(0);
      }
    }
  }
  __syncthreads();
  const T alpha = T(o.alpha);
  const T *Wb = W + o.b_base;
  T *Cb = C + o.c_base;
  const int lane = tid & 31, warp = tid >> 5;
  constexpr int NW = FT_THREADS / 32;
  __shared__ __align__(16) T wslot[NW][32 * CB];     // per-warp staged W rows
  T *wsl = wslot[warp];
  // items: (output block j, column block cb), enumerated block by block
  int j = t.out_b, cb = 0, skip = warp;
  while (j < t.out_e) {
    const int nc = fout[j].ncols;
    const int ncb = (nc + CB - 1) / CB;
    if (skip < ncb - cb) { cb += skip; break; }
    skip -= ncb - cb;
    cb = 0;
    ++j;
  }
  while (j < t.out_e) {
    const qc_fout ob = fout[j];
    const int nc = ob.ncols;
    const int c0 = cb * CB;
    const int nb = min(CB, nc - c0);
    T acc[FPL][CB];
#pragma unroll
    for (int q = 0; q < FPL; ++q)
#pragma unroll
      for (int i = 0; i < CB; ++i) acc[q][i] = T(0);
    for (int p = ob.pair_b; p < ob.pair_e; ++p) {
      const qc_fpair pr = fpair[p];
      const T *w = Wb + pr.w_off + c0;
      const T *a = As + pr.srow * FT + lane;
      // the W rows of this pair, 32 at a time: lane l stages row r0+l (8 columns,
      // zero beyond the block) in this warp's shared slot; the FMAs then read them
      // as broadcasts, so no global load sits inside the multiply loop
      for (int r0 = 0; r0 < pr.rows; r0 += 32) {
        const int nr = min(32, pr.rows - r0);
        __syncwarp();
        if (lane < nr) {
          const T *wr = w + (long long)(r0 + lane) * nc;
#pragma unroll
          for (int i = 0; i < CB; ++i) wsl[lane * CB + i] = (i < nb) ? __ldg(wr + i) : T(0);
        }
        __syncwarp();
#pragma unroll 2
        for (int r = 0; r < nr; ++r) {
          T av[FPL];
#pragma unroll
          for (int q = 0; q < FPL; ++q) av[q] = a[(r0 + r) * FT + 32 * q];
          T wv[CB];
#pragma unroll
          for (int i = 0; i < CB; ++i) wv[i] = wsl[r * CB + i];
#pragma unroll
          for (int i = 0; i < CB; ++i)
#pragma unroll
            for (int q = 0; q < FPL; ++q) acc[q][i] = fma(av[q], wv[i], acc[q][i]);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < FPL; ++q) {
      const int fl = lane + 32 * q;
      if (fl < nf) {
        const int fg = t.f0 + fl;
        if (ob.colmajor) {
          T *dst = Cb + ob.c_off + (long long)c0 * t.F + fg;
#pragma unroll
          for (int i = 0; i < CB; ++i)
            if (i < nb) dst[(long long)i * t.F] = alpha * acc[q][i];
        } else {
          T *dst = Cb + ob.c_off + (long long)(fg / ob.flo) * ob.fhs + (long long)(fg % ob.flo) * nc + c0;
#pragma unroll
          for (int i = 0; i < CB; ++i)
            if (i < nb) dst[i] = alpha * acc[q][i];
        }
      }
    }
    // advance NW items
    int adv = NW;
    while (j < t.out_e && adv > 0) {
      const int ncb = (fout[j].ncols + CB - 1) / CB;
      if (cb + adv < ncb) { cb += adv; adv = 0; break; }
      adv -= ncb - cb;
      cb = 0;
      ++j;
    }
  }
}

// dst[dst_off + i0*s0 + i1*s1 + i2*s2] = src[src_off + (i0*d1 + i1)*d2 + i2] for every
// block (blockIdx.x, grid-stride over its elements) and operator (blockIdx.y).
template <typename TD>
__global__ void __launch_bounds__(256)
k_block_permute(const qc_bperm *__restrict__ descs, const qc_op *__restrict__ ops, const double *__restrict__ src,
                TD *__restrict__ dst) {
  const qc_bperm d = descs[blockIdx.x];
  const int op = d.op_b + (int)blockIdx.y;
  if (op >= d.op_e) return;
  const qc_op o = ops[op];
  const double *s = src + o.a_base + d.src_off;
  TD *t = dst + o.c_base + d.dst_off;
  const long long n = (long long)d.d0 * d.d1 * d.d2;
  const int d12 = d.d1 * d.d2;
  for (long long e = threadIdx.x; e < n; e += blockDim.x) {
    const int i0 = (int)(e / d12), rem = (int)(e % d12);
    const int i1 = rem / d.d2, i2 = rem % d.d2;
    t[(long long)i0 * d.s0 + (long long)i1 * d.s1 + (long long)i2 * d.s2] = (TD)s[e];
  }
}

template <typename T>
int launch_fiber(const void *tasks, long long ntasks, int opspan, const void *fin, const void *fout,
                 const void *fpair, const void *ops, int max_rows, int fiber_tile, const T *A, const T *W, T *C,
                 cudaStream_t s) {
  if (ntasks <= 0) return QC_OK;
  if (ntasks > 0x7fffffffLL || opspan < 1 || opspan > 65535 || max_rows < 1) return QC_ERR_ARG;
  if (fiber_tile != 32 && fiber_tile != 64) return QC_ERR_ARG;
  const size_t smem = (size_t)max_rows * fiber_tile * sizeof(T);
  if (smem > 200 * 1024) return QC_ERR_ARG;
  dim3 grid((unsigned)ntasks, (unsigned)opspan);
  const qc_ftask *tk = (const qc_ftask *)tasks;
  // the kernels also hold 8-16 KB of static shared memory (per-warp W rows): allow the
  // full dynamic range once per instantiation
  static bool attr_set[2] = {false, false};
  const int v = (fiber_tile == 32) ? 0 : 1;
  if (!attr_set[v]) {
    cudaError_t ea = (v == 0) ? cudaFuncSetAttribute(k_fiber<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     200 * 1024)
                              : cudaFuncSetAttribute(k_fiber<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     200 * 1024);
    if (ea != cudaSuccess) {
      fprintf(stderr, "[qcgpu] qc_fiber: %s\n", cudaGetErrorString(ea));
      return QC_ERR_CUDA;
    }
    attr_set[v] = true;
  }
  if (fiber_tile == 32) {
    k_fiber<T, 1><<<grid, FT_THREADS, smem, s>>>(tk, (const qc_fin *)fin, (const qc_fout *)fout,
                                                 (const qc_fpair *)fpair, (const qc_op *)ops, A, W, C);
  } else {
    k_fiber<T, 2><<<grid, FT_THREADS, smem, s>>>(tk, (const qc_fin *)fin, (const qc_fout *)fout,
                                                 (const qc_fpair *)fpair, (const qc_op *)ops, A, W, C);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "[qcgpu] qc_fiber: %s\n", cudaGetErrorString(e));
    return QC_ERR_CUDA;
  }
  return QC_OK;
}

}  // namespace

extern "C" int qc_block_permute(const void *descs, long long ndescs, int opspan, const void *ops, const double *src,
                                void *dst, int dst_f32, void *stream) {
  if (ndescs <= 0) return QC_OK;
  if (ndescs > 0x7fffffffLL || opspan < 1 || opspan > 65535) return QC_ERR_ARG;
  dim3 grid((unsigned)ndescs, (unsigned)opspan);
  cudaStream_t s = (cudaStream_t)stream;
  if (dst_f32)
    k_block_permute<float><<<grid, 256, 0, s>>>((const qc_bperm *)descs, (const qc_op *)ops, src, (float *)dst);
  else
    k_block_permute<double><<<grid, 256, 0, s>>>((const qc_bperm *)descs, (const qc_op *)ops, src, (double *)dst);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "[qcgpu] qc_block_permute: %s\n", cudaGetErrorString(e));
    return QC_ERR_CUDA;
  }
  return QC_OK;
}

extern "C" int qc_fiber_f64(const void *tasks, long long ntasks, int opspan, const void *fin, const void *fout,
                            const void *fpair, const void *ops, int max_rows, int fiber_tile, const double *A,
                            const double *W, double *C, void *stream) {
  return launch_fiber<double>(tasks, ntasks, opspan, fin, fout, fpair, ops, max_rows, fiber_tile, A, W, C,
                              (cudaStream_t)stream);
}

extern "C" int qc_fiber_f32(const void *tasks, long long ntasks, int opspan, const void *fin, const void *fout,
                            const void *fpair, const void *ops, int max_rows, int fiber_tile, const float *A,
                            const float *W, float *C, void *stream) {
  return launch_fiber<float>(tasks, ntasks, opspan, fin, fout, fpair, ops, max_rows, fiber_tile, A, W, C,
                             (cudaStream_t)stream);
}
