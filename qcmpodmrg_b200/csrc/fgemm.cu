// Dense fiber-group GEMM for the two W contractions of sigma (the .W_i and .W_{i+1}
// stages of HVecQt, source/mpo_dmrg_kernelQt.py:301-306).
//
// In those contractions an output block (fibers f = (l, r) x columns c = MPO bond x
// physical index) is a sum over input blocks times small W blocks.  The blocks that
// share their fiber sectors form a group, and inside a group every output block reads
// every input block, so the group is one dense product
//     C_g[F x CT] = alpha * A_g[F x R] . W_g[R x CT]
// with R = the input blocks' contracted rows, CT = the output blocks' columns and
// W_g the group's W blocks laid out once per dot as a dense panel (qc_wpanel_*).
//
// A work item is one tile of FT fibers of one group for a range of operators.  A
// persistent grid of 128-thread CTAs walks the (item, operator) sequence with two
// shared-memory buffers: while one (item, operator) is multiplied, the next one's A
// tile, W panel and column records are in flight (cp.async, zero fill past the tile).
// Each thread owns 4 fibers x mc columns (mc = 4 or 8) of the C tile: per contracted
// row it reads one 16-byte A vector and mc/4 16-byte W vectors from shared memory for
// 4*mc FMAs.  Every A and C element crosses HBM once; the W panels stay in L2.
#include <cuda_runtime.h>
#include <cstdio>
#include "qc_types.h"

namespace {

constexpr int FG_THREADS = 128;

__device__ __forceinline__ void cp_async4(void *dst, const void *src, bool valid) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src, bool valid) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_elem(float *dst, const float *src, bool valid) {
  cp_async4(dst, valid ? src : nullptr, valid);
}
__device__ __forceinline__ void cp_async_elem(double *dst, const double *src, bool valid) {
  cp_async8(dst, valid ? src : nullptr, valid);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// four consecutive elements from shared memory (16-byte aligned)
__device__ __forceinline__ void lds4(const float *p, float *v) {
  const float4 a = *reinterpret_cast<const float4 *>(p);
  v[0] = a.x;
  v[1] = a.y;
  v[2] = a.z;
  v[3] = a.w;
}
__device__ __forceinline__ void lds4(const double *p, double *v) {
  const double2 a = *reinterpret_cast<const double2 *>(p), b = *reinterpret_cast<const double2 *>(p + 2);
  v[0] = a.x;
  v[1] = a.y;
  v[2] = b.x;
  v[3] = b.y;
}

// One (item, operator) step of a CTA: the item, its group and the operator's bases.
struct FgStep {
  qc_fgitem it;
  qc_fggrp g;
  long long a_base, c_base;
  double alpha;
  int op;
};

__device__ __forceinline__ void fg_load_op(FgStep &st, const qc_op *__restrict__ ops) {
  const qc_op o = ops[st.op];
  st.a_base = o.a_base;
  st.c_base = o.c_base;
  st.alpha = o.alpha;
}

// The row records a warp stages (rows warp, warp + 4, ...): lane l holds those of the
// warp's rows l and l + 32, loaded in one round trip when a new item begins.
struct FgRows {
  long long off[2], fs[2];
};

__device__ __forceinline__ void fg_load_rows(FgRows &rr, const qc_fggrp &g, const qc_fgrow *__restrict__ rows) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int r = warp + (FG_THREADS / 32) * (lane + 32 * h);
    if (r < g.R) {
      const qc_fgrow w = rows[g.row_b + r];
      rr.off[h] = w.off;
      rr.fs[h] = w.fs;
    } else {
      rr.off[h] = 0;
      rr.fs[h] = 0;
    }
  }
}

// Stage a step into one buffer: the A tile [R][FT] (row r, fiber f at
// A + a_base + row.off + (f0 + f) * row.fs; zero for f >= nf), the operator's W panel
// [R][CTs] and the group's column records.  No global load on the way: the row records
// come from the warp's registers (shuffles), the rest is cp.async.
template <typename T>
__device__ __forceinline__ void fg_stage(const FgStep &st, const FgRows &rr, const qc_fgcol *__restrict__ cols,
                                         const T *__restrict__ A, const T *__restrict__ Wp, T *as, T *ws,
                                         qc_fgcol *cs) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const qc_fggrp &g = st.g;
  const T *Ab = A + st.a_base;
  const int FT = g.FT, nf = st.it.nf;
  const int nrw = (g.R - warp + (FG_THREADS / 32) - 1) / (FG_THREADS / 32);     // rows of this warp
  for (int j = 0; j < nrw; ++j) {
    const int h = j >> 5, src_lane = j & 31;
    const long long off = __shfl_sync(0xffffffffu, h ? rr.off[1] : rr.off[0], src_lane);
    const long long fs = __shfl_sync(0xffffffffu, h ? rr.fs[1] : rr.fs[0], src_lane);
    const int r = warp + (FG_THREADS / 32) * j;
    const T *src = Ab + off + (long long)st.it.f0 * fs;
    T *dst = as + r * FT;
    for (int f = lane; f < FT; f += 32) cp_async_elem(dst + f, src + (long long)f * fs, f < nf);
  }
  const T *wsrc = Wp + st.it.wpan + (long long)(st.op - st.it.op_b) * st.it.wstride;
  const int nw16 = g.R * g.CTs * (int)sizeof(T) / 16;
  for (int e = tid; e < nw16; e += FG_THREADS)
    cp_async16(reinterpret_cast<char *>(ws) + 16 * e, reinterpret_cast<const char *>(wsrc) + 16 * e);
  const int nc16 = g.CT * (int)(sizeof(qc_fgcol) / 16);
  for (int e = tid; e < nc16; e += FG_THREADS)
    cp_async16(reinterpret_cast<char *>(cs) + 16 * e, reinterpret_cast<const char *>(cols + g.col_b) + 16 * e);
}

// One thread tile: fibers 4*fc .. 4*fc+3 of the item x columns col0 .. col0+MC-1.  The W
// panel stores an 8-column tile as two 4-column halves, half q of chunk cc at
// q * CTs/2 + 4*cc, so the chunks one load instruction reads are contiguous (no bank
// conflicts); w0 points at half 0 of the tile's chunk, qstride = CTs/2.
template <typename T, int MC>
__device__ __forceinline__ void fg_tile(const T *as, const T *w0, int qstride, const qc_fgcol *cs,
                                        const qc_fggrp &g, int f0, int nf, int fc, int col0, T alpha, T *Cb) {
  T acc[4][MC];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int c = 0; c < MC; ++c) acc[i][c] = T(0);
  const T *a = as + 4 * fc;
  const int FT = g.FT, CTs = g.CTs, R = g.R;
#pragma unroll 4
  for (int r = 0; r < R; ++r) {
    T av[4], wv[MC];
    lds4(a + r * FT, av);
#pragma unroll
    for (int q = 0; q < MC / 4; ++q) lds4(w0 + r * CTs + q * qstride, wv + 4 * q);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int c = 0; c < MC; ++c) acc[i][c] = fma(av[i], wv[c], acc[i][c]);
  }
  // fibers -> (f / flo, f % flo), advanced one fiber at a time
  const int fl0 = 4 * fc;
  const int fg0 = f0 + fl0;
  int qf[4], rf[4];
  if (g.flo >= g.F) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      qf[i] = 0;
      rf[i] = fg0 + i;
    }
  } else {
    int q = fg0 / g.flo, rm = fg0 - q * g.flo;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      qf[i] = q;
      rf[i] = rm;
      if (++rm == g.flo) {
        rm = 0;
        ++q;
      }
    }
  }
#pragma unroll
  for (int c = 0; c < MC; ++c) {
    const int col = col0 + c;
    if (col < g.CT) {
      const qc_fgcol cl = cs[col];
      T *dst = Cb + cl.off;
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (fl0 + i < nf) dst[(long long)qf[i] * cl.fhs + (long long)rf[i] * cl.fs] = alpha * acc[i][c];
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(FG_THREADS, 4)
k_fgemm(const qc_fgitem *__restrict__ items, int nitems, const qc_fggrp *__restrict__ groups,
        const qc_fgrow *__restrict__ rows, const qc_fgcol *__restrict__ cols, const qc_op *__restrict__ ops,
        int max_a, int max_w, int max_ct, const T *__restrict__ A, const T *__restrict__ Wp, T *__restrict__ C) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  qc_fgcol *const cs0 = reinterpret_cast<qc_fgcol *>(smem_raw);   // [2][max_ct]
  T *const as0 = reinterpret_cast<T *>(cs0 + 2 * max_ct);         // [2][max_a]
  T *const ws0 = as0 + 2 * max_a;                                 // [2][max_w]
  // this CTA's steps: items blockIdx.x, + gridDim.x, ..., each for its operators in order.
  // Records are fetched ahead: the next step's item and operator before the multiply, its
  // group and row records (only when a new item begins) right after it.
  const int G = (int)gridDim.x;
  int ci = blockIdx.x;
  if (ci >= nitems) return;
  FgStep cur;
  cur.it = items[ci];
  cur.op = cur.it.op_b;
  cur.g = groups[cur.it.group];
  fg_load_op(cur, ops);
  FgRows rr;
  fg_load_rows(rr, cur.g, rows);
  fg_stage<T>(cur, rr, cols, A, Wp, as0, ws0, cs0);
  cp_async_commit();
  // step 1
  FgStep nxt;
  int ni = ci;
  nxt.it = cur.it;
  nxt.g = cur.g;
  nxt.op = cur.op + 1;
  bool nxt_new = false;
  if (nxt.op >= cur.it.op_e) {
    ni = ci + G;
    nxt_new = true;
    if (ni < nitems) {
      nxt.it = items[ni];
      nxt.op = nxt.it.op_b;
      nxt.g = groups[nxt.it.group];
    }
  }
  bool has_nxt = ni < nitems;
  if (has_nxt) {
    fg_load_op(nxt, ops);
    if (nxt_new) fg_load_rows(rr, nxt.g, rows);
  }
  for (int k = 0;; ++k) {
    const int buf = k & 1;
    if (has_nxt)
      fg_stage<T>(nxt, rr, cols, A, Wp, as0 + (buf ^ 1) * max_a, ws0 + (buf ^ 1) * max_w,
                  cs0 + (buf ^ 1) * max_ct);
    cp_async_commit();
    // the step after next: item (if a new one) and operator records now
    FgStep n2;
    int n2i = ni;
    bool n2_new = false, has_n2 = false;
    if (has_nxt) {
      n2.it = nxt.it;
      n2.g = nxt.g;
      n2.op = nxt.op + 1;
      if (n2.op >= nxt.it.op_e) {
        n2i = ni + G;
        n2_new = true;
        if (n2i < nitems) {
          n2.it = items[n2i];
          n2.op = n2.it.op_b;
        }
      }
      has_n2 = n2i < nitems;
      if (has_n2 && !n2_new) fg_load_op(n2, ops);
    }
    cp_async_wait<1>();
    __syncthreads();
    {
      const qc_fggrp &g = cur.g;
      const T alpha = T(cur.alpha);
      T *Cb = C + cur.c_base;
      const T *as = as0 + buf * max_a;
      const T *ws = ws0 + buf * max_w;
      const qc_fgcol *cs = cs0 + buf * max_ct;
      const int chunks = g.CTs / g.mc;
      const int ntile = ((cur.it.nf + 3) >> 2) * chunks;
      for (int m = threadIdx.x; m < ntile; m += FG_THREADS) {
        const int fc = m / chunks, cc = m - fc * chunks;
        if (g.mc == 4) {
          fg_tile<T, 4>(as, ws + 4 * cc, 0, cs, g, cur.it.f0, cur.it.nf, fc, 4 * cc, alpha, Cb);
        } else if (sizeof(T) == 4) {
          fg_tile<T, 8>(as, ws + 4 * cc, g.CTs / 2, cs, g, cur.it.f0, cur.it.nf, fc, 8 * cc, alpha, Cb);
        } else {      // FP64: an 8-column tile as two 4-column tiles (register budget)
          fg_tile<T, 4>(as, ws + 4 * cc, 0, cs, g, cur.it.f0, cur.it.nf, fc, 8 * cc, alpha, Cb);
          fg_tile<T, 4>(as, ws + g.CTs / 2 + 4 * cc, 0, cs, g, cur.it.f0, cur.it.nf, fc, 8 * cc + 4, alpha, Cb);
        }
      }
    }
    // a new item two steps ahead: its group, operator and row records (the row records of
    // the step staged above are no longer needed)
    if (has_n2 && n2_new) {
      n2.g = groups[n2.it.group];
      fg_load_op(n2, ops);
      fg_load_rows(rr, n2.g, rows);
    }
    __syncthreads();
    if (!has_nxt) break;
    cur = nxt;
    nxt = n2;
    ni = n2i;
    has_nxt = has_n2;
  }
  cp_async_wait<0>();
}

template <typename T>
__global__ void k_wpanel(const T *__restrict__ src, const long long *__restrict__ idx, T *__restrict__ dst,
                         long long n) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long j = idx[e];
    dst[e] = j >= 0 ? src[j] : T(0);
  }
}

size_t fg_smem(int max_a, int max_w, int max_ct, size_t elem) {
  return 2 * (size_t)max_ct * sizeof(qc_fgcol) + 2 * ((size_t)max_a + (size_t)max_w) * elem;
}

template <typename T>
int launch_fgemm(const void *items, long long nitems, const void *groups, const void *rows, const void *cols,
                 const void *ops, int max_a, int max_w, int max_ct, const T *A, const T *Wp, T *C, cudaStream_t s) {
  if (nitems <= 0) return QC_OK;
  if (nitems > 0x7fffffffLL || !items || !groups || !ops || max_a < 4 || max_w < 0 || max_ct < 0 ||
      (max_a % 4) || (max_w % 4))
    return QC_ERR_ARG;
  const size_t smem = fg_smem(max_a, max_w, max_ct, sizeof(T));
  if (smem > 220 * 1024) return QC_ERR_ARG;
  static int attr_smem = 0, nsm = 0;
  if ((int)smem > attr_smem) {
    cudaError_t ea = cudaFuncSetAttribute(k_fgemm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ea != cudaSuccess) {
      fprintf(stderr, "[qcgpu] qc_fgemm: %s\n", cudaGetErrorString(ea));
      return QC_ERR_CUDA;
    }
    attr_smem = (int)smem;
  }
  if (nsm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  }
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fgemm<T>, FG_THREADS, smem);
  if (per_sm < 1) per_sm = 1;
  long long g = (long long)nsm * per_sm;
  if (g > nitems) g = nitems;
  k_fgemm<T><<<(int)g, FG_THREADS, smem, s>>>((const qc_fgitem *)items, (int)nitems, (const qc_fggrp *)groups,
                                               (const qc_fgrow *)rows, (const qc_fgcol *)cols, (const qc_op *)ops,
                                               max_a, max_w, max_ct, A, Wp, C);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "[qcgpu] qc_fgemm: %s\n", cudaGetErrorString(e));
    return QC_ERR_CUDA;
  }
  return QC_OK;
}

template <typename T>
int launch_wpanel(const T *src, const long long *idx, T *dst, long long n, cudaStream_t s) {
  if (n <= 0) return QC_OK;
  long long blocks = (n + 255) / 256;
  if (blocks > 4096) blocks = 4096;
  k_wpanel<T><<<(int)blocks, 256, 0, s>>>(src, idx, dst, n);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "[qcgpu] qc_wpanel: %s\n", cudaGetErrorString(e));
    return QC_ERR_CUDA;
  }
  return QC_OK;
}

// W panels assembled from their W blocks (one CTA per (block, operator)), into panels the
// caller zero-filled; every index is checked against the two buffers' sizes.
template <typename T>
__global__ void k_wpanel_pairs(const T *__restrict__ W, long long wsize, const qc_wpair *__restrict__ recs,
                               long long nrec, const qc_op *__restrict__ ops, T *__restrict__ P, long long psize) {
  const int o = (int)blockIdx.y;
  for (long long k = blockIdx.x; k < nrec; k += gridDim.x) {
    const qc_wpair w = recs[k];
    if (o >= w.nops) continue;
    const long long sb = ops[w.op_b + o].b_base + w.src;
    const long long db = w.dst + (long long)o * w.opstride;
    const int n = w.nr * w.ncol, half = w.width >> 1;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      const int r = e / w.ncol, j = e - r * w.ncol;
      const int c = w.j0 + j;
      const int pc = (w.mc == 8) ? ((c & 7) >> 2) * half + (c >> 3) * 4 + (c & 3) : c;
      const long long d = db + (long long)(w.r0 + r) * w.width + pc;
      const long long si = sb + (long long)r * w.src_ld + j;
      if (d >= 0 && d < psize && si >= 0 && si < wsize) P[d] = W[si];
    }
  }
}

template <typename T>
int launch_wpanel_pairs(const T *W, long long wsize, const void *recs, long long nrec, int maxops, const void *ops,
                        T *P, long long psize, cudaStream_t s) {
  if (nrec <= 0) return QC_OK;
  if (!W || !recs || !ops || !P || maxops < 1 || maxops > 65535 || wsize < 0 || psize < 0) return QC_ERR_ARG;
  const long long gx = nrec < (1LL << 30) ? nrec : (1LL << 30);
  k_wpanel_pairs<T><<<dim3((unsigned)gx, (unsigned)maxops), 128, 0, s>>>(W, wsize, (const qc_wpair *)recs, nrec,
                                                                         (const qc_op *)ops, P, psize);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "[qcgpu] qc_wpanel_pairs: %s\n", cudaGetErrorString(e));
    return QC_ERR_CUDA;
  }
  return QC_OK;
}

}  // namespace

extern "C" int qc_wpanel_pairs_f64(const double *W, long long wsize, const void *recs, long long nrec, int maxops,
                                   const void *ops, double *P, long long psize, void *stream) {
  return launch_wpanel_pairs<double>(W, wsize, recs, nrec, maxops, ops, P, psize, (cudaStream_t)stream);
}

extern "C" int qc_wpanel_pairs_f32(const float *W, long long wsize, const void *recs, long long nrec, int maxops,
                                   const void *ops, float *P, long long psize, void *stream) {
  return launch_wpanel_pairs<float>(W, wsize, recs, nrec, maxops, ops, P, psize, (cudaStream_t)stream);
}

extern "C" int qc_fgemm_f64(const void *items, long long nitems, const void *groups, const void *rows,
                            const void *cols, const void *ops, int max_a, int max_w, int max_ct, const double *A,
                            const double *Wp, double *C, void *stream) {
  return launch_fgemm<double>(items, nitems, groups, rows, cols, ops, max_a, max_w, max_ct, A, Wp, C,
                              (cudaStream_t)stream);
}

extern "C" int qc_fgemm_f32(const void *items, long long nitems, const void *groups, const void *rows,
                            const void *cols, const void *ops, int max_a, int max_w, int max_ct, const float *A,
                            const float *Wp, float *C, void *stream) {
  return launch_fgemm<float>(items, nitems, groups, rows, cols, ops, max_a, max_w, max_ct, A, Wp, C,
                             (cudaStream_t)stream);
}

extern "C" int qc_wpanel_f64(const double *src, const long long *idx, double *dst, long long n, void *stream) {
  return launch_wpanel<double>(src, idx, dst, n, (cudaStream_t)stream);
}

extern "C" int qc_wpanel_f32(const float *src, const long long *idx, float *dst, long long n, void *stream) {
  return launch_wpanel<float>(src, idx, dst, n, (cudaStream_t)stream);
}
