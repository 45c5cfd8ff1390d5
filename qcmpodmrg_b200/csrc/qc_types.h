// Work-item records shared by the plan compiler (host) and the kernels (device).
#pragma once
#include <cstdint>

// One output tile of one output block.  Element (m, n) of the block lives at
// c_off + (m / mlo) * c_mh + (m % mlo) * c_ml + (n / nlo) * c_nh + (n % nlo) * c_nl.
struct alignas(16) qc_task {
  long long c_off;
  int M, N;
  int m0, n0;
  int mlo, nlo;
  int c_mh, c_ml, c_nh, c_nl;
  int cb, ce;          // contribution range [cb, ce)
  int op_b, op_e;      // per-operator mode: operators [op_b, op_e) of the operator table
};
static_assert(sizeof(qc_task) == 64, "qc_task is 64 bytes");

// One block-pair product accumulated into every tile of its output block.
// A(m, k) at a_off + (m / mlo) * a_mh + (m % mlo) * a_ml + (k / klo) * a_kh + (k % klo) * a_kl
// B(k, n) at b_off + (k / klo) * b_kh + (k % klo) * b_kl + (n / nlo) * b_nh + (n % nlo) * b_nl
struct alignas(16) qc_contrib {
  long long a_off, b_off;
  double alpha;
  int K, klo;
  int a_mh, a_ml, a_kh, a_kl;
  int b_kh, b_kl, b_nh, b_nl;
  int op_b, op_e;      // summed mode: operators [op_b, op_e) whose products accumulate here
};
static_assert(sizeof(qc_contrib) == 80, "qc_contrib is 80 bytes");

// Per-operator base offsets of a stage: operator o reads A at a_base + a_off,
// B at b_base + b_off, writes C at c_base + c_off and scales by alpha * c.alpha.
struct alignas(16) qc_op {
  long long a_base, b_base, c_base;
  double alpha;
};
static_assert(sizeof(qc_op) == 32, "qc_op is 32 bytes");

#define QC_OK 0
#define QC_ERR_ARG -1
#define QC_ERR_CAPACITY -2
#define QC_ERR_CUDA -3
#define QC_ERR_LAYOUT -4
#define QC_ERR_HALFINT -5

// Kinds of work-item groups in a compiled plan (the records a group's task array holds).
#define QC_GROUP_BGEMM 1   // qc_task + qc_contrib (packed-layout grouped GEMM, k_bgemm)
#define QC_GROUP_PANEL 2   // qc_ptask (dense panel GEMM, k_pgemm)
#define QC_GROUP_FIBER 3   // qc_ftask + qc_fin/qc_fout/qc_fpair (fiber-group kernel, k_fiber)

// ---- fiber-group work items (the W contractions of sigma) -------------------
// A fiber group is a set of output blocks that share their "fiber" index
// f = (l, r) and read the same input blocks; one task = one tile of fibers.
struct alignas(16) qc_ftask {
  int f0, F;           // first fiber of the tile, fibers in the group
  int in_b, in_e;      // input blocks [in_b, in_e) of qc_fin
  int out_b, out_e;    // output blocks [out_b, out_e) of qc_fout
  int op_b, op_e;      // operators (grid.y indexes this range)
};
static_assert(sizeof(qc_ftask) == 32, "qc_ftask is 32 bytes");

struct alignas(16) qc_fin {
  long long a_off;     // input block offset (relative to the operator's A base)
  int rows;            // extent of the contracted index
  int fiber_major;     // 0: block stored [rows][F]; 1: stored [F][rows]
  int srow;            // first shared-memory row
  int pad;
};
static_assert(sizeof(qc_fin) == 32, "qc_fin is 32 bytes");

struct alignas(16) qc_fout {
  long long c_off;     // output block offset (relative to the operator's C base)
  int fhs;             // (f, c) at c_off + (f / flo)*fhs + (f % flo)*ncols + c, or,
  int colmajor;        // when colmajor is set, at c_off + c*F + f (block stored [ncols][F])
  int ncols;
  int pair_b, pair_e;  // contributions [pair_b, pair_e) of qc_fpair (empty: the block is zeroed)
  int flo;             // >= F for a block stored [F][ncols]
};
static_assert(sizeof(qc_fout) == 32, "qc_fout is 32 bytes");

struct alignas(16) qc_fpair {
  long long w_off;     // W block offset (relative to the operator's B base); (a, c) at w_off + a*ncols + c
  int srow;            // shared-memory rows of the input block
  int rows;
};
static_assert(sizeof(qc_fpair) == 16, "qc_fpair is 16 bytes");

// ---- block permute-copy (per-dot operand repacks) ---------------------------
// Copies one rank-3 block stored row-major [d0][d1][d2] at src_off to
// dst_off + i0*s0 + i1*s1 + i2*s2 (offsets relative to the operator's A / C base
// of the operator table; grid.y indexes the operators [op_b, op_e)).
struct alignas(16) qc_bperm {
  long long src_off, dst_off;
  int d0, d1, d2;
  int s0, s1, s2;
  int op_b, op_e;
  int pad0, pad1, pad2, pad3;
};
static_assert(sizeof(qc_bperm) == 64, "qc_bperm is 64 bytes");


// ---- dense panel GEMM work items (qc_pgemm_*) -------------------------------
// C[row(m) + n] = sum_k A[a_off + m*lda + k] * B[b_off + k*N + n] for the output
// tile rows [m0, m0+TM) x cols [n0, n0+TN) (lda = K when 0), with row(m) = c_off + m*N, or
// crow_table[crow + m] when crow >= 0 (rows scattered to separate blocks);
// offsets relative to the operator's bases; grid.y indexes the operators [op_b, op_e).
struct alignas(16) qc_ptask {
  long long a_off, b_off, c_off;
  int M, N, K;
  int m0, n0;
  int op_b, op_e;
  int crow;
  int lda;             // row stride of A (0: K)
};
static_assert(sizeof(qc_ptask) == 64, "qc_ptask is 64 bytes");

// ---- tensor-core panel GEMM work units (qc_tcpanel_*) ------------------------
// One unit = one 128-row x up-to-BN-column output tile of one operator:
//   C[row(m), n0 + n] = alpha * sum_k A[m, k] * B[n0 + n, k]    (m < m_valid, n < n_valid)
// A and B are read by TMA through tensor maps (maps[a_map], maps[b_map]) of this GPU's
// own buffers: A rows a_c1 .. a_c1+127 of operator slice a_c2, B rows b_c1 .. of slice
// b_c2, both K-major (k contiguous), nk stages of 32 k.  Epilogue, row-table form: row m
// goes to C + ops[op].c_base + crow[c_off + m] + b_c1 (rows scattered through a row table);
// segment form: the tile's columns are nseg segments (qc_tcseg records from c_off), column
// c of segment s and tile row m going to C + c_base + seg.off + (a_c1 + m) * seg.ldc + c - seg.col0.
struct alignas(16) qc_tcunit {
  int a_map, b_map;
  int a_c1, b_c1;
  int a_c2, b_c2;
  int nk;
  int m_valid;
  int n_valid;
  int op;
  int nseg, pad1;
  long long c_off;
  long long pad2;
};

struct alignas(16) qc_tcseg {
  long long off;       // element offset (relative to the operator's C base) of the segment's row 0
  int col0;            // first tile column of the segment
  int ncol;            // columns of the segment
  int ldc;             // row stride of the segment's destination
  int pad0, pad1, pad2;
};
static_assert(sizeof(qc_tcseg) == 32, "qc_tcseg is 32 bytes");
static_assert(sizeof(qc_tcunit) == 64, "qc_tcunit is 64 bytes");

// One tensor map to encode on the host (cuTensorMapEncodeTiled, FP32 elements).
struct alignas(16) qc_tmdesc {
  long long addr;        // global address, 16-byte aligned
  int rank;              // 2 .. 5
  int swizzle;           // CUtensorMapSwizzle value (3 = 128-byte swizzle)
  long long dims[5];     // elements per dimension (dimension 0 contiguous)
  long long strides[4];  // byte strides of dimensions 1 .. rank-1 (multiples of 16)
  int box[5];            // box extent per dimension (box[0] * 4 <= 128 with 128-byte swizzle)
  int pad;
};
static_assert(sizeof(qc_tmdesc) == 112, "qc_tmdesc is 112 bytes");

// ---- dense fiber-group GEMM (k_fgemm) -------------------------------------------
// Every output block of a fiber group reads every input block of the group, so one
// group is one dense product  C_g[F x CT] = A_g[F x R] . W_g[R x CT]: A_g's R rows are
// the input blocks' contracted rows, W_g's CT columns the output blocks' columns, and
// W_g is the group's W blocks laid out as one dense panel (zeros where a pair is
// absent).  A work item is one tile of fibers of one group for a range of operators.
struct alignas(16) qc_fggrp {
  long long row_b;     // first row record (qc_fgrow) of the group
  long long col_b;     // first column record (qc_fgcol) of the group
  int F;               // fibers of the group
  int R;               // rows (contracted extent summed over the input blocks)
  int CT;              // columns (summed over the output blocks)
  int CTs;             // CT padded to a multiple of mc: row stride of the W panel
  int FT;              // fibers per tile (multiple of 4): row stride of the staged A tile
  int mc;              // columns per thread tile (4 or 8)
  int flo;             // two-level fiber split of the outputs (>= F: none)
  int pad;
};
static_assert(sizeof(qc_fggrp) == 48, "qc_fggrp is 48 bytes");

struct alignas(16) qc_fgrow {
  long long off;       // A element (row, fiber f) at a_base + off + f * fs
  long long fs;
};
static_assert(sizeof(qc_fgrow) == 16, "qc_fgrow is 16 bytes");

struct alignas(16) qc_fgcol {
  long long off;       // C element (fiber f, column) at c_base + off + (f / flo) * fhs + (f % flo) * fs
  long long fhs;
  long long fs;
  long long pad;
};
static_assert(sizeof(qc_fgcol) == 32, "qc_fgcol is 32 bytes");

struct alignas(16) qc_fgitem {
  long long wpan;      // W panel of operator op_b (element offset; multiple of 4)
  int group;           // qc_fggrp index
  int f0, nf;          // first fiber of the tile, fibers in the tile (<= FT)
  int op_b, op_e;      // operators; operator op's panel is wpan + (op - op_b) * wstride
  int wstride;         // multiple of 4
};
static_assert(sizeof(qc_fgitem) == 32, "qc_fgitem is 32 bytes");

// One W block of a dense fiber-group W panel: for operators o < nops (of op_b ..), rows
// r < nr, columns j < ncol: P[dst + o * opstride + (r0 + r) * width + perm(j0 + j)] =
// W[b_base(op_b + o) + src + r * src_ld + j]; perm places column c of an 8-column thread
// tile as the kernel reads it (two 4-column halves, width / 2 apart) when mc == 8.
struct alignas(16) qc_wpair {
  long long dst, opstride, src;
  int width, mc, r0, nr, j0, ncol, src_ld, op_b, nops, pad;
};
static_assert(sizeof(qc_wpair) == 64, "qc_wpair is 64 bytes");
