/*
 * qcmpodmrg_b200 -- C ABI of the B200 two-site MPO-DMRG hot path.
 *
 * Two shared libraries are built from qcmpodmrg_b200/csrc:
 *   libqsym.so   drop-in for the reference's ctypes/qsym.c (same symbol, same
 *                signature), loaded by source/sysutil_include.py:14-17.
 *   libqcgpu.so  block maps, plan compiler and the sm_100a kernels.
 *
 * Conventions: plain pointers and sizes; device pointers are CUDA device
 * addresses; `stream` is a cudaStream_t passed as void*.  Every function
 * returns an int status (QC_OK = 0, negative on error) except where a count is
 * documented; qc_last_error() returns the message of the last failure on the
 * calling thread.  Nothing here calls exit().
 */
#ifndef QCMPODMRG_B200_H
#define QCMPODMRG_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define QC_OK 0
#define QC_ERR_ARG -1
#define QC_ERR_CAPACITY -2
#define QC_ERR_CUDA -3
#define QC_ERR_LAYOUT -4
#define QC_ERR_HALFINT -5

/* Kinds of work-item groups in a compiled plan. */
#define QC_GROUP_BGEMM 1   /* qc_task + qc_contrib (packed-layout grouped GEMM) */
#define QC_GROUP_PANEL 2   /* qc_ptask (dense panel GEMM) */
#define QC_GROUP_FIBER 3   /* qc_ftask + qc_fin / qc_fout / qc_fpair (fiber-group kernel) */

/* ---------------------------------------------------------------- libqsym.so */

/* Replaces ctypes/qsym.c:5-22 symAllowed (and symAllowed2..8, :24-480).
 * allowed[idx] = 1 iff sum_{status[i]==0} q_i - sum_{status[i]==1} q_i == 0
 * over the row-major Cartesian product of the sectors of a0..a(rank-1)
 * (each a_i is [ndims[i]][nqnum] doubles).  Quantum numbers must be
 * multiples of 1/2; the comparison is done exactly on 2q as integers.
 * Unlike the reference, rank 8 iterates its last index over ndims[7]
 * (qsym.c:436 loops over ndims[6]).  Returns 0, or QC_ERR_* without exiting. */
int symAllowed(int rank, int nqnum, int *ndims, int *status, int *allowed,
               double *a0, double *a1, double *a2, double *a3,
               double *a4, double *a5, double *a6, double *a7);

/* ---------------------------------------------------------------- libqcgpu.so */

int qc_version(void);
const char *qc_last_error(void);

/* Integer allowed-block mask (the same map as symAllowed, on 2q as int32).
 * qsyms2: concatenation over i of [nsyms[i]][nqnum] int32 values of 2q.
 * Replaces qtensor_util.blks_allowed1 (source/qtensor/qtensor_util.py:70-90). */
int qc_sym_allowed(int rank, int nqnum, const int *nsyms, const int *status,
                   const int *qsyms2, int *allowed);

/* Same mask computed on the GPU (qsyms2_dev, allowed_dev device pointers). */
int qc_sym_allowed_gpu(int rank, int nqnum, const int *nsyms, const int *status,
                       const int *qsyms2_dev, int *allowed_dev, void *stream);

/* Packed layout of a block-sparse tensor: replaces qtensor.fromQsyms
 * (source/qtensor/qtensor.py:272-346).  ndims: concatenation over i of the
 * nsyms[i] sector dimensions.  Outputs over nblks = prod(nsyms):
 * iblks (1-based index of allowed blocks, 0 otherwise), ioff (packed offset,
 * 0 for forbidden blocks), ndim (block size, for all blocks).
 * *size_allowed and *nallowed receive the totals. */
int qc_block_layout(int rank, const int *nsyms, const long long *ndims,
                    const int *allowed, int *iblks, long long *ioff, long long *ndim,
                    long long *size_allowed, long long *nallowed);

/* Davidson-diagonal gather map of a two-site wavefunction layout (rank 4: l, n1, n2, r with
 * four 1-dim physical sectors): gat[packed position] = index into the dense diagonal
 * [16][ldim][rdim], every index numbered sector by sector (HDiagQt's diag[prjmap],
 * source/mpo_dmrg_kernelQt.py:119-122).  blocks: the nblk allowed flat block indices; ndims:
 * the sector sizes of the four indices back to back; ioff: packed offset of every flat block;
 * size: the layout's element count (bounds check).  Host function. */
int qc_psi_diag_gather(long long nblk, const long long *blocks, const int *nsyms,
                       const long long *ndims, const long long *ioff, long long ldim,
                       long long rdim, long long size, long long *gat);

/* Block-pair list of a contraction: replaces the pair loop of
 * qtensor.tensordotSYM (source/qtensor/qtensor.py:617-636).  For every
 * allowed output block (out_iblks over the external sectors e1+e2, row-major)
 * and every internal sector tuple (row-major over the contracted axes in the
 * order of ax1) with both input blocks allowed, writes one triple
 * (out_block, in1_block, in2_block) of flat block indices.
 * Returns the number of triples (written only if <= cap), or < 0 on error. */
long long qc_contract_pairs(int r1, const int *nsyms1, const int *iblks1,
                            int r2, const int *nsyms2, const int *iblks2,
                            int nax, const int *ax1, const int *ax2,
                            const int *out_iblks, long long *triples, long long cap);

/* Plan compiler: turns pair triples into GPU work items for qc_bgemm_*.
 * Each operand (1, 2, out) is described by its sector grid nsyms[rank], the
 * concatenated sector dimensions ndims (int64) and the per-block packed
 * offsets off[nblks] (from qc_block_layout).  For each operator o (nops of
 * them) the element offsets base1[o], base2[o], baseo[o] are added and the
 * product is scaled by alpha[o].  group_ops != 0 merges the contributions of
 * all operators into one output (sum over o, used for sigma).  tile_m/tile_n
 * is the output tile.  Writes up to task_cap tasks (qc_task, 64 B) and
 * contrib_cap contributions (qc_contrib, 80 B).  Returns the number of
 * contributions and stores the number of tasks in *ntasks and the algorithmic
 * FLOP count (2*M*N*K summed over contributions) in *flops; if a capacity is
 * too small nothing is written and the required counts are returned. */
long long qc_compile_pairs(int r1, const int *nsyms1, const long long *ndims1, const long long *off1,
                           int r2, const int *nsyms2, const long long *ndims2, const long long *off2,
                           int ro, const int *nsymso, const long long *ndimso, const long long *offo,
                           int nax, const int *ax1, const int *ax2,
                           long long npairs, const long long *triples,
                           int nops, const long long *base1, const long long *base2,
                           const long long *baseo, const double *alpha, int group_ops,
                           int tile_m, int tile_n,
                           void *tasks, long long task_cap, void *contribs, long long contrib_cap,
                           long long *ntasks, double *flops);

/* Grouped block GEMM, FP64 (DFMA): the engine behind one stage of HVecQt /
 * renormQt_H00 / HDiagQt (source/mpo_dmrg_kernelQt.py:238-317, 642-697,
 * 77-119), i.e. the tensordotCAL loop (source/qtensor/qtensor.py:642-659) for
 * all operators and block pairs of a stage in one launch.
 * tasks (qc_task, 64 B), contribs (qc_contrib, 80 B) and ops (qc_op, 32 B:
 * a_base, b_base, c_base, alpha per operator) are device arrays; the layout
 * is documented in qcmpodmrg_b200/csrc/qc_types.h.
 * summed == 0: each task writes one tile per operator of its range; the grid
 *              is ntasks x opspan CTAs, opspan = the longest operator range;
 * summed != 0: each task writes one tile summed over the operators of every
 * contribution's range (opspan ignored).
 * tile_cfg: output tile / threads: 0 = 64x64/256, 1 = 128x32/256, 2 = 256x16/256,
 * 3 = 32x32/64, 4 = 64x16/64, 5 = 128x64/256. */
int qc_bgemm_f64(const void *tasks_dev, long long ntasks, int opspan, const void *contribs_dev,
                 const void *ops_dev, int summed, const double *A, const double *B, double *C,
                 int tile_cfg, void *stream);

/* Same engine with FP32 operands and FP32 accumulation (mixed-precision sigma). */
int qc_bgemm_f32(const void *tasks_dev, long long ntasks, int opspan, const void *contribs_dev,
                 const void *ops_dev, int summed, const float *A, const float *B, float *C,
                 int tile_cfg, void *stream);

/* The same contraction on the 5th-generation tensor cores: tcgen05.mma
 * kind::tf32 with FP32 accumulators in tensor memory, FP32 operands rounded to
 * TF32 when staged in shared memory, FP32 output.  Per-operator mode only
 * (summed must be 0) and only tile_cfg 5 (128 x 64 output tiles).  Waits are
 * bounded; a timed-out wait is reported by qc_tc_status(). */
int qc_bgemm_tf32(const void *tasks_dev, long long ntasks, int opspan, const void *contribs_dev,
                  const void *ops_dev, int summed, const float *A, const float *B, float *C,
                  int tile_cfg, void *stream);

/* Same as qc_bgemm_tf32 with split operands: each FP32 value x is staged as
 * hi = tf32(x) and lo = tf32(x - hi), and the tile accumulates
 * hi*hi + hi*lo + lo*hi (three tcgen05.mma per K-step), which keeps FP32-level
 * accuracy (relative error about 2^-21) on the tensor cores. */
int qc_bgemm_tf32x3(const void *tasks_dev, long long ntasks, int opspan, const void *contribs_dev,
                    const void *ops_dev, int summed, const float *A, const float *B, float *C,
                    int tile_cfg, void *stream);

/* Dense panel GEMM: for every task (qc_ptask, 64 B) and operator o in
 * [op_b, op_e) (grid.y, at most opspan):
 *   C[o.c_base + row(m) + n] = o.alpha * sum_k A[o.a_base + a_off + m*K + k] * B[o.b_base + b_off + k*N + n]
 * for the tile m0 <= m < m0+128, n0 <= n < n0+TN, where row(m) = c_off + m*N, or
 * crow[task.crow + m] (device int64 table, may be null if unused) when task.crow >= 0.
 * Used for the L.psi and .R
 * contractions of HVecQt (source/mpo_dmrg_kernelQt.py:301, 306-316) once L and R
 * are permuted into per-sector panels (qc_block_permute).  tile_cfg: 0 = 128x64,
 * 1 = 128x32, 2 = 128x16. */
int qc_pgemm_f64(const void *tasks_dev, long long ntasks, int opspan, const void *ops_dev,
                 const long long *crow_dev, const double *A, const double *B, double *C, int tile_cfg,
                 void *stream);
int qc_pgemm_f32(const void *tasks_dev, long long ntasks, int opspan, const void *ops_dev,
                 const long long *crow_dev, const float *A, const float *B, float *C, int tile_cfg,
                 void *stream);

/* 0 if no tensor-core launch has reported a timed-out wait, 1 otherwise
 * (synchronous: reads a device flag), negative on a CUDA error. */
int qc_tc_status(void);

/* Fiber-group contraction for the two MPO-site contractions of HVecQt
 * (the .W_i and .W_{i+1} tensordots, source/mpo_dmrg_kernelQt.py:301-306; a
 * specialisation of tensordotCAL, source/tools/qtensor.py:623-660, for an
 * operand-2 block that is a small MPO-bond x MPO-bond matrix).
 *
 * For every task (qc_ftask, 32 B): fibers f0 .. min(f0+32, F) of one fiber group,
 * operators op_b .. op_e (grid.y, at most opspan).  Input blocks fin[in_b..in_e)
 * (qc_fin, 32 B: offset, rows, storage order [rows][F] or [F][rows], first row in
 * the staged tile) are staged once; each output block fout[out_b..out_e)
 * (qc_fout, 32 B: offset, fiber strides fhs/flo, column-major flag, ncols, pair range)
 * is written as
 *   C[c_base + c_off + (f/flo)*fhs + (f%flo)*ncols + c]      (colmajor = 0)
 *   C[c_base + c_off + c*F + f]                              (colmajor = 1)
 *       = alpha * sum_pairs sum_r in[srow+r][f] * W[b_base + w_off + r*ncols + c]
 * (an empty pair range writes zeros)
 * with pairs fpair[pair_b..pair_e) (qc_fpair, 16 B).  fiber_tile (32 or 64) is
 * the number of fibers per task (the tasks' f0 step); max_rows >= the staged rows
 * of every task (shared memory max_rows*fiber_tile*sizeof(T), at most 200 KiB).
 * Null A/W/C with absolute element addresses in ops is allowed. */
/* Per-dot operand repack: for every descriptor (qc_bperm, 64 B) and operator
 * o in [op_b, op_e) (grid.y, at most opspan), copies the block stored row-major
 * [d0][d1][d2] at src + ops[o].a_base + src_off to
 * dst + ops[o].c_base + dst_off + i0*s0 + i1*s1 + i2*s2, converting to FP32 when
 * dst_f32 != 0.  Used to lay environments out as the contiguous GEMM panels of
 * the sigma contractions (a permutation of the blocks of the reference's packed
 * qtensor.value, source/tools/qtensor.py:272-346). */
int qc_block_permute(const void *descs_dev, long long ndescs, int opspan, const void *ops_dev,
                     const double *src, void *dst, int dst_f32, void *stream);

int qc_fiber_f64(const void *tasks_dev, long long ntasks, int opspan, const void *fin_dev,
                 const void *fout_dev, const void *fpair_dev, const void *ops_dev, int max_rows,
                 int fiber_tile, const double *A, const double *W, double *C, void *stream);
int qc_fiber_f32(const void *tasks_dev, long long ntasks, int opspan, const void *fin_dev,
                 const void *fout_dev, const void *fpair_dev, const void *ops_dev, int max_rows,
                 int fiber_tile, const float *A, const float *W, float *C, void *stream);

/* Dense fiber-group GEMM (default form of the .W_i / .W_{i+1} contractions,
 * kernelQt.py:301-306): inside a fiber group every output block reads every input block,
 * so group g is C_g[F x CT] = alpha * A_g[F x R] . W_g[R x CT].  items_dev: qc_fgitem
 * records (32 B: one tile of fibers of one group, a range of operators); groups_dev:
 * qc_fggrp (48 B); rows_dev: qc_fgrow (16 B, A_g row r at a_base + off + f * fs);
 * cols_dev: qc_fgcol (32 B, C_g column at c_base + off + (f / flo) * fhs + (f % flo) * fs);
 * Wp: the W panels (qc_wpanel_*).  max_a / max_w (multiples of 4) and max_ct bound the
 * items' staged A tile (R x FT), W panel (R x CTs) and columns.  Persistent CTAs of 128
 * threads, two cp.async buffers.  Returns QC_ERR_ARG when the buffers exceed 220 KB of
 * shared memory. */
int qc_fgemm_f64(const void *items_dev, long long nitems, const void *groups_dev, const void *rows_dev,
                 const void *cols_dev, const void *ops_dev, int max_a, int max_w, int max_ct, const double *A,
                 const double *Wp, double *C, void *stream);
int qc_fgemm_f32(const void *items_dev, long long nitems, const void *groups_dev, const void *rows_dev,
                 const void *cols_dev, const void *ops_dev, int max_a, int max_w, int max_ct, const float *A,
                 const float *Wp, float *C, void *stream);
/* W panels of the dense fiber-group GEMM: dst[i] = idx[i] >= 0 ? src[idx[i]] : 0 (once per dot). */
int qc_wpanel_f64(const double *src, const long long *idx_dev, double *dst, long long n, void *stream);
int qc_wpanel_f32(const float *src, const long long *idx_dev, float *dst, long long n, void *stream);
/* W panels of the dense fiber-group GEMM assembled from their W blocks (the form the plan
 * compiler emits; the W blocks are those of the pair lists of tensordotSYM for
 * top2 = tensordot(top1, W_i) / top3 = tensordot(top2, W_j), kernelQt.py:301-306):
 * recs_dev holds nrec qc_wpair records (64 B; see qc_types.h), maxops the largest operator
 * count of a record, ops_dev the stage's operator table (b_base: the operator's W).  P
 * (psize elements) must be zero-filled by the caller; W holds wsize elements.  Indices
 * outside either buffer are skipped. */
int qc_wpanel_pairs_f64(const double *W, long long wsize, const void *recs_dev, long long nrec, int maxops,
                        const void *ops_dev, double *P, long long psize, void *stream);
int qc_wpanel_pairs_f32(const float *W, long long wsize, const void *recs_dev, long long nrec, int maxops,
                        const void *ops_dev, float *P, long long psize, void *stream);

/* ---------------------------------------------- tensor-core panel GEMM (TMA + tcgen05)
 * Replaces the pair loops of top1 = tensordot(L, psi) and top4 = tensordot(top3, R)
 * (source/mpo_dmrg_kernelQt.py:269-273, 302-306; tensordotCAL, qtensor.py:642-659) in the
 * split-TF32 precision: per work unit (qc_tcunit, 64 B) a 128-row tile C = A . B^T with A
 * and B read by TMA through tensor maps (maps_dev: CUtensorMap records encoded by
 * qc_tmap_encode) of this GPU's own buffers, K-major, 128-byte swizzle; FP32 output. */
/* Encodes n tensor maps (qc_tmdesc records, FP32 elements) into out_maps (n x 128 bytes, host). */
int qc_tmap_encode(int n, const void *descs, void *out_maps);
/* Row form: A raw FP32 (split into TF32 hi/lo in the kernel), B pre-split planes; row m of a
 * unit goes to C + ops[op].c_base + crow[c_off + m] + b_c1 (the .R contraction into sigma). */
int qc_tcpanel_f32(const void *units_dev, long long nunits, const void *maps_dev, const void *ops_dev,
                   const long long *crow_dev, float *C, void *stream);
/* Segment form: A and B pre-split planes; a unit's columns are nseg qc_tcseg segments, each
 * with its own destination and row stride (the L.psi contraction into the T1 panels). */
int qc_tcpanel_seg_f32(const void *units_dev, long long nunits, const void *maps_dev, const void *ops_dev,
                       const void *segs_dev, float *C, void *stream);
/* hi[i] = tf32(x[i]) in place, lo[i] = tf32(x[i] - hi[i]) (n values). */
int qc_tf32_split(float *hi, float *lo, long long n, void *stream);
/* hi[i] = tf32(x[idx[i]]), lo[i] = tf32(x[idx[i]] - hi[i]) from an FP64 vector (idx < 0: 0). */
int qc_gather_split_f32(const double *x, const long long *idx, long long n, float *hi, float *lo, void *stream);
/* 1 if a tensor-core panel launch reported a timed-out wait since the last clear, else 0. */
int qc_tcpanel_status(int clear);

/* dst[i] = src[idx[i]] (FP64), i < n.  Used for diag[prjmap] (kernelQt.py:122) and, with
 * spin projection, for projectionNMs of the N-symmetry sigma back to the (N, Sz) layout
 * (qtensor.py:546-560, called at kernelQt.py:310 and :445). */
int qc_gather_f64(const double *src, const long long *idx, double *dst, long long n, void *stream);
/* dst[idx[i]] = src[i] (FP64) after zeroing dst[0..ndst).  With spin projection this is
 * reduceQsymsToN of the wavefunction and of site tensors (qtensor.py:528-543, called at
 * kernelQt.py:160, :382, :638 and :775): the same elements, zero in the blocks that only
 * N symmetry allows. */
int qc_scatter_f64(const double *src, const long long *idx, double *dst, long long n,
                   long long ndst, void *stream);

/* out[i] = sum_{o < nops} part[o*n + i] in fixed order (per-operator partial sigma
 * vectors -> sigma; the sum over p of HVecQt, kernelQt.py:316). */
int qc_reduce_ops_f64(const double *part, int nops, long long n, double *out, void *stream);
int qc_reduce_ops_f32(const float *part, int nops, long long n, float *out, void *stream);

/* Precision conversions used by the mixed-precision path. */
int qc_convert_f64_to_f32(const double *src, float *dst, long long n, void *stream);
int qc_convert_f32_to_f64(const float *src, double *dst, long long n, void *stream);

/* ---------------------------------------------- learned Davidson preconditioner
 * No counterpart in the reference; it plugs in where pdvdson applies its
 * diagonal preconditioner (source/tools/pdvdson.py:275-278).  A 3-layer MLP
 * (F inputs <= 32, width 256, 2 outputs) with BF16 weights [out][in] and FP32
 * biases, activations and accumulation.  All pointers are device pointers. */
/* Y[B,2] = MLP(X[B,F]); H1, H2 [B,256] receive the hidden activations. */
int qc_mlp_forward(int B, int F, const float *X, const void *W1, const float *b1, const void *W2,
                   const float *b2, const void *W3, const float *b3, float *H1, float *H2, float *Y,
                   void *stream);
/* Accumulates (+=) the FP32 gradients of every weight and bias for dL/dY[B,2]. */
int qc_mlp_backward(int B, int F, const float *X, const void *W2, const void *W3, const float *H1,
                    const float *H2, const float *dY, float *dW1, float *db1, float *dW2, float *db2,
                    float *dW3, float *db3, void *stream);
/* One Adam step on FP32 master weights w (n values); refreshes the BF16 copy wbf16 if non-NULL. */
int qc_adam_step(int n, float *w, void *wbf16, const float *g, float *m, float *v, float lr, float beta1,
                 float beta2, float eps, int step, float grad_scale, void *stream);
/* c[i] = r[i] * exp(Y[2b]) / (|d[i] - e| + exp(Y[2b+1])), b = blk[i]  (FP64 vectors). */
int qc_precond_apply(long long n, const double *r, const double *d, double e, const int *blk,
                     const float *Y, double *c, void *stream);

/* Sigma without any device allocation.  This entry point has no counterpart in
 * the reference; it exists for host codes that own the GPU memory budget and
 * cannot hand out intermediate buffers (or must not trigger cudaMalloc's
 * device-wide synchronisation mid-iteration).  It runs the same four
 * qc_bgemm_f64 contractions and the operator sum as the regular path, with the
 * intermediates held in a fixed 32 MiB device array inside the library
 * (present on every GPU that loads it, until process exit).
 * Only plans whose every group is a packed-layout grouped GEMM are accepted
 * (group_kind[g] == QC_GROUP_BGEMM; in Python SigmaOperator(use_fiber=False,
 * panel1=False), see SigmaOperator.work_groups).  The default sigma plan, with
 * dense-panel and fiber-group stages, is refused with QC_ERR_ARG before any
 * work is queued.  The work lists are trusted as compiled by this library for
 * the given t1 / t2 / t3.
 *   groups: ngroups work-item groups of the compiled sigma plan, ordered by
 *     stage 0..3 (L.psi, .W_i, .W_{i+1}, .R); for each: stage, device task and
 *     contribution arrays, task count, operator span, tile configuration, kind;
 *   stage_ops[4]: device operator tables of the four stages;
 *   L, Wi, Wj, R: device environment / site-operator values; x: device input;
 *   y: device output (ndim0 doubles); t1, t2, t3: intermediate sizes (doubles).
 * Needs t1 + t2 + t3 + nops*ndim0 doubles (each region padded to 256 bytes);
 * larger dots return QC_ERR_CAPACITY before queueing any work.  All calls on a
 * device share the array and leave their data in it: calls that overlap on the
 * GPU race and must be serialised by the caller.  The first call on each device
 * looks up the array's device address with that device current; make it before
 * any stream capture.  Allocates nothing (no cudaMalloc/cudaFree). */
int qc_sigma_f64_noalloc(int ngroups, const int *group_stage, const void *const *group_tasks,
                         const long long *group_ntasks, const int *group_opspan,
                         const void *const *group_contribs, const int *group_cfg,
                         const int *group_kind, const void *const *stage_ops, const double *L,
                         const double *Wi,
                         const double *Wj, const double *R, const double *x, double *y, int nops,
                         long long ndim0, long long t1, long long t2, long long t3, void *stream);

#ifdef __cplusplus
}
#endif
#endif
