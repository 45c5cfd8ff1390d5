// Sigma product (all four contractions plus the sum over operators) for callers
// that cannot allocate device memory.
//
// Some host codes that would call this library own the whole GPU memory budget
// themselves (a parent application that pools or reserves device memory up
// front, or a solver that must not trigger cudaMalloc's implicit device-wide
// synchronisation in the middle of an iteration).  They can pass inputs and
// outputs but cannot provide the intermediate buffers that the regular sigma
// path (qc_bgemm_f64, four launches with caller-allocated scratch) needs.
// This entry point keeps those intermediates in one fixed device array that is
// part of the library image instead: nothing is allocated per call.
//
// Limits and sharing rules:
//  * only plans made entirely of packed-layout grouped-GEMM groups are accepted
//    (QC_GROUP_BGEMM: qc_task / qc_contrib records, the operands in the packed
//    block layout; in Python, SigmaOperator(use_fiber=False, panel1=False)).
//    Each group carries its kind; a plan with dense-panel or fiber-group stages
//    (the default sigma plan) reads other operands through other records and is
//    refused with QC_ERR_ARG before any work is queued.  The work lists
//    themselves are trusted: they must come from this library's plan compiler
//    for these t1 / t2 / t3 sizes;
//  * the array holds QC_NOALLOC_SCRATCH_DOUBLES doubles (32 MiB); every GPU that
//    loads the library holds that much device memory until the process exits;
//  * one call needs t1 + t2 + t3 + nops * ndim0 doubles (plus 256-byte padding
//    per region); larger problems are rejected with QC_ERR_CAPACITY before any
//    work is queued;
//  * all calls on a device share the array and it keeps the last call's
//    contents: calls that overlap on the GPU (different streams, or different
//    host threads without ordering) race on it and must be serialised by the
//    caller;
//  * the device address of the array is looked up once per device (with that
//    device current) on the first call; make that first call before any
//    stream capture begins.
#include <cuda_runtime.h>
#include <cstdio>
#include <mutex>
#include <string>
#include "qc_types.h"

#define QC_NOALLOC_SCRATCH_DOUBLES (4LL * 1024 * 1024)

static __device__ __align__(256) double g_noalloc_scratch[QC_NOALLOC_SCRATCH_DOUBLES];

int qc_internal_bgemm_f64(const void *tasks, long long ntasks, int opspan, const void *contribs, const void *ops,
                          int summed, const double *A, const double *B, double *C, int cfg, cudaStream_t s);
int qc_internal_reduce_f64(const double *part, int nops, long long n, double *out, cudaStream_t s);

static thread_local std::string g_noalloc_err;
static std::mutex g_noalloc_mu;
static double *g_noalloc_ptr[128] = {nullptr};

// Failures return a negative QC_ERR_* code and print the reason on stderr.
static int noalloc_fail(int code, const std::string &msg) {
  g_noalloc_err = msg;
  fprintf(stderr, "[qcgpu] %s\n", msg.c_str());
  return code;
}

static int scratch_base(double **out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128)
    return noalloc_fail(QC_ERR_CUDA, "qc_sigma_f64_noalloc: no current CUDA device");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return noalloc_fail(QC_ERR_CUDA, std::string("qc_sigma_f64_noalloc: cudaGetSymbolAddress: ") +
                                           cudaGetErrorString(e));
    g_noalloc_ptr[dev] = (double *)p;
  }
  *out = g_noalloc_ptr[dev];
  return QC_OK;
}

static inline long long pad256(long long n) { return (n + 31) & ~31LL; }   // 32 doubles = 256 bytes

extern "C" int qc_sigma_f64_noalloc(int ngroups, const int *group_stage, const void *const *group_tasks,
                                    const long long *group_ntasks, const int *group_opspan,
                                    const void *const *group_contribs, const int *group_cfg,
                                    const int *group_kind, const void *const *stage_ops, const double *L, const double *Wi,
                                    const double *Wj, const double *R, const double *x, double *y, int nops,
                                    long long ndim0, long long t1, long long t2, long long t3, void *stream) {
  if (ngroups < 0 || !group_stage || !group_tasks || !group_ntasks || !group_opspan || !group_contribs ||
      !group_cfg || !group_kind || !stage_ops || nops < 1 || ndim0 < 1 || t1 < 0 || t2 < 0 || t3 < 0)
    return noalloc_fail(QC_ERR_ARG, "qc_sigma_f64_noalloc: bad arguments");
  const long long need = pad256(t1) + pad256(t2) + pad256(t3) + pad256((long long)nops * ndim0);
  if (need > QC_NOALLOC_SCRATCH_DOUBLES)
    return noalloc_fail(QC_ERR_CAPACITY, "qc_sigma_f64_noalloc: this dot needs " + std::to_string(need) +
                                             " scratch doubles, the static array holds " +
                                             std::to_string(QC_NOALLOC_SCRATCH_DOUBLES));
  for (int g = 0; g < ngroups; ++g) {
    if (group_stage[g] < 0 || group_stage[g] > 3 || (g > 0 && group_stage[g] < group_stage[g - 1]))
      return noalloc_fail(QC_ERR_ARG, "qc_sigma_f64_noalloc: groups must be ordered by stage 0..3");
    if (group_kind[g] != QC_GROUP_BGEMM)
      return noalloc_fail(QC_ERR_ARG, "qc_sigma_f64_noalloc: group " + std::to_string(g) + " is of kind " +
                                          std::to_string(group_kind[g]) +
                                          "; only packed-layout grouped-GEMM plans (QC_GROUP_BGEMM) are accepted");
  }
  double *base = nullptr;
  int rc = scratch_base(&base);
  if (rc != QC_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  double *T1 = base, *T2 = T1 + pad256(t1), *T3 = T2 + pad256(t2), *P = T3 + pad256(t3);
  // the per-operator partial vectors must start at zero (blocks without contributions)
  if (cudaMemsetAsync(P, 0, sizeof(double) * (size_t)nops * (size_t)ndim0, s) != cudaSuccess)
    return noalloc_fail(QC_ERR_CUDA, "qc_sigma_f64_noalloc: cudaMemsetAsync");
  for (int g = 0; g < ngroups; ++g) {
    const int st = group_stage[g];
    const double *A = st == 0 ? L : (st == 1 ? T1 : (st == 2 ? T2 : T3));
    const double *B = st == 0 ? x : (st == 1 ? Wi : (st == 2 ? Wj : R));
    double *C = st == 0 ? T1 : (st == 1 ? T2 : (st == 2 ? T3 : P));
    rc = qc_internal_bgemm_f64(group_tasks[g], group_ntasks[g], group_opspan[g], group_contribs[g], stage_ops[st],
                               0, A, B, C, group_cfg[g], s);
    if (rc != QC_OK) return noalloc_fail(rc, "qc_sigma_f64_noalloc: kernel launch failed");
  }
  rc = qc_internal_reduce_f64(P, nops, ndim0, y, s);
  if (rc != QC_OK) return noalloc_fail(rc, "qc_sigma_f64_noalloc: reduction launch failed");
  return QC_OK;
}
