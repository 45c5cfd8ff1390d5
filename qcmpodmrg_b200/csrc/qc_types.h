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
