// Drop-in replacement for the reference's native block-mask routine
// (ctypes/qsym.c:5-480, loaded by source/sysutil_include.py:14-17 and called
// from source/qtensor/qtensor_util.py:70-90 with up to eight sector arrays).
//
// Same symbol, same signature, same output; the arithmetic is exact integer
// arithmetic on 2q instead of a floating-point |sum| < 1e-10 test, which is
// equivalent for quantum numbers that are multiples of 1/2 (N and Sz).
#include <cmath>
#include <vector>
#include "qc_types.h"

extern "C" int qc_sym_allowed(int rank, int nqnum, const int *nsyms, const int *status,
                              const int *qsyms2, int *allowed);

extern "C" int symAllowed(int rank, int nqnum, int *ndims, int *status, int *allowed,
                          double *a0, double *a1, double *a2, double *a3,
                          double *a4, double *a5, double *a6, double *a7) {
  double *a[8] = {a0, a1, a2, a3, a4, a5, a6, a7};
  if (rank < 1 || rank > 8 || nqnum < 1 || !ndims || !status || !allowed) return QC_ERR_ARG;
  std::vector<int> q2;
  for (int r = 0; r < rank; ++r) {
    if (!a[r] || ndims[r] <= 0) return QC_ERR_ARG;
    for (long long i = 0; i < (long long)ndims[r] * nqnum; ++i) {
      double t = 2.0 * a[r][i];
      double rt = std::nearbyint(t);
      if (std::fabs(t - rt) > 1e-8) return QC_ERR_HALFINT;
      q2.push_back((int)rt);
    }
  }
  return qc_sym_allowed(rank, nqnum, ndims, status, q2.data(), allowed);
}
