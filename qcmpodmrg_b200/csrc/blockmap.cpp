// Host-side block maps and plan compiler (integer arithmetic only).
//
// qc_sym_allowed    <- ctypes/qsym.c:5-480 / qtensor_util.py:70-90 (mask of allowed blocks)
// qc_block_layout   <- source/qtensor/qtensor.py:272-346 (fromQsyms packed layout)
// qc_contract_pairs <- source/qtensor/qtensor.py:563-637 (tensordotSYM pair list)
// qc_compile_pairs  <- the tensordotCAL loop (qtensor.py:642-659), re-expressed as
//                      GPU work items (one task per output tile, one contribution
//                      per block pair) for every operator of a stage at once.
#include <cstring>
#include <string>
#include <vector>
#include <cmath>
#include "qc_types.h"

static thread_local std::string g_err;
static int set_err(int code, const std::string &msg) { g_err = msg; return code; }

extern "C" const char *qc_last_error(void) { return g_err.c_str(); }
extern "C" int qc_version(void) { return 1; }

// Row-major odometer over `rank` indices with extents n[].
static inline bool odo_next(std::vector<int> &i, const int *n, int rank) {
  for (int r = rank - 1; r >= 0; --r) {
    if (++i[r] < n[r]) return true;
    i[r] = 0;
  }
  return false;
}

extern "C" int qc_sym_allowed(int rank, int nqnum, const int *nsyms, const int *status,
                              const int *qsyms2, int *allowed) {
  if (rank < 1 || rank > 16 || nqnum < 1 || nqnum > 4 || !nsyms || !status || !qsyms2 || !allowed)
    return set_err(QC_ERR_ARG, "qc_sym_allowed: bad arguments");
  std::vector<long long> first(rank + 1, 0);
  long long nblks = 1;
  for (int r = 0; r < rank; ++r) {
    if (nsyms[r] <= 0) {
      return set_err(QC_ERR_ARG, "qc_sym_allowed: empty index");
    }
    first[r + 1] = first[r] + nsyms[r];
    nblks *= nsyms[r];
  }
  // Partial sums along the odometer: acc[r][q] = sum over indices < r.
  std::vector<int> idx(rank, 0);
  std::vector<long long> acc((rank + 1) * nqnum, 0);
  auto refresh = [&](int from) {
    for (int r = from; r < rank; ++r) {
      const int *q = qsyms2 + (first[r] + idx[r]) * nqnum;
      int sgn = status[r] ? -1 : 1;
      for (int k = 0; k < nqnum; ++k) acc[(r + 1) * nqnum + k] = acc[r * nqnum + k] + sgn * q[k];
    }
  };
  refresh(0);
  for (long long b = 0; b < nblks; ++b) {
    int ok = 1;
    for (int k = 0; k < nqnum; ++k) ok &= (acc[rank * nqnum + k] == 0);
    allowed[b] = ok;
    // advance odometer, recompute partial sums from the changed digit
    int r = rank - 1;
    while (r >= 0) {
      if (++idx[r] < nsyms[r]) break;
      idx[r] = 0;
      --r;
    }
    if (r < 0) break;
    refresh(r);
  }
  return QC_OK;
}

extern "C" int qc_block_layout(int rank, const int *nsyms, const long long *ndims, const int *allowed,
                               int *iblks, long long *ioff, long long *ndim, long long *size_allowed,
                               long long *nallowed) {
  if (rank < 1 || !nsyms || !ndims || !allowed || !iblks || !ioff || !ndim)
    return set_err(QC_ERR_ARG, "qc_block_layout: bad arguments");
  std::vector<long long> first(rank + 1, 0);
  long long nblks = 1;
  for (int r = 0; r < rank; ++r) { first[r + 1] = first[r] + nsyms[r]; nblks *= nsyms[r]; }
  std::vector<int> idx(rank, 0);
  long long off = 0, na = 0;
  for (long long b = 0; b < nblks; ++b) {
    long long sz = 1;
    for (int r = 0; r < rank; ++r) sz *= ndims[first[r] + idx[r]];
    ndim[b] = sz;
    if (allowed[b]) {
      iblks[b] = (int)(b + 1);
      ioff[b] = off;
      off += sz;
      ++na;
    } else {
      iblks[b] = 0;
      ioff[b] = 0;
    }
    odo_next(idx, nsyms, rank);
  }
  if (size_allowed) *size_allowed = off;
  if (nallowed) *nallowed = na;
  return QC_OK;
}

extern "C" long long qc_contract_pairs(int r1, const int *nsyms1, const int *iblks1,
                                       int r2, const int *nsyms2, const int *iblks2,
                                       int nax, const int *ax1, const int *ax2,
                                       const int *out_iblks, long long *triples, long long cap) {
  if (r1 < 1 || r2 < 1 || nax < 0 || nax > r1 || nax > r2)
    return set_err(QC_ERR_ARG, "qc_contract_pairs: bad ranks");
  std::vector<int> in1(r1, 0), in2(r2, 0);
  for (int j = 0; j < nax; ++j) {
    if (ax1[j] < 0 || ax1[j] >= r1 || ax2[j] < 0 || ax2[j] >= r2 || nsyms1[ax1[j]] != nsyms2[ax2[j]])
      return set_err(QC_ERR_ARG, "qc_contract_pairs: bad axes");
    in1[ax1[j]] = 1; in2[ax2[j]] = 1;
  }
  std::vector<int> e1, e2, ns_ext, ns_int;
  for (int i = 0; i < r1; ++i) if (!in1[i]) e1.push_back(i);
  for (int i = 0; i < r2; ++i) if (!in2[i]) e2.push_back(i);
  for (int i : e1) ns_ext.push_back(nsyms1[i]);
  for (int i : e2) ns_ext.push_back(nsyms2[i]);
  for (int j = 0; j < nax; ++j) ns_int.push_back(nsyms1[ax1[j]]);
  // row-major strides of the input block grids
  std::vector<long long> st1(r1), st2(r2);
  { long long s = 1; for (int i = r1 - 1; i >= 0; --i) { st1[i] = s; s *= nsyms1[i]; } }
  { long long s = 1; for (int i = r2 - 1; i >= 0; --i) { st2[i] = s; s *= nsyms2[i]; } }
  const int rout = (int)ns_ext.size();
  long long nout = 1;
  for (int n : ns_ext) nout *= n;
  long long nint = 1;
  for (int n : ns_int) nint *= n;
  long long cnt = 0;
  std::vector<int> oi(rout > 0 ? rout : 1, 0), ii(nax > 0 ? nax : 1, 0);
  for (long long ob = 0; ob < nout; ++ob) {
    if (rout == 0 || out_iblks[ob]) {
      long long base1 = 0, base2 = 0;
      for (size_t k = 0; k < e1.size(); ++k) base1 += oi[k] * st1[e1[k]];
      for (size_t k = 0; k < e2.size(); ++k) base2 += oi[e1.size() + k] * st2[e2[k]];
      std::fill(ii.begin(), ii.end(), 0);
      for (long long ib = 0; ib < nint; ++ib) {
        long long b1 = base1, b2 = base2;
        for (int j = 0; j < nax; ++j) { b1 += ii[j] * st1[ax1[j]]; b2 += ii[j] * st2[ax2[j]]; }
        int v1 = iblks1[b1], v2 = iblks2[b2];
        if (v1 && v2) {
          if (cnt < cap && triples) {
            triples[3 * cnt] = ob;
            triples[3 * cnt + 1] = v1 - 1;
            triples[3 * cnt + 2] = v2 - 1;
          }
          ++cnt;
        }
        if (nax > 0) odo_next(ii, ns_int.data(), nax);
      }
    }
    if (rout > 0) odo_next(oi, ns_ext.data(), rout);
  }
  return cnt;
}

// ----------------------------------------------------------------------------
// Plan compiler
// ----------------------------------------------------------------------------
namespace {
struct IdxMap {   // up to two non-trivial axes: index = hi * lo_ext + lo
  int ext = 1, lo_ext = 1;
  long long s_hi = 0, s_lo = 0;
};

// Row-major strides of a block with dims d[0..r).
static void strides(const long long *d, int r, long long *s) {
  long long t = 1;
  for (int i = r - 1; i >= 0; --i) { s[i] = t; t *= d[i]; }
}

// Build a map over the listed axes, keeping those of extent > 1 (at most two).
// pos[] receives the positions (within axes) of the kept axes.
static inline bool make_map(const long long *d, const long long *s, const int *axes, int naxes, IdxMap &m,
                            int *pos, int &npos) {
  npos = 0;
  for (int k = 0; k < naxes; ++k)
    if (d[axes[k]] > 1) {
      if (npos == 2) return false;
      pos[npos++] = k;
    }
  m = IdxMap();
  if (npos == 1) { m.ext = (int)d[axes[pos[0]]]; m.lo_ext = m.ext; m.s_lo = s[axes[pos[0]]]; }
  if (npos == 2) {
    m.ext = (int)(d[axes[pos[0]]] * d[axes[pos[1]]]); m.lo_ext = (int)d[axes[pos[1]]];
    m.s_hi = s[axes[pos[0]]]; m.s_lo = s[axes[pos[1]]];
  }
  return true;
}
// Strides of an operand's axes at the kept positions.
static inline void strides_at(const long long *s, const int *axes, const int *pos, int npos, long long &hi,
                              long long &lo) {
  hi = lo = 0;
  if (npos == 1) lo = s[axes[pos[0]]];
  if (npos == 2) { hi = s[axes[pos[0]]]; lo = s[axes[pos[1]]]; }
}
}  // namespace

// Block dims of flat block b of a tensor with sector grid nsyms and concatenated sector dims.
static inline void block_dims(long long b, int r, const int *nsyms, const long long *first,
                              const long long *ndims, long long *d) {
  for (int i = r - 1; i >= 0; --i) {
    const long long s = b % nsyms[i];
    b /= nsyms[i];
    d[i] = ndims[first[i] + s];
  }
}

extern "C" long long qc_compile_pairs(int r1, const int *nsyms1, const long long *ndims1, const long long *off1,
                                      int r2, const int *nsyms2, const long long *ndims2, const long long *off2,
                                      int ro, const int *nsymso, const long long *ndimso, const long long *offo,
                                      int nax, const int *ax1, const int *ax2,
                                      long long npairs, const long long *triples,
                                      int nops, const long long *base1, const long long *base2,
                                      const long long *baseo, const double *alpha, int group_ops,
                                      int tile_m, int tile_n,
                                      void *tasks_v, long long task_cap, void *contribs_v, long long contrib_cap,
                                      long long *ntasks_out, double *flops_out) {
  if (r1 < 1 || r2 < 1 || ro < 0 || nax < 0 || nops < 1 || tile_m < 1 || tile_n < 1)
    return set_err(QC_ERR_ARG, "qc_compile_pairs: bad arguments");
  if (r1 > 16 || r2 > 16 || ro > 16) return set_err(QC_ERR_ARG, "qc_compile_pairs: rank > 16");
  long long f1[17] = {0}, f2[17] = {0}, fo[17] = {0};
  for (int i = 0; i < r1; ++i) f1[i + 1] = f1[i] + nsyms1[i];
  for (int i = 0; i < r2; ++i) f2[i + 1] = f2[i] + nsyms2[i];
  for (int i = 0; i < ro; ++i) fo[i + 1] = fo[i] + nsymso[i];
  int in1[16] = {0}, in2[16] = {0};
  int i1[16], i2[16], e1[16], e2[16], om[16], on[16];
  int ne1 = 0, ne2 = 0;
  for (int j = 0; j < nax; ++j) { i1[j] = ax1[j]; i2[j] = ax2[j]; in1[ax1[j]] = 1; in2[ax2[j]] = 1; }
  for (int i = 0; i < r1; ++i) if (!in1[i]) e1[ne1++] = i;
  for (int i = 0; i < r2; ++i) if (!in2[i]) e2[ne2++] = i;
  if (ne1 + ne2 != ro) return set_err(QC_ERR_ARG, "qc_compile_pairs: output rank");
  for (int k = 0; k < ne1; ++k) om[k] = k;
  for (int k = 0; k < ne2; ++k) on[k] = ne1 + k;
  qc_task *tasks = (qc_task *)tasks_v;
  qc_contrib *contribs = (qc_contrib *)contribs_v;
  const int nouter = group_ops ? 1 : nops;
  const long long nc_total = npairs * nops;
  // ---- counting pass (cheap): tasks per output block group
  long long nt_total = 0;
  double flops = 0.0;
  for (long long p = 0; p < npairs;) {
    const long long ob = triples[3 * p];
    long long q = p;
    long long dO[16], sO[16];
    block_dims(ob, ro, nsymso, fo, ndimso, dO);
    strides(dO, ro, sO);
    IdxMap mm, nn;
    int pm[2], pn[2], npm, npn;
    if (!make_map(dO, sO, om, ne1, mm, pm, npm) || !make_map(dO, sO, on, ne2, nn, pn, npn))
      return set_err(QC_ERR_LAYOUT, "qc_compile_pairs: more than two non-trivial axes in M or N");
    while (q < npairs && triples[3 * q] == ob) {
      long long d1[16];
      block_dims(triples[3 * q + 1], r1, nsyms1, f1, ndims1, d1);
      long long K = 1;
      for (int j = 0; j < nax; ++j) K *= d1[i1[j]];
      flops += 2.0 * (double)mm.ext * (double)nn.ext * (double)K * nops;
      ++q;
    }
    nt_total += (long long)((mm.ext + tile_m - 1) / tile_m) * ((nn.ext + tile_n - 1) / tile_n) * nouter;
    p = q;
  }
  if (ntasks_out) *ntasks_out = nt_total;
  if (flops_out) *flops_out = flops;
  if (!tasks || !contribs || nt_total > task_cap || nc_total > contrib_cap) return nc_total;
  // ---- fill pass
  long long nt = 0, nc = 0;
  for (int oo = 0; oo < nouter; ++oo) {
    for (long long p = 0; p < npairs;) {
      const long long ob = triples[3 * p];
      long long dO[16], sO[16];
      block_dims(ob, ro, nsymso, fo, ndimso, dO);
      strides(dO, ro, sO);
      IdxMap mm, nn;
      int pm[2], pn[2], npm, npn;
      make_map(dO, sO, om, ne1, mm, pm, npm);
      make_map(dO, sO, on, ne2, nn, pn, npn);
      const long long cb = nc;
      const int ilo = group_ops ? 0 : oo, ihi = group_ops ? nops : oo + 1;
      long long q = p;
      for (int op = ilo; op < ihi; ++op) {
        for (q = p; q < npairs && triples[3 * q] == ob; ++q) {
          const long long j1 = triples[3 * q + 1], j2 = triples[3 * q + 2];
          long long d1[16], d2[16], s1[16], s2[16];
          block_dims(j1, r1, nsyms1, f1, ndims1, d1);
          block_dims(j2, r2, nsyms2, f2, ndims2, d2);
          strides(d1, r1, s1);
          strides(d2, r2, s2);
          IdxMap kk;
          int pk[2], npk;
          if (!make_map(d1, s1, i1, nax, kk, pk, npk))
            return set_err(QC_ERR_LAYOUT, "qc_compile_pairs: more than two non-trivial contracted axes");
          qc_contrib &c = contribs[nc++];
          std::memset(&c, 0, sizeof(c));
          c.a_off = base1[op] + off1[j1];
          c.b_off = base2[op] + off2[j2];
          c.alpha = alpha[op];
          c.K = kk.ext;
          c.klo = kk.lo_ext;
          long long hi, lo;
          strides_at(s1, e1, pm, npm, hi, lo); c.a_mh = (int)hi; c.a_ml = (int)lo;
          strides_at(s1, i1, pk, npk, hi, lo); c.a_kh = (int)hi; c.a_kl = (int)lo;
          strides_at(s2, i2, pk, npk, hi, lo); c.b_kh = (int)hi; c.b_kl = (int)lo;
          strides_at(s2, e2, pn, npn, hi, lo); c.b_nh = (int)hi; c.b_nl = (int)lo;
        }
      }
      const long long ce = nc;
      const int outop = group_ops ? 0 : oo;
      for (int m0 = 0; m0 < mm.ext; m0 += tile_m) {
        for (int n0 = 0; n0 < nn.ext; n0 += tile_n) {
          qc_task &t = tasks[nt++];
          std::memset(&t, 0, sizeof(t));
          t.c_off = baseo[outop] + offo[ob];
          t.M = mm.ext; t.N = nn.ext; t.m0 = m0; t.n0 = n0;
          t.mlo = mm.lo_ext; t.nlo = nn.lo_ext;
          t.c_mh = (int)mm.s_hi; t.c_ml = (int)mm.s_lo; t.c_nh = (int)nn.s_hi; t.c_nl = (int)nn.s_lo;
          t.cb = (int)cb; t.ce = (int)ce;
        }
      }
      p = q;
    }
  }
  return nc;
}

// Packed two-site wavefunction position -> index of the dense diagonal [16][ldim][rdim]
// (HDiagQt's diag[prjmap], source/mpo_dmrg_kernelQt.py:119-122, with every index numbered
// sector by sector).  The layout is rank 4 (l, n1, n2, r) with one-dimensional physical
// sectors; block (sl, n, m, sr) of size dl x dr starts at ioff[block].
extern "C" int qc_psi_diag_gather(long long nblk, const long long *blocks, const int *nsyms,
                                  const long long *ndims, const long long *ioff, long long ldim,
                                  long long rdim, long long size, long long *gat) {
  if (nblk < 0 || !nsyms || !ndims || !ioff || !gat || (nblk > 0 && !blocks))
    return set_err(QC_ERR_ARG, "qc_psi_diag_gather: bad arguments");
  const long long n0 = nsyms[0], n1 = nsyms[1], n2 = nsyms[2], n3 = nsyms[3];
  const long long *d0 = ndims, *d1 = ndims + n0, *d2 = d1 + n1, *d3 = d2 + n2;
  std::vector<long long> so0(n0 + 1, 0), so3(n3 + 1, 0);
  for (long long s = 0; s < n0; ++s) so0[s + 1] = so0[s] + d0[s];
  for (long long s = 0; s < n3; ++s) so3[s + 1] = so3[s] + d3[s];
  if (so0[n0] != ldim || so3[n3] != rdim || n1 != 4 || n2 != 4)
    return set_err(QC_ERR_ARG, "qc_psi_diag_gather: layout does not match the dense diagonal");
  for (long long s = 0; s < 4; ++s)
    if (d1[s] != 1 || d2[s] != 1) return set_err(QC_ERR_ARG, "qc_psi_diag_gather: physical sectors not 1-dim");
  for (long long b = 0; b < nblk; ++b) {
    long long f = blocks[b];
    const long long sr = f % n3; f /= n3;
    const long long m = f % n2; f /= n2;
    const long long n = f % n1; f /= n1;
    const long long sl = f;
    if (sl < 0 || sl >= n0) return set_err(QC_ERR_ARG, "qc_psi_diag_gather: block index out of range");
    const long long dl = d0[sl], dr = d3[sr], o = ioff[blocks[b]];
    if (o < 0 || o + dl * dr > size) return set_err(QC_ERR_ARG, "qc_psi_diag_gather: block outside the layout");
    const long long base = (n * 4 + m) * ldim * rdim + so0[sl] * rdim + so3[sr];
    for (long long u = 0; u < dl; ++u)
      for (long long v = 0; v < dr; ++v) gat[o + u * dr + v] = base + u * rdim + v;
  }
  return QC_OK;
}
