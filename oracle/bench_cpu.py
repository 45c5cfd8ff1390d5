"""ORACLE (test infrastructure): CPU timing samples for bench.py.

Only bench.py's CPU-baseline leg and its --impl reference arm import this.
Both time the oracle (the NumPy restatement of HVecQt / HDiagQt /
renormQt_H00, source/mpo_dmrg_kernelQt.py) on this host's cores.
"""
import os
import time

import numpy

from .blocks import QTensor, classification
from .kernels import SigmaOracle, hdiag, RenormOracle, boundary_env
from .mpo import QPHYS, build_mpo, site_operator

# Davidson matrix-vector products per dot at K=24, D=500 (the FP64 GPU arm of the same
# workload, the algorithm of the reference's pdvdson: 355 products over the 46 dots of one
# sweep after the ramp and three warm-up sweeps).
MATVECS_PER_DOT = 7.7


def _qt(status, qsyms, ndims, values=None, rng=None):
    q = QTensor(status).from_qsyms(len(qsyms), qsyms, ndims, allocate=True)
    # contiguous index lists: sector s of index i covers positions [off, off + ndims[i][s])
    q.idlst = []
    for nd in q.ndims:
        off = numpy.concatenate([[0], numpy.cumsum(nd)[:-1]])
        q.idlst.append([list(range(int(o), int(o + n))) for o, n in zip(off, nd)])
    if values is not None:
        q.value = numpy.asarray(values, dtype=numpy.float64)
    elif rng is not None:
        q.value = rng.standard_normal(q.size_allowed)
    return q


def oracle_dot(d, isite):
    """Oracle sigma of the product's current dot (its environments copied to the host)."""
    L, R = d.lenv[isite - 1], d.renv[isite + 2]
    Wi, Wj = d.mpo[isite], d.mpo[isite + 1]

    def conv(ts, i):
        l = ts.layouts[i]
        return _qt(l.status, l.qsyms, l.ndims, ts.op_values(i).cpu().numpy())

    ql, qr = d.qnuml[isite], d.qnumr[isite + 2]
    cls = [classification(q) for q in (ql, QPHYS, QPHYS, d.qkey - qr)]
    qtmp = QTensor([False, False, False, True]).from_qsyms(4, [c[0] for c in cls], [c[1] for c in cls],
                                                           allocate=False)
    n = d.nops
    sig = SigmaOracle(qtmp, d.qkey, [conv(L, i) for i in range(n)], [conv(R, i) for i in range(n)],
                      [conv(Wi, i) for i in range(n)], [conv(Wj, i) for i in range(n)],
                      list(range(n)), numpy.ones(n), isite)
    lay, idl, s, dg = d.dot_operators(isite)
    x = numpy.random.default_rng(0).standard_normal(qtmp.size_allowed)
    return sig, x, s.flops


def oracle_sp_dot(d, isite):
    """Oracle H and S products (HVecQt with ifs2proj, SVecQt) of a spin-projected dot."""
    from .spin import sigma_sp, svec
    L, R = d.lenv[isite - 1], d.renv[isite + 2]
    PL, PR = d.plenv[isite - 1], d.prenv[isite + 2]
    Wi, Wj = d.mpo[isite], d.mpo[isite + 1]

    def conv(ts):
        return [_qt(l.status, l.qsyms, l.ndims, ts.op_values(i).cpu().numpy()) for i, l in enumerate(ts.layouts)]

    ql, qr = d.qnuml[isite], d.qnumr[isite + 2]
    cls = [classification(q) for q in (ql, QPHYS, QPHYS, d.qkey - qr)]
    qtmp = QTensor([False, False, False, True]).from_qsyms(4, [c[0] for c in cls], [c[1] for c in cls],
                                                           allocate=False)
    hv = sigma_sp(qtmp, d.qkey, conv(L), conv(R), conv(Wi), conv(Wj), list(d.opers), d.hpwts, isite)
    pops = conv(d.pops)
    sv = svec(qtmp, d.qkey, conv(PL), conv(PR), pops, d.qwts, isite)
    lay, idl, s, dg = d.dot_operators(isite)
    s2, sd = d.dot_projector(isite)
    x = numpy.random.default_rng(0).standard_normal(qtmp.size_allowed)
    return (lambda v: (hv(v), sv(v))), x, s.flops + s2.flops


_CACHE = {}


def _with_idlst(q):
    if q.idlst is None:
        q.idlst = []
        for nd in q.ndims:
            off = numpy.concatenate([[0], numpy.cumsum(nd)[:-1]])
            q.idlst.append([list(range(int(o), int(o + n))) for o, n in zip(off, nd)])
    return q


def _dot_sample(K, D, isite):
    """Oracle sigma, diagonal and L renormalisation at dot (isite, isite+1) of the synthetic
    D-state (random environments of the right block structure); returns the three times."""
    ham, W, mps, rm = _CACHE["ham"], _CACHE["W"], _CACHE["mps"], _CACHE["rmps"]
    for i in (isite, isite + 1):
        if i not in W:
            W[i] = [_with_idlst(site_operator(p, ham.sbas, i, ham.int1e, ham.int2e)) for p in range(ham.sbas)]
    rng = numpy.random.default_rng(5 + isite)
    qkey = numpy.array([float(K), 0.0])
    nops = ham.sbas
    ql = mps["qnum%d" % isite]
    qr = rm["qnum%d" % (K - isite - 2)]
    # environment layouts: a-bond of the neighbouring site operators, MPS bonds (status T,F,T)
    cl, cr = classification(ql), classification(qr)
    lenv = [_qt([True, False, True], [W[isite][p].qsyms[0], cl[0], cl[0]], [W[isite][p].ndims[0], cl[1], cl[1]],
                rng=rng) for p in range(nops)]
    renv = [_qt([True, False, True], [-W[isite + 1][p].qsyms[1], cr[0], cr[0]],
                [W[isite + 1][p].ndims[1], cr[1], cr[1]], rng=rng) for p in range(nops)]
    cls = [classification(q) for q in (ql, QPHYS, QPHYS, qkey - qr)]
    qtmp = QTensor([False, False, False, True]).from_qsyms(4, [c[0] for c in cls], [c[1] for c in cls],
                                                           allocate=False)
    sig = SigmaOracle(qtmp, qkey, lenv, renv, W[isite], W[isite + 1], list(range(nops)), numpy.ones(nops), isite)
    x = rng.standard_normal(qtmp.size_allowed)
    t0 = time.time()
    sig(x)
    t_hvec = time.time() - t0
    prj = qtmp.prjmap([c[2] for c in cls])
    dims = (len(ql), 16, len(qr), len(ql) * 16 * len(qr))
    t0 = time.time()
    hdiag(prj, dims, lenv, renv, W[isite], W[isite + 1], numpy.ones(nops))
    t_diag = time.time() - t0
    site = QTensor([False, False, True]).from_dense(rng.standard_normal((len(ql), 4, len(ql) * 4)),
                                                    [ql, QPHYS, (ql[:, None, :] + QPHYS[None]).reshape(-1, 2)])
    t0 = time.time()
    RenormOracle(list(range(nops)), isite, "L")(site, lenv, W[isite])
    t_ren = time.time() - t0
    return t_hvec, t_diag, t_ren


# dots sampled by the successive steps of the reference arm: spread over one half of the
# chain (the synthetic state's bond dimensions are symmetric about its middle)
def _dot_order(K):
    half = list(range(0, K // 2))
    order = []
    seen = set()
    for i in [K // 2 - 1, K // 4, 1, 3 * K // 8, K // 8] + half:
        if 0 <= i <= K - 2 and i not in seen:
            seen.add(i)
            order.append(i)
    return order


def reference_step(args, warm=False, step=0):
    """One bounded sample of the K=24, D=500 sweep on the host: at one dot of a synthetic
    D=500 state (successive steps visit successive dots of half the chain, mid-chain first),
    one oracle sigma matvec, one diagonal and one renormalisation.  Returns the dot's cost
    (MATVECS_PER_DOT sigma + diagonal + renormalisation) and the sweep estimate from every
    dot sampled so far: the cost of each of the 2 (K - 1) dots of a sweep interpolated
    linearly in the dot position from the sampled ones (mirrored about the middle)."""
    from qcmpodmrg_b200.hamiltonian import make_hamiltonian
    from qcmpodmrg_b200.synthetic import random_mps
    K, D = args.sites, args.dmax
    if "ham" not in _CACHE:
        ham = make_hamiltonian(K, K, 1, 3.0)
        _CACHE["ham"] = ham
        _CACHE["W"] = {}
        _CACHE["mps"] = random_mps(K, K, D, seed=1)
        _CACHE["rmps"] = random_mps(K, K, D, seed=2)
        _CACHE["samples"] = {}
    if warm:
        return None
    order = _dot_order(K)
    isite = order[step % len(order)]
    t_hvec, t_diag, t_ren = _dot_sample(K, D, isite)
    cost = MATVECS_PER_DOT * t_hvec + t_diag + t_ren
    _CACHE["samples"][isite] = cost
    pos = sorted(_CACHE["samples"])
    vals = [_CACHE["samples"][i] for i in pos]
    dots = numpy.arange(K - 1)
    mirrored = numpy.minimum(dots, K - 2 - dots)
    per_dot = numpy.interp(mirrored, pos, vals)
    est = 2.0 * float(per_dot.sum())
    return {"sweep_s_est": est, "cores": os.cpu_count(), "dot": isite, "dot_cost_s": cost,
            "sample": "dot %d of a synthetic D=%d state: sigma %.1f s, diagonal %.1f s, renormalisation %.1f s; "
                      "sweep = sum over the 2(K-1) dots of (%.1f sigma + diagonal + renormalisation), each dot's "
                      "cost interpolated from the %d dots sampled (mirrored about the middle)"
                      % (isite, D, t_hvec, t_diag, t_ren, MATVECS_PER_DOT, len(pos))}
