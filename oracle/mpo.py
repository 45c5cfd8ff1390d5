"""ORACLE (test infrastructure only): the H_p = a_p^+ V_p site operators.

Restates source/mpo_dmrg_opers.py:91-260 (dense W factors), mpo_dmrg_const.py
(2x2 matrices) and source/qtensor/qtensor_opers.py:72-90,153-193,358-408
(operator classes and bond quantum numbers).  The MPO bond is sorted by
(N, Sz) numerically (stable); the reference sorts by the printed string of the
same pairs.  Both orders group equal quantum numbers contiguously and give the
same operator, so sigma, diagonal and energies are unchanged.
"""
import numpy

from .blocks import QTensor

SGN = numpy.array([[1., 0.], [0., -1.]])
IDN = numpy.eye(2)
CRE = numpy.array([[0., 0.], [1., 0.]])
ANN = numpy.array([[0., 1.], [0., 0.]])
NII = numpy.array([[0., 0.], [0., 1.]])
QPHYS = numpy.array([[0., 0.], [1., -0.5], [1., 0.5], [2., 0.]])
SPINS = (0.5, -0.5)


def case(porb, isite, ncsite=1):
    """qtensor_opers.case: symmetry class of operator p relative to the dot."""
    s = porb % 2
    if porb // 2 < isite:
        return 0 + s
    if porb // 2 == isite:
        return 2 + s
    if ncsite == 1 or porb // 2 == isite + 1:
        return 4 + s
    return 6 + s


def wfac_spin(nsite, i, hq, v):
    """Dense W factor of V_p at spin-orbital site i (genWfacSpin)."""
    n1 = 1 if i == 0 else 2 * (nsite + 1)
    n2 = 1 if i == nsite - 1 else 2 * (nsite + 1)
    w = numpy.zeros((n1, n2, 2, 2))
    dl, dr = i, nsite - i - 1
    last = n2 - 1
    rs = numpy.arange(i + 1, nsite)
    if i == nsite - 1:
        w[0, 0] = hq[i] * ANN
        w[1, 0] = CRE
        w[2, 0] = ANN
        for j in range(i):
            w[3 + j, 0] = v[i, j, i] * NII
        w[n1 - 1, 0] = IDN
        return w
    w[0, 0] = SGN
    for k, r in enumerate(rs):
        w[0, 1 + dr + k] = -v[i, i, r] * NII
    w[0, 1 + 2 * dr + dl] = -ANN
    w[0, 2 + 2 * dr + 2 * dl] = CRE
    w[0, last] = hq[i] * ANN
    if i == 0:
        return w
    w[1, last] = CRE
    for k in range(dr):
        w[2 + k, 1 + k] = SGN
    w[2 + dr, last] = ANN
    for k in range(dr):
        w[3 + dr + k, 1 + dr + k] = SGN
    o6 = 3 + 2 * dr
    for l in range(i):
        for k, r in enumerate(rs):
            w[o6 + l, 1 + k] = v[r, l, i] * ANN        # -v * annt with annt = -ann
            w[o6 + l, 1 + dr + k] = v[i, l, r] * CRE
        w[o6 + l, 1 + 2 * dr + l] = IDN
        w[o6 + l, last] = v[i, l, i] * NII
    o7 = 3 + 2 * dr + dl
    for l in range(i):
        for k, r in enumerate(rs):
            w[o7 + l, 1 + dr + k] = -v[l, i, r] * ANN
        w[o7 + l, 2 + 2 * dr + dl + l] = IDN
    w[n1 - 1, last] = IDN
    return w


def elem_spin(p, i):
    if i < p:
        return SGN
    if i == p:
        return CRE
    return IDN


def hfac_spin(p, nsite, i, hq, v):
    w = wfac_spin(nsite, i, hq, v)
    return numpy.matmul(elem_spin(p, i), w)        # ij,abjk->abik


def link(op1, op2):
    """abij,bckl -> a c (ik) (jl)  (mpo_dmrg_opers.linkTwoOpers)."""
    t = numpy.tensordot(op1, op2, axes=([1], [0])).transpose(0, 3, 1, 4, 2, 5)
    s = t.shape
    return t.reshape(s[0], s[1], s[2] * s[3], s[4] * s[5])


def hfac_spatial(p, nsite, isite, hq, v):
    return link(hfac_spin(p, nsite, 2 * isite, hq, v), hfac_spin(p, nsite, 2 * isite + 1, hq, v))


def wqnums_right(nsite, i, sz):
    """Right-bond quantum numbers of spin site i (genWfacSpinQnumsRight)."""
    q = [[0., 0.]]
    q += [[-2., -sz - SPINS[k % 2]] for k in range(i + 1, nsite)]
    q += [[0., -sz + SPINS[k % 2]] for k in range(i + 1, nsite)]
    q += [[-1., -SPINS[k % 2]] for k in range(i + 1)]
    q += [[1., SPINS[k % 2]] for k in range(i + 1)]
    q += [[-1., -sz]]
    return numpy.array(q)


def wqnums(nsite, i, isz):
    sz = SPINS[isz]
    ql = numpy.array([[0., 0.]]) if i == 0 else wqnums_right(nsite, i - 1, sz)
    qr = numpy.array([[-1., -sz]]) if i == nsite - 1 else wqnums_right(nsite, i, sz)
    return ql, qr


def elem_qnums(p, i):
    spin = SPINS[p % 2]
    if i < p:
        return numpy.array([0., 0.]), numpy.array([0., 0.])
    if i == p:
        return numpy.array([0., 0.]), numpy.array([1., spin])
    return numpy.array([1., spin]), numpy.array([1., spin])


def sort_key_order(q):
    """Stable numeric order of bond quantum numbers (N first, then Sz)."""
    q2 = numpy.rint(2 * q).astype(numpy.int64)
    return numpy.lexsort((q2[:, 1], q2[:, 0]))


def site_operator(p, nsite_spin, isite, int1e, int2e):
    """H_p site tensor at spatial site isite as a QTensor [a, b, n, n'] (genHRfacSpatialQt)."""
    dense = hfac_spatial(p, nsite_spin, isite, int1e[p], int2e[p])
    ql1, _ = elem_qnums(p, 2 * isite)
    _, qr1 = elem_qnums(p, 2 * isite + 1)
    ql2, _ = wqnums(nsite_spin, 2 * isite, p % 2)
    _, qr2 = wqnums(nsite_spin, 2 * isite + 1, p % 2)
    ql = ql2 + ql1
    qr = qr2 + qr1
    il = sort_key_order(ql)
    ir = sort_key_order(qr)
    dense = dense[numpy.ix_(il, ir)]
    qt = QTensor([False, True, False, True])
    qt.from_dense(dense, [ql[il], qr[ir], QPHYS, QPHYS], collect=[True, True, False, False])
    return qt


def build_mpo(ham):
    """All site operators: mpo[isite][iop] for iop = spin orbital p (one rank holds all)."""
    K = ham.nsite
    return [[site_operator(p, ham.sbas, i, ham.int1e, ham.int2e) for p in range(ham.sbas)]
            for i in range(K)]
