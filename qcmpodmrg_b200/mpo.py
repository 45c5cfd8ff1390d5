"""Host-side construction of the H_p = a_p^+ V_p site operators.

The operator algebra is the reference's (source/mpo_dmrg_opers.py:91-260 for
the dense W factors and the a_p^+ string, source/qtensor/qtensor_opers.py:
153-193 for the MPO-bond quantum numbers, :358-408 for the spatial-site
operator in block form with uncollected physical indices).  The 2x2 one-site
matrices are those of source/mpo_dmrg_const.py.  The MPO bond is ordered by
(N, Sz) numerically; the reference orders it by the printed string of the
same pairs.  Any order that keeps equal quantum numbers contiguous gives the
same operator, so sigma, diagonal and energies are unchanged.

Everything here runs once per calculation (not per matvec).
"""
import numpy

from .qtensor import Layout, classification

SGN = numpy.array([[1., 0.], [0., -1.]])
IDN = numpy.eye(2)
CRE = numpy.array([[0., 0.], [1., 0.]])
ANN = numpy.array([[0., 1.], [0., 0.]])
NII = numpy.array([[0., 0.], [0., 1.]])
QPHYS = numpy.array([[0., 0.], [1., -0.5], [1., 0.5], [2., 0.]])
SPINS = (0.5, -0.5)
W_STATUS = numpy.array([False, True, False, True])


def case(porb, isite, ncsite=1):
    """Symmetry class of operator p relative to the dot (qtensor_opers.case, :72-90).

    Operators of one class share every block structure, so one set of block-pair
    lists serves all of them.
    """
    s = porb % 2
    if porb // 2 < isite:
        return s
    if porb // 2 == isite:
        return 2 + s
    if ncsite == 1 or porb // 2 == isite + 1:
        return 4 + s
    return 6 + s


def _wfac(nsite, i, hq, v):
    """Dense W factor of V_p at spin-orbital site i (mpo_dmrg_opers.genWfacSpin)."""
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
        w[3:3 + i, 0] = v[i, :i, i][:, None, None] * NII
        w[n1 - 1, 0] = IDN
        return w
    w[0, 0] = SGN
    w[0, 1 + dr:1 + 2 * dr] = -v[i, i, rs][:, None, None] * NII
    w[0, 1 + 2 * dr + dl] = -ANN
    w[0, 2 + 2 * dr + 2 * dl] = CRE
    w[0, last] = hq[i] * ANN
    if i == 0:
        return w
    w[1, last] = CRE
    k = numpy.arange(dr)
    w[2 + k, 1 + k] = SGN
    w[2 + dr, last] = ANN
    w[3 + dr + k, 1 + dr + k] = SGN
    o6, o7 = 3 + 2 * dr, 3 + 2 * dr + dl
    ls = numpy.arange(i)
    # rows of the left-complementary channels (creation/annihilation strings to the left)
    w[o6:o6 + i, 1:1 + dr] = v[numpy.ix_(rs, ls, [i])][:, :, 0].T[:, :, None, None] * ANN
    w[o6:o6 + i, 1 + dr:1 + 2 * dr] = v[i][numpy.ix_(ls, rs)][:, :, None, None] * CRE
    w[o6 + ls, 1 + 2 * dr + ls] = IDN
    w[o6:o6 + i, last] = v[i, ls, i][:, None, None] * NII
    w[o7:o7 + i, 1 + dr:1 + 2 * dr] = -v[numpy.ix_(ls, [i], rs)][:, 0, :][:, :, None, None] * ANN
    w[o7 + ls, 2 + 2 * dr + dl + ls] = IDN
    w[n1 - 1, last] = IDN
    return w


def _hfac_spin(p, nsite, i, hq, v):
    e = SGN if i < p else (CRE if i == p else IDN)
    return numpy.matmul(e, _wfac(nsite, i, hq, v))


def _link(op1, op2):
    t = numpy.tensordot(op1, op2, axes=([1], [0]))        # a i j c k l
    t = t.transpose(0, 3, 1, 4, 2, 5)                    # a c i k j l
    s = t.shape
    return t.reshape(s[0], s[1], s[2] * s[3], s[4] * s[5])


def _wq_right(nsite, i, sz):
    q = [[0., 0.]]
    q += [[-2., -sz - SPINS[k % 2]] for k in range(i + 1, nsite)]
    q += [[0., -sz + SPINS[k % 2]] for k in range(i + 1, nsite)]
    q += [[-1., -SPINS[k % 2]] for k in range(i + 1)]
    q += [[1., SPINS[k % 2]] for k in range(i + 1)]
    q += [[-1., -sz]]
    return numpy.array(q)


def _wq(nsite, i, isz):
    sz = SPINS[isz]
    ql = numpy.array([[0., 0.]]) if i == 0 else _wq_right(nsite, i - 1, sz)
    qr = numpy.array([[-1., -sz]]) if i == nsite - 1 else _wq_right(nsite, i, sz)
    return ql, qr


def _elem_q(p, i):
    spin = SPINS[p % 2]
    if i < p:
        return numpy.zeros(2), numpy.zeros(2)
    if i == p:
        return numpy.zeros(2), numpy.array([1., spin])
    return numpy.array([1., spin]), numpy.array([1., spin])


def _order(q):
    q2 = numpy.rint(2 * q).astype(numpy.int64)
    return numpy.lexsort((q2[:, 1], q2[:, 0]))


_PRJ = {}


def site_operator(p, nsite_spin, isite, int1e, int2e):
    """H_p at spatial site isite: (Layout, packed values, bond idlst) -- genHRfacSpatialQt."""
    hq, v = int1e[p], int2e[p]
    dense = _link(_hfac_spin(p, nsite_spin, 2 * isite, hq, v), _hfac_spin(p, nsite_spin, 2 * isite + 1, hq, v))
    ql1, _ = _elem_q(p, 2 * isite)
    _, qr1 = _elem_q(p, 2 * isite + 1)
    ql2, _ = _wq(nsite_spin, 2 * isite, p % 2)
    _, qr2 = _wq(nsite_spin, 2 * isite + 1, p % 2)
    ql, qr = ql2 + ql1, qr2 + qr1
    il, ir = _order(ql), _order(qr)
    dense = dense[numpy.ix_(il, ir)]
    cl = classification(ql[il])
    cr = classification(qr[ir])
    phys = classification(QPHYS, collect=False)
    lay = Layout(W_STATUS, [cl[0], cr[0], phys[0], phys[0]], [cl[1], cr[1], phys[1], phys[1]])
    key = (id(lay), tuple(len(x) for x in cl[2]), tuple(len(x) for x in cr[2]))
    hit = _PRJ.get(key)
    if hit is not None and hit[0] is lay:
        prj = hit[1]
    else:
        prj = lay.prjmap([cl[2], cr[2], phys[2], phys[2]])
        _PRJ[key] = (lay, prj)          # the layout is held, so its id cannot be recycled
    return lay, dense.ravel()[prj].copy()


def build_mpo(ham, isites=None):
    """Layouts and packed values of H_p (p = 0..2K-1) at every spatial site."""
    K = ham.nsite
    out = {}
    for i in (range(K) if isites is None else isites):
        lays, vals = [], []
        for p in range(ham.sbas):
            l, v = site_operator(p, ham.sbas, i, ham.int1e, ham.int2e)
            lays.append(l)
            vals.append(v)
        out[i] = (lays, vals)
    return out
