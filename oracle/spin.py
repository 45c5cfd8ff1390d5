"""ORACLE (test infrastructure only): spin projection (SP-MPS), restated in NumPy.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs may import this
module; the product never does.  With spin projection the wavefunction is
optimised for Hc = S c E with the projector P = sum_g w_g R(theta_g) onto total
spin S (Sz fixed), R(theta) = exp(-i theta S_y):

  smalld          Wigner small-d d^j_{m'm}(beta)        source/tools/smalld.py:8-43
  s2quad          quadrature (theta_g, w_g)             source/mpo_dmrg_util.py:35-89
  exp_isy_phi     one-site R(theta), 4x4                source/mpo_dmrg_opers.py:228-243
  rotation_op     R(theta) as a bond-1 MPO site tensor  source/qtensor/qtensor_opers.py:457-469
  sp_site_operator  H_p R(theta_g) site tensor, (N)-only quantum numbers
                                                        source/mpo_dmrg_opers.py:253-260,
                                                        source/qtensor/qtensor_opers.py:358-408
  sigma_sp / svec / hdiag / renorm: the H and S kernels with the wavefunction reduced
  to N symmetry and projected back to (N, Sz)           source/mpo_dmrg_kernelQt.py:153-319
                                                        (ifs2proj branches), :322-450, :770-854
  gdavidson       generalised Davidson Hc = Sce         source/tools/pgdvdson.py:60-330
  SPOracleDMRG    the two-site sweep with projection    source/mpo_dmrg_util.py:193-214 (initOps),
                                                        source/mpo_dmrg_dot.py:40-70,
                                                        source/mpo_dmrg_kernel.py:347-377 (renorm)

Operators are ordered as the reference partitions them on one rank
(source/mpo_dmrg_class.py:219-222, tools/parallel_util.py:39-42): index
x -> (p, g) = (x // npts, x % npts), weight qwts[g].
"""
import math

import numpy
import scipy.linalg
import scipy.special

from .blocks import QTensor, Contraction, classification
from .kernels import SigmaOracle, hdiag, RenormOracle, flip_right
from .mpo import QPHYS, case, hfac_spatial, elem_qnums, wqnums
from .solver import _ortho
from .dmrg import OracleDMRG

QPHYS_N = QPHYS[:, 0:1].copy()


# ----------------------------------------------------------------- quadrature
def smalld(j, mp, ms, beta):
    """Wigner small-d d^j_{mp,ms}(beta) by the explicit sum over s (tools/smalld.py)."""
    r = [x - math.floor(x) for x in (j, mp, ms)]
    if abs(r[0] - r[1]) > 1e-10 or abs(r[1] - r[2]) > 1e-10 or abs(r[0] - r[2]) > 1e-10:
        return 0.0
    g = scipy.special.gamma
    pre = math.sqrt(g(j + mp + 1) * g(j - mp + 1) * g(j + ms + 1) * g(j - ms + 1))
    cb, sb = math.cos(beta / 2.0), math.sin(beta / 2.0)
    val = 0.0
    for s in numpy.arange(0.0, 2 * j + 0.1):
        if j + ms - s > -0.1 and mp - ms + s > -0.1 and j - mp - s > -0.1:
            term = math.pow(-1.0, mp - ms + s)
            term /= g(j + ms - s + 1) * g(s + 1) * g(mp - ms + s + 1) * g(j - mp - s + 1)
            term *= math.pow(cb, 2 * j + ms - mp - 2 * s) * math.pow(sb, mp - ms + 2 * s)
            val += term
    return pre * val


def s2quad(npts, sval=0.0, sz=0.0, quad="GaussLegendre"):
    """Quadrature points theta_g in [0, pi] and weights for P_S (mpo_dmrg_util.s2quad)."""
    assert sval + 1.e-4 > abs(sz)
    if quad == "GaussLegendre":
        x, w = numpy.polynomial.legendre.leggauss(npts)
        xts = numpy.array([math.acos(v) for v in x])
        fac = numpy.array([smalld(sval, sz, sz, t) for t in xts])
        wts = (2. * sval + 1.) / 2.0 * (fac * w)
    elif quad == "Simpson":
        n = npts - 1
        assert n % 2 == 0 and n > 0
        h = numpy.pi / (3.0 * n)
        c = numpy.zeros(npts)
        c[0::2] = 2.0
        c[1::2] = 4.0
        c[0] = c[-1] = 1.0
        xts = numpy.linspace(0, numpy.pi, num=npts)
        wts = c * h * numpy.array([(2. * sval + 1.) / 2.0 * math.sin(t) * smalld(sval, sz, sz, t) for t in xts])
    else:
        raise ValueError(quad)
    return xts, wts


# ----------------------------------------------------------------- operators
def exp_isy_phi(phi):
    """exp(-i phi S_y) on one spatial orbital |0>, |b>, |a>, |ab> (genExpISyPhiMat)."""
    m = numpy.zeros((4, 4))
    m[0, 0] = m[3, 3] = 1.0
    c, s = math.cos(0.5 * phi), math.sin(0.5 * phi)
    m[1, 1] = m[2, 2] = c
    m[1, 2] = s
    m[2, 1] = -s
    return m


def rotation_op(phi):
    """R(phi) as the [1, 1, 4, 4] site tensor with N-only quantum numbers (genExpISyPhiQt)."""
    q = QTensor([False, True, False, True])
    q.from_dense(exp_isy_phi(phi).reshape(1, 1, 4, 4), [[[0.]], [[0.]], QPHYS_N, QPHYS_N],
                 collect=[False] * 4)
    return q


def sort_n_order(q):
    """Stable order by particle number (the reference sorts the printed N-only pairs;
    both keep equal N contiguous in their original relative order)."""
    return numpy.argsort(numpy.rint(2 * q[:, 0]).astype(numpy.int64), kind="stable")


def sp_site_operator(p, phi, nsite_spin, isite, int1e, int2e):
    """H_p R(phi) at spatial site isite with N-only bond / physical quantum numbers."""
    dense = hfac_spatial(p, nsite_spin, isite, int1e[p], int2e[p])
    dense = numpy.tensordot(dense, exp_isy_phi(phi), axes=([3], [0]))
    ql1, _ = elem_qnums(p, 2 * isite)
    _, qr1 = elem_qnums(p, 2 * isite + 1)
    ql2, _ = wqnums(nsite_spin, 2 * isite, p % 2)
    _, qr2 = wqnums(nsite_spin, 2 * isite + 1, p % 2)
    ql = (ql2 + ql1)[:, 0:1]
    qr = (qr2 + qr1)[:, 0:1]
    il, ir = sort_n_order(ql), sort_n_order(qr)
    qt = QTensor([False, True, False, True])
    qt.from_dense(dense[numpy.ix_(il, ir)], [ql[il], qr[ir], QPHYS_N, QPHYS_N],
                  collect=[True, True, False, False])
    return qt


def sp_opers(sbas, npts):
    return [(x // npts, x % npts) for x in range(sbas * npts)]


def build_mpo_sp(ham, qpts):
    """mpo[isite][x] = H_p R(theta_g) for x -> (p, g) (dumpMPO_H with ifs2proj)."""
    ops = sp_opers(ham.sbas, len(qpts))
    return [[sp_site_operator(p, qpts[g], ham.sbas, i, ham.int1e, ham.int2e) for (p, g) in ops]
            for i in range(ham.nsite)]


def boundary_env_n(nop):
    """genBopsQt with N-only quantum numbers (mpo_dmrg_initQt.py:58-66)."""
    out = []
    for _ in range(nop):
        q = QTensor([True, False, True])
        q.from_dense(numpy.ones((1, 1, 1)), [[[0.]]] * 3)
        out.append(q)
    return out


# ----------------------------------------------------------------- kernels
class ProjectedSigma(SigmaOracle):
    """sigma = P_(N,Sz) sum_x w_x R_x W_x[i+1] W_x[i] L_x (psi reduced to N).

    HVecQt with ifs2proj (the R environment flipped with qkey[:1], kernelQt.py:297-298,
    the result projected back with projectionNMs, :309-311) and, with the projector's
    environments and R(theta) operators, SVecQt (kernelQt.py:373-450).
    """

    def __init__(self, qtmp, qkey, lenv, renv, wi, wj, opers, wts, isite):
        qkey = numpy.asarray(qkey, dtype=numpy.float64)[:1]
        super(ProjectedSigma, self).__init__(qtmp, qkey, lenv, renv, wi, wj, opers, wts, isite)

    def reduce(self, x):
        psi = self.qtmp.copy_structure()
        psi.value = numpy.asarray(x, dtype=numpy.float64).copy()
        return psi.reduce_to_n()

    def __call__(self, x):
        psi_n = self.reduce(x)
        y = numpy.zeros(self.qtmp.size_allowed)
        for iop in range(len(self.opers)):
            c1, c2, c3, c4 = self._plans(iop, psi_n)
            R = flip_right(self.renv[iop], self.qkey)
            t4 = c4.run(c3.run(c2.run(c1.run(self.lenv[iop], psi_n), self.wi[iop]), self.wj[iop]), R)
            y += self.hpwts[iop] * t4.projection_nms(self.qtmp.qsyms).value
        return y

    def count_flops(self, x=None):
        """Pair-GEMM FLOPs of the four contractions on the N-reduced wavefunction."""
        psi_n = self.reduce(numpy.zeros(self.qtmp.size_allowed))
        tot = 0
        for iop in range(len(self.opers)):
            c1, c2, c3, c4 = self._plans(iop, psi_n)
            R = flip_right(self.renv[iop], self.qkey)
            tot += c1.flops(self.lenv[iop], psi_n) + c2.flops(c1.out, self.wi[iop])
            tot += c3.flops(c2.out, self.wj[iop]) + c4.flops(c3.out, R)
        return tot

    def _plans(self, iop, psi):
        key = case(self.opers[iop], self.isite, 2)
        if key not in self.templates:
            L, W1, W2 = self.lenv[iop], self.wi[iop], self.wj[iop]
            R = flip_right(self.renv[iop], self.qkey)
            c1 = Contraction().plan(L, psi, ([2], [0]))
            c2 = Contraction().plan(c1.out, W1, ([0, 2], [0, 3]))
            c3 = Contraction().plan(c2.out, W2, ([1, 3], [3, 0]))
            c4 = Contraction().plan(c3.out, R, ([1, 3], [2, 0]))
            assert c4.out.size_allowed == psi.size_allowed
            self.templates[key] = (c1, c2, c3, c4)
        return self.templates[key]


def sigma_sp(qtmp, qkey, lenv, renv, wi, wj, opers_p, hpwts, isite):
    return ProjectedSigma(qtmp, qkey, lenv, renv, wi, wj, opers_p, hpwts, isite)


def svec(qtmp, qkey, plenv, prenv, pops, qwts, isite):
    """SVecQt: one template for all R(theta) operators (kernelQt.py:385-395)."""
    return ProjectedSigma(qtmp, qkey, plenv, prenv, pops, pops, [0] * len(pops), qwts, isite)


def sdiag(prjmap, dims, plenv, prenv, pops, qwts):
    """SDiagQt two-site (kernelQt.py:348-363)."""
    return hdiag(prjmap, dims, plenv, prenv, pops, pops, qwts)


def renorm_p(site_n, penv, pops, isite, status):
    """renormQt_S00: the projector's environments (kernelQt.py:770-854)."""
    return RenormOracle([0] * len(pops), isite, status)(site_n, penv, pops)


# ----------------------------------------------------------------- solver
def _gen_ortho(vbas, crit_indp):
    """pgdvdson.genOrthoBas: normalise the first row, orthonormalise the rest against it."""
    vbas = numpy.array(vbas, dtype=numpy.float64)
    vbas[0] = vbas[0] / numpy.linalg.norm(vbas[0])
    if vbas.shape[0] == 1:
        return vbas[0:1].copy()
    n, v2 = _ortho(vbas[0:1], vbas[1:], crit_indp)
    return numpy.vstack((vbas[0:1], v2)) if n else vbas[0:1].copy()


def gdavidson(hvec, svec_, diag, neig=1, v0=None, crit_e=1.e-8, crit_vec=1.e-8, maxcycle=20,
              crit_indp=1.e-12, lshift=1.e-4, nfac=10, trace=None):
    """pgdvdson.eigenSolver.solve_iter with iop=4 and no start-vector noise.

    Returns (eigs, vecs, nmvp); the vectors are S-normalised (x^T S x = 1)."""
    ndim = len(diag)
    if v0 is None:
        d = diag + 1.e-12 * numpy.arange(1, 1 + ndim) / float(ndim)
        vbas = numpy.zeros((neig, ndim))
        vbas[numpy.arange(neig), numpy.argsort(d)[:neig]] = 1.0
    else:
        vbas = numpy.array(v0, dtype=numpy.float64).reshape(neig, ndim)
    vbas = _gen_ortho(vbas, crit_indp)
    wbas = numpy.array([hvec(v) for v in vbas])
    sbas = numpy.array([svec_(v) for v in vbas])
    nmvp = len(vbas)
    eigs = numpy.zeros(neig) + 1.e3
    for niter in range(1, maxcycle):
        tmpH = vbas.dot(wbas.T)
        tmpS = vbas.dot(sbas.T)
        tmpH = 0.5 * (tmpH + tmpH.T)
        tmpS = 0.5 * (tmpS + tmpS.T)
        eig, vr = scipy.linalg.eigh(tmpH, tmpS)
        vr = vr[:, :neig].T.copy()
        teig = eig[:neig]
        econv = [abs(teig[i] - eigs[i]) <= crit_e for i in range(neig)]
        eigs = teig.copy()
        rbas = vr.dot(wbas) - numpy.diag(eigs).dot(vr.dot(sbas))
        rindx, rconv = [], []
        for i in range(neig):
            rconv.append(numpy.linalg.norm(rbas[i]) <= crit_vec)
            if not rconv[-1] and not econv[i]:
                rindx.append(i)
        if trace is not None:       # (iteration, subspace size, matvecs, eigenvalues, residual norms)
            trace.append((niter, vbas.shape[0], nmvp, eigs.copy(), numpy.linalg.norm(rbas, axis=1)))
        if len(rindx) == 0 or niter == maxcycle - 1:
            return eigs, vr.dot(vbas), nmvp
        if vbas.shape[0] > nfac * neig:
            pr = numpy.identity(vbas.shape[0])[:neig, :] - vr
            vr = _gen_ortho(numpy.vstack((vr, pr[rindx, :])), crit_indp)
            vbas, wbas, sbas = vr.dot(vbas), vr.dot(wbas), vr.dot(sbas)
        for i in range(neig):
            if not rconv[i]:
                rbas[i] = rbas[i] / (numpy.abs(diag - eigs[i]) + lshift)
        nindp, vbas2 = _ortho(vbas, rbas[rindx, :], crit_indp)
        if nindp == 0:
            raise RuntimeError("generalised Davidson: unable to generate a new direction")
        wbas2 = numpy.array([hvec(v) for v in vbas2])
        sbas2 = numpy.array([svec_(v) for v in vbas2])
        nmvp += nindp
        vbas = numpy.vstack((vbas, vbas2))
        wbas = numpy.vstack((wbas, wbas2))
        sbas = numpy.vstack((sbas, sbas2))
    return eigs, vr.dot(vbas), nmvp


# ----------------------------------------------------------------- sweep
class SPOracleDMRG(OracleDMRG):
    """The two-site Qt sweep with spin projection (ifs2proj, one MPI rank)."""

    def __init__(self, ham, npts, sval=0.0, sz=0.0):
        self.qpts, self.qwts = s2quad(npts, sval, sz)
        super(SPOracleDMRG, self).__init__(ham, mpo=build_mpo_sp(ham, self.qpts))
        self.npts = npts
        self.qkey = numpy.array([float(ham.nelec), float(sz)])
        ops = sp_opers(ham.sbas, npts)
        self.opers = [p for (p, g) in ops]
        self.nops = len(ops)
        self.hpwts = numpy.array([self.qwts[g] for (p, g) in ops])
        self.pops = [rotation_op(t) for t in self.qpts]

    def load_mps(self, init):
        K = self.nsite
        self.qnuml = [numpy.array(init["qnum%d" % i], dtype=numpy.float64).reshape(-1, 2) for i in range(K + 1)]
        self.qnumr = [None] * (K + 1)
        self.qnumr[K] = numpy.array([[0., 0.]])
        self.lmps = []
        for i in range(K):
            q = QTensor([False, False, True])
            q.from_dense(numpy.asarray(init["site%d" % i], dtype=numpy.float64),
                         [self.qnuml[i], QPHYS, self.qnuml[i + 1]])
            self.lmps.append(q)
        self.rmps = [None] * K
        self.renv = {K: boundary_env_n(self.nops)}
        self.lenv = {-1: boundary_env_n(self.nops)}
        self.prenv = {K: boundary_env_n(self.npts)}
        self.plenv = {-1: boundary_env_n(self.npts)}
        for i in range(K):
            s = self.lmps[i].reduce_to_n()
            self.lenv[i] = RenormOracle(self.opers, i, "L")(s, self.lenv[i - 1], self.mpo[i])
            self.plenv[i] = renorm_p(s, self.plenv[i - 1], self.pops, i, "L")
        self.psi0 = None

    def solve_dot(self, isite, status, dmax, crit_e):
        ql = self.qnuml[isite]
        qr = self.qnumr[isite + 2]
        ldim, rdim = len(ql), len(qr)
        dims = (ldim, 16, rdim, ldim * 16 * rdim)
        qtmp = QTensor([False, False, False, True])
        cls = [classification(q) for q in (ql, QPHYS, QPHYS, self.qkey - qr)]
        qtmp.from_qsyms(4, [c[0] for c in cls], [c[1] for c in cls])
        prjmap = qtmp.prjmap([c[2] for c in cls])
        lenv, renv = self.lenv[isite - 1], self.renv[isite + 2]
        wi, wj = self.mpo[isite], self.mpo[isite + 1]
        diag = hdiag(prjmap, dims, lenv, renv, wi, wj, self.hpwts)
        hv = sigma_sp(qtmp, self.qkey, lenv, renv, wi, wj, self.opers, self.hpwts, isite)
        sv = svec(qtmp, self.qkey, self.plenv[isite - 1], self.prenv[isite + 2], self.pops, self.qwts, isite)
        v0 = None if self.psi0 is None else self.psi0[0:1, prjmap].copy()
        eig, vec, nmvp = gdavidson(hv, sv, diag, 1, v0, crit_e=crit_e, crit_vec=self.crit_vec)
        self.nhvec += nmvp
        civec = numpy.zeros((1, dims[3]))
        civec[:, prjmap] = vec
        res = self.decimate(civec, isite, status, dims, dmax)
        return eig, nmvp, res, dims, lenv, renv

    def renormalize(self, isite, status, q):
        s = q.reduce_to_n()
        if status == "L":
            self.lenv[isite] = RenormOracle(self.opers, isite, "L")(s, self.lenv[isite - 1], self.mpo[isite])
            self.plenv[isite] = renorm_p(s, self.plenv[isite - 1], self.pops, isite, "L")
        else:
            self.renv[isite] = RenormOracle(self.opers, isite, "R")(s, self.renv[isite + 1], self.mpo[isite])
            self.prenv[isite] = renorm_p(s, self.prenv[isite + 1], self.pops, isite, "R")
