"""ORACLE (test infrastructure only): sigma, diagonal and renormalisation.

Restates, for the two-site dot and maxslc = 1:
  HVecQt        source/mpo_dmrg_kernelQt.py:153-319 (two-site branch :238-317)
  HDiagQt       source/mpo_dmrg_kernelQt.py:30-127  (two-site branch :77-119)
  renormQt_H00  source/mpo_dmrg_kernelQt.py:633-767
  pRDMQt        source/mpo_dmrg_kernelQt.py:453-626 (noise term, status L/R)
  genBopsQt     source/mpo_dmrg_initQt.py:49-85 (boundary operators)
Operators are indexed by spin orbital p with weights hpwts[p] (= 1 for plain H).
Templates (pair lists) are cached per symmetry class exactly like the
reference's ``ista`` dictionaries, which is what makes one plan valid for every
operator of a class.
"""
import numpy

from .blocks import QTensor, Contraction
from .mpo import case


def boundary_env(nop):
    """genBopsQt: a 1x1x1 operator with zero quantum numbers for every p."""
    out = []
    for _ in range(nop):
        q = QTensor([True, False, True])
        q.from_dense(numpy.ones((1, 1, 1)), [[[0., 0.]]] * 3)
        out.append(q)
    return out


def flip_right(rop, qkey):
    """R operators seen from the left: qsyms -> [-q0, qkey-q1, qkey-q2] (kernelQt.py:297-300)."""
    q = QTensor(rop.status)
    q.from_qsyms(rop.rank, [-rop.qsyms[0], qkey - rop.qsyms[1], qkey - rop.qsyms[2]], rop.ndims, allocate=False)
    q.value = rop.value
    q.idlst = rop.idlst
    return q


def flip_horizontal(cop):
    """W seen from the right: negate and flip the two bond indices (kernelQt.py:723-727)."""
    q = QTensor(numpy.array([not cop.status[0], not cop.status[1], cop.status[2], cop.status[3]]))
    q.from_qsyms(cop.rank, [-cop.qsyms[0], -cop.qsyms[1], cop.qsyms[2], cop.qsyms[3]], cop.ndims, allocate=False)
    q.value = cop.value
    q.idlst = cop.idlst
    return q


class SigmaOracle(object):
    """H_eff * psi for the two-site dot (isite, isite+1)."""

    def __init__(self, qtmp, qkey, lenv, renv, wi, wj, opers, hpwts, isite):
        self.qtmp, self.qkey = qtmp, numpy.asarray(qkey, dtype=numpy.float64)
        self.lenv, self.renv, self.wi, self.wj = lenv, renv, wi, wj
        self.opers, self.hpwts, self.isite = opers, hpwts, isite
        self.templates = {}
        self.flops = 0

    def _plans(self, iop, psi):
        key = case(self.opers[iop], self.isite, 2)
        if key not in self.templates:
            L, W1, W2 = self.lenv[iop], self.wi[iop], self.wj[iop]
            R = flip_right(self.renv[iop], self.qkey)
            c1 = Contraction().plan(L, psi, ([2], [0]))
            c2 = Contraction().plan(c1.out, W1, ([0, 2], [0, 3]))
            c3 = Contraction().plan(c2.out, W2, ([1, 3], [3, 0]))
            c4 = Contraction().plan(c3.out, R, ([1, 3], [2, 0]))
            assert c4.out.size_allowed == self.qtmp.size_allowed
            self.templates[key] = (c1, c2, c3, c4)
        return self.templates[key]

    def __call__(self, x):
        psi = self.qtmp.copy_structure()
        psi.value = numpy.asarray(x, dtype=numpy.float64)
        y = numpy.zeros(self.qtmp.size_allowed)
        for iop in range(len(self.opers)):
            c1, c2, c3, c4 = self._plans(iop, psi)
            R = flip_right(self.renv[iop], self.qkey)
            t1 = c1.run(self.lenv[iop], psi)
            t2 = c2.run(t1, self.wi[iop])
            t3 = c3.run(t2, self.wj[iop])
            t4 = c4.run(t3, R)
            y += self.hpwts[iop] * t4.value
        return y

    def count_flops(self, x=None):
        psi = self.qtmp.copy_structure()
        tot = 0
        for iop in range(len(self.opers)):
            c1, c2, c3, c4 = self._plans(iop, psi)
            R = flip_right(self.renv[iop], self.qkey)
            tot += c1.flops(self.lenv[iop], psi)
            tot += c2.flops(c1.out, self.wi[iop])
            tot += c3.flops(c2.out, self.wj[iop])
            tot += c4.flops(c3.out, R)
        return tot


def hdiag(prjmap, dims, lenv, renv, wi, wj, hpwts):
    """HDiagQt two-site: diag[l,n,m,r] = sum_p w_p L[a,l,l] Wi[a,b,n,n] Wj[b,c,m,m] R[c,r,r]."""
    ldim, cdim, rdim, ndim = dims
    diag = numpy.zeros(ndim)
    for iop in range(len(lenv)):
        ld = lenv[iop].to_dense_diag()
        cd = wi[iop].to_dense_diag()
        wd = wj[iop].to_dense_diag()
        rd = renv[iop].to_dense_diag()
        t = numpy.tensordot(ld, cd, axes=([0], [0]))
        t = numpy.tensordot(t, wd, axes=([1], [0]))
        t = numpy.tensordot(t, rd, axes=([2], [0]))
        diag += hpwts[iop] * t.reshape(ndim)
    return diag[prjmap].copy()


class RenormOracle(object):
    """renormQt_H00: new environment for every operator after a decimation."""

    def __init__(self, opers, isite, status):
        self.opers, self.isite, self.status = opers, isite, status
        self.templates = {}

    def __call__(self, site, env, cops):
        out = []
        for iop in range(len(cops)):
            key = case(self.opers[iop], self.isite)
            if self.status == "L":
                cop = cops[iop]
                if key not in self.templates:
                    c1 = Contraction().plan(site, env[iop], ([0], [1]))
                    c2 = Contraction().plan(cop, c1.out, ([0, 2], [2, 0]))
                    c3 = Contraction().plan(c2.out, site, ([1, 3], [1, 0]))
                    self.templates[key] = (c1, c2, c3)
                c1, c2, c3 = self.templates[key]
                t = c3.run(c2.run(cop, c1.run(site, env[iop])), site)
                t.idlst = [cop.idlst[1], site.idlst[2], site.idlst[2]]
            else:
                cop = flip_horizontal(cops[iop])
                if key not in self.templates:
                    c1 = Contraction().plan(site, env[iop], ([2], [1]))
                    c2 = Contraction().plan(cop, c1.out, ([1, 2], [2, 1]))
                    c3 = Contraction().plan(c2.out, site, ([1, 3], [1, 2]))
                    self.templates[key] = (c1, c2, c3)
                c1, c2, c3 = self.templates[key]
                t = c3.run(c2.run(cop, c1.run(site, env[iop])), site)
                t.idlst = [cop.idlst[0], site.idlst[0], site.idlst[0]]
            out.append(t)
        return out


def prdm_noise(civec, status, lenv_or_renv, cops, qkey, opers, isite, ncsite, dims, noise):
    """pRDMQt-equivalent noise term sum_p (L.psi.W)(L.psi.W)^+ (dense restatement).

    civec: dense two-site wavefunction [ldim, 4, 4*rdim] for 'L' or [ldim*4, 4, rdim] for 'R'.
    Used by the decimation when noise > 0 (mpo_dmrg_dotutil.py:294-313).
    """
    ldim, cdim, rdim, ndim = dims
    rdm = None
    for iop in range(len(cops)):
        W = cops[iop].to_dense()
        E = lenv_or_renv[iop].to_dense()
        if status == "L":
            t = numpy.tensordot(E, civec, axes=([2], [0]))          # L[p,i,a] B[a,n,b] -> [p,i,n,b]
            t = numpy.tensordot(t, W, axes=([0, 2], [0, 3]))       # -> [i,b,q,m]
            t = t.transpose(0, 3, 1, 2)
            s = t.shape
            t = t.reshape(s[0] * s[1], s[2] * s[3])
            m = t.dot(t.T) * noise
        else:
            t = numpy.tensordot(civec, E, axes=([2], [2]))          # B[a,n,b] R[q,j,b] -> [a,n,q,j]
            t = numpy.tensordot(W, t, axes=([1, 3], [2, 1]))       # W[p,q,m,n] -> [p,m,a,j]
            t = t.transpose(0, 2, 1, 3)
            s = t.shape
            t = t.reshape(s[0] * s[1], s[2] * s[3])
            m = t.T.dot(t) * noise
        rdm = m if rdm is None else rdm + m
    return rdm
