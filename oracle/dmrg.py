"""ORACLE (test infrastructure only): the Qt two-site sweep around the hot path.

Restates the reference's control flow for ifQt=True, ncsite=2, maxslc=1, one
symmetry sector, one MPI rank:
  mpo_dmrg_class.default        source/mpo_dmrg_class.py:329-434 (sweep R then L)
  mpo_dmrg_util.initOps         source/mpo_dmrg_util.py:193-214 (genBopsQt R, genHopsQt L)
  mpo_dmrg_opt.sweep            source/mpo_dmrg_opt.py:31-101, updateSite :319-350,
                                updateBoundary :353-383, checkOpers :151-188
  mpo_dmrg_dot.ci_solver        source/mpo_dmrg_dot.py:24-112
  dotutil setupQtmpCI/decimation/genGuess  source/mpo_dmrg_dotutil.py:173-184,269-476,479-540
Environments are kept in memory instead of HDF5 files.
"""
import time

import numpy

from .blocks import QTensor, classification
from .kernels import SigmaOracle, hdiag, RenormOracle, boundary_env, prdm_noise
from .mpo import QPHYS, build_mpo
from .solver import davidson, rdm_blkdiag


def dpt(q1, q2):
    return numpy.array([numpy.asarray(a) + numpy.asarray(b) for a in q1 for b in q2])


class OracleDMRG(object):
    def __init__(self, ham, mpo=None):
        self.ham = ham
        self.nsite = ham.nsite
        self.nops = ham.sbas
        self.opers = list(range(ham.sbas))
        self.hpwts = numpy.ones(self.nops)
        self.mpo = mpo if mpo is not None else build_mpo(ham)
        self.qkey = numpy.array([float(ham.nelec), 0.0])
        self.crit_vec = 1.e-8
        self.thresh = -1.e-14
        self.noise = 0.0
        self.ifguess = True
        self.log = []
        self.nmvp_total = 0
        self.timings = {"hvec": 0.0, "hdiag": 0.0, "renorm": 0.0, "decim": 0.0}
        self.nhvec = 0

    # ---------------- set-up -----------------
    def load_mps(self, init):
        """init: dict with qnum0..qnumK (arrays [n,2]) and site0..site{K-1} dense [l,4,r]."""
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
        # initOps: R boundary, then all L environments from the L-MPS (genHopsQt 'L')
        self.renv = {K: boundary_env(self.nops)}
        self.lenv = {-1: boundary_env(self.nops)}
        for i in range(K):
            self.lenv[i] = RenormOracle(self.opers, i, "L")(self.lmps[i], self.lenv[i - 1], self.mpo[i])
        self.psi0 = None

    # ---------------- one dot -----------------
    def solve_dot(self, isite, status, dmax, crit_e):
        K = self.nsite
        ql = self.qnuml[isite]
        qr = self.qnumr[isite + 2]
        ldim, rdim = len(ql), len(qr)
        dims = (ldim, 16, rdim, ldim * 16 * rdim)
        qtmp = QTensor([False, False, False, True])
        cls = [classification(q) for q in (ql, QPHYS, QPHYS, self.qkey - qr)]
        qtmp.from_qsyms(4, [c[0] for c in cls], [c[1] for c in cls])
        idlst = [c[2] for c in cls]
        prjmap = qtmp.prjmap(idlst)
        lenv, renv = self.lenv[isite - 1], self.renv[isite + 2]
        wi, wj = self.mpo[isite], self.mpo[isite + 1]
        t0 = time.time()
        diag = hdiag(prjmap, dims, lenv, renv, wi, wj, self.hpwts)
        self.timings["hdiag"] += time.time() - t0
        sig = SigmaOracle(qtmp, self.qkey, lenv, renv, wi, wj, self.opers, self.hpwts, isite)

        def hv(x):
            t = time.time()
            y = sig(x)
            self.timings["hvec"] += time.time() - t
            self.nhvec += 1
            return y

        v0 = None if self.psi0 is None else self.psi0[0:1, prjmap].copy()
        eig, vec, nmvp = davidson(hv, diag, 1, v0, crit_e=crit_e, crit_vec=self.crit_vec)
        civec = numpy.zeros((1, dims[3]))
        civec[:, prjmap] = vec
        t0 = time.time()
        res = self.decimate(civec, isite, status, dims, dmax)
        self.timings["decim"] += time.time() - t0
        return eig, nmvp, res, dims, lenv, renv

    def decimate(self, civecs, isite, status, dims, dmax):
        ldim, cdim, rdim, ndim = dims
        neig = civecs.shape[0]
        if status == "L":
            lcdim, crdim = ldim * 4, 4 * rdim
            c = civecs.reshape(neig, lcdim, crdim)
            rdm = sum(c[i].dot(c[i].T) for i in range(neig))
            if self.noise >= 1.e-10:
                rdm = rdm + prdm_noise(civecs[0].reshape(ldim, 4, crdim), "L", self.lenv[isite - 1],
                                       self.mpo[isite], self.qkey, self.opers, isite, 2, dims, self.noise)
            classes = dpt(self.qnuml[isite], QPHYS)
        else:
            lcdim, crdim = ldim * 4, 4 * rdim
            c = civecs.reshape(neig, lcdim, crdim)
            rdm = sum(c[i].T.dot(c[i]) for i in range(neig))
            if self.noise >= 1.e-10:
                rdm = rdm + prdm_noise(civecs[0].reshape(lcdim, 4, rdim), "R", self.renv[isite + 2],
                                       self.mpo[isite + 1], self.qkey, self.opers, isite, 2, dims, self.noise)
            classes = dpt(QPHYS, self.qnumr[isite + 2])
        tr = numpy.trace(rdm)
        if abs(tr) < 1.e-12:
            rdm = rdm + numpy.identity(rdm.shape[0]) / float(rdm.shape[0])
        else:
            rdm = rdm / tr
        dwts, qred, rot, sigs = rdm_blkdiag(rdm, classes, self.thresh, dmax)
        nres = len(qred)
        if status == "L":
            site = rot.reshape(ldim, 4, nres).copy()
            srotR = numpy.array([rot.T.dot(c[i]).reshape(nres, 4, rdim) for i in range(neig)])
        else:
            site = rot.reshape(4, rdim, nres).transpose(2, 0, 1).copy()
            srotR = numpy.array([c[i].dot(rot).reshape(ldim, 4, nres) for i in range(neig)])
        return dwts, numpy.array(qred, dtype=numpy.float64), site, srotR, civecs

    # ---------------- sweeps -----------------
    def sweep(self, status, dmax, crit_e):
        K = self.nsite
        actlst = list(range(0, K - 1)) if status == "L" else list(range(K - 2, -1, -1))
        elst, dlst, nmvp = [], [], 0
        for isite in actlst:
            eig, nm, (dwts, qred, site, srotR, civecs), dims, lenv, renv = self.solve_dot(isite, status, dmax, crit_e)
            nmvp += nm
            elst.append(eig[0])
            dlst.append(dwts)
            t0 = time.time()
            if status == "L":
                self.qnuml[isite + 1] = qred
                q = QTensor([False, False, True])
                q.from_dense(site, [self.qnuml[isite], QPHYS, qred])
                self.lmps[isite] = q
                self.renormalize(isite, "L", q)
            else:
                j = isite + 1
                self.qnumr[j] = qred
                q = QTensor([True, False, False])
                q.from_dense(site, [qred, QPHYS, self.qnumr[j + 1]])
                self.rmps[j] = q
                self.renormalize(j, "R", q)
            self.timings["renorm"] += time.time() - t0
            self.guess(isite, status, actlst, civecs, srotR)
            self.log.append({"status": status, "isite": isite, "e": float(eig[0]), "dwt": float(dwts),
                             "nmvp": int(nm), "bond": int(len(qred))})
        # sweep_updateBoundary
        smat = srotR[0]
        smat = smat / numpy.linalg.norm(smat)
        if status == "L":
            q = QTensor([False, False, True])
            q.from_dense(smat, [qred, QPHYS, self.qkey.reshape(1, 2)])
            self.lmps[K - 1] = q
            self.qnuml[K] = self.qkey.reshape(1, 2).copy()
        else:
            q = QTensor([True, False, False])
            q.from_dense(smat, [self.qkey.reshape(1, 2), QPHYS, qred])
            self.rmps[0] = q
            self.qnumr[0] = self.qkey.reshape(1, 2).copy()
        eav_i = int(numpy.argmin(elst))
        self.nmvp_total += nmvp
        return nmvp, elst[eav_i], dlst[eav_i], elst, dlst

    def renormalize(self, isite, status, q):
        """renorm (mpo_dmrg_kernel.py:347-377): new environments of site isite."""
        if status == "L":
            self.lenv[isite] = RenormOracle(self.opers, isite, "L")(q, self.lenv[isite - 1], self.mpo[isite])
        else:
            self.renv[isite] = RenormOracle(self.opers, isite, "R")(q, self.renv[isite + 1], self.mpo[isite])

    def guess(self, isite, status, actlst, civecs, srotR):
        if not self.ifguess:
            return
        if isite == actlst[-1]:
            self.psi0 = civecs.copy()
        elif status == "R":
            t = self.lmps[isite - 1].to_dense()
            self.psi0 = numpy.array([numpy.tensordot(t, srotR[i], axes=([2], [0])).ravel()
                                     for i in range(srotR.shape[0])])
        else:
            t = self.rmps[isite + 2].to_dense()
            self.psi0 = numpy.array([numpy.tensordot(srotR[i], t, axes=([2], [0])).ravel()
                                     for i in range(srotR.shape[0])])

    def run(self, init_mps, dmax, nsweeps, tol=1.e-7, noise=0.0):
        """mpo_dmrg_class.default with schedule.fixed(ncsite=2, maxM=dmax, tol=tol, noise=noise)."""
        self.noise = noise
        self.load_mps(init_mps)
        eav, dwt, esweeps, nmvps = [], [], [], []
        eold = 1.e3
        for isweep in range(nsweeps):
            n1, e1, d1, el1, dl1 = self.sweep("R", dmax, tol)
            n2, e2, d2, el2, dl2 = self.sweep("L", dmax, tol)
            nmvps.append(n1 + n2)
            esweeps += el1 + el2
            if e1 < e2:
                eav.append(e1)
                dwt.append(d1)
            else:
                eav.append(e2)
                dwt.append(d2)
            if abs(eav[-1] - eold) < tol:
                break
            eold = eav[-1]
        return {"eav": numpy.array(eav), "dwt": numpy.array(dwt), "esweeps": numpy.array(esweeps),
                "nmvp": numpy.array(nmvps)}
