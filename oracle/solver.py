"""ORACLE (test infrastructure only): Davidson solver and RDM decimation.

davidson()      restates source/tools/pdvdson.py:90-330 (eigenSolver.solve_iter,
                iop=4 preconditioner, restart to span{x, x_old-x} when the
                subspace exceeds nfac*neig) with genOrthoBas/dvdson_ortho
                (:336-390, 5-pass Gram-Schmidt) and genV0 (:81-87).
rdm_blkdiag()   restates source/mpo_dmrg_qparser.py:106-183: eigh per
                symmetry class, global descending sort (numpy argsort, the same
                tie-breaking as the reference), truncation by thresh and Dcut,
                discarded weight, re-sort of kept states by quantum number.
"""
import numpy
import scipy.linalg


def _ortho(vbas, rbas, crit_indp, times=5):
    rbas = rbas.copy()
    for _ in range(times):
        rbas = rbas - (rbas.dot(vbas.T)).dot(vbas)
    out = []
    for i in range(rbas.shape[0]):
        r = rbas[i].copy()
        n = numpy.linalg.norm(r)
        if n <= crit_indp:
            continue
        r = r / n
        r = r / numpy.linalg.norm(r)
        out.append(r)
        v2 = numpy.array(out)
        for _ in range(times):
            rbas[i:] -= (rbas[i:].dot(vbas.T)).dot(vbas)
            rbas[i:] -= (rbas[i:].dot(v2.T)).dot(v2)
    v2 = numpy.array(out).reshape(len(out), rbas.shape[1])
    return len(out), v2


def gen_v0(diag, neig):
    n = len(diag)
    d = diag + 1.e-12 * numpy.arange(1, 1 + n) / float(n)
    idx = numpy.argsort(d)[:neig]
    v0 = numpy.zeros((neig, n))
    v0[numpy.arange(neig), idx] = 1.0
    return v0


def davidson(hvec, diag, neig=1, v0=None, crit_e=1.e-8, crit_vec=1.e-8, maxcycle=20,
             crit_indp=1.e-12, lshift=1.e-4, nfac=10, precond=None):
    """Returns (eigs, vecs, nmvp).  ``precond(r, diag, e) -> correction`` overrides iop=4."""
    ndim = len(diag)
    vbas = gen_v0(diag, neig) if v0 is None else numpy.array(v0, dtype=numpy.float64).reshape(neig, ndim)
    vbas[0] = vbas[0] / numpy.linalg.norm(vbas[0])
    if neig > 1:
        n, v2 = _ortho(vbas[0:1], vbas[1:], crit_indp)
        vbas[1:] = v2
    nmvp = 0
    wbas = numpy.array([hvec(v) for v in vbas])
    nmvp += len(vbas)
    eigs = numpy.zeros(neig) + 1.e3
    nsub = neig
    for niter in range(1, maxcycle):
        tmpH = vbas.dot(wbas.T)
        tmpH = 0.5 * (tmpH + tmpH.T)
        eig, vr = scipy.linalg.eigh(tmpH)
        vr = vr[:, :neig].T.copy()
        teig = eig[:neig]
        econv = [abs(teig[i] - eigs[i]) <= crit_e for i in range(neig)]
        eigs = teig.copy()
        rbas = vr.dot(wbas) - numpy.diag(eigs).dot(vr.dot(vbas))
        rindx = []
        rconv = []
        for i in range(neig):
            rn = numpy.linalg.norm(rbas[i])
            rconv.append(rn <= crit_vec)
            if not rconv[-1] and not econv[i]:
                rindx.append(i)
        if len(rindx) == 0 or niter == maxcycle - 1:
            return eigs, vr.dot(vbas), nmvp
        if nsub > nfac * neig:
            pr = numpy.identity(nsub)[:neig, :] - vr
            nindp, vr2 = _ortho(vr, pr[rindx, :], crit_indp)
            if nindp != 0:
                vr = numpy.vstack((vr, vr2))
            vbas = vr.dot(vbas)
            wbas = vr.dot(wbas)
        for i in range(neig):
            if rconv[i]:
                continue
            if precond is None:
                rbas[i] = rbas[i] / (numpy.abs(diag - eigs[i]) + lshift)
            else:
                rbas[i] = precond(rbas[i], diag, eigs[i])
        nindp, vbas2 = _ortho(vbas, rbas[rindx, :], crit_indp)
        if nindp == 0:
            raise RuntimeError("Davidson: unable to generate a new direction")
        wbas2 = numpy.array([hvec(v) for v in vbas2])
        nmvp += nindp
        vbas = numpy.vstack((vbas, vbas2))
        wbas = numpy.vstack((wbas, wbas2))
        nsub = vbas.shape[0]
    return eigs, vr.dot(vbas), nmvp


def rdm_blkdiag(rho, classes, thresh, dcut=-1):
    """Returns (dwts, qsyms kept, rotL[:, kept], sigs kept)."""
    groups = {}
    order = []
    for idx, val in enumerate(classes):
        key = tuple(float(x) for x in val)
        if key not in groups:
            groups[key] = []
            order.append(key)
        groups[key].append(idx)
    nrows = rho.shape[0]
    qsym, rot, sig = [], [], []
    for key in order:
        rows = groups[key]
        s2, u = scipy.linalg.eigh(rho[numpy.ix_(rows, rows)])
        s2 = numpy.abs(s2)
        qsym += [list(key)] * len(s2)
        col = numpy.zeros((nrows, len(s2)))
        col[rows, :] = u
        rot.append(col)
        sig.append(s2)
    rot = numpy.hstack(rot)
    sig = numpy.hstack(sig)
    sig = sig / numpy.sum(sig)
    indx = numpy.argsort(sig)[::-1]
    nres = len(sig)
    tsig = sig[indx]
    for i in range(nres):
        if tsig[i] < thresh * 1.01:
            nres = i
            break
    if nres == 0:
        nres = 1
    if dcut > 0:
        nres = min(nres, dcut)
    indx = indx[:nres]
    sig = sig[indx].copy()
    dwts = 1.0 - numpy.sum(sig)
    qsym = [qsym[i] for i in indx]
    rot = rot[:, indx]
    o = sorted(range(nres), key=lambda x: qsym[x])
    qsym = [qsym[i] for i in o]
    return dwts, qsym, rot[:, o].copy(), sig[o].copy()
