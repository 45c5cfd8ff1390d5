"""Davidson eigensolver on the GPU in FP64 (pdvdson.eigenSolver.solve_iter).

Follows source/tools/pdvdson.py:90-330: start vector from the diagonal
(genV0, :81-87) or the guess, Rayleigh-Ritz in the subspace, residuals,
convergence when every residual norm <= crit_vec or its eigenvalue changed by
<= crit_e, restart to span{x, x_old - x} once the subspace exceeds nfac*neig,
preconditioner iop=4  r / (|diag - e| + 1e-4)  (:275-278) unless a
preconditioner object is supplied, and 5-pass Gram-Schmidt (dvdson_ortho,
:350-390).  All vectors stay on the device; the subspace eigenproblem is a
cuSOLVER eigh.  The matrix-vector product is called one vector at a time, as
the reference's HVecs does (:67-78).
"""
import torch

# a start vector of smaller norm carries no usable direction (a projected guess whose
# weight lies outside the dot's blocks is rounding noise)
V0_MIN_NORM = 1.e-8


def _ortho(vbas, rbas, crit_indp, times=5):
    rbas = rbas.clone()
    for _ in range(times):
        rbas = rbas - (rbas @ vbas.T) @ vbas
    out = []
    for i in range(rbas.shape[0]):
        r = rbas[i].clone()
        n = torch.linalg.norm(r)
        if float(n) <= crit_indp:
            continue
        r = r / n
        r = r / torch.linalg.norm(r)
        out.append(r)
        v2 = torch.stack(out)
        for _ in range(times):
            rbas[i:] -= (rbas[i:] @ vbas.T) @ vbas
            rbas[i:] -= (rbas[i:] @ v2.T) @ v2
    if not out:
        return 0, None
    return len(out), torch.stack(out)


def gen_v0(diag, neig):
    n = diag.numel()
    d = diag + 1.e-12 * torch.arange(1, 1 + n, dtype=diag.dtype, device=diag.device) / float(n)
    idx = torch.argsort(d)[:neig]
    v0 = torch.zeros((neig, n), dtype=diag.dtype, device=diag.device)
    v0[torch.arange(neig, device=diag.device), idx] = 1.0
    return v0


class DavidsonResult(object):
    def __init__(self, eigs, vecs, nmvp, niter, rnorms):
        self.eigs, self.vecs, self.nmvp, self.niter, self.rnorms = eigs, vecs, nmvp, niter, rnorms


def davidson(hvec, diag, neig=1, v0=None, crit_e=1.e-8, crit_vec=1.e-8, maxcycle=20, crit_indp=1.e-12,
             lshift=1.e-4, nfac=10, precond=None, record=None):
    """Lowest ``neig`` eigenpairs of the operator ``hvec`` (device FP64 vectors)."""
    gen = davidson_steps(diag, neig, v0, crit_e, crit_vec, maxcycle, crit_indp, lshift, nfac, precond, record)
    try:
        x = next(gen)
        while True:
            x = gen.send(hvec(x))
    except StopIteration as stop:
        return stop.value


def davidson_steps(diag, neig=1, v0=None, crit_e=1.e-8, crit_vec=1.e-8, maxcycle=20, crit_indp=1.e-12,
                   lshift=1.e-4, nfac=10, precond=None, record=None):
    """The same solver as a generator: yields every vector to multiply, receives H x,
    and returns the DavidsonResult -- so many independent solves can share one
    batched matrix-vector launch per step."""
    ndim = diag.numel()
    if neig > ndim:
        raise ValueError("neig > ndim")
    vbas = gen_v0(diag, neig) if v0 is None else v0.reshape(neig, ndim).to(torch.float64).clone()
    n0 = float(torch.linalg.norm(vbas[0]))
    if not n0 > V0_MIN_NORM:
        # the guess has (numerically) no weight in this dot's blocks: the reference's
        # genOrthoBas would divide by ~0 here; start from the diagonal instead (genV0)
        vbas = gen_v0(diag, neig)
        n0 = 1.0
    vbas[0] = vbas[0] / n0
    if neig > 1:
        n, v2 = _ortho(vbas[0:1], vbas[1:], crit_indp)
        if n + 1 != neig:
            raise RuntimeError("insufficient orthonormal start basis")
        vbas[1:] = v2
    ws_ = []
    for v in vbas:
        ws_.append((yield v))
    wbas = torch.stack(ws_)
    nmvp = neig
    eigs = torch.full((neig,), 1.e3, dtype=torch.float64, device=diag.device)
    rnorms = []
    for niter in range(1, maxcycle):
        h = vbas @ wbas.T
        h = 0.5 * (h + h.T)
        e, u = torch.linalg.eigh(h)
        vr = u[:, :neig].T.contiguous()
        teig = e[:neig]
        econv = (teig - eigs).abs() <= crit_e
        eigs = teig.clone()
        xbas = vr @ vbas
        rbas = vr @ wbas - eigs[:, None] * xbas
        rn = torch.linalg.norm(rbas, dim=1)
        hh = torch.cat([rn, econv.to(rn.dtype)]).cpu().tolist()      # one device->host copy per step
        rn_h = hh[:neig]
        ec_h = [v != 0.0 for v in hh[neig:]]
        rnorms.append(rn_h)
        rconv = [x <= crit_vec for x in rn_h]
        rindx = [i for i in range(neig) if not rconv[i] and not ec_h[i]]
        if len(rindx) == 0 or niter == maxcycle - 1:
            return DavidsonResult(eigs.cpu().numpy(), xbas, nmvp, niter, rnorms)
        nsub = vbas.shape[0]
        if nsub > nfac * neig:
            pr = torch.eye(nsub, dtype=torch.float64, device=diag.device)[:neig, :] - vr
            nindp, vr2 = _ortho(vr, pr[rindx, :], crit_indp)
            if nindp:
                vr = torch.cat([vr, vr2])
            vbas = vr @ vbas
            wbas = vr @ wbas
        for i in range(neig):
            if rconv[i]:
                continue
            if record is not None:      # raw residual, before preconditioning
                record(rbas[i], diag, eigs[i], xbas[i])
            if precond is None:
                rbas[i] = rbas[i] / ((diag - eigs[i]).abs() + lshift)
            else:
                rbas[i] = precond(rbas[i], diag, eigs[i], xbas[i])
        nindp, vbas2 = _ortho(vbas, rbas[rindx, :], crit_indp)
        if nindp == 0:
            raise RuntimeError("Davidson: unable to generate a new direction")
        ws_ = []
        for v in vbas2:
            ws_.append((yield v))
        wbas2 = torch.stack(ws_)
        nmvp += nindp
        vbas = torch.cat([vbas, vbas2])
        wbas = torch.cat([wbas, wbas2])
    return DavidsonResult(eigs.cpu().numpy(), vr @ vbas, nmvp, maxcycle, rnorms)


def _gen_ortho(vbas, crit_indp):
    """First row normalised, the others orthonormalised against it and each other
    (pgdvdson.genOrthoBas, source/tools/pgdvdson.py:362-374)."""
    v0 = vbas[0:1] / torch.linalg.norm(vbas[0])
    if vbas.shape[0] == 1:
        return v0
    n, v2 = _ortho(v0, vbas[1:], crit_indp)
    return torch.cat([v0, v2]) if n else v0


def _eigh_general(h, s):
    """Generalised symmetric eigenproblem h x = e s x with s positive definite, by the
    Cholesky reduction s = C C^T: eigenvectors normalised to x^T s x = 1 (as LAPACK sygvd)."""
    c, info = torch.linalg.cholesky_ex(s)
    if int(info) != 0:
        raise RuntimeError("generalised Davidson: the subspace metric is not positive definite")
    a = torch.linalg.solve_triangular(c, h, upper=False)
    a = torch.linalg.solve_triangular(c, a.T, upper=False)
    a = 0.5 * (a + a.T)
    e, y = torch.linalg.eigh(a)
    x = torch.linalg.solve_triangular(c.T, y, upper=True)
    return e, x


def gdavidson(hvec, svec, diag, neig=1, v0=None, crit_e=1.e-8, crit_vec=1.e-8, maxcycle=20, crit_indp=1.e-12,
              lshift=1.e-4, nfac=10):
    """Lowest ``neig`` solutions of H x = e S x (pgdvdson.eigenSolver.solve_iter,
    source/tools/pgdvdson.py:90-330): the subspace problem is generalised, residuals are
    H x - e S x, the restart keeps span{x, x_old - x} orthonormalised by genOrthoBas, the
    preconditioner is iop=4 and the start vectors carry no noise.  The returned vectors
    are S-normalised.  Both products are called one vector at a time (HSVecs, :63-75)."""
    ndim = diag.numel()
    if neig > ndim:
        raise ValueError("neig > ndim")
    vbas = gen_v0(diag, neig) if v0 is None else v0.reshape(neig, ndim).to(torch.float64).clone()
    vbas = _gen_ortho(vbas, crit_indp)
    wbas = torch.stack([hvec(v) for v in vbas])
    sbas = torch.stack([svec(v) for v in vbas])
    nmvp = vbas.shape[0]
    eigs = torch.full((neig,), 1.e3, dtype=torch.float64, device=diag.device)
    rnorms = []
    for niter in range(1, maxcycle):
        h = vbas @ wbas.T
        s = vbas @ sbas.T
        e, u = _eigh_general(0.5 * (h + h.T), 0.5 * (s + s.T))
        vr = u[:, :neig].T.contiguous()
        teig = e[:neig]
        econv = (teig - eigs).abs() <= crit_e
        eigs = teig.clone()
        rbas = vr @ wbas - eigs[:, None] * (vr @ sbas)
        rn_h = torch.linalg.norm(rbas, dim=1).cpu().tolist()
        ec_h = econv.cpu().tolist()
        rnorms.append(rn_h)
        rconv = [x <= crit_vec for x in rn_h]
        rindx = [i for i in range(neig) if not rconv[i] and not ec_h[i]]
        if len(rindx) == 0 or niter == maxcycle - 1:
            return DavidsonResult(eigs.cpu().numpy(), vr @ vbas, nmvp, niter, rnorms)
        nsub = vbas.shape[0]
        if nsub > nfac * neig:
            pr = torch.eye(nsub, dtype=torch.float64, device=diag.device)[:neig, :] - vr
            vr = _gen_ortho(torch.cat([vr, pr[rindx, :]]), crit_indp)
            vbas, wbas, sbas = vr @ vbas, vr @ wbas, vr @ sbas
        for i in range(neig):
            if not rconv[i]:
                rbas[i] = rbas[i] / ((diag - eigs[i]).abs() + lshift)
        nindp, vbas2 = _ortho(vbas, rbas[rindx, :], crit_indp)
        if nindp == 0:
            raise RuntimeError("generalised Davidson: unable to generate a new direction")
        wbas2 = torch.stack([hvec(v) for v in vbas2])
        sbas2 = torch.stack([svec(v) for v in vbas2])
        nmvp += nindp
        vbas = torch.cat([vbas, vbas2])
        wbas = torch.cat([wbas, wbas2])
        sbas = torch.cat([sbas, sbas2])
    return DavidsonResult(eigs.cpu().numpy(), vr @ vbas, nmvp, maxcycle, rnorms)
