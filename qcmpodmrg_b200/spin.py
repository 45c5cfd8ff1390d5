"""Spin projection (SP-MPS): H c = S c E with S the projector onto total spin S.

The projector is a quadrature over spin rotations, P = sum_g w_g R(theta_g) with
R(theta) = exp(-i theta S_y) a bond-1 MPO (source/mpo_dmrg_util.py:35-89 for the
quadrature, source/mpo_dmrg_opers.py:228-260 for R and H_p R).  A rotation
conserves only the particle number, so every operator of the projected problem
carries N-only quantum numbers:

  H_eff c   HVecQt with ifs2proj   source/mpo_dmrg_kernelQt.py:153-319
  S c       SVecQt                 source/mpo_dmrg_kernelQt.py:373-450
  diagonals HDiagQt / SDiagQt      source/mpo_dmrg_kernelQt.py:30-127, 322-370
  renorm    renormQt_H00 + _S00    source/mpo_dmrg_kernelQt.py:633-854
  solver    pgdvdson               source/tools/pgdvdson.py:60-330

The wavefunction stays in its (N, Sz) packed layout.  Reducing it to N
symmetry keeps every sector and only adds blocks that are zero
(qtensor.reduceQsymsToN, source/qtensor/qtensor.py:528-543), so on the device
the reduction is one scatter into the N-only layout and the projection back
(projectionNMs, :546-560) one gather through the same index map.  Between the
two, the sigma of the projected operators runs on the same plans and kernels as
the plain two-site sigma, with the operator set x -> (p, g) = (x // npts,
x % npts) weighted by w_g (source/mpo_dmrg_class.py:219-240).
"""
import math
import time

import numpy
import torch

from . import kernels as K
from .kernels import SigmaOperator, DiagOperator, Renormalizer, TensorSet, _ragged
from .mpo import QPHYS, W_STATUS, _hfac_spin, _link, _elem_q, _wq
from .qtensor import Layout, classification
from .dmrg import DMRG, PSI_STATUS, L_STATUS, SiteTensor
from .davidson import gdavidson

QPHYS_N = QPHYS[:, 0:1].copy()


# ------------------------------------------------------------------ quadrature
def smalld(j, mp, ms, beta):
    """Wigner small-d element d^j_{mp,ms}(beta) from its explicit finite sum."""
    frac = [x - math.floor(x) for x in (j, mp, ms)]
    if max(frac) - min(frac) > 1e-10:
        return 0.0
    pre = math.sqrt(math.gamma(j + mp + 1) * math.gamma(j - mp + 1) * math.gamma(j + ms + 1)
                    * math.gamma(j - ms + 1))
    c, s_ = math.cos(0.5 * beta), math.sin(0.5 * beta)
    tot = 0.0
    k = 0.0
    while k <= 2 * j + 0.05:
        if j + ms - k > -0.1 and mp - ms + k > -0.1 and j - mp - k > -0.1:
            den = (math.gamma(j + ms - k + 1) * math.gamma(k + 1) * math.gamma(mp - ms + k + 1)
                   * math.gamma(j - mp - k + 1))
            tot += (math.pow(-1.0, mp - ms + k) / den * math.pow(c, 2 * j + ms - mp - 2 * k)
                    * math.pow(s_, mp - ms + 2 * k))
        k += 1.0
    return pre * tot


def s2quad(npts, sval=0.0, sz=0.0, quad="GaussLegendre"):
    """Rotation angles theta_g in [0, pi] and weights of P_S = (2S+1)/2 int d^S_{sz,sz}(theta)
    R(theta) sin(theta) dtheta (mpo_dmrg_util.s2quad, Gauss-Legendre in cos(theta) or Simpson)."""
    if sval + 1.e-4 <= abs(sz):
        raise ValueError("|Sz| exceeds S")
    if quad == "GaussLegendre":
        x, w = numpy.polynomial.legendre.leggauss(npts)
        pts = numpy.array([math.acos(v) for v in x])
        wts = (2. * sval + 1.) / 2.0 * (numpy.array([smalld(sval, sz, sz, t) for t in pts]) * w)
    elif quad == "Simpson":
        n = npts - 1
        if n <= 0 or n % 2:
            raise ValueError("Simpson needs an odd number of points")
        c = numpy.where(numpy.arange(npts) % 2 == 1, 4.0, 2.0)
        c[0] = c[-1] = 1.0
        pts = numpy.linspace(0, numpy.pi, num=npts)
        f = numpy.array([(2. * sval + 1.) / 2.0 * math.sin(t) * smalld(sval, sz, sz, t) for t in pts])
        wts = c * (numpy.pi / (3.0 * n)) * f
    else:
        raise ValueError("unknown quadrature %r" % quad)
    return pts, wts


# ------------------------------------------------------------------ operators
def exp_isy_phi(phi):
    """exp(-i phi S_y) on one spatial orbital, basis |0>, |b>, |a>, |ab> (real)."""
    c, s_ = math.cos(0.5 * phi), math.sin(0.5 * phi)
    return numpy.array([[1., 0., 0., 0.], [0., c, s_, 0.], [0., -s_, c, 0.], [0., 0., 0., 1.]])


_PHYS_N = classification(QPHYS_N, collect=False)


def _packed(lay, idl, dense):
    return dense.ravel()[lay.prjmap(idl)].copy()


def rotation_set(qpts, device):
    """R(theta_g) for every quadrature point as a TensorSet of [1, 1, 4, 4] site tensors."""
    one = classification(numpy.zeros((1, 1)), collect=False)
    lay = Layout(W_STATUS, [one[0], one[0], _PHYS_N[0], _PHYS_N[0]], [one[1], one[1], _PHYS_N[1], _PHYS_N[1]])
    idl = [one[2], one[2], _PHYS_N[2], _PHYS_N[2]]
    vals = [_packed(lay, idl, exp_isy_phi(t).reshape(1, 1, 4, 4)) for t in qpts]
    return TensorSet([lay] * len(qpts), vals, device=device)


def _order_n(q):
    """Stable order by particle number: equal N contiguous, original order inside."""
    return numpy.argsort(numpy.rint(2 * q[:, 0]).astype(numpy.int64), kind="stable")


def _sp_site_block(p, nsite_spin, isite, int1e, int2e):
    """H_p at spatial site isite with its MPO bond ordered by N (stable), and the N-only
    layout every H_p R(theta) shares: (dense [A, B, 4, 4] in that order, layout, packing map)."""
    hq, v = int1e[p], int2e[p]
    dense = _link(_hfac_spin(p, nsite_spin, 2 * isite, hq, v), _hfac_spin(p, nsite_spin, 2 * isite + 1, hq, v))
    ql1, _ = _elem_q(p, 2 * isite)
    _, qr1 = _elem_q(p, 2 * isite + 1)
    ql2, _ = _wq(nsite_spin, 2 * isite, p % 2)
    _, qr2 = _wq(nsite_spin, 2 * isite + 1, p % 2)
    ql, qr = (ql2 + ql1)[:, 0:1], (qr2 + qr1)[:, 0:1]
    il, ir = _order_n(ql), _order_n(qr)
    cl, cr = classification(ql[il]), classification(qr[ir])
    lay = Layout(W_STATUS, [cl[0], cr[0], _PHYS_N[0], _PHYS_N[0]], [cl[1], cr[1], _PHYS_N[1], _PHYS_N[1]])
    prj = lay.prjmap([cl[2], cr[2], _PHYS_N[2], _PHYS_N[2]])
    return numpy.ascontiguousarray(dense[numpy.ix_(il, ir)]), lay, prj


def sp_site_operator(p, phi, nsite_spin, isite, int1e, int2e):
    """H_p R(phi) at spatial site isite with N-only quantum numbers: (Layout, packed values)."""
    dense, lay, prj = _sp_site_block(p, nsite_spin, isite, int1e, int2e)
    return lay, numpy.tensordot(dense, exp_isy_phi(phi), axes=([3], [0])).ravel()[prj].copy()


def sp_opers(sbas, npts):
    """Operator x -> (p, g), the reference's one-rank partition of npts * sbas operators."""
    return [(x // npts, x % npts) for x in range(sbas * npts)]


def build_mpo_sp(ham, qpts, isites=None):
    """Layouts and values of H_p R(theta_g) for every operator at every spatial site.

    H_p, its bond order and its layout are built once per (p, site); the rotations of
    all quadrature points are applied to it in one contraction."""
    npts = len(qpts)
    rot = numpy.stack([exp_isy_phi(t) for t in qpts]).transpose(1, 0, 2).reshape(4, 4 * npts)   # [m, (g k)]
    out = {}
    for i in (range(ham.nsite) if isites is None else isites):
        lays, vals = [], []
        for p in range(ham.sbas):
            dense, lay, prj = _sp_site_block(p, ham.sbas, i, ham.int1e, ham.int2e)
            a, b = dense.shape[:2]
            allg = (dense.reshape(-1, 4) @ rot).reshape(a, b, 4, npts, 4).transpose(3, 0, 1, 2, 4).reshape(npts, -1)
            for g in range(npts):
                lays.append(lay)
                vals.append(allg[g][prj].copy())
        out[i] = (lays, vals)
    return out


def boundary_set_n(nops, device):
    """Boundary environments (genBopsQt) with N-only quantum numbers."""
    lay = Layout([True, False, True], [numpy.zeros((1, 1))] * 3, [numpy.ones(1, dtype=numpy.int64)] * 3)
    return TensorSet([lay] * nops, [numpy.ones(1)] * nops, device=device)


# ------------------------------------------------------------------ reduction maps
def reduce_layout(lay):
    """The same sectors with N-only quantum numbers (every (N, Sz) block stays a block)."""
    return Layout(lay.status, [q[:, 0:1] for q in lay.qsyms], lay.ndims)


def reduce_map(lay, lay_n):
    """Packed position in ``lay`` -> packed position in ``lay_n`` of the same element."""
    idx = lay.idx_allowed
    if len(idx) == 0:
        return numpy.zeros(0, dtype=numpy.int64)
    if not lay_n.allowed[idx].all():
        raise ValueError("reduced layout lacks a block of the (N, Sz) layout")
    b, e = _ragged(lay.ndim[idx])
    out = numpy.empty(lay.size, dtype=numpy.int64)
    out[lay.ioff[idx][b] + e] = lay_n.ioff[idx][b] + e
    return out


class ProjectedOperator(object):
    """y = P_(N,Sz) A_N (reduce x) for an operator A_N on the N-only layout.

    ``inner`` is a SigmaOperator on the reduced layout; the reduction is a scatter
    (qc_scatter_f64, zeros elsewhere) and the projection a gather (qc_gather_f64)."""

    def __init__(self, ws, inner, red):
        self.ws, self.inner = ws, inner
        self.red = torch.from_numpy(red).to(ws.device)
        self.ndim0 = len(red)
        self.nn = inner.ndim0
        self.flops = inner.flops

    def __call__(self, x, y=None, precision=None):
        xn = self.ws.get("sp_xn", self.nn, torch.float64)[:self.nn]
        K.scatter(x, self.red, xn)
        yn = self.inner(xn, precision=precision)
        if y is None:
            y = torch.empty(self.ndim0, dtype=torch.float64, device=self.ws.device)
        return K.gather(yn, self.red, y)

    def release(self):
        self.inner.release()


# ------------------------------------------------------------------ sweep
class SPDMRG(DMRG):
    """Two-site DMRG for the spin-projected state (ifs2proj=True, one rank).

    Environments of the npts*2K operators H_p R(theta_g) and of the npts projector
    terms R(theta_g) live in HBM; each dot solves H c = S c E with the generalised
    Davidson on the GPU and renormalises both environment sets after the decimation."""

    ifs2proj = True

    def __init__(self, ham, npts, sval=0.0, sz=0.0, device="cuda", w_path="fiber", quad="GaussLegendre",
                 prune_zero_blocks=True, precision="f64"):
        """precision: "f64", or "f32" for FP32 H and S products in the generalised Davidson
        followed by an FP64 check of the solution (FP64 iterations when it fails)."""
        if precision not in ("f64", "f32"):
            raise ValueError("spin projection runs in f64 or f32 (mixed)")
        self.npts, self.sval, self.quad = int(npts), float(sval), quad
        self.prune_zero_blocks = prune_zero_blocks
        super(SPDMRG, self).__init__(ham, device=device, precision=precision, w_path=w_path, sz=sz)

    def _setup_operators(self, ham):
        self.qpts, self.qwts = s2quad(self.npts, self.sval, self.sz, self.quad)
        ops = sp_opers(ham.sbas, self.npts)
        self.nops = len(ops)
        self.opers = [p for (p, g) in ops]
        self.hpwts = numpy.array([self.qwts[g] for (p, g) in ops])
        self.qkey = numpy.array([float(ham.nelec), self.sz])
        mpo = build_mpo_sp(ham, self.qpts)
        self.mpo = {i: TensorSet(l, v, device=self.device) for i, (l, v) in mpo.items()}
        self.pops = rotation_set(self.qpts, self.device)
        self.popers = [0] * self.npts         # one symmetry class for all projector terms

    def _reduced_site(self, st):
        lay_n = reduce_layout(st.layout)
        vals = torch.empty(lay_n.size, dtype=torch.float64, device=self.device)
        K.scatter(st.values, torch.from_numpy(reduce_map(st.layout, lay_n)).to(self.device), vals)
        return lay_n, vals

    def load_mps(self, init):
        Kn = self.nsite
        dev = self.device
        self.qnuml = [numpy.array(init["qnum%d" % i], dtype=numpy.float64).reshape(-1, 2) for i in range(Kn + 1)]
        self.qnumr = [None] * (Kn + 1)
        self.qnumr[Kn] = numpy.zeros((1, 2))
        self.lmps = [SiteTensor(init["site%d" % i], [self.qnuml[i], QPHYS, self.qnuml[i + 1]], L_STATUS, dev)
                     for i in range(Kn)]
        self.rmps = [None] * Kn
        self.lenv = {-1: boundary_set_n(self.nops, dev)}
        self.renv = {Kn: boundary_set_n(self.nops, dev)}
        self.plenv = {-1: boundary_set_n(self.npts, dev)}
        self.prenv = {Kn: boundary_set_n(self.npts, dev)}
        for i in range(Kn):
            self.renormalize(i, "L", self.lmps[i])
        self.psi0 = None

    def renormalize(self, j, status, st):
        """renormQt_H00 and renormQt_S00 on the N-reduced site tensor."""
        lay_n, vals = self._reduced_site(st)
        if status == "L":
            rn = Renormalizer(self.ws, j, "L", lay_n, self.lenv[j - 1], self.mpo[j], self.opers)
            self.lenv[j] = rn(vals)
            rp = Renormalizer(self.ws, j, "L", lay_n, self.plenv[j - 1], self.pops, self.popers)
            self.plenv[j] = rp(vals)
        else:
            rn = Renormalizer(self.ws, j, "R", lay_n, self.renv[j + 1], self.mpo[j], self.opers)
            self.renv[j] = rn(vals)
            rp = Renormalizer(self.ws, j, "R", lay_n, self.prenv[j + 1], self.pops, self.popers)
            self.prenv[j] = rp(vals)
        return rn.flops + rp.flops

    def _noise_layout(self, lay):
        """pRDMQt contracts the N-reduced wavefunction (kernelQt.py:493, :572)."""
        lay_n = reduce_layout(lay)
        self._noise_red = (lay, lay_n, torch.from_numpy(reduce_map(lay, lay_n)).to(self.device))
        return lay_n, self.qkey[:1]

    def _noise_values(self, lay, vals):
        lay0, lay_n, red = self._noise_red
        out = torch.empty(lay_n.size, dtype=torch.float64, device=self.device)
        return K.scatter(vals.contiguous(), red, out)

    def _mixed_gdavidson(self, sig, sv, diag, v0, crit_e):
        """Generalised Davidson with FP32 H and S products, then one FP64 pair of products:
        the FP64 Rayleigh quotient e = x.Hx / x.Sx is accurate to second order in the
        vector's error.  Accepted when the FP64 residual |Hx - e Sx| (x S-normalised) is at
        most 1e-4 or at most twice the FP32 solve's own residual plus 1e-5, or when the FP32
        solve converged by the reference's criteria and e agrees with its Ritz value within
        1e-6 Eh; otherwise FP64 iterations continue from x."""
        from .dmrg import ACCEPT_DE
        r1 = gdavidson(sig, sv, diag, 1, v0, crit_e=crit_e, crit_vec=max(self.crit_vec, 1e-5))
        x = r1.vecs[0]
        hx, sx = sig(x, precision="f64"), sv(x, precision="f64")
        xsx = float(torch.dot(x, sx))
        if xsx <= 0.0:
            raise RuntimeError("spin projection: the FP32 solution has no weight in the projected space")
        e64 = float(torch.dot(x, hx)) / xsx
        rn = float(torch.linalg.norm(hx - e64 * sx)) / xsx ** 0.5
        self.stats["nmvp_f64"] = self.stats.get("nmvp_f64", 0) + 1
        self.stats["nmvp_low"] = self.stats.get("nmvp_low", 0) + r1.nmvp
        converged = r1.niter < 19
        # as in DMRG._mixed_davidson: an FP64 residual no larger than twice the FP32 solver's
        # own (plus its floor) means the FP32 products did not bias the vector
        rn_low = float(r1.rnorms[-1][0]) if r1.rnorms else float("inf")
        unbiased = rn <= 2.0 * rn_low + 1e-5
        if rn <= max(self.crit_vec, 1e-4) or unbiased or (converged and abs(e64 - float(r1.eigs[0])) <= ACCEPT_DE):
            r1.eigs = numpy.array([e64])
            r1.vecs = (x / xsx ** 0.5).reshape(1, -1)
            r1.nmvp += 1
            return r1
        r2 = gdavidson(lambda v: sig(v, precision="f64"), lambda v: sv(v, precision="f64"), diag, 1,
                       x.reshape(1, -1), crit_e=crit_e, crit_vec=self.crit_vec)
        self.stats["nmvp_f64"] += r2.nmvp
        r2.nmvp += r1.nmvp + 1
        return r2

    def _psi_layout(self, isite):
        ql, qr = self.qnuml[isite], self.qnumr[isite + 2]
        cls = [classification(q) for q in (ql, QPHYS, QPHYS, self.qkey - qr)]
        lay = Layout(PSI_STATUS, [c[0] for c in cls], [c[1] for c in cls])
        return lay, [c[2] for c in cls]

    def _live(self, lay):
        """Blocks of the N-reduced wavefunction that can be non-zero: the (N, Sz) ones (the
        reference also contracts the zero blocks; skipping them changes no result)."""
        return lay.allowed.astype(bool) if self.prune_zero_blocks else None

    def dot_operators(self, isite):
        """H_eff (projected) and its diagonal for the dot; the plan is compiled per dot."""
        lay, idl = self._psi_layout(isite)
        lay_n = reduce_layout(lay)
        red = reduce_map(lay, lay_n)
        L, R = self.lenv[isite - 1], self.renv[isite + 2]
        Wi, Wj = self.mpo[isite], self.mpo[isite + 1]
        inner = SigmaOperator(self.ws, isite, lay_n, L, R, Wi, Wj, self.qkey[:1], self.opers, self.hpwts,
                              self.precision, live=self._live(lay), **self.sigma_opts)
        sig = ProjectedOperator(self.ws, inner, red)
        dg = DiagOperator(self.ws, isite, lay, L, R, Wi, Wj, self.qkey, self.opers, self.hpwts)
        return lay, idl, sig, dg

    def dot_projector(self, isite):
        """S (projected) and its diagonal for the dot (SVecQt / SDiagQt)."""
        lay, idl = self._psi_layout(isite)
        lay_n = reduce_layout(lay)
        red = reduce_map(lay, lay_n)
        PL, PR = self.plenv[isite - 1], self.prenv[isite + 2]
        inner = SigmaOperator(self.ws, isite, lay_n, PL, PR, self.pops, self.pops, self.qkey[:1], self.popers,
                              self.qwts, self.precision, live=self._live(lay), **self.sigma_opts)
        sv = ProjectedOperator(self.ws, inner, red)
        sd = DiagOperator(self.ws, isite, lay, PL, PR, self.pops, self.pops, self.qkey, self.popers, self.qwts)
        return sv, sd

    def _solve_dot_host(self, isite, status, dmax, crit_e):
        """The same dot through mpo_dmrg_kernel.HDiag/HVec/SVec with host (NumPy) vectors
        and the generalised Davidson on the host, as the reference's pgdvdson calls them."""
        from . import mpo_dmrg_kernel as MK
        dev = self.device
        info = [self, isite, 2, [[self.lenv[isite - 1], self.renv[isite + 2], self.plenv[isite - 1],
                                  self.prenv[isite + 2]]], status, True]
        t0 = time.time()
        lay, idl, sig, dg = MK._ops(self, isite)
        sv, sd = MK._sops(self, isite)
        prj_h = lay.prjmap(idl)
        self.stats["plan_s"] += time.time() - t0
        ndim0 = lay.size
        ldim, rdim = len(self.qnuml[isite]), len(self.qnumr[isite + 2])
        dims = (ldim, 16, rdim, ldim * 16 * rdim)
        diag = torch.from_numpy(MK.HDiag(info, ndim0, prj_h))
        self.d2h_bytes += 8 * ndim0

        def host(fn):
            def apply(x):
                y = fn(x.numpy(), info, ndim0, prj_h)
                self.h2d_bytes += 8 * ndim0
                self.d2h_bytes += 8 * ndim0
                return torch.from_numpy(y)
            return apply

        v0 = None
        if self.psi0 is not None:
            v0 = self.psi0[0:1].reshape(1, -1)[:, torch.from_numpy(prj_h).to(self.psi0.device)].cpu()
        t0 = time.time()
        res = gdavidson(host(MK.HVec), host(MK.SVec), diag, 1, v0, crit_e=crit_e, crit_vec=self.crit_vec)
        self.stats["hvec_s"] += time.time() - t0
        self.stats["nmvp"] += res.nmvp
        self.stats["sigma_flops"] += res.nmvp * (sig.flops + sv.flops)
        civec = torch.zeros((1, dims[3]), dtype=torch.float64, device=dev)
        civec[:, torch.from_numpy(prj_h).to(dev)] = res.vecs.to(dev)
        self.h2d_bytes += 8 * ndim0
        t0 = time.time()
        out = self.decimate(civec, isite, status, dims, dmax)
        torch.cuda.synchronize(dev)
        self.stats["decim_s"] += time.time() - t0
        return res, out, dims, sig

    def solve_dot(self, isite, status, dmax, crit_e):
        if self.host_api:
            return self._solve_dot_host(isite, status, dmax, crit_e)
        dev = self.device
        t0 = time.time()
        lay, idl, sig, dg = self.dot_operators(isite)
        sv, sd = self.dot_projector(isite)
        prj = torch.from_numpy(lay.prjmap(idl)).to(dev)
        self.stats["plan_s"] += time.time() - t0
        ldim, rdim = len(self.qnuml[isite]), len(self.qnumr[isite + 2])
        dims = (ldim, 16, rdim, ldim * 16 * rdim)
        t0 = time.time()
        diag = dg()
        torch.cuda.synchronize(dev)
        self.stats["hdiag_s"] += time.time() - t0
        self.stats["diag_flops"] += dg.flops
        v0 = None
        if self.psi0 is not None:
            v0 = self.psi0[0:1].reshape(1, -1)[:, prj].contiguous()
        t0 = time.time()
        if self.precision == "f64":
            res = gdavidson(sig, sv, diag, 1, v0, crit_e=crit_e, crit_vec=self.crit_vec)
        else:
            res = self._mixed_gdavidson(sig, sv, diag, v0, crit_e)
        torch.cuda.synchronize(dev)
        self.stats["hvec_s"] += time.time() - t0
        self.stats["nmvp"] += res.nmvp
        self.stats["sigma_flops"] += res.nmvp * (sig.flops + sv.flops)
        civec = torch.zeros((1, dims[3]), dtype=torch.float64, device=dev)
        civec[:, prj] = res.vecs
        t0 = time.time()
        out = self.decimate(civec, isite, status, dims, dmax)
        torch.cuda.synchronize(dev)
        self.stats["decim_s"] += time.time() - t0
        return res, out, dims, sig

