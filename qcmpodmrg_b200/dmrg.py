"""Two-site Qt DMRG driver with device-resident environments.

Mirrors the reference's control flow around the hot path (ifQt=True,
ncsite=2, one symmetry sector):
  default(sc, fmps)     source/mpo_dmrg_class.py:329-434  -> DMRG.run
  initOps / genHopsQt   source/mpo_dmrg_util.py:193-214, mpo_dmrg_initQt.py:88-271 -> load_mps
  sweep                 source/mpo_dmrg_opt.py:31-101 (+ updateSite :319-350, updateBoundary :353-383)
  ci_solver             source/mpo_dmrg_dot.py:24-112 (setupQtmpCI dotutil.py:173-184)
  decimation            source/mpo_dmrg_dotutil.py:269-476 with rdm_blkdiag (mpo_dmrg_qparser.py:106-183)
                        and the pRDM noise term (pRDMQt, mpo_dmrg_kernelQt.py:453-626) when noise > 0
  genGuess              source/mpo_dmrg_dotutil.py:479-540
The spin-projected variant (ifs2proj) is qcmpodmrg_b200.spin.SPDMRG.
Environments L_p / R_p of every operator live in HBM (TensorSet) instead of
per-site HDF5 files; the sigma/diagonal/renormalisation plans are built once
per dot.  Davidson, the RDM and its eigendecomposition run in FP64 on the GPU;
the global sort of RDM eigenvalues runs on the host with NumPy so ties break
exactly as in the reference.
"""
import time

import numpy
import torch

from .kernels import SigmaOperator, DiagOperator, Renormalizer, TensorSet, Workspace, NoiseRDM
from .mpo import QPHYS, build_mpo
from .qtensor import Layout, classification
from .davidson import davidson

L_STATUS = numpy.array([False, False, True])
R_STATUS = numpy.array([True, False, False])
PSI_STATUS = numpy.array([False, False, False, True])


def dpt(q1, q2):
    q1 = numpy.asarray(q1, dtype=numpy.float64)
    q2 = numpy.asarray(q2, dtype=numpy.float64)
    return (q1[:, None, :] + q2[None, :, :]).reshape(-1, q1.shape[1])


def noise_psi_layout(ql, qr, qkey, status):
    """The wavefunction as the rank-3 tensor pRDMQt contracts (setupQtmpPRDM,
    source/mpo_dmrg_dotutil.py:543-569): [l, n1, (n2 r)] for 'L', [(l n1), n2, r] for
    'R', merged indices classified by their quantum numbers.  Returns the layout, its
    sector -> dense-position lists, and those of the dense density matrix's indices."""
    if status == "L":
        qn = [ql, QPHYS, qkey - dpt(QPHYS, qr)]
    else:
        qn = [dpt(ql, QPHYS), QPHYS, qkey - qr]
    cls = [classification(q) for q in qn]
    lay = Layout([False, False, True], [c[0] for c in cls], [c[1] for c in cls])
    idl = [c[2] for c in cls]
    dense_idl = [idl[0], idl[1], idl[0], idl[1]] if status == "L" else [idl[1], idl[2], idl[1], idl[2]]
    return lay, idl, dense_idl


ACCEPT_DE = 1e-6      # Eh: FP64 vs low-precision Ritz value agreement that accepts a mixed solve


class SiteTensor(object):
    """A site tensor in packed layout on the device (plus its dense form)."""

    def __init__(self, dense, qnums, status, device):
        cls = [classification(q) for q in qnums]
        self.layout = Layout(status, [c[0] for c in cls], [c[1] for c in cls])
        self.idlst = [c[2] for c in cls]
        prj = torch.from_numpy(self.layout.prjmap(self.idlst)).to(device)
        if not torch.is_tensor(dense):
            dense = torch.from_numpy(numpy.ascontiguousarray(dense, dtype=numpy.float64)).to(device)
        self.dense = dense.reshape(tuple(int(n) for n in self.layout.shape))
        self.values = self.dense.reshape(-1)[prj].contiguous()


def boundary_set(nops, device):
    lay = Layout([True, False, True], [numpy.zeros((1, 2))] * 3, [numpy.ones(1, dtype=numpy.int64)] * 3)
    return TensorSet([lay] * nops, [numpy.ones(1)] * nops, device=device)


class DMRG(object):
    """Two-site MPO-DMRG with every hot-path contraction on the GPU."""

    ifs2proj = False          # spin projection: qcmpodmrg_b200.spin.SPDMRG

    def __init__(self, ham, device="cuda", precision="f64", preconditioner=None, w_path="fiber", plan_cache=True,
                 sz=0.0):
        """sz: the target Sz of the (N, Sz) sector (the reference's qsectors key [N, Sz])."""
        n2s = int(round(2 * float(sz)))
        if abs(2 * float(sz) - n2s) > 1e-9 or (n2s - int(ham.nelec)) % 2 != 0 or abs(float(sz)) > ham.nelec / 2.0:
            raise ValueError("sz=%g is not an Sz of %d electrons (2*Sz must have the parity of N and "
                             "|Sz| <= N/2)" % (float(sz), int(ham.nelec)))
        self.ham = ham
        self.sz = float(sz)
        self.device = torch.device(device)
        self.nsite = ham.nsite
        self.precision = precision
        self.preconditioner = preconditioner
        # kernels of the two MPO-site contractions of sigma: "generic" grouped GEMM,
        # "fiber" (fiber-group kernel per contraction) or "fused" (two-site W blocks)
        self.sigma_opts = {"generic": {"use_fiber": False}, "fiber": {"use_fiber": True, "fuse_w": False},
                           "fused": {"use_fiber": True, "fuse_w": True}}[w_path]
        self.crit_vec = 1.e-8
        self.thresh = -1.e-14
        self.noise = 0.0          # weight of the pRDM noise term in the decimation (schedule noise)
        self.ifguess = True
        self.ws = Workspace(self.device)
        self.plan_cache = {}          # oldest first
        # compiled plans of dots whose sectors did not change are reused with the new
        # environments (the work lists depend only on block layouts and the sigma options);
        # runs with and without reuse give bitwise the same energies and discarded weights
        self.plan_cache_size = 2 * self.nsite if plan_cache else 0
        t0 = time.time()
        self._setup_operators(ham)
        self.t_mpo = time.time() - t0
        self.log = []
        self.stats = {"hvec_s": 0.0, "hdiag_s": 0.0, "renorm_s": 0.0, "decim_s": 0.0, "plan_s": 0.0,
                      "nmvp": 0, "sigma_flops": 0.0, "renorm_flops": 0.0, "diag_flops": 0.0}
        self.events = False
        # host_api: drive the dot through the reference-facing functions with host
        # (NumPy) vectors, as the reference's pdvdson does (used for end-to-end timing)
        self.host_api = False
        self.recorder = None      # callback(residual, diag, e, x) fed by Davidson (preconditioner training)
        self.h2d_bytes = 0
        self.d2h_bytes = 0
        # list: every low-precision dot solve is repeated in plain FP64 from the same start
        # vector and both energies are appended here (off when None)
        self.shadow = None
        # mixed precision: one FP64 Davidson step after every accepted low-precision solve.
        # Off: at K=24, D=500 it cost one more FP64 product per dot (1.36x instead of 1.43x
        # over FP64) and did not bring converged D=200 energies closer to the FP64 run's
        self.fp64_step = False

    # ------------------------------------------------------------- set-up
    def _setup_operators(self, ham):
        """H = sum_p H_p, one operator per spin orbital (mpo_dmrg_class.partition, one rank)."""
        self.nops = ham.sbas
        self.opers = list(range(ham.sbas))
        self.hpwts = numpy.ones(self.nops)
        self.qkey = numpy.array([float(ham.nelec), self.sz])
        mpo = build_mpo(ham)
        self.mpo = {i: TensorSet(l, v, device=self.device) for i, (l, v) in mpo.items()}

    def load_mps(self, init):
        K = self.nsite
        dev = self.device
        self.qnuml = [numpy.array(init["qnum%d" % i], dtype=numpy.float64).reshape(-1, 2) for i in range(K + 1)]
        self.qnumr = [None] * (K + 1)
        self.qnumr[K] = numpy.zeros((1, 2))
        self.lmps = [SiteTensor(init["site%d" % i], [self.qnuml[i], QPHYS, self.qnuml[i + 1]], L_STATUS, dev)
                     for i in range(K)]
        self.rmps = [None] * K
        self.lenv = {-1: boundary_set(self.nops, dev)}
        self.renv = {K: boundary_set(self.nops, dev)}
        for i in range(K):
            rn = Renormalizer(self.ws, i, "L", self.lmps[i].layout, self.lenv[i - 1], self.mpo[i], self.opers)
            self.lenv[i] = rn(self.lmps[i].values)
        self.psi0 = None

    # ------------------------------------------------------------- one dot
    def dot_operators(self, isite):
        ql, qr = self.qnuml[isite], self.qnumr[isite + 2]
        cls = [classification(q) for q in (ql, QPHYS, QPHYS, self.qkey - qr)]
        lay = Layout(PSI_STATUS, [c[0] for c in cls], [c[1] for c in cls])
        idl = [c[2] for c in cls]
        L, R = self.lenv[isite - 1], self.renv[isite + 2]
        Wi, Wj = self.mpo[isite], self.mpo[isite + 1]
        # compiled plans depend only on block layouts (interned by content): a dot whose
        # wavefunction and environment sectors are unchanged reuses them
        # the key is built from object ids; a hit is confirmed by identity against the layout
        # objects the entry holds (so no id can be recycled by a new layout while cached)
        key = (isite, id(lay), tuple(id(x) for x in L.layouts), tuple(id(x) for x in R.layouts),
               self.precision, tuple(sorted(self.sigma_opts.items())))
        for (_, _, _, s_, d_) in self.plan_cache.values():     # cached plans keep no environment alive
            s_.release()
            d_.release()
        hit = self.plan_cache.get(key)
        if (hit is not None and hit[0] is lay and all(a is b for a, b in zip(hit[1], L.layouts))
                and all(a is b for a, b in zip(hit[2], R.layouts))):
            sig, dg = hit[3], hit[4]
            sig.rebind(L, R)
            dg.rebind(L, R)
            self.stats["plan_hits"] = self.stats.get("plan_hits", 0) + 1
            return lay, idl, sig, dg
        sig = SigmaOperator(self.ws, isite, lay, L, R, Wi, Wj, self.qkey, self.opers, self.hpwts, self.precision,
                            **self.sigma_opts)
        wp = self.stats.setdefault("w_paths", {})
        for k, v in sig.w_paths.items():
            wp[k] = wp.get(k, 0) + v
        dg = DiagOperator(self.ws, isite, lay, L, R, Wi, Wj, self.qkey, self.opers, self.hpwts)
        self.plan_cache[key] = (lay, tuple(L.layouts), tuple(R.layouts), sig, dg)
        while len(self.plan_cache) > self.plan_cache_size:
            self.plan_cache.pop(next(iter(self.plan_cache)))
        self.stats["plan_misses"] = self.stats.get("plan_misses", 0) + 1
        return lay, idl, sig, dg

    def solve_dot(self, isite, status, dmax, crit_e):
        if self.host_api:
            return self._solve_dot_host(isite, status, dmax, crit_e)
        dev = self.device
        t0 = time.time()
        lay, idl, sig, dg = self.dot_operators(isite)
        if lay.size == 0:
            raise RuntimeError("dot (%d, %d), sweep %s: the wavefunction has no allowed block (left bond sectors "
                               "%s, right bond sectors %s, target %s)" % (
                                   isite, isite + 1, status, numpy.unique(self.qnuml[isite], axis=0).tolist(),
                                   numpy.unique(self.qnumr[isite + 2], axis=0).tolist(), self.qkey.tolist()))
        prj = torch.from_numpy(lay.prjmap(idl)).to(dev)
        self.stats["plan_s"] += time.time() - t0
        ldim, rdim = len(self.qnuml[isite]), len(self.qnumr[isite + 2])
        dims = (ldim, 16, rdim, ldim * 16 * rdim)
        torch.cuda.synchronize(dev)
        t0 = time.time()
        diag = dg()
        torch.cuda.synchronize(dev)
        self.stats["hdiag_s"] += time.time() - t0
        self.stats["diag_flops"] += dg.flops
        nmv = [0]

        def hv(x):
            nmv[0] += 1
            return sig(x)

        v0 = None
        if self.psi0 is not None:
            v0 = self.psi0[0:1].reshape(1, -1)[:, prj].contiguous()
        learned = hasattr(self.preconditioner, "set_layout")
        if learned:
            self.preconditioner.set_layout(lay)
            self.recorder = self.preconditioner.record
        t0 = time.time()
        if self.precision == "f64":
            res = davidson(hv, diag, 1, v0, crit_e=crit_e, crit_vec=self.crit_vec, precond=self.preconditioner,
                           record=self.recorder)
        else:
            res = self._mixed_davidson(hv, lambda v: sig(v, precision="f64"), diag, v0, crit_e)
            if hasattr(sig, "check_device_status"):
                sig.check_device_status()
        torch.cuda.synchronize(dev)
        self.stats["hvec_s"] += time.time() - t0
        if self.shadow is not None and self.precision != "f64":
            # the plain FP64 solve of the same dot from the same start vector (accuracy
            # check: same operators, same inputs); its result does not enter the sweep
            r64 = davidson(lambda v: sig(v, precision="f64"), diag, 1, v0, crit_e=crit_e, crit_vec=self.crit_vec)
            self.shadow.append({"isite": isite, "status": status, "e_f64": float(r64.eigs[0]),
                                "e_mixed": float(res.eigs[0]), "nmvp_f64": int(r64.nmvp),
                                "nmvp_mixed": int(res.nmvp), "niter_f64": int(r64.niter),
                                "niter_mixed": int(res.niter)})
        self.stats["nmvp"] += res.nmvp
        self.stats["sigma_flops"] += res.nmvp * sig.flops
        if learned:
            self.preconditioner.end_dot(res.vecs[0])
        civec = torch.zeros((1, dims[3]), dtype=torch.float64, device=dev)
        civec[:, prj] = res.vecs
        t0 = time.time()
        out = self.decimate(civec, isite, status, dims, dmax)
        torch.cuda.synchronize(dev)
        self.stats["decim_s"] += time.time() - t0
        return res, out, dims, sig

    # ---- split dot step (used by the batched multi-instance driver)
    def dot_begin(self, isite, crit_e):
        """Plans, diagonal and a Davidson generator for the dot; returns a context."""
        from .davidson import davidson_steps
        lay, idl, sig, dg = self.dot_operators(isite)
        prj = torch.from_numpy(lay.prjmap(idl)).to(self.device)
        diag = dg()
        v0 = None
        if self.psi0 is not None:
            v0 = self.psi0[0:1].reshape(1, -1)[:, prj].contiguous()
        gen = davidson_steps(diag, 1, v0, crit_e=crit_e, crit_vec=self.crit_vec)
        return {"isite": isite, "lay": lay, "prj": prj, "sig": sig, "gen": gen, "diag": diag}

    def dot_end(self, ctx, res, status, dmax, actlst, elst, dlst):
        isite = ctx["isite"]
        dev = self.device
        ldim, rdim = len(self.qnuml[isite]), len(self.qnumr[isite + 2])
        dims = (ldim, 16, rdim, ldim * 16 * rdim)
        self.stats["nmvp"] += res.nmvp
        self.stats["sigma_flops"] += res.nmvp * ctx["sig"].flops
        civec = torch.zeros((1, dims[3]), dtype=torch.float64, device=dev)
        civec[:, ctx["prj"]] = res.vecs
        dwts, qred, site, srotR, civecs = self.decimate(civec, isite, status, dims, dmax)
        elst.append(float(res.eigs[0]))
        dlst.append(float(dwts))
        self._update(isite, status, qred, site)
        self.guess(isite, status, actlst, civecs, srotR)
        return qred, srotR

    def _update(self, isite, status, qred, site):
        dev = self.device
        if status == "L":
            self.qnuml[isite + 1] = qred
            st = SiteTensor(site, [self.qnuml[isite], QPHYS, qred], L_STATUS, dev)
            self.lmps[isite] = st
            self.stats["renorm_flops"] += self.renormalize(isite, "L", st)
        else:
            j = isite + 1
            self.qnumr[j] = qred
            st = SiteTensor(site, [qred, QPHYS, self.qnumr[j + 1]], R_STATUS, dev)
            self.rmps[j] = st
            self.stats["renorm_flops"] += self.renormalize(j, "R", st)

    def renormalize(self, j, status, st):
        """New environments of site j from its site tensor (renorm, mpo_dmrg_kernel.py:347-377);
        returns the FLOPs launched."""
        if status == "L":
            rn = Renormalizer(self.ws, j, "L", st.layout, self.lenv[j - 1], self.mpo[j], self.opers)
            self.lenv[j] = rn(st.values)
        else:
            rn = Renormalizer(self.ws, j, "R", st.layout, self.renv[j + 1], self.mpo[j], self.opers)
            self.renv[j] = rn(st.values)
        return rn.flops

    def boundary(self, status, qred, srotR):
        K = self.nsite
        dev = self.device
        smat = srotR[0] / torch.linalg.norm(srotR[0])
        qk = self.qkey.reshape(1, 2).copy()
        if status == "L":
            self.lmps[K - 1] = SiteTensor(smat, [qred, QPHYS, qk], L_STATUS, dev)
            self.qnuml[K] = qk
        else:
            self.rmps[0] = SiteTensor(smat, [qk, QPHYS, qred], R_STATUS, dev)
            self.qnumr[0] = qk

    def _mixed_davidson(self, hv, hv64, diag, v0, crit_e):
        """Davidson with low-precision sigma (hv), then FP64 refinement (hv64).

        Phase 1 iterates with the FP32/TF32 sigma until the energy change is below
        crit_e or the residual below the precision's floor.  Phase 2 applies the
        FP64 sigma to the final vector: its Rayleigh quotient has an error of second
        order in the vector's error.  The vector is accepted when its FP64 residual is
        at most 1e-4, or at most twice the low-precision one plus the precision's floor
        (the low-precision sigma did not bias the vector beyond the point where the FP64
        solver itself stops, by its criteria or at the same iteration cap), or when phase 1
        converged and the FP64 Rayleigh quotient agrees with the low-precision Ritz value
        within ACCEPT_DE; otherwise FP64 Davidson
        iterations (reference criteria) continue from that vector.  With fp64_step on, an
        accepted vector gets one more Davidson step on FP64 products.  Vectors are
        device tensors, or host tensors when hv / hv64 are the host-buffer entry points.
        """
        # residual floor of the low-precision sigma (relative sigma error ~1e-7 FP32,
        # ~1e-3 TF32), and the FP64 residual accepted without FP64 iterations: the
        # FP64 Rayleigh quotient then has an error of order residual^2 / gap
        floor = 2e-4 if self.precision == "tf32" else 1e-5
        accept = 1e-4
        r1 = davidson(hv, diag, 1, v0, crit_e=crit_e, crit_vec=max(self.crit_vec, floor),
                      precond=self.preconditioner, record=self.recorder)
        x = r1.vecs[0] / torch.linalg.norm(r1.vecs[0])
        y = hv64(x)
        e64 = float(torch.dot(x, y))
        rn = float(torch.linalg.norm(y - e64 * x))
        self.stats["nmvp_f64"] = self.stats.get("nmvp_f64", 0) + 1
        self.stats["nmvp_low"] = self.stats.get("nmvp_low", 0) + r1.nmvp
        converged = r1.niter < 19             # phase 1 met its criteria (not the iteration cap)
        # residual the low-precision solver saw for its final vector: when the FP64 residual
        # is no larger than that (plus the precision's floor), the low-precision products did
        # not bias the vector beyond the point where the FP64 solver itself stops -- also when
        # phase 1 ended at the iteration cap, where the FP64 solver stops as well
        rn_low = float(r1.rnorms[-1][0]) if r1.rnorms else float("inf")
        unbiased = rn <= 2.0 * rn_low + floor
        if rn <= max(self.crit_vec, accept) or unbiased or (converged and abs(e64 - float(r1.eigs[0])) <= ACCEPT_DE):
            r1.nmvp += 1
            if self.fp64_step and rn > self.crit_vec:
                # one FP64 Davidson step from the accepted vector (Rayleigh-Ritz in the span of
                # the vector and its preconditioned FP64 residual): the last step the FP64
                # solver takes runs on FP64 products
                x, e64 = self._fp64_step(hv64, diag, x, y, e64)
                self.stats["nmvp_f64"] += 1
                r1.nmvp += 1
            r1.eigs = numpy.array([e64])
            r1.vecs = x.reshape(1, -1)
            return r1
        r2 = davidson(hv64, diag, 1, x.reshape(1, -1), crit_e=crit_e, crit_vec=self.crit_vec,
                      precond=self.preconditioner)
        self.stats["nmvp_f64"] += r2.nmvp
        r2.nmvp += r1.nmvp + 1
        return r2

    def _fp64_step(self, hv64, diag, x, y, e):
        """One FP64 Davidson step from the normalised vector x (y = H x in FP64, e its
        Rayleigh quotient): the residual preconditioned as the solver does it (iop=4, or
        the preconditioner of the run), orthogonalised against x, one FP64 product, and
        the lower Ritz pair of the 2 x 2 projected problem.  Returns (vector, energy)."""
        r = y - e * x
        if self.preconditioner is None:
            d = r / ((diag.to(r.device) - e).abs() + 1.e-4)
        else:
            d = self.preconditioner(r, diag, torch.tensor(e, dtype=torch.float64, device=r.device), x)
        for _ in range(2):
            d = d - torch.dot(x, d) * x
        nd = float(torch.linalg.norm(d))
        if not nd > 1.e-14:
            return x, e
        d = d / nd
        yd = hv64(d)
        hh = torch.stack([torch.dot(d, y), torch.dot(x, yd), torch.dot(d, yd)]).cpu().numpy()
        h = numpy.array([[e, 0.5 * (hh[0] + hh[1])], [0.5 * (hh[0] + hh[1]), hh[2]]])
        w, u = numpy.linalg.eigh(h)
        x2 = float(u[0, 0]) * x + float(u[1, 0]) * d
        x2 = x2 / torch.linalg.norm(x2)
        return x2, float(w[0])

    def _solve_dot_host(self, isite, status, dmax, crit_e):
        """The same dot, through mpo_dmrg_kernel.HDiag/HVec with host buffers."""
        from . import mpo_dmrg_kernel as K
        dev = self.device
        info = [self, isite, 2, [[self.lenv[isite - 1], self.renv[isite + 2]]], status, True]
        t0 = time.time()
        lay, idl, sig, dg = K._ops(self, isite)
        prj_h = lay.prjmap(idl)
        self.stats["plan_s"] += time.time() - t0
        ndim0 = lay.size
        ldim, rdim = len(self.qnuml[isite]), len(self.qnumr[isite + 2])
        dims = (ldim, 16, rdim, ldim * 16 * rdim)
        diag = torch.from_numpy(K.HDiag(info, ndim0, prj_h))
        self.d2h_bytes += 8 * ndim0

        def hv(x):
            y = K.HVec(x.numpy(), info, ndim0, prj_h)
            self.h2d_bytes += 8 * ndim0
            self.d2h_bytes += 8 * ndim0
            return torch.from_numpy(y)

        v0 = None
        if self.psi0 is not None:
            v0 = self.psi0[0:1].reshape(1, -1)[:, torch.from_numpy(prj_h).to(self.psi0.device)].cpu()
        t0 = time.time()
        if self.precision == "f64":
            res = davidson(hv, diag, 1, v0, crit_e=crit_e, crit_vec=self.crit_vec)
        else:               # the same mixed-precision solve, FP64 products through the same entry point

            def hv64(x):
                y = K.HVec(x.numpy(), info, ndim0, prj_h, precision="f64")
                self.h2d_bytes += 8 * ndim0
                self.d2h_bytes += 8 * ndim0
                return torch.from_numpy(y)

            learned = self.preconditioner
            self.preconditioner = None if hasattr(learned, "set_layout") else learned
            try:
                res = self._mixed_davidson(hv, hv64, diag, v0, crit_e)
            finally:
                self.preconditioner = learned
        self.stats["hvec_s"] += time.time() - t0
        self.stats["nmvp"] += res.nmvp
        self.stats["sigma_flops"] += res.nmvp * sig.flops
        civec = torch.zeros((1, dims[3]), dtype=torch.float64, device=dev)
        civec[:, torch.from_numpy(prj_h).to(dev)] = res.vecs.to(dev)
        self.h2d_bytes += 8 * ndim0
        t0 = time.time()
        out = self.decimate(civec, isite, status, dims, dmax)
        torch.cuda.synchronize(dev)
        self.stats["decim_s"] += time.time() - t0
        return res, out, dims, sig

    def prdm(self, civecs, isite, status, dims):
        """Density matrix of the half of the dot being kept, sum_i C_i C_i^T, plus
        noise * the pRDM noise term of every state when noise >= 1e-10 (pRDMQt,
        source/mpo_dmrg_kernelQt.py:453-626; decimation, mpo_dmrg_dotutil.py:294-330)."""
        ldim, cdim, rdim, ndim = dims
        neig = civecs.shape[0]
        c = civecs.reshape(neig, ldim * 4, 4 * rdim)
        nz = self.noise_operator(isite, status) if self.noise >= 1.e-10 else None
        rdm = None
        for i in range(neig):
            m = c[i] @ c[i].T if status == "L" else c[i].T @ c[i]
            rdm = m if rdm is None else rdm + m
            if nz is not None:
                op, lay, prj = nz
                rdm = rdm + self.noise * op(self._noise_values(lay, civecs[i].reshape(-1)[prj]))
        return rdm

    def noise_operator(self, isite, status):
        """NoiseRDM for the dot, the rank-3 wavefunction layout and its dense->packed map."""
        lay, idl, dense_idl = noise_psi_layout(self.qnuml[isite], self.qnumr[isite + 2], self.qkey, status)
        if status == "L":
            E, W, j = self.lenv[isite - 1], self.mpo[isite], isite
        else:
            E, W, j = self.renv[isite + 2], self.mpo[isite + 1], isite + 1
        lay_op, qkey = self._noise_layout(lay)
        op = NoiseRDM(self.ws, j, status, lay_op, E, W, self.opers, qkey, dense_idl)
        self.stats["prdm_flops"] = self.stats.get("prdm_flops", 0.0) + op.flops
        return op, lay, torch.from_numpy(lay.prjmap(idl)).to(self.device)

    def _noise_layout(self, lay):
        return lay, self.qkey

    def _noise_values(self, lay, vals):
        return vals

    def decimate(self, civecs, isite, status, dims, dmax):
        ldim, cdim, rdim, ndim = dims
        neig = civecs.shape[0]
        lcdim, crdim = ldim * 4, 4 * rdim
        c = civecs.reshape(neig, lcdim, crdim)
        rdm = self.prdm(civecs, isite, status, dims)
        if status == "L":
            classes = dpt(self.qnuml[isite], QPHYS)
        else:
            classes = dpt(QPHYS, self.qnumr[isite + 2])
        tr = float(torch.trace(rdm))
        if abs(tr) < 1.e-12:
            rdm = rdm + torch.eye(rdm.shape[0], dtype=rdm.dtype, device=rdm.device) / float(rdm.shape[0])
        else:
            rdm = rdm / tr
        dwts, qred, rot, sigs = self.rdm_blkdiag(rdm, classes, dmax)
        nres = len(qred)
        if status == "L":
            site = rot.reshape(ldim, 4, nres)
            srotR = torch.stack([(rot.T @ c[i]).reshape(nres, 4, rdim) for i in range(neig)])
        else:
            site = rot.reshape(4, rdim, nres).permute(2, 0, 1).contiguous()
            srotR = torch.stack([(c[i] @ rot).reshape(ldim, 4, nres) for i in range(neig)])
        return dwts, qred, site, srotR, civecs

    def rdm_blkdiag(self, rho, classes, dcut):
        """Block eigh per (N, Sz) class on the GPU; global sort/truncation on the host."""
        q2 = numpy.rint(2 * classes).astype(numpy.int64)
        keys, first = [], {}
        for i, k in enumerate(map(tuple, q2)):
            if k not in first:
                first[k] = []
                keys.append(k)
            first[k].append(i)
        nrows = rho.shape[0]
        # classes the wavefunction has no weight in give exactly zero blocks: their
        # eigenpairs are (0, unit vectors), as LAPACK returns them for a zero matrix; the
        # device eigensolver is not called on them (on the B200 it returned NaN for an
        # all-zero 41 x 41 block, which poisoned the global sort)
        zero_row = (rho.abs().amax(dim=1) == 0).cpu().numpy() if nrows else numpy.zeros(0, dtype=bool)
        qsym, cols, sig = [], [], []
        for k in keys:
            rows = torch.tensor(first[k], dtype=torch.int64, device=rho.device)
            n = len(first[k])
            if zero_row[first[k]].all():
                s2 = torch.zeros(n, dtype=rho.dtype, device=rho.device)
                u = torch.eye(n, dtype=rho.dtype, device=rho.device)
            else:
                blk = rho[rows][:, rows]
                s2, u = torch.linalg.eigh(blk)
            qsym += [list(numpy.array(k) / 2.0)] * len(first[k])
            col = torch.zeros((nrows, len(first[k])), dtype=rho.dtype, device=rho.device)
            col[rows, :] = u
            cols.append(col)
            sig.append(s2.abs())
        rot = torch.cat(cols, dim=1)
        sig_h = torch.cat(sig).cpu().numpy()
        sig_h = sig_h / numpy.sum(sig_h)
        indx = numpy.argsort(sig_h)[::-1]
        nres = len(sig_h)
        tsig = sig_h[indx]
        for i in range(nres):
            if tsig[i] < self.thresh * 1.01:
                nres = i
                break
        if nres == 0:
            nres = 1
        if dcut > 0:
            nres = min(nres, dcut)
        indx = indx[:nres]
        s = sig_h[indx].copy()
        dwts = 1.0 - numpy.sum(s)
        qk = [qsym[i] for i in indx]
        o = sorted(range(nres), key=lambda x: qk[x])
        sel = numpy.asarray(indx)[o].copy()
        qred = numpy.array([qk[i] for i in o], dtype=numpy.float64)
        rot = rot[:, torch.from_numpy(sel).to(rot.device)].contiguous()
        return dwts, qred, rot, s[o]

    # ------------------------------------------------------------- sweeps
    def sweep(self, status, dmax, crit_e):
        K = self.nsite
        dev = self.device
        actlst = list(range(0, K - 1)) if status == "L" else list(range(K - 2, -1, -1))
        elst, dlst, nmvp = [], [], 0
        for isite in actlst:
            res, (dwts, qred, site, srotR, civecs), dims, sig = self.solve_dot(isite, status, dmax, crit_e)
            nmvp += res.nmvp
            elst.append(float(res.eigs[0]))
            dlst.append(float(dwts))
            t0 = time.time()
            if status == "L":
                self.qnuml[isite + 1] = qred
                st = SiteTensor(site, [self.qnuml[isite], QPHYS, qred], L_STATUS, dev)
                self.lmps[isite] = st
                rflops = self.renormalize(isite, "L", st)
            else:
                j = isite + 1
                self.qnumr[j] = qred
                st = SiteTensor(site, [qred, QPHYS, self.qnumr[j + 1]], R_STATUS, dev)
                self.rmps[j] = st
                rflops = self.renormalize(j, "R", st)
            # no synchronisation here: the next dot's plans are compiled on the host while
            # the renormalisation runs (renorm_s is host time: plan + launches)
            self.stats["renorm_s"] += time.time() - t0
            self.stats["renorm_flops"] += rflops
            self.guess(isite, status, actlst, civecs, srotR)
            self.log.append({"status": status, "isite": isite, "e": elst[-1], "dwt": dlst[-1],
                             "nmvp": int(res.nmvp), "bond": int(len(qred)), "ndim0": int(sig.ndim0),
                             "sigma_gflop": sig.flops / 1e9})
        smat = srotR[0] / torch.linalg.norm(srotR[0])
        qk = self.qkey.reshape(1, 2).copy()
        if status == "L":
            self.lmps[K - 1] = SiteTensor(smat, [qred, QPHYS, qk], L_STATUS, dev)
            self.qnuml[K] = qk
        else:
            self.rmps[0] = SiteTensor(smat, [qk, QPHYS, qred], R_STATUS, dev)
            self.qnumr[0] = qk
        i = int(numpy.argmin(elst))
        return nmvp, elst[i], dlst[i], elst, dlst

    def guess(self, isite, status, actlst, civecs, srotR):
        if not self.ifguess:
            return
        if isite == actlst[-1]:
            self.psi0 = civecs.clone()
        elif status == "R":
            t = self.lmps[isite - 1].dense
            self.psi0 = torch.stack([torch.tensordot(t, srotR[i], dims=([2], [0])).reshape(-1)
                                     for i in range(srotR.shape[0])])
        else:
            t = self.rmps[isite + 2].dense
            self.psi0 = torch.stack([torch.tensordot(srotR[i], t, dims=([2], [0])).reshape(-1)
                                     for i in range(srotR.shape[0])])

    def snapshot(self):
        """The state between two sweeps (after a left-to-right sweep): left-canonical site
        tensors, bond quantum numbers and the next dot's start vector (device copies)."""
        st = {"site%d" % i: self.lmps[i].dense.clone() for i in range(self.nsite)}
        st.update({"qnum%d" % i: self.qnuml[i].copy() for i in range(self.nsite + 1)})
        st["psi0"] = None if self.psi0 is None else self.psi0.clone()
        return st

    def restore(self, st):
        """Return to a snapshot: environments rebuilt from the site tensors (genHopsQt)."""
        self.load_mps(st)
        self.psi0 = None if st["psi0"] is None else st["psi0"].clone()

    def run(self, init_mps, dmax, nsweeps, tol=1.e-7, callback=None, noise=0.0):
        """schedule.fixed(ncsite=2, maxM=dmax, tol=tol, noise=noise): sweeps R then L until |dE| < tol."""
        self.noise = float(noise)
        last = numpy.asarray(init_mps["qnum%d" % self.nsite], dtype=numpy.float64).reshape(-1, 2)
        if last.shape[0] != 1 or numpy.abs(last[0] - self.qkey).max() > 1e-9:
            raise ValueError("the start MPS ends in the sector %s, the target sector is %s"
                             % (last.tolist(), self.qkey.tolist()))
        self.load_mps(init_mps)
        eav, dwt, esweeps, nmvps = [], [], [], []
        eold = 1.e3
        for isweep in range(nsweeps):
            t0 = time.time()
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
            if callback is not None:
                callback(isweep, eav[-1], time.time() - t0)
            if abs(eav[-1] - eold) < tol:
                break
            eold = eav[-1]
        return {"eav": numpy.array(eav), "dwt": numpy.array(dwt), "esweeps": numpy.array(esweeps),
                "nmvp": numpy.array(nmvps)}
