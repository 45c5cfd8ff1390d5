"""Spin projection on the product's plans, with the kernels interpreted on the CPU:
the projected H / S operators, their diagonals, both renormalisations and a sweep
reproduce the reference's outputs (tests/golden/*SP_K*.npz)."""
import numpy
import pytest
import torch

from helpers import load, record_sp_operators, record_sp_renormalizers
from emulate import patch_stage_run
from qcmpodmrg_b200.hamiltonian import make_hamiltonian


@pytest.mark.parametrize("tag,w_path,prune", [("SP_K4", "generic", True), ("SP_K4", "fiber", True),
                                               ("SP_K4", "fiber", False), ("SP_K5", "generic", True),
                                               ("SP_K5", "fiber", True), ("SPS_K4", "fiber", True)])
def test_sp_operators_emulated(tag, w_path, prune, monkeypatch):
    patch_stage_run(monkeypatch)
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, sv, dg, sd, ws = record_sp_operators(r, "cpu", use_fiber=(w_path == "fiber"), prune=prune)
        y = sig(torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64))).numpy()
        assert numpy.abs(y - r["hvec_y"]).max() <= 1e-12 * max(1.0, numpy.abs(r["hvec_y"]).max())
        s = sv(torch.from_numpy(numpy.asarray(r["svec_x"], dtype=numpy.float64))).numpy()
        assert numpy.abs(s - r["svec_y"]).max() <= 1e-13
        assert numpy.abs(dg().numpy() - r["hdiag"]).max() <= 1e-12
        assert numpy.abs(sd().numpy() - r["sdiag"]).max() <= 1e-13


def test_sp_pruning_skips_zero_block_work(monkeypatch):
    """Skipping the pairs of the zero blocks leaves results unchanged and removes work."""
    patch_stage_run(monkeypatch)
    r = load("kernels_SP_K4.npz")["records"][-1]
    a = record_sp_operators(r, "cpu", prune=True)
    b = record_sp_operators(r, "cpu", prune=False)
    x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64))
    for i in (0, 1):
        assert numpy.abs(a[i](x).numpy() - b[i](x).numpy()).max() <= 1e-13
        assert a[i].flops < b[i].flops


@pytest.mark.parametrize("tag", ["SP_K4", "SP_K5"])
def test_sp_renormalizers_emulated(tag, monkeypatch):
    patch_stage_run(monkeypatch)
    for r in load("kernels_%s.npz" % tag)["records"]:
        rn, rp, vals = record_sp_renormalizers(r, "cpu")
        site = torch.from_numpy(vals)
        for op, ref in ((rn, r["renorm_out"]), (rp, r["renorm_pout"])):
            out = op(site)
            for i, b in enumerate(ref):
                assert out.layouts[i].size == len(b["value"])
                assert numpy.abs(out.op_values(i).numpy() - b["value"]).max() <= 1e-12


def test_gdavidson_device_matches_oracle():
    from oracle.spin import gdavidson as ogd
    from qcmpodmrg_b200.davidson import gdavidson
    rng = numpy.random.default_rng(1)
    n = 90
    h = rng.uniform(-1, 1, (n, n))
    h = numpy.diag(numpy.arange(n) * 0.5) + h + h.T
    s = rng.uniform(0, 1, (n, n))
    s = numpy.diag(rng.uniform(0.8, 1.0, n)) + 0.05 * (s + s.T)
    ht, st = torch.from_numpy(h), torch.from_numpy(s)
    r = gdavidson(lambda x: ht @ x, lambda x: st @ x, torch.from_numpy(numpy.diag(h).copy()), 1, crit_e=1e-12,
                  crit_vec=1e-9, maxcycle=60)
    e, v, nm = ogd(lambda x: h @ x, lambda x: s @ x, numpy.diag(h).copy(), 1, crit_e=1e-12, crit_vec=1e-9,
                   maxcycle=60)
    assert abs(r.eigs[0] - e[0]) < 1e-11 and r.nmvp == nm
    x = r.vecs[0].numpy()
    assert abs(x @ s @ x - 1.0) < 1e-12


def test_sp_sweep_emulated(monkeypatch):
    """One R+L sweep of the spin-projected K=4 run: every dot's energy as the reference's."""
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.spin import SPDMRG
    sw = load("sweep_SP_K4.npz")
    ham = make_hamiltonian(int(sw["K"]), int(sw["N"]), int(sw["seed"]), None)
    d = SPDMRG(ham, int(sw["npts"]), device="cpu")
    out = d.run(sw["init_mps"], int(sw["D"]), 1)
    n = len(out["esweeps"])
    assert n == 2 * (int(sw["K"]) - 1)
    assert numpy.abs(out["esweeps"] - sw["esweeps"][:n]).max() <= 1e-8
    assert abs(out["eav"][0] - sw["eav"][0]) <= 1e-8
    assert out["nmvp"][0] == sw["nmvp"][0]


def test_sp_dropin_matches_oracle_on_same_dot(monkeypatch):
    """mpo_dmrg_kernel.HVec/SVec/HDiag/SDiag/renorm on a spin-projected DMRG equal the oracle
    computing the same dot from the same MPS (environments built independently)."""
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    _dropin_vs_oracle("cpu")


def _dropin_vs_oracle(device):
    from oracle import spin as ospin
    from oracle.blocks import QTensor, classification
    from oracle.mpo import QPHYS
    from oracle.kernels import hdiag
    from qcmpodmrg_b200 import mpo_dmrg_kernel as MK
    from qcmpodmrg_b200.spin import SPDMRG
    sw = load("sweep_SP_K5.npz")
    ham = make_hamiltonian(int(sw["K"]), int(sw["N"]), int(sw["seed"]), sw["decay"])
    npts = int(sw["npts"])
    d = SPDMRG(ham, npts, device=device)
    d.load_mps(sw["init_mps"])
    o = ospin.SPOracleDMRG(ham, npts)
    o.load_mps(sw["init_mps"])
    K = int(sw["K"])
    isite = K - 2                     # first dot of the R sweep: L environments from the MPS
    qtmp = QTensor([False, False, False, True])
    cls = [classification(q) for q in (o.qnuml[isite], QPHYS, QPHYS, o.qkey - o.qnumr[isite + 2])]
    qtmp.from_qsyms(4, [c[0] for c in cls], [c[1] for c in cls])
    prjmap = qtmp.prjmap([c[2] for c in cls])
    ndim0 = qtmp.size_allowed
    x = numpy.random.default_rng(5).standard_normal(ndim0)
    info = [d, isite, 2, [[d.lenv[isite - 1], d.renv[isite + 2]]], "R", True]
    L, R = o.lenv[isite - 1], o.renv[isite + 2]
    Wi, Wj = o.mpo[isite], o.mpo[isite + 1]
    PL, PR = o.plenv[isite - 1], o.prenv[isite + 2]
    yh = ospin.sigma_sp(qtmp, o.qkey, L, R, Wi, Wj, o.opers, o.hpwts, isite)(x)
    ys = ospin.svec(qtmp, o.qkey, PL, PR, o.pops, o.qwts, isite)(x)
    assert numpy.abs(MK.HVec(x, info, ndim0, prjmap) - yh).max() <= 1e-12 * max(1.0, numpy.abs(yh).max())
    assert numpy.abs(MK.SVec(x, info, ndim0, prjmap) - ys).max() <= 1e-13
    ldim, rdim = len(o.qnuml[isite]), len(o.qnumr[isite + 2])
    dims = (ldim, 16, rdim, ldim * 16 * rdim)
    assert numpy.abs(MK.HDiag(info, ndim0, prjmap) - hdiag(prjmap, dims, L, R, Wi, Wj, o.hpwts)).max() <= 1e-12
    sd = ospin.sdiag(prjmap, dims, PL, PR, o.pops, o.qwts)
    assert numpy.abs(MK.SDiag(info, ndim0, prjmap) - sd).max() <= 1e-13
    # the reference's own consistency check (checkDiagQt, kernelQt.py:129-150): the
    # effective operators are symmetric and their diagonals are HDiag / SDiag
    if ndim0 <= 64:
        eye = numpy.identity(ndim0)
        for vec, dia in ((MK.HVec, MK.HDiag), (MK.SVec, MK.SDiag)):
            m = numpy.array([vec(e, info, ndim0, prjmap) for e in eye]).T
            assert numpy.abs(m - m.T).max() <= 1e-12
            assert numpy.abs(numpy.diag(m) - dia(info, ndim0, prjmap)).max() <= 1e-12
    # renorm of the L environments of site 0 from the MPS: H and projector sets
    flstN = [[None, None]]
    MK.renorm(d, 0, 2, None, flstN, d.lmps[0], "L")
    for E, ref in ((flstN[0][0], o.lenv[0]), (flstN[0][1], o.plenv[0])):
        for i, q in enumerate(ref):
            assert numpy.abs(E.op_values(i).cpu().numpy() - q.value).max() <= 1e-12


def test_sp_mixed_sweep_emulated(monkeypatch):
    """FP32 H and S products with the FP64 check: the K=4 spin-projected first half sweep
    reaches the reference's energies within 1e-6 Eh (intermediates rounded to FP32 by the
    interpreter)."""
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.spin import SPDMRG
    sw = load("sweep_SP_K4.npz")
    ham = make_hamiltonian(int(sw["K"]), int(sw["N"]), int(sw["seed"]), None)
    d = SPDMRG(ham, int(sw["npts"]), device="cpu", precision="f32")
    d.load_mps(sw["init_mps"])
    n, e, dw, el, dl = d.sweep("R", int(sw["D"]), 1e-7)       # the first half sweep
    assert numpy.abs(numpy.array(el) - sw["esweeps"][:len(el)]).max() <= 1e-6
    assert d.stats.get("nmvp_low", 0) > 0 and d.stats.get("nmvp_f64", 0) > 0


def test_sp_triplet_reaches_fci_triplet(monkeypatch):
    """Projection onto S=1 (Sz=0, 3 points, every state kept): the sweep lands on the lowest
    triplet of exact diagonalisation, not on the singlet ground state."""
    from helpers import fci_spin_states
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.spin import SPDMRG
    sw = load("sweep_SP_K4.npz")
    ham = make_hamiltonian(4, 4, 1, None)
    w, s2 = fci_spin_states(ham)
    e_t = w[numpy.flatnonzero(numpy.abs(s2 - 2.0) < 1e-6)[0]]
    assert abs(s2[0]) < 1e-6 and e_t > w[0] + 0.1          # the ground state is a singlet
    out = SPDMRG(ham, 3, sval=1.0, sz=0.0, device="cpu").run(sw["init_mps"], 16, 1)
    assert abs(out["eav"][0] - e_t) <= 1e-8


def test_sp_host_api_sweep_emulated(monkeypatch):
    """The spin-projected dot driven through mpo_dmrg_kernel.HVec/SVec/HDiag with host vectors
    (the reference's calling convention) gives the reference's first half sweep."""
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.spin import SPDMRG
    sw = load("sweep_SP_K4.npz")
    ham = make_hamiltonian(int(sw["K"]), int(sw["N"]), int(sw["seed"]), None)
    d = SPDMRG(ham, int(sw["npts"]), device="cpu")
    d.host_api = True
    d.load_mps(sw["init_mps"])
    n, e, dw, el, dl = d.sweep("R", int(sw["D"]), 1e-7)       # the first half sweep
    assert numpy.abs(numpy.array(el) - sw["esweeps"][:len(el)]).max() <= 1e-8
    assert d.h2d_bytes > 0 and d.d2h_bytes > 0


def test_sp_simpson_sweep_emulated(monkeypatch):
    """Simpson's rule with 5 points (an inexact projector): the first half sweep's dot
    energies equal the reference's, quadrature error included."""
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.spin import SPDMRG
    sw = load("sweep_SPS_K4.npz")
    ham = make_hamiltonian(int(sw["K"]), int(sw["N"]), int(sw["seed"]), None)
    d = SPDMRG(ham, int(sw["npts"]), device="cpu", quad="Simpson")
    d.load_mps(sw["init_mps"])
    n, e, dw, el, dl = d.sweep("R", int(sw["D"]), 1e-7)       # the first half sweep
    assert numpy.abs(numpy.array(el) - sw["esweeps"][:len(el)]).max() <= 1e-8


def test_sp_half_integer_spin_reaches_fci_doublet(monkeypatch):
    """Odd electron number (K=4, N=3) projected onto S=1/2, Sz=1/2 from the occupation-number
    start: one sweep lands on the lowest doublet of exact diagonalisation."""
    from helpers import fci_spin_states
    from qcmpodmrg_b200.synthetic import product_mps
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.spin import SPDMRG
    ham = make_hamiltonian(4, 3, 1, None)
    w, s2 = fci_spin_states(ham)                 # Sz = -1/2 determinants: S(S+1) = s2 - 1/4
    e_d = w[numpy.flatnonzero(numpy.abs(s2 - 0.25 - 0.75) < 1e-6)[0]]
    out = SPDMRG(ham, 4, sval=0.5, sz=0.5, device="cpu").run(product_mps(ham), 16, 1)
    assert abs(out["eav"][0] - e_d) <= 1e-8
