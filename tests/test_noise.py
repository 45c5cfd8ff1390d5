"""The decimation's pRDM noise term (pRDMQt with noise > 0, the reference's default
schedules): oracle and product against the reference's own outputs
(tests/golden/*NZ*_K*.npz, made by make_golden.py --noise)."""
import numpy
import pytest
import torch

from helpers import load, record_noise
from emulate import patch_stage_run
from oracle.blocks import from_dict
from oracle.kernels import prdm_noise
from qcmpodmrg_b200.hamiltonian import make_hamiltonian

TAGS = ["NZ_K5", "NZ_K6", "NZSP_K5"]


def _ham(fx):
    return make_hamiltonian(int(fx["K"]), int(fx["N"]), int(fx["seed"]), None if fx["decay"] < 0 else fx["decay"])


@pytest.mark.parametrize("tag", TAGS)
def test_oracle_prdm_matches_reference(tag):
    for r in load("kernels_%s.npz" % tag)["records"]:
        c = numpy.asarray(r["prdm_cimat"])
        ldim, cdim, rdim, ndim = [int(x) for x in r["dims"]]
        isite = int(r["key"][2])
        opers = [int(x) for x in r["opers"]]
        if int(r["key"][1]) == 0:
            m = c.reshape(c.shape[0], c.shape[1] * c.shape[2], -1)
            cc = sum(m[i] @ m[i].T for i in range(len(m)))
            nz = prdm_noise(c[0].reshape(ldim, 4, 4 * rdim), "L", [from_dict(d) for d in r["envL"]],
                            [from_dict(d) for d in r["mpo_i"]], r["qkey"], opers, isite, 2, tuple(r["dims"]),
                            r["noise"])
        else:
            m = c.reshape(c.shape[0], c.shape[1], -1)
            cc = sum(m[i].T @ m[i] for i in range(len(m)))
            nz = prdm_noise(c[0].reshape(ldim * 4, 4, rdim), "R", [from_dict(d) for d in r["envR"]],
                            [from_dict(d) for d in r["mpo_j"]], r["qkey"], opers, isite, 2, tuple(r["dims"]),
                            r["noise"])
        assert numpy.abs(cc + nz - r["prdm_out"]).max() <= 1e-15


def _first_sweep_matches(out, fx):
    """Every dot energy of the first R+L sweep, its averaged energy, weight and matvecs."""
    n = len(out["esweeps"])
    assert n == 2 * (int(fx["K"]) - 1)
    assert numpy.abs(out["esweeps"] - fx["esweeps"][:n]).max() <= 1e-8
    assert abs(out["eav"][0] - fx["eav"][0]) <= 1e-8 and abs(out["dwt"][0] - fx["dwt"][0]) <= 1e-10
    assert out["nmvp"][0] == fx["nmvp"][0]


def test_oracle_sweep_with_noise_matches_reference():
    from oracle.dmrg import OracleDMRG
    fx = load("sweep_NZ_K5.npz")
    _first_sweep_matches(OracleDMRG(_ham(fx)).run(fx["init_mps"], int(fx["D"]), 1, noise=float(fx["noise"])), fx)


@pytest.mark.parametrize("tag", TAGS)
def test_noise_rdm_emulated(tag, monkeypatch):
    patch_stage_run(monkeypatch)
    for r in load("kernels_%s.npz" % tag)["records"]:
        op, vals, cc = record_noise(r, "cpu")
        got = cc + r["noise"] * op(vals).numpy()
        assert numpy.abs(got - r["prdm_out"]).max() <= 1e-15


def test_dropin_prdm_with_noise_emulated(monkeypatch):
    """mpo_dmrg_kernel.pRDM on the product DMRG equals C C^T + noise * the oracle's noise
    term on the same dot (environments built independently from the same MPS)."""
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    _dropin_prdm_vs_oracle("cpu")


def _dropin_prdm_vs_oracle(device):
    from oracle.dmrg import OracleDMRG
    from qcmpodmrg_b200.dmrg import DMRG
    from qcmpodmrg_b200 import mpo_dmrg_kernel as MK
    fx = load("sweep_NZ_K5.npz")
    ham = _ham(fx)
    d = DMRG(ham, device=device)
    d.noise = float(fx["noise"])
    d.load_mps(fx["init_mps"])
    o = OracleDMRG(ham)
    o.load_mps(fx["init_mps"])
    K = int(fx["K"])
    isite = K - 2
    ldim, rdim = len(o.qnuml[isite]), len(o.qnumr[isite + 2])
    dims = (ldim, 16, rdim, ldim * 16 * rdim)
    # a wavefunction of the dot's symmetry sector (elements outside it are dropped by both)
    from oracle.blocks import QTensor, classification
    from oracle.mpo import QPHYS
    qtmp = QTensor([False, False, False, True])
    cls = [classification(q) for q in (o.qnuml[isite], QPHYS, QPHYS, o.qkey - o.qnumr[isite + 2])]
    qtmp.from_qsyms(4, [x[0] for x in cls], [x[1] for x in cls])
    prj = qtmp.prjmap([x[2] for x in cls])
    c = numpy.zeros(ldim * 16 * rdim)
    c[prj] = numpy.random.default_rng(11).standard_normal(len(prj))
    c = c.reshape(1, ldim, 4, 4 * rdim)
    m = c.reshape(1, ldim * 4, 4 * rdim)
    want = m[0] @ m[0].T + prdm_noise(c[0], "L", o.lenv[isite - 1], o.mpo[isite], o.qkey, o.opers, isite, 2,
                                       dims, d.noise)
    got = MK.pRDM(c, [d, isite, 2, None, "L", True])
    assert numpy.abs(got - want).max() <= 1e-12 * numpy.abs(want).max()
    c = c.reshape(1, ldim * 4, 4, rdim)
    m = c.reshape(1, ldim * 4, 4 * rdim)
    want = m[0].T @ m[0] + prdm_noise(c[0], "R", o.renv[isite + 2], o.mpo[isite + 1], o.qkey, o.opers, isite,
                                       2, dims, d.noise)
    got = MK.pRDM(c, [d, isite, 2, None, "R", True])
    assert numpy.abs(got - want).max() <= 1e-12 * numpy.abs(want).max()


def test_sweep_with_noise_emulated(monkeypatch):
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.dmrg import DMRG
    fx = load("sweep_NZ_K5.npz")
    _first_sweep_matches(DMRG(_ham(fx), device="cpu").run(fx["init_mps"], int(fx["D"]), 1,
                                                          noise=float(fx["noise"])), fx)


def test_sp_half_sweep_with_noise_emulated(monkeypatch):
    """Spin projection and the noise term together (the reference's K=5, 3-point run with
    noise 1e-4): every dot energy of the first right-to-left half sweep and its matvecs."""
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.spin import SPDMRG
    fx = load("sweep_NZSP_K5.npz")
    d = SPDMRG(_ham(fx), int(fx["npts"]), device="cpu")
    d.noise = float(fx["noise"])
    d.load_mps(fx["init_mps"])
    n, e, dw, el, dl = d.sweep("R", int(fx["D"]), 1e-7)
    assert numpy.abs(numpy.array(el) - fx["esweeps"][:len(el)]).max() <= 1e-8
