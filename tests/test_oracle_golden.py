"""Pin the oracle against outputs of the reference itself (tests/golden, made by make_golden.py)."""
import numpy
import pytest

from helpers import load
from oracle.blocks import from_dict, sym_allowed
from oracle.kernels import SigmaOracle, hdiag, RenormOracle
from oracle.dmrg import OracleDMRG
from qcmpodmrg_b200.hamiltonian import make_hamiltonian, fci_energy


def test_oracle_symallowed_matches_reference_libqsym():
    for c in load("qsym_cases.npz")["cases"]:
        qs = [numpy.asarray(q).reshape(int(n), -1) for q, n in zip(c["qsyms"], c["ndims"])]
        got = sym_allowed(numpy.asarray(c["ndims"]), numpy.asarray(c["status"]).astype(bool), qs)
        assert numpy.array_equal(got, c["allowed"])


@pytest.mark.parametrize("tag", ["K4", "K5", "K6", "K5N2", "K5N8"])
def test_oracle_kernels_match_reference(tag):
    fx = load("kernels_%s.npz" % tag)
    assert len(fx["records"]) >= 1
    for r in fx["records"]:
        qtmp = from_dict(r["qtmp"])
        L = [from_dict(d) for d in r["envL"]]
        R = [from_dict(d) for d in r["envR"]]
        Wi = [from_dict(d) for d in r["mpo_i"]]
        Wj = [from_dict(d) for d in r["mpo_j"]]
        opers = [int(x) for x in numpy.atleast_1d(r["opers"])]
        isite = int(r["key"][2])
        sig = SigmaOracle(qtmp, r["qkey"], L, R, Wi, Wj, opers, numpy.atleast_1d(r["hpwts"]), isite)
        y = sig(r["hvec_x"])
        assert numpy.abs(y - r["hvec_y"]).max() <= 1e-12 * max(1.0, numpy.abs(r["hvec_y"]).max())
        d = hdiag(numpy.asarray(r["prjmap"]), tuple(int(x) for x in r["dims"]), L, R, Wi, Wj,
                  numpy.atleast_1d(r["hpwts"]))
        assert numpy.abs(d - r["hdiag"]).max() <= 1e-12
        st = "L" if int(r["key"][1]) == 0 else "R"
        site = from_dict(r["renorm_site"])
        if st == "L":
            out = RenormOracle(opers, isite, "L")(site, L, Wi)
        else:
            out = RenormOracle(opers, isite + 1, "R")(site, R, Wj)
        for a, b in zip(out, r["renorm_out"]):
            assert a.size_allowed == len(b["value"])
            assert numpy.abs(a.value - b["value"]).max() <= 1e-12


@pytest.mark.parametrize("tag", ["K4", "K5"])
def test_oracle_sweeps_match_reference(tag):
    fx = load("sweep_%s.npz" % tag)
    decay = None if fx["decay"] < 0 else fx["decay"]
    ham = make_hamiltonian(int(fx["K"]), int(fx["N"]), int(fx["seed"]), decay)
    nsw = min(int(fx["nsweeps"]), 3)             # the K=5 run is converged after three
    out = OracleDMRG(ham).run(fx["init_mps"], int(fx["D"]), nsw)
    n = len(out["eav"])
    assert numpy.abs(out["eav"] - fx["eav"][:n]).max() <= 1e-8
    assert numpy.abs(out["dwt"] - fx["dwt"][:n]).max() <= 1e-10
    assert numpy.array_equal(out["nmvp"], fx["nmvp"][:n])
    if tag == "K5":
        # the reference run with the MPO bond cut into three slices (maxslc=3) follows
        # another trajectory in the first sweep and joins it by the third
        sl = load("sweep_SL_K5.npz")
        assert abs(out["eav"][2] - sl["eav"][2]) <= 1e-10


def test_reference_reaches_fci_at_full_bond():
    """Independent physics check: D large enough => the reference's energy equals FCI."""
    fx = load("sweep_K4.npz")
    ham = make_hamiltonian(4, 4, 1)
    assert abs(fx["eav"][-1] - fci_energy(ham)) < 1e-9
