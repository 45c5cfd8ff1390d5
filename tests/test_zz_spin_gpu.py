"""GPU parity of spin projection (SP-MPS): the projected H and S operators, their
diagonals, both renormalisations, the drop-in functions and whole sweeps against
the reference's outputs (tests/golden/*SP_K*.npz), the oracle and exact
diagonalisation (S=1, S=1/2); also the plain sweep in an odd-N sector.

Tolerances: operators 1e-12 relative (FP64, summation order differs from NumPy);
the K=4 run keeps every state (D=16), so its energies are held to 1e-8 and its
discarded weights to 1e-10.  The K=5, D=12 run truncates among RDM eigenvalues
that are zero to rounding, where which states are kept depends on last-bit
differences of the eigensolvers; its final energy is held to 1e-6 (the oracle,
on LAPACK like the reference, lands 2e-8 from it).
"""
import numpy
import pytest
import torch

from helpers import load, record_sp_operators, record_sp_renormalizers
from qcmpodmrg_b200.hamiltonian import make_hamiltonian

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["SP_K4", "SP_K5"])
@pytest.mark.parametrize("w_path,prune", [("generic", True), ("fiber", True), ("fiber", False)])
def test_gpu_sp_operators(tag, w_path, prune, cuda):
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, sv, dg, sd, ws = record_sp_operators(r, cuda, use_fiber=(w_path == "fiber"), prune=prune)
        x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64)).to(cuda)
        y = sig(x).cpu().numpy()
        assert numpy.abs(y - r["hvec_y"]).max() <= 1e-12 * max(1.0, numpy.abs(r["hvec_y"]).max())
        xs = torch.from_numpy(numpy.asarray(r["svec_x"], dtype=numpy.float64)).to(cuda)
        s = sv(xs).cpu().numpy()
        assert numpy.abs(s - r["svec_y"]).max() <= 1e-13
        assert numpy.abs(dg().cpu().numpy() - r["hdiag"]).max() <= 1e-12
        assert numpy.abs(sd().cpu().numpy() - r["sdiag"]).max() <= 1e-13


@pytest.mark.parametrize("tag", ["SP_K4", "SP_K5"])
def test_gpu_sp_renormalizers(tag, cuda):
    for r in load("kernels_%s.npz" % tag)["records"]:
        rn, rp, vals = record_sp_renormalizers(r, cuda)
        site = torch.from_numpy(vals).to(cuda)
        for op, ref in ((rn, r["renorm_out"]), (rp, r["renorm_pout"])):
            out = op(site)
            for i, b in enumerate(ref):
                assert out.layouts[i].size == len(b["value"])
                assert numpy.abs(out.op_values(i).cpu().numpy() - b["value"]).max() <= 1e-12


def test_gpu_sp_dropin_matches_oracle(cuda):
    from test_spin_emulated import _dropin_vs_oracle
    _dropin_vs_oracle(cuda)


def test_gpu_sp_sweeps_match_reference(cuda):
    from qcmpodmrg_b200.spin import SPDMRG
    sw = load("sweep_SP_K4.npz")
    ham = make_hamiltonian(int(sw["K"]), int(sw["N"]), int(sw["seed"]), None)
    out = SPDMRG(ham, int(sw["npts"]), device=cuda).run(sw["init_mps"], int(sw["D"]), int(sw["nsweeps"]))
    assert numpy.abs(out["eav"] - sw["eav"]).max() <= 1e-8
    assert numpy.abs(out["dwt"] - sw["dwt"]).max() <= 1e-10
    assert numpy.abs(out["esweeps"] - sw["esweeps"]).max() <= 1e-8


def test_gpu_sp_truncated_sweeps_converge_to_reference(cuda):
    from qcmpodmrg_b200.spin import SPDMRG
    sw = load("sweep_SP_K5.npz")
    ham = make_hamiltonian(int(sw["K"]), int(sw["N"]), int(sw["seed"]), sw["decay"])
    out = SPDMRG(ham, int(sw["npts"]), device=cuda).run(sw["init_mps"], int(sw["D"]), int(sw["nsweeps"]))
    assert abs(out["eav"][-1] - sw["eav"][-1]) <= 1e-6
    assert numpy.abs(out["eav"] - sw["eav"][:len(out["eav"])]).max() <= 1e-5


def test_gpu_sp_mixed_precision(cuda):
    """FP32 H and S products with the FP64 check reach the reference's K=4 energies to 1e-6 Eh."""
    from qcmpodmrg_b200.spin import SPDMRG
    sw = load("sweep_SP_K4.npz")
    ham = make_hamiltonian(int(sw["K"]), int(sw["N"]), int(sw["seed"]), None)
    d = SPDMRG(ham, int(sw["npts"]), device=cuda, precision="f32")
    out = d.run(sw["init_mps"], int(sw["D"]), int(sw["nsweeps"]))
    assert numpy.abs(out["eav"] - sw["eav"][:len(out["eav"])]).max() <= 1e-6
    assert d.stats.get("nmvp_low", 0) > 0


def test_gpu_sp_triplet_reaches_fci_triplet(cuda):
    from helpers import fci_spin_states
    from qcmpodmrg_b200.spin import SPDMRG
    sw = load("sweep_SP_K4.npz")
    ham = make_hamiltonian(4, 4, 1, None)
    w, s2 = fci_spin_states(ham)
    e_t = w[numpy.flatnonzero(numpy.abs(s2 - 2.0) < 1e-6)[0]]
    out = SPDMRG(ham, 3, sval=1.0, sz=0.0, device=cuda).run(sw["init_mps"], 16, 2)
    assert abs(out["eav"][-1] - e_t) <= 1e-8


def test_gpu_sp_half_integer_spin(cuda):
    """K=4, N=3 projected onto S=1/2, Sz=1/2: the lowest doublet of exact diagonalisation."""
    from helpers import fci_spin_states
    from qcmpodmrg_b200.spin import SPDMRG
    from qcmpodmrg_b200.synthetic import product_mps
    ham = make_hamiltonian(4, 3, 1, None)
    w, s2 = fci_spin_states(ham)
    e_d = w[numpy.flatnonzero(numpy.abs(s2 - 1.0) < 1e-6)[0]]
    out = SPDMRG(ham, 4, sval=0.5, sz=0.5, device=cuda).run(product_mps(ham), 16, 2)
    assert abs(out["eav"][-1] - e_d) <= 1e-8


def test_gpu_odd_electron_number_sector(cuda):
    """Plain (unprojected) sweeps in the N=3, Sz=1/2 sector reach the exact ground energy."""
    from qcmpodmrg_b200.dmrg import DMRG
    from qcmpodmrg_b200.hamiltonian import fci_energy
    from qcmpodmrg_b200.synthetic import product_mps
    ham = make_hamiltonian(4, 3, 1, None)
    out = DMRG(ham, device=cuda, sz=0.5).run(product_mps(ham), 16, 2)
    assert abs(out["eav"][-1] - fci_energy(ham)) <= 1e-8
