"""GPU end-to-end: FP64 two-site sweeps reproduce the reference's energies (1e-8 Eh)
and discarded weights (1e-10) from the same initial MPS.

Where a truncation cuts between exactly degenerate RDM eigenvalues (Sz = +-1/2
partner sectors of an Sz = 0 state), which state is kept depends on last-bit
differences of two eigensolvers (LAPACK in the reference, cuSOLVER here); the
choice moves the energy of that sweep by about the discarded weight and is
undone by the next sweep.  Converged (final-sweep) energies and discarded
weights are held to 1e-8 / 1e-10; earlier sweeps to 1e-5.

The K=12, N=12, D=100 six-sweep run (C1) stops before convergence (discarded
weight ~6e-3 per sweep) and its Davidson solves stop at |de| <= 1e-7.  Its trajectory
is set by rounding noise: from the occupation-number start the Davidson vector of a dot
can lie in a subspace that H leaves invariant (a spin sector of the start state), and
only rounding noise takes the solver out of it.  Exact diagonalisation of the dot
Hamiltonians shows it: at the ninth dot of the first sweep the reference's own solver
returns -17.4394 Eh where the dot's lowest eigenvalue is -18.8792 Eh; the reference
leaves the subspace four dots later, the CPU interpreter of the kernels not within the
first sweep, the B200 at yet another dot, and each then follows its own unconverged
trajectory.  So the test holds the dots before the first truncation to 1e-10
(bit-level agreement of sigma, Davidson and decimation), and the sweep energies only as
variational upper bounds of one another: the GPU run's last sweep at least as low as
the reference's up to C1_TOL_FINAL, and within C1_TOL_E of it.  The converged
comparison is test_sweeps_config1_converged.
"""
import os

import numpy
import pytest

from helpers import load, GOLDEN
from qcmpodmrg_b200.hamiltonian import make_hamiltonian

pytestmark = pytest.mark.gpu


C1_TOL_E = 1e-2       # unconverged runs: spread of the last sweep's energy between trajectories
C1_TOL_FINAL = 5e-4   # the GPU's last sweep may lie above the reference's by at most this
C1_EXACT_DOTS = 7     # dots of the first sweep before the first truncating decimation


@pytest.mark.parametrize("tag", ["K4", "K5", "K6", "K5N2", "K5N8"])
def test_sweeps_match_reference(tag, cuda):
    if not os.path.exists(os.path.join(GOLDEN, "sweep_%s.npz" % tag)):
        pytest.skip("fixture not generated")
    from qcmpodmrg_b200.dmrg import DMRG
    fx = load("sweep_%s.npz" % tag)
    decay = None if fx["decay"] < 0 else fx["decay"]
    ham = make_hamiltonian(int(fx["K"]), int(fx["N"]), int(fx["seed"]), decay)
    out = DMRG(ham, device=cuda).run(fx["init_mps"], int(fx["D"]), int(fx["nsweeps"]))
    n = min(len(out["eav"]), len(fx["eav"]))
    assert abs(out["eav"][n - 1] - fx["eav"][n - 1]) <= 1e-8
    assert abs(out["dwt"][n - 1] - fx["dwt"][n - 1]) <= 1e-10
    assert numpy.abs(out["eav"][:n] - fx["eav"][:n]).max() <= 1e-5
    if tag == "K5" and n >= 3 and os.path.exists(os.path.join(GOLDEN, "sweep_SL_K5.npz")):
        # the maxslc=3 reference run, held like the other sweeps before the last
        assert abs(out["eav"][2] - load("sweep_SL_K5.npz")["eav"][2]) <= 1e-5


def test_sweeps_config1_partial(cuda):
    if not os.path.exists(os.path.join(GOLDEN, "sweep_C1.npz")):
        pytest.skip("fixture not generated")
    from qcmpodmrg_b200.dmrg import DMRG
    fx = load("sweep_C1.npz")
    decay = None if fx["decay"] < 0 else fx["decay"]
    ham = make_hamiltonian(int(fx["K"]), int(fx["N"]), int(fx["seed"]), decay)
    out = DMRG(ham, device=cuda).run(fx["init_mps"], int(fx["D"]), int(fx["nsweeps"]))
    e_ref = numpy.asarray(fx["esweeps"])
    e_gpu = numpy.asarray(out["esweeps"])
    assert numpy.abs(e_gpu[:C1_EXACT_DOTS] - e_ref[:C1_EXACT_DOTS]).max() <= 1e-10
    print("C1 6 sweeps: GPU", list(out["eav"]), "reference", list(fx["eav"]))
    assert out["eav"][-1] <= fx["eav"][-1] + C1_TOL_FINAL
    assert abs(out["eav"][-1] - fx["eav"][-1]) <= C1_TOL_E



def test_sweeps_config1_converged(cuda):
    """Config 1 (K=12, N=12, D=100), Davidson and sweep tolerance 1e-9, 16 sweeps, from the
    reference's start MPS.  Neither run reaches the 1e-9 sweep tolerance within the 16
    sweeps (the reference's energy still falls by ~1e-7 per sweep at the end; its run took
    3.5 h on the CPU), and after the first truncation through degenerate RDM eigenvalues
    the two FP64 runs follow different, equally valid trajectories.  Both energies are
    variational upper bounds, so the test holds the GPU run to be at least as low as the
    reference after the same sweeps (1e-8) and within 1e-4 Eh of it."""
    if not os.path.exists(os.path.join(GOLDEN, "sweep_C1C.npz")):
        pytest.skip("fixture not generated")
    from qcmpodmrg_b200.dmrg import DMRG
    fx = load("sweep_C1C.npz")
    decay = None if fx["decay"] < 0 else fx["decay"]
    ham = make_hamiltonian(int(fx["K"]), int(fx["N"]), int(fx["seed"]), decay)
    out = DMRG(ham, device=cuda).run(fx["init_mps"], int(fx["D"]), int(fx["nsweeps"]), tol=float(fx["tol"]))
    print("C1 16 sweeps: GPU %.10f (dwt %.3e)  reference %.10f (dwt %.3e)" % (
        out["eav"][-1], out["dwt"][-1], fx["eav"][-1], fx["dwt"][-1]))
    assert out["eav"][-1] <= fx["eav"][-1] + 1e-8
    assert fx["eav"][-1] - out["eav"][-1] <= 1e-4
