"""The drop-in boundary exercised from the reference's side: the reference's own sweep
(mpo_dmrg_class.default -> mpo_dmrg_opt.sweep -> mpo_dmrg_dot.ci_solver -> pdvdson) with
its kernel dispatcher patched as INTEGRATION.md shows, so that HVec / HDiag / renorm of
every two-site Qt dot run on qcmpodmrg_b200 (the reference's qtensor sites handed to
renorm as they are), reaches the energies and discarded weights of the unpatched
reference run recorded in the fixtures.

Needs the converted reference (tests/golden/convert_reference.py -> baseline/_ref).  On
the CPU the device operators run through the NumPy interpreter of their work items; on
the B200 through the CUDA kernels."""
import os

import numpy
import pytest

from helpers import load, GOLDEN

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "baseline", "_ref", "qcmpodmrg")
needs_ref = pytest.mark.skipif(not os.path.isdir(REF), reason="converted reference not present (baseline/_ref)")


def _run(tag, device):
    import reference_runner as rr
    from qcmpodmrg_b200.hamiltonian import make_hamiltonian
    from qcmpodmrg_b200.dmrg import DMRG
    fx = load("sweep_%s.npz" % tag)
    decay = None if fx["decay"] < 0 else float(fx["decay"])
    K, N = int(fx["K"]), int(fx["N"])

    def factory(init_mps):
        d = DMRG(make_hamiltonian(K, N, int(fx["seed"]), decay), device=device)
        d.load_mps(init_mps)
        return d

    res, _ = rr.run_reference(K=K, N=N, D=int(fx["D"]), nsweeps=int(fx["nsweeps"]), seed=int(fx["seed"]),
                              decay=decay, targets=(), record_envs=False, gpu=factory)
    eav, dwt = numpy.asarray(res["eav"]), numpy.asarray(res["dwt"])
    assert len(eav) == len(fx["eav"])
    # converged (final) sweep to 1e-8 Eh / 1e-10; earlier sweeps to 1e-5 (a truncation through
    # degenerate RDM eigenvalues may keep the other partner state for one sweep)
    assert abs(eav[-1] - fx["eav"][-1]) <= 1e-8
    assert abs(dwt[-1] - fx["dwt"][-1]) <= 1e-10
    assert numpy.abs(eav - fx["eav"]).max() <= 1e-5


@needs_ref
@pytest.mark.parametrize("tag", ["K4", "K5"])
def test_reference_sweep_on_emulated_kernels(tag, monkeypatch):
    from emulate import patch_stage_run
    patch_stage_run(monkeypatch)
    _run(tag, "cpu")


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["K4", "K5", "K6"])
def test_reference_sweep_on_gpu_kernels(tag, cuda):
    _run(tag, cuda)
