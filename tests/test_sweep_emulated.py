"""Whole two-site sweeps of the product driver, with the kernels interpreted on the
CPU, reproduce the reference's energies (validates driver + plans without a GPU)."""
import numpy
import pytest
import torch

from helpers import load
from emulate import patch_stage_run
from qcmpodmrg_b200.hamiltonian import make_hamiltonian


@pytest.mark.parametrize("tag", ["K4"])
def test_sweeps_emulated(tag, monkeypatch):
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.dmrg import DMRG
    fx = load("sweep_%s.npz" % tag)
    decay = None if fx["decay"] < 0 else fx["decay"]
    ham = make_hamiltonian(int(fx["K"]), int(fx["N"]), int(fx["seed"]), decay)
    d = DMRG(ham, device="cpu")
    out = d.run(fx["init_mps"], int(fx["D"]), int(fx["nsweeps"]))
    assert numpy.abs(out["eav"] - fx["eav"]).max() <= 1e-8
    assert numpy.abs(out["dwt"] - fx["dwt"]).max() <= 1e-10
    # later sweeps revisit dots with unchanged sectors: their compiled plans are reused
    assert d.stats.get("plan_hits", 0) > 0
