"""Whole two-site sweeps of the product driver, with the kernels interpreted on the
CPU, reproduce the reference's energies (validates driver + plans without a GPU)."""
import numpy
import pytest
import torch

from helpers import load
from emulate import patch_stage_run
from qcmpodmrg_b200.hamiltonian import make_hamiltonian


@pytest.mark.parametrize("tag", ["K4", "K5N2", "K5N8"])
def test_sweeps_emulated(tag, monkeypatch):
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.dmrg import DMRG
    fx = load("sweep_%s.npz" % tag)
    decay = None if fx["decay"] < 0 else fx["decay"]
    ham = make_hamiltonian(int(fx["K"]), int(fx["N"]), int(fx["seed"]), decay)
    d = DMRG(ham, device="cpu", plan_cache=True)
    out = d.run(fx["init_mps"], int(fx["D"]), int(fx["nsweeps"]))
    assert numpy.abs(out["eav"] - fx["eav"]).max() <= 1e-8
    assert numpy.abs(out["dwt"] - fx["dwt"]).max() <= 1e-10
    # later sweeps revisit dots with unchanged sectors: their compiled plans are reused
    assert d.stats.get("plan_hits", 0) > 0


def test_plan_cache_requires_identical_layouts(monkeypatch):
    """A cached plan is reused only for the very layout objects it was compiled for:
    an entry whose key matches but whose layouts are other objects (a recycled id)
    is rebuilt, not reused."""
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.dmrg import DMRG
    fx = load("sweep_K4.npz")
    ham = make_hamiltonian(int(fx["K"]), int(fx["N"]), int(fx["seed"]), None if fx["decay"] < 0 else fx["decay"])
    d = DMRG(ham, device="cpu", plan_cache=True)
    d.load_mps(fx["init_mps"])
    d.sweep("R", int(fx["D"]), 1e-8)
    lay, idl, sig, dg = d.dot_operators(1)
    key = next(k for k in d.plan_cache if k[0] == 1)
    entry = d.plan_cache[key]
    fake_L = tuple(object() for _ in entry[1])          # same key, other objects
    d.plan_cache[key] = (entry[0], fake_L) + entry[2:]
    misses = d.stats.get("plan_misses", 0)
    lay2, idl2, sig2, dg2 = d.dot_operators(1)
    assert sig2 is not sig and d.stats["plan_misses"] == misses + 1
    lay3, idl3, sig3, dg3 = d.dot_operators(1)           # the rebuilt entry is reused
    assert sig3 is sig2


def test_odd_electron_number_sector(monkeypatch):
    """N=3 in K=4 orbitals, sector Sz=1/2, from the occupation-number start: the sweeps reach
    exact diagonalisation's ground energy (the Sz=+1/2 and -1/2 spectra coincide)."""
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.dmrg import DMRG
    from qcmpodmrg_b200.hamiltonian import fci_energy
    from qcmpodmrg_b200.synthetic import product_mps
    ham = make_hamiltonian(4, 3, 1, None)
    out = DMRG(ham, device="cpu", sz=0.5).run(product_mps(ham), 16, 2)
    assert abs(out["eav"][-1] - fci_energy(ham)) <= 1e-8


def test_mixed_precision_sweep_emulated(monkeypatch):
    """The mixed-precision solve (low-precision Davidson, one FP64 product for the energy and
    the residual check, and the optional closing FP64 Davidson step) with the tensor-core plan, on the CPU
    interpreter (whose split-TF32 products are exact): the reference's converged energies."""
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.dmrg import DMRG
    fx = load("sweep_K5N8.npz")
    ham = make_hamiltonian(int(fx["K"]), int(fx["N"]), int(fx["seed"]), None if fx["decay"] < 0 else fx["decay"])
    d = DMRG(ham, device="cpu", precision="tf32x3")
    d.fp64_step = True                 # the optional closing FP64 step too
    out = d.run(fx["init_mps"], int(fx["D"]), int(fx["nsweeps"]))
    assert abs(out["eav"][-1] - fx["eav"][-1]) <= 1e-8
    assert d.stats["nmvp_low"] > d.stats["nmvp_f64"] > 0


def test_plan_cache_keys_on_the_sigma_options(monkeypatch):
    """A cached plan is reused only under the sigma options it was compiled with: another
    fiber-GEMM schedule (as the autotuner sets it) compiles a new plan, the same one hits."""
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.dmrg import DMRG
    fx = load("sweep_K4.npz")
    ham = make_hamiltonian(int(fx["K"]), int(fx["N"]), int(fx["seed"]), None if fx["decay"] < 0 else fx["decay"])
    d = DMRG(ham, device="cpu")
    d.load_mps(fx["init_mps"])
    d.sweep("R", int(fx["D"]), 1e-8)
    lay, idl, sig, dg = d.dot_operators(1)
    assert d.dot_operators(1)[2] is sig                      # same options: reused
    d.sigma_opts["fg_budget"] = (2048, 2048)
    sig2 = d.dot_operators(1)[2]
    assert sig2 is not sig                                   # other schedule: compiled anew
    assert d.dot_operators(1)[2] is sig2
