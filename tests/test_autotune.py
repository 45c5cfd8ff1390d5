"""The measured choice of the fiber-GEMM schedule (qcmpodmrg_b200.autotune) on the CPU
interpreter of the kernels: every candidate budget compiles a plan whose sigma is bitwise
the default plan's (the schedule changes no summation order), the fastest candidate is
recorded in the run's sigma options, and later plans are compiled with it."""
import numpy
import torch

from helpers import load
from emulate import patch_stage_run
from qcmpodmrg_b200.hamiltonian import make_hamiltonian


def test_fiber_budget_candidates_agree_and_choice_applies(monkeypatch):
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda *a, **k: "cpu-interpreter")
    from qcmpodmrg_b200 import autotune
    from qcmpodmrg_b200.dmrg import DMRG
    fx = load("sweep_K6.npz")
    ham = make_hamiltonian(int(fx["K"]), int(fx["N"]), int(fx["seed"]), None if fx["decay"] < 0 else fx["decay"])
    d = DMRG(ham, device="cpu", precision="f64")
    d.load_mps(fx["init_mps"])
    d.sweep("R", int(fx["D"]), 1e-8)
    d.sweep("L", int(fx["D"]), 1e-8)
    cost = {}

    def fake_time(sig, x, precision, repeats):
        # a deterministic stand-in for the CUDA-event time: fewer fiber items is "faster"
        n = sum(len(st.h_items) for st in _fiber_stages(sig))
        cost[n] = cost.get(n, 0) + 1
        return float(n), sig(x, precision=precision)

    monkeypatch.setattr(autotune, "_time_sigma", fake_time)
    autotune._CACHE.clear()
    cands = ((4096, 4096), (64, 64), (16, 4096), (4096, 16))
    rep = autotune.tune_fiber_budget(d, 2, candidates=cands)
    assert len(rep["table"]) == len(cands)
    assert rep["choice"] == min(rep["table"], key=lambda t: t[1])[0]
    # the small budgets cut groups into more items: the candidates really differ
    assert len(set(ms for _, ms in rep["table"])) > 1
    lay, idl, sig, dg = d.dot_operators(2)
    for st in _fiber_stages(sig):
        assert (st.a_budget, st.w_budget) == tuple(rep["choice"])


def _fiber_stages(sig):
    from qcmpodmrg_b200.engine import FiberStage, CompositeStage
    out = []

    def walk(st):
        if isinstance(st, CompositeStage):
            for x in st.subs:
                walk(x)
        elif isinstance(st, FiberStage) and st.ntasks and st.fgemm:
            out.append(st)
    for st in sig.stages:
        walk(st)
    return out
