"""The plan compiler + work lists, executed by a NumPy interpreter of the kernel
semantics, reproduce the reference's HVecQt / HDiagQt / renormQt_H00 (no GPU)."""
import numpy
import pytest
import torch

from helpers import load, record_operators, record_renormalizer
from emulate import patch_stage_run
from qcmpodmrg_b200.engine import CompositeStage, Stage


@pytest.mark.parametrize("tag", ["K4", "K5", "K6", "K5N2", "K5N8"])
def test_sigma_diag_renorm_emulated(tag, monkeypatch):
    patch_stage_run(monkeypatch)
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, dg, ws = record_operators(r, "cpu")
        x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64))
        y = sig(x).numpy()
        ref = numpy.asarray(r["hvec_y"])
        assert numpy.abs(y - ref).max() <= 1e-12 * max(1.0, numpy.abs(ref).max())
        d = dg().numpy()
        assert numpy.abs(d - numpy.asarray(r["hdiag"])).max() <= 1e-12
        rn, site = record_renormalizer(r, "cpu")
        out = rn(torch.from_numpy(site))
        for i, b in enumerate(r["renorm_out"]):
            got = out.op_values(i).numpy()
            assert len(got) == len(b["value"])
            assert numpy.abs(got - b["value"]).max() <= 1e-12


@pytest.mark.parametrize("tag", ["K5", "K6"])
def test_sigma_fiber_fused_emulated(tag, monkeypatch):
    """Fiber-group kernel with the two MPO-site contractions fused (two-site W blocks)."""
    patch_stage_run(monkeypatch)
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, dg, ws = record_operators(r, "cpu", use_fiber=True)
        assert sig.fused is not None
        x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64))
        ref = numpy.asarray(r["hvec_y"])
        assert numpy.abs(sig(x).numpy() - ref).max() <= 1e-12 * max(1.0, numpy.abs(ref).max())


@pytest.mark.parametrize("tag", ["K5", "K6"])
def test_sigma_fiber_unfused_emulated(tag, monkeypatch):
    """Fiber-group kernel for .W_i and .W_{i+1} as two separate stages (no two-site W)."""
    patch_stage_run(monkeypatch)
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, dg, ws = record_operators(r, "cpu", use_fiber=True, fuse_w=False)
        assert any(isinstance(s, CompositeStage) for s in sig.stages)
        assert sig.fused is None
        x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64))
        ref = numpy.asarray(r["hvec_y"])
        assert numpy.abs(sig(x).numpy() - ref).max() <= 1e-12 * max(1.0, numpy.abs(ref).max())


@pytest.mark.parametrize("tag", ["K5", "K6"])
def test_sigma_tensor_core_panels_emulated(tag, monkeypatch):
    """Panel GEMMs routed to the tensor-core tile class (TF32 modes) keep the same work-item semantics."""
    patch_stage_run(monkeypatch)
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, dg, ws = record_operators(r, "cpu", precision="tf32x3", use_fiber=True)
        x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64))
        ref = numpy.asarray(r["hvec_y"])
        y = sig(x, precision="f64").numpy()
        assert numpy.abs(y - ref).max() <= 1e-12 * max(1.0, numpy.abs(ref).max())


@pytest.mark.parametrize("tag", ["K5", "K6", "K5N8"])
def test_sigma_tma_tensor_core_units_emulated(tag, monkeypatch):
    """L.psi and .R as tensor-core work units (tensor-map boxes, column segments of the T1
    panels, row table, padded rows, transposed R panels, psi panels) have the semantics of
    HVecQt's top1 / top4 (interpreter, FP32 buffers)."""
    patch_stage_run(monkeypatch)
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, dg, ws = record_operators(r, "cpu", precision="tf32x3", use_fiber=True, fuse_w=False)
        assert sig.tc4 is not None and sig.tc4.ntasks > 0
        assert sig.tc1 is not None and sig.tc1.ntasks > 0
        x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64))
        ref = numpy.asarray(r["hvec_y"])
        y = sig(x).numpy()
        assert numpy.linalg.norm(y - ref) <= 2e-6 * numpy.linalg.norm(ref)


@pytest.mark.parametrize("tag", ["K5", "K6", "K5N8"])
def test_sigma_fgemm_slices_and_small_tiles_emulated(tag, monkeypatch):
    """Dense fiber-group GEMM with W panels cut into column slices and fiber tiles of a few
    fibers (small shared-memory budgets), T2 column by column: same sigma."""
    from qcmpodmrg_b200 import engine
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(engine, "FG_W_BUDGET", 40)
    monkeypatch.setattr(engine, "FG_A_BUDGET", 96)
    sliced = 0
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, dg, ws = record_operators(r, "cpu", use_fiber=True, fuse_w=False)
        for st in sig.stages:
            for s in getattr(st, "subs", [st]):
                if isinstance(s, engine.FiberStage) and s.ntasks:
                    g = s.h_groups
                    assert (g["R"].astype(numpy.int64) * g["FT"] <= max(96, 4 * g["R"].max())).all()
                    key = numpy.stack([g["row_b"], g["F"], g["R"]], 1)[g["R"] > 0]
                    sliced += len(key) - len(numpy.unique(key, axis=0))     # records cut from one group
        x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64))
        ref = numpy.asarray(r["hvec_y"])
        assert numpy.abs(sig(x).numpy() - ref).max() <= 1e-12 * max(1.0, numpy.abs(ref).max())
    assert sliced > 0
