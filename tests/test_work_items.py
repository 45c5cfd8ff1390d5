"""Structural invariants of the compiled work items (no GPU): every element a
fiber-group or panel-GEMM launch writes lies inside its destination buffer and is
written exactly once (no two tasks, tiles or operators write the same element),
and every element a task reads lies inside its source buffer.  These are the
properties that keep the kernels free of out-of-bounds and racing writes."""
import numpy
import pytest
import torch

from helpers import load, record_operators, record_sp_operators
from emulate import patch_stage_run
from qcmpodmrg_b200.engine import CompositeStage, FiberStage, PanelStage, PANEL_TILES


def _subs(st):
    return st.subs if isinstance(st, CompositeStage) else [st]


def _fiber_writes(fs):
    out = []
    for t in fs.h_tasks:
        nf = min(fs.tile, int(t["F"]) - int(t["f0"]))
        f = int(t["f0"]) + numpy.arange(nf)
        for op in range(int(t["op_b"]), int(t["op_e"])):
            cb = int(fs.host_ops[op]["c_base"])
            for ob in fs.h_fout[int(t["out_b"]):int(t["out_e"])]:
                nc = int(ob["ncols"])
                rows = cb + int(ob["c_off"]) + (f // int(ob["flo"])) * int(ob["fhs"]) + (f % int(ob["flo"])) * nc
                out.append((rows[:, None] + numpy.arange(nc)[None, :]).ravel())
    return numpy.concatenate(out) if out else numpy.zeros(0, dtype=numpy.int64)


def _fiber_reads(fs):
    hi = []
    for t in fs.h_tasks:
        nf = min(fs.tile, int(t["F"]) - int(t["f0"]))
        for op in range(int(t["op_b"]), int(t["op_e"])):
            ab = int(fs.host_ops[op]["a_base"])
            for b in fs.h_fin[int(t["in_b"]):int(t["in_e"])]:
                assert int(b["srow"]) + int(b["rows"]) <= fs.max_rows
                last_f = int(t["f0"]) + nf - 1
                if b["fiber_major"]:
                    hi.append(ab + int(b["a_off"]) + last_f * int(b["rows"]) + int(b["rows"]) - 1)
                else:
                    hi.append(ab + int(b["a_off"]) + (int(b["rows"]) - 1) * int(t["F"]) + last_f)
    return max(hi) if hi else -1


def _panel_writes(ps):
    out = []
    for (cfg, tk, _, _) in ps.groups:
        tm, tn = PANEL_TILES[cfg]
        for t in tk:
            m = int(t["m0"]) + numpy.arange(min(tm, int(t["M"]) - int(t["m0"])))
            n = int(t["n0"]) + numpy.arange(min(tn, int(t["N"]) - int(t["n0"])))
            rows = ps.h_crow[int(t["crow"]) + m] if t["crow"] >= 0 else int(t["c_off"]) + m * int(t["N"])
            for op in range(int(t["op_b"]), int(t["op_e"])):
                cb = int(ps.host_ops[op]["c_base"])
                out.append((cb + rows[:, None] + n[None, :]).ravel())
    return numpy.concatenate(out) if out else numpy.zeros(0, dtype=numpy.int64)


def _check_sigma_writes(sig):
    ndst = {"sigma1": sig.tot[0], "sigma2": sig.tot[1], "sigma3": sig.tot[2], "sigma23": sig.tot[2],
            "sigma4": sig.nops * sig.ndim0}
    stages = list(sig.stages) + ([sig.fused] if sig.fused is not None else [])
    for st in stages:
        for sub in _subs(st):
            if isinstance(sub, FiberStage) and sub.ntasks:
                w = _fiber_writes(sub)
                assert w.min() >= 0 and w.max() < ndst[sub.name], sub.name
                assert len(numpy.unique(w)) == len(w), "overlapping writes in " + sub.name
                src = {"sigma2": sig.tot[0], "sigma3": sig.tot[1], "sigma23": sig.tot[0]}[sub.name]
                assert _fiber_reads(sub) < src, sub.name
            if isinstance(sub, PanelStage) and sub.groups:
                w = _panel_writes(sub)
                assert w.min() >= 0 and w.max() < ndst[sub.name], sub.name
                assert len(numpy.unique(w)) == len(w), "overlapping writes in " + sub.name


@pytest.mark.parametrize("tag", ["K4", "K5", "K6"])
@pytest.mark.parametrize("fuse", [False, True])
def test_fiber_and_panel_writes_in_bounds_and_disjoint(tag, fuse, monkeypatch):
    patch_stage_run(monkeypatch)
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, _, _ = record_operators(r, "cpu", use_fiber=True, fuse_w=fuse)
        _check_sigma_writes(sig)


@pytest.mark.parametrize("tag", ["SP_K4", "SP_K5"])
def test_spin_projected_plans_write_in_bounds_and_disjoint(tag, monkeypatch):
    """The same invariants for the N-symmetry plans of the projected H and S operators,
    and the reduction map stays inside the reduced vector."""
    patch_stage_run(monkeypatch)
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, sv, _, _, _ = record_sp_operators(r, "cpu", use_fiber=True)
        for op in (sig, sv):
            _check_sigma_writes(op.inner)
            red = op.red.numpy()
            assert red.min() >= 0 and red.max() < op.nn and len(numpy.unique(red)) == len(red)


@pytest.mark.parametrize("tag", ["K5", "K6"])
def test_panel_layouts_cover_the_intermediates_once(tag, monkeypatch):
    """T1 panels hold every T1 block of the L.psi pairs once; T3 panels every T3 block
    the .R contraction needs once (their extents tile the panel sizes exactly)."""
    patch_stage_run(monkeypatch)
    from qcmpodmrg_b200.engine import panel_sigma1, panel_sigma4
    from qcmpodmrg_b200.qtensor import Contraction, flip_right
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, _, _ = record_operators(r, "cpu", use_fiber=True, fuse_w=False)
        psi = sig.psi
        for i in range(sig.nops):
            Ll = sig.L.layouts[i]
            c1 = Contraction(Ll, psi, ([2], [0]))
            pan = panel_sigma1(Ll, psi, c1.triples, c1.out.nblks)
            assert pan is not None
            ob = c1.triples[:, 0]
            size = c1.out.ndim[ob]
            cover = numpy.zeros(pan["t1size"], dtype=numpy.int64)
            for o, n in zip(pan["t1off"][ob], size):
                cover[o:o + n] += 1
            assert (cover == 1).all()


@pytest.mark.parametrize("tag", ["K5", "K6"])
def test_persistent_fiber_staging_in_bounds(tag, monkeypatch):
    """Persistent fiber kernel: one work record per (task, operator); every group's metadata
    blob fits max_blob and repeats the group's records (outputs' pair ranges rebased); inside
    an item the W blocks of its pairs get disjoint shared-memory areas (rows padded to 4)
    within max_w, and the 8-wide W reads of the last column block stay inside max_w + 8."""
    from emulate import decode_blob
    patch_stage_run(monkeypatch)
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, _, _ = record_operators(r, "cpu", use_fiber=True, fuse_w=False)
        for st in sig.stages:
            for sub in _subs(st):
                if not (isinstance(sub, FiberStage) and sub.ntasks):
                    continue
                t = sub.h_tasks
                live = t["out_e"] > t["out_b"]
                assert len(sub.h_work) == int((t["op_e"] - t["op_b"])[live].sum())
                assert int(sub.h_work["blob_len"].max()) <= sub.max_blob
                assert (sub.h_work["blob"] + sub.h_work["blob_len"]).max() <= len(sub.h_blob)
                for wk in sub.h_work[:: max(1, len(sub.h_work) // 200)]:
                    fins, fouts, pairs = decode_blob(sub, wk)
                    assert fouts["pair_b"].min() >= 0 and fouts["pair_e"].max() <= len(pairs)
                    if len(fins):                  # groups of zero-filled outputs stage nothing
                        assert (fins["srow"] + fins["rows"]).max() <= sub.max_rows
                    spans = []
                    for fo in fouts:
                        ncp = (int(fo["ncols"]) + 3) // 4 * 4
                        for p in pairs[int(fo["pair_b"]):int(fo["pair_e"])]:
                            lo, hi = int(p["wsm"]), int(p["wsm"]) + int(p["rows"]) * ncp
                            assert lo % 4 == 0 and hi <= sub.max_w
                            last = lo + (int(p["rows"]) - 1) * ncp + ((int(fo["ncols"]) - 1) // 8) * 8 + 7
                            assert last < sub.max_w + 8
                            spans.append((lo, hi))
                    spans.sort()
                    assert all(a[1] <= b[0] for a, b in zip(spans, spans[1:]))
