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
from qcmpodmrg_b200.engine import fg_col_perm, CompositeStage, FiberStage, PanelStage, PANEL_TILES


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
                if ob["colmajor"]:
                    out.append((cb + int(ob["c_off"]) + numpy.arange(nc)[None, :] * int(t["F"]) + f[:, None]).ravel())
                    continue
                rows = cb + int(ob["c_off"]) + (f // int(ob["flo"])) * int(ob["fhs"]) + (f % int(ob["flo"])) * nc
                out.append((rows[:, None] + numpy.arange(nc)[None, :]).ravel())
    return numpy.concatenate(out) if out else numpy.zeros(0, dtype=numpy.int64)


def _fgemm_writes_reads(fs):
    """Elements the dense fiber-group GEMM writes (from its own tables) and its highest read."""
    out, hi = [], -1
    for it in fs.h_items:
        g = fs.h_groups[int(it["group"])]
        f = int(it["f0"]) + numpy.arange(int(it["nf"]))
        cols = fs.h_cols[int(g["col_b"]):int(g["col_b"]) + int(g["CT"])]
        rows = fs.h_rows[int(g["row_b"]):int(g["row_b"]) + int(g["R"])]
        flo = int(g["flo"])
        for op in range(int(it["op_b"]), int(it["op_e"])):
            o = fs.host_ops[op]
            out.append((int(o["c_base"]) + cols["off"][None, :] + (f // flo)[:, None] * cols["fhs"][None, :]
                        + (f % flo)[:, None] * cols["fs"][None, :]).ravel())
            if len(rows):
                hi = max(hi, int((int(o["a_base"]) + rows["off"] + int(f[-1]) * rows["fs"]).max()))
                assert int((int(o["a_base"]) + rows["off"]).min()) >= 0
    return (numpy.concatenate(out) if out else numpy.zeros(0, dtype=numpy.int64)), hi


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
                if sub.fgemm:
                    wg, hi = _fgemm_writes_reads(sub)
                    assert numpy.array_equal(numpy.sort(wg), numpy.sort(w)), sub.name
                    assert hi < src, sub.name
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


@pytest.mark.parametrize("tag", ["K5", "K6", "K5N8"])
def test_dense_fiber_group_tables(tag, monkeypatch):
    """Dense fiber-group GEMM tables: items tile every group's fibers exactly once for its
    operator range; every item's staged A tile, W panel and columns fit the launch's
    max_a / max_w / max_ct (and the shared memory of both precisions); W panels stay inside
    the gathered panel buffer at 16-byte offsets; T2 is written column by column and read
    back with contiguous fibers."""
    patch_stage_run(monkeypatch)
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, _, _ = record_operators(r, "cpu", use_fiber=True, fuse_w=False)
        for st in sig.stages:
            for sub in _subs(st):
                if not (isinstance(sub, FiberStage) and sub.ntasks):
                    continue
                assert sub.fgemm
                it, gr = sub.h_items, sub.h_groups
                g = gr[it["group"]]
                assert (it["nf"] >= 1).all() and (it["nf"] <= g["FT"]).all() and (g["FT"] % 4 == 0).all()
                assert (g["R"].astype(numpy.int64) * g["FT"] <= sub.max_a).all()
                assert (g["R"].astype(numpy.int64) * g["CTs"] <= sub.max_w).all()
                assert (g["CT"] <= sub.max_ct).all() and (g["CTs"] % g["mc"] == 0).all()
                assert sub.max_a % 4 == 0 and sub.max_w % 4 == 0
                for elem in (4, 8):
                    assert 2 * sub.max_ct * 32 + 2 * (sub.max_a + sub.max_w) * elem <= 220 * 1024
                assert (it["wpan"] % 4 == 0).all() and (it["wstride"] % 4 == 0).all()
                last = it["wpan"] + (it["op_e"] - 1 - it["op_b"]).astype(numpy.int64) * it["wstride"] + \
                    g["R"].astype(numpy.int64) * g["CTs"]
                assert last.max() <= sub.wpanel_size
                # W blocks: inside the panels and the W tensor set, every panel element
                # written at most once per operator, columns inside the panel width
                wp = sub.h_wpairs
                assert (wp["j0"] >= 0).all() and (wp["j0"] + wp["ncol"] <= wp["width"]).all()
                assert (wp["nr"] >= 1).all() and (wp["ncol"] >= 1).all() and (wp["nops"] >= 1).all()
                count = numpy.zeros(sub.wpanel_size, dtype=numpy.int64)
                wtot = int(sub.host_ops["b_base"].max()) + 1
                for w in wp:
                    rr = numpy.arange(int(w["nr"]))[:, None]
                    jj = numpy.arange(int(w["ncol"]))[None, :]
                    pc = fg_col_perm(int(w["j0"]) + jj, int(w["width"]), int(w["mc"]))
                    for o in range(int(w["nops"])):
                        dd = int(w["dst"]) + o * int(w["opstride"]) + (int(w["r0"]) + rr) * int(w["width"]) + pc
                        numpy.add.at(count, dd.ravel(), 1)
                        si = int(sub.host_ops[int(w["op_b"]) + o]["b_base"]) + int(w["src"]) + \
                            rr * int(w["src_ld"]) + jj
                        assert si.min() >= 0
                    assert int(w["src"]) + (int(w["nr"]) - 1) * int(w["src_ld"]) + int(w["ncol"]) - 1 >= 0
                assert count.max() <= 1
                assert wtot >= 1
                for k in numpy.unique(it["group"]):
                    sel = it[it["group"] == k]
                    cover = numpy.zeros(int(gr[k]["F"]), dtype=numpy.int64)
                    for x in sel:
                        cover[int(x["f0"]):int(x["f0"]) + int(x["nf"])] += 1
                    assert (cover == 1).all()
                if sub.name == "sigma2":
                    assert (sub.h_fout["colmajor"] == 1).all()
                if sub.name == "sigma3":
                    assert (sub.h_fin["fiber_major"] == 0).all()
