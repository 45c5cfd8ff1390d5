"""NumPy interpreter of the qc_bgemm work-item semantics (test infrastructure).

Lets the plan compiler (task/contribution lists) be checked on a machine without
a GPU: C[tile] = sum_c alpha_c * A_c[M-tile, :] @ B_c[:, N-tile], with the
two-level index maps documented in qcmpodmrg_b200/csrc/qc_types.h.
"""
import numpy


def _idx(i, lo, s_hi, s_lo):
    return (i // lo) * s_hi + (i % lo) * s_lo


def _f64(t):
    """A device buffer as float64 NumPy (scratch may hold never-written FP32 bit patterns)."""
    with numpy.errstate(invalid="ignore", over="ignore"):
        return t.detach().cpu().numpy().astype(numpy.float64)


def patch_stage_run(monkeypatch):
    """Route Stage.run through the interpreter (tile extents follow the stage's tile config)."""
    import torch
    from qcmpodmrg_b200 import engine, kernels

    def run(self, A, B, C, kind="f64", stream=None):
        if self.ntasks == 0:
            return
        a = _f64(A)
        b = _f64(B)
        c = _f64(C)
        for cfg, tk, ct in self.host_groups:
            tm, tn = engine.TILES[cfg]
            _run_tiled(tk, ct, self.host_ops, self.summed, a, b, c, tm, tn)
        C.copy_(torch.from_numpy(c).to(C.dtype))

    monkeypatch.setattr(engine.Stage, "run", run)

    def frun(self, A, B, C, kind="f64", stream=None):
        if self.ntasks == 0:
            return
        a = _f64(A)
        w = _f64(B)
        c = _f64(C)
        if self.fgemm:
            _run_fgemm(self, a, w, c)
        else:
            _run_fiber(self, a, w, c)
        C.copy_(torch.from_numpy(c).to(C.dtype))

    monkeypatch.setattr(engine.FiberStage, "run", frun)

    def prun(self, A, B, C, kind="f64", stream=None):
        a = _f64(A)
        b = _f64(B)
        c = _f64(C)
        for (cfg, tk, _, _) in self.groups:
            tm, tn = engine.PANEL_TILES[cfg]
            for t in tk:
                for op in range(t["op_b"], t["op_e"]):
                    o = self.host_ops[op]
                    M, N, K = int(t["M"]), int(t["N"]), int(t["K"])
                    lda = int(t["lda"]) or K
                    Am = a[o["a_base"] + t["a_off"] + numpy.arange(M)[:, None] * lda + numpy.arange(K)[None, :]]
                    Bm = b[o["b_base"] + t["b_off"]:][:K * N].reshape(K, N)
                    m1, n1 = min(M, t["m0"] + tm), min(N, t["n0"] + tn)
                    blk = o["alpha"] * (Am[t["m0"]:m1] @ Bm[:, t["n0"]:n1])
                    if t["crow"] >= 0:         # rows scattered through the row table
                        rows = self.h_crow[t["crow"] + numpy.arange(t["m0"], m1)]
                        idx = o["c_base"] + rows[:, None] + numpy.arange(t["n0"], n1)[None, :]
                        c[idx] = blk
                    else:
                        cm = c[o["c_base"] + t["c_off"]:][:M * N].reshape(M, N)
                        cm[t["m0"]:m1, t["n0"]:n1] = blk
        C.copy_(torch.from_numpy(c).to(C.dtype))

    monkeypatch.setattr(engine.PanelStage, "run", prun)

    def block_permute(descs, ndescs, opspan, ops, src, dst):
        d = descs.cpu().numpy().view(engine.BPERM_DT)
        o = ops.cpu().numpy().view(engine.OP_DT)
        a = _f64(src)
        c = _f64(dst)
        for x in d:
            for op in range(x["op_b"], x["op_e"]):
                blk = a[o[op]["a_base"] + x["src_off"]:][:x["d0"] * x["d1"] * x["d2"]].reshape(x["d0"], x["d1"], x["d2"])
                i0, i1, i2 = numpy.meshgrid(numpy.arange(x["d0"]), numpy.arange(x["d1"]), numpy.arange(x["d2"]),
                                            indexing="ij")
                c[o[op]["c_base"] + x["dst_off"] + i0 * x["s0"] + i1 * x["s1"] + i2 * x["s2"]] = blk
        dst.copy_(torch.from_numpy(c).to(dst.dtype))
        return dst

    monkeypatch.setattr(kernels, "block_permute", block_permute)
    from qcmpodmrg_b200 import kernels

    def gather(src, idx, out):
        out.copy_(src[idx])
        return out

    def convert(src, out):
        n = min(src.numel(), out.numel())
        out[:n].copy_(src[:n].to(out.dtype))
        return out

    monkeypatch.setattr(kernels, "gather", gather)

    def scatter(src, idx, out):
        out.zero_()
        out[idx] = src[:idx.numel()]
        return out

    monkeypatch.setattr(kernels, "scatter", scatter)

    def reduce_ops(part, nops, n, out):
        out[:n].copy_(part[:nops * n].reshape(nops, n).sum(0).to(out.dtype))
        return out

    monkeypatch.setattr(kernels, "reduce_ops", reduce_ops)
    monkeypatch.setattr(kernels, "convert", convert)

    def tf32_split(hi, lo):          # exact in the interpreter: hi keeps x, lo = 0
        lo.zero_()
        return hi, lo

    monkeypatch.setattr(kernels, "tf32_split", tf32_split)

    def gather_split(x, idx, hi, lo):
        i = idx.cpu().numpy()
        v = numpy.where(i >= 0, _f64(x)[numpy.maximum(i, 0)], 0.0)
        hi.copy_(torch.from_numpy(v).to(hi.dtype))
        lo.zero_()
        return hi, lo

    monkeypatch.setattr(kernels, "gather_split", gather_split)

    def tcrun(self, A, B, C, kind="tf32x3", stream=None):
        a = _f64(A)
        b = _f64(B)
        c = _f64(C)
        _run_tcpanel(self, a, b, c)
        C.copy_(torch.from_numpy(c).to(C.dtype))

    monkeypatch.setattr(engine.TCPanelStage, "run", tcrun)


def _run_fiber(st, A, W, C):
    """Reference semantics of k_fiber: out[f, c] = alpha * sum_pairs sum_r in[r, f] * W[r, c]."""
    FT = st.tile
    for t in st.h_tasks:
        nf = min(FT, t["F"] - t["f0"])
        for op in range(t["op_b"], t["op_e"]):
            o = st.host_ops[op]
            rows = {}
            for fi in st.h_fin[t["in_b"]:t["in_e"]]:
                base = o["a_base"] + fi["a_off"]
                r = numpy.arange(fi["rows"])[:, None]
                f = t["f0"] + numpy.arange(nf)[None, :]
                idx = base + (f * fi["rows"] + r if fi["fiber_major"] else r * t["F"] + f)
                rows[int(fi["srow"])] = A[idx]
            for fo in st.h_fout[t["out_b"]:t["out_e"]]:
                acc = numpy.zeros((nf, fo["ncols"]))
                for p in st.h_fpair[fo["pair_b"]:fo["pair_e"]]:
                    blk = rows[int(p["srow"])]
                    wi = o["b_base"] + p["w_off"] + numpy.arange(p["rows"])[:, None] * fo["ncols"] + \
                        numpy.arange(fo["ncols"])[None, :]
                    acc += blk.T @ W[wi]
                fg = t["f0"] + numpy.arange(nf)
                cc = numpy.arange(fo["ncols"])[None, :]
                if fo["colmajor"]:
                    ci = o["c_base"] + fo["c_off"] + cc * t["F"] + fg[:, None]
                else:
                    ci = o["c_base"] + fo["c_off"] + ((fg // fo["flo"]) * fo["fhs"] + (fg % fo["flo"]) * fo["ncols"])[:, None] \
                        + cc
                C[ci] = o["alpha"] * acc


def _run_tiled(tasks, contribs, ops, summed, A, B, C, tm, tn):
    for t in tasks:
        ms = numpy.arange(t["m0"], min(t["m0"] + tm, t["M"]))
        ns = numpy.arange(t["n0"], min(t["n0"] + tn, t["N"]))
        outer = [None] if summed else list(range(t["op_b"], t["op_e"]))
        for oi in outer:
            acc = numpy.zeros((len(ms), len(ns)))
            for c in contribs[t["cb"]:t["ce"]]:
                ks = numpy.arange(c["K"])
                ao = c["a_off"] + _idx(ms, t["mlo"], c["a_mh"], c["a_ml"])[:, None] + \
                    _idx(ks, c["klo"], c["a_kh"], c["a_kl"])[None, :]
                bo = c["b_off"] + _idx(ks, c["klo"], c["b_kh"], c["b_kl"])[:, None] + \
                    _idx(ns, t["nlo"], c["b_nh"], c["b_nl"])[None, :]
                oprange = range(c["op_b"], c["op_e"]) if summed else [oi]
                for op in oprange:
                    o = ops[op]
                    acc += o["alpha"] * c["alpha"] * (A[o["a_base"] + ao] @ B[o["b_base"] + bo])
            cbase = 0 if summed else ops[oi]["c_base"]
            co = cbase + t["c_off"] + _idx(ms, t["mlo"], t["c_mh"], t["c_ml"])[:, None] + \
                _idx(ns, t["nlo"], t["c_nh"], t["c_nl"])[None, :]
            C[co] = acc


def _run_tcpanel(st, A, B, C):
    """Reference semantics of qc_tcpanel_f32: per unit, C[row table rows, n0 + n] = alpha * A . B^T,
    A and B addressed through the unit's tensor-map specifications (B as hi + lo planes)."""
    for u in st.h_units:
        wa, offa, dima, stra, _ = st.map_specs[int(u["a_map"])]
        wb, offb, dimb, strb, _ = st.map_specs[int(u["b_map"])]
        assert wa == "A" and wb == "B"
        K = int(dima[0])
        assert int(dimb[0]) == K
        m = int(u["a_c1"]) + numpy.arange(int(u["m_valid"]))
        n = int(u["b_c1"]) + numpy.arange(int(u["n_valid"]))
        assert m.max() < dima[1] and n.max() < dimb[1] and u["a_c2"] < dima[2] and u["b_c2"] < dimb[2]
        k = numpy.arange(K)
        ia = offa + int(u["a_c2"]) * stra[1] + m[:, None] * stra[0] + k[None, :]
        ib = offb + int(u["b_c2"]) * strb[1] + n[:, None] * strb[0] + k[None, :]
        am = A[ia] + (A[ia + stra[2]] if len(dima) == 4 else 0.0)       # pre-split A: hi + lo planes
        bm = B[ib] + B[ib + strb[2]]
        o = st.host_ops[int(u["op"])]
        tile = o["alpha"] * (am @ bm.T)
        if st.h_segs is None:
            rows = st.d_crow.cpu().numpy()[int(u["c_off"]) + numpy.arange(int(u["m_valid"]))] + int(u["b_c1"])
            idx = o["c_base"] + rows[:, None] + numpy.arange(int(u["n_valid"]))[None, :]
            C[idx] = tile
        else:
            for sg in st.h_segs[int(u["c_off"]):int(u["c_off"]) + int(u["nseg"])]:
                c = numpy.arange(int(sg["ncol"]))
                mm = numpy.arange(int(u["m_valid"]))
                idx = o["c_base"] + sg["off"] + (int(u["a_c1"]) + mm[:, None]) * int(sg["ldc"]) + c[None, :]
                C[idx] = tile[:, int(sg["col0"]) + c]


def wpanel_pairs(st, W):
    """Reference semantics of qc_wpanel_pairs: the zero-filled W panels with every W block
    of every record copied in for each operator of its range (columns permuted)."""
    from qcmpodmrg_b200.engine import fg_col_perm
    P = numpy.zeros(max(st.wpanel_size, 4), dtype=W.dtype)
    for w in st.h_wpairs:
        r = numpy.arange(int(w["nr"]))[:, None]
        j = numpy.arange(int(w["ncol"]))[None, :]
        pc = fg_col_perm(int(w["j0"]) + j, int(w["width"]), int(w["mc"]))
        for o in range(int(w["nops"])):
            sb = int(st.host_ops[int(w["op_b"]) + o]["b_base"]) + int(w["src"])
            d = int(w["dst"]) + o * int(w["opstride"]) + (int(w["r0"]) + r) * int(w["width"]) + pc
            P[d] = W[sb + r * int(w["src_ld"]) + j]
    return P


def _run_fgemm(st, A, W, C):
    """Reference semantics of k_fgemm, from its items, group / row / column records and
    W panel map only: C_g tile = alpha * A_g tile . W_g for every (item, operator)."""
    from qcmpodmrg_b200.engine import fg_col_perm
    P = wpanel_pairs(st, W)
    for it in st.h_items:
        g = st.h_groups[int(it["group"])]
        R, CT, CTs = int(g["R"]), int(g["CT"]), int(g["CTs"])
        assert int(it["nf"]) <= int(g["FT"]) and R * int(g["FT"]) <= st.max_a and R * CTs <= st.max_w
        assert CT <= st.max_ct and int(it["wpan"]) % 4 == 0 and int(it["wstride"]) % 4 == 0 and CTs % int(g["mc"]) == 0
        f = int(it["f0"]) + numpy.arange(int(it["nf"]))
        rows = st.h_rows[int(g["row_b"]):int(g["row_b"]) + R]
        cols = st.h_cols[int(g["col_b"]):int(g["col_b"]) + CT]
        flo = int(g["flo"])
        for op in range(int(it["op_b"]), int(it["op_e"])):
            o = st.host_ops[op]
            a = A[o["a_base"] + rows["off"][:, None] + f[None, :] * rows["fs"][:, None]]       # [R, nf]
            w0 = int(it["wpan"]) + (op - int(it["op_b"])) * int(it["wstride"])
            w = P[w0:w0 + R * CTs].reshape(R, CTs)[:, fg_col_perm(numpy.arange(CT), CTs, int(g["mc"]))]
            tile = o["alpha"] * (a.T @ w)                                                   # [nf, CT]
            ci = o["c_base"] + cols["off"][None, :] + (f // flo)[:, None] * cols["fhs"][None, :] + \
                (f % flo)[:, None] * cols["fs"][None, :]
            C[ci] = tile
