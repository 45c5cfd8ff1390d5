"""Device operators of the two-site hot path: sigma, diagonal, renormalisation.

  SigmaOperator  <- HVecQt        source/mpo_dmrg_kernelQt.py:153-319 (two-site :238-317)
  DiagOperator   <- HDiagQt       source/mpo_dmrg_kernelQt.py:30-127  (two-site :77-119)
  Renormalizer   <- renormQt_H00  source/mpo_dmrg_kernelQt.py:633-767 (also genHopsQt,
                                  source/mpo_dmrg_initQt.py:88-271, which is the same chain)

The reference loops over operators p, MPO slices and block pairs in Python and
calls numpy.tensordot per pair.  Here the operator loop is folded into the
work lists: each of the four sigma contractions (L.psi, .W_i, .W_{i+1}, .R) is
one launch over all operators and all block pairs, with intermediates in HBM
scratch and the sum over operators done inside the last launch (no atomics).
Block-pair lists are built per symmetry class of the operator, as the
reference caches its templates per class.
"""
import numpy
import torch

from . import native
from .native import check
from .engine import (Stage, compile_classes, add_parts, live_blocks, prune, op_table, TASK_DT, CONTRIB_DT, LOG,
                     compile_fiber, FiberStage, CompositeStage, panel_sigma1, compile_panels, BPERM_DT, PanelStage,
                     fiber_stages, panel_sigma4, upload)
from .mpo import case
from .qtensor import Contraction, Layout, flip_right, flip_horizontal


class Workspace(object):
    """Grow-only device scratch buffers shared by all operators of a context."""

    def __init__(self, device):
        self.device = device
        self.bufs = {}

    def get(self, name, numel, dtype):
        b = self.bufs.get((name, dtype))
        if b is None or b.numel() < numel:
            self.bufs.pop((name, dtype), None)
            b = torch.empty(max(int(numel), 1) + 64, dtype=dtype, device=self.device)
            self.bufs[(name, dtype)] = b
        return b


class TensorSet(object):
    """Per-operator block tensors (environments or site operators) back to back in one buffer."""

    def __init__(self, layouts, values, offsets=None, device=None):
        self.layouts = list(layouts)
        if offsets is None:
            sizes = numpy.array([l.size for l in self.layouts], dtype=numpy.int64)
            offsets = numpy.concatenate([[0], numpy.cumsum(sizes)[:-1]]).astype(numpy.int64)
        self.offsets = numpy.asarray(offsets, dtype=numpy.int64)
        self.total = int(self.offsets[-1] + self.layouts[-1].size) if self.layouts else 0
        if isinstance(values, (list, tuple)):
            host = numpy.concatenate([numpy.asarray(v, dtype=numpy.float64) for v in values]) \
                if values else numpy.zeros(0)
            values = torch.from_numpy(host).to(device)
        self.values = values
        self._f32 = None

    def f32(self):
        if self._f32 is None or self._f32.data_ptr() == 0:
            self._f32 = self.values.to(torch.float32)
        return self._f32

    def op_values(self, i):
        o = int(self.offsets[i])
        return self.values[o:o + self.layouts[i].size]

    def nbytes(self):
        return self.values.numel() * self.values.element_size()


def _stream(device):
    return torch.cuda.current_stream(device).cuda_stream


def block_permute(descs, ndescs, opspan, ops, src, dst):
    """Per-dot block permutation of an FP64 tensor set into dst (FP64 or FP32), qc_block_permute."""
    check(native.lib().qc_block_permute(descs.data_ptr(), ndescs, opspan, ops.data_ptr(), src.data_ptr(),
                                        dst.data_ptr(), int(dst.dtype == torch.float32), _stream(dst.device)),
          "qc_block_permute")
    LOG.launches += 1
    return dst


def gather(src, idx, out):
    """out[i] = src[idx[i]] on the device (qc_gather_f64)."""
    check(native.lib().qc_gather_f64(src.data_ptr(), idx.data_ptr(), out.data_ptr(), out.numel(),
                                     _stream(out.device)), "qc_gather_f64")
    LOG.launches += 1
    return out


def scatter(src, idx, out):
    """out = 0; out[idx[i]] = src[i] on the device (qc_scatter_f64)."""
    check(native.lib().qc_scatter_f64(src.data_ptr(), idx.data_ptr(), out.data_ptr(), idx.numel(), out.numel(),
                                      _stream(out.device)), "qc_scatter_f64")
    LOG.launches += 1
    return out


def convert(src, out):
    """FP64 <-> FP32 conversion on the device."""
    lib = native.lib()
    n = min(src.numel(), out.numel())
    if src.dtype == torch.float64:
        check(lib.qc_convert_f64_to_f32(src.data_ptr(), out.data_ptr(), n, _stream(out.device)), "convert")
    else:
        check(lib.qc_convert_f32_to_f64(src.data_ptr(), out.data_ptr(), n, _stream(out.device)), "convert")
    LOG.launches += 1
    return out


def gather_split(x, idx, hi, lo):
    """hi[i] = tf32(x[idx[i]]), lo[i] = tf32(x[idx[i]] - hi[i]); idx < 0 gives 0 (qc_gather_split_f32)."""
    check(native.lib().qc_gather_split_f32(x.data_ptr(), idx.data_ptr(), idx.numel(), hi.data_ptr(), lo.data_ptr(),
                                           _stream(hi.device)), "qc_gather_split_f32")
    LOG.launches += 1
    return hi, lo


def tf32_split(hi, lo):
    """hi = tf32(x), lo = tf32(x - hi) for the FP32 values x held in hi (qc_tf32_split)."""
    check(native.lib().qc_tf32_split(hi.data_ptr(), lo.data_ptr(), hi.numel(), _stream(hi.device)),
          "qc_tf32_split")
    LOG.launches += 1
    return hi, lo


def reduce_ops(part, nops, n, out):
    """out = sum over operators of the per-operator partial vectors (qc_reduce_ops_*)."""
    lib = native.lib()
    fn = lib.qc_reduce_ops_f64 if part.dtype == torch.float64 else lib.qc_reduce_ops_f32
    check(fn(part.data_ptr(), nops, n, out.data_ptr(), _stream(out.device)), "qc_reduce_ops")
    LOG.launches += 1
    return out


def _groups(opers, isite, ncsite):
    g = {}
    for iop, p in enumerate(opers):
        g.setdefault(case(p, isite, ncsite), []).append(iop)
    return g


def _ncols(c, triples):
    """N extent (product of the operand-2 external dims) of the output blocks a stage writes."""
    if len(triples) == 0:
        return numpy.array([64])
    ne1 = c.l1.rank - len(c.axes[0])
    ob = numpy.unique(triples[:, 0])
    return numpy.prod(c.out.block_dims(ob)[:, ne1:], axis=1)


def unit_phys_t2(lay):
    """True when every block of the intermediate T2 = T1 . W_i, axes (l', n2, r, b, n1'),
    has extent 1 on its two physical axes (1 and 4)."""
    if lay.rank != 5 or len(lay.idx_allowed) == 0:
        return False
    d = lay.block_dims(lay.idx_allowed)
    return bool(numpy.all(d[:, 1] == 1) and numpy.all(d[:, 4] == 1))


def pair_flops(c, t):
    """2*M*N*K summed over the block pairs of one contraction (one operator)."""
    if len(t) == 0:
        return 0.0
    ne1 = c.l1.rank - len(c.axes[0])
    d = c.out.block_dims(t[:, 0]).astype(numpy.float64)
    k = c.l1.block_dims(t[:, 1])[:, c.axes[0]].astype(numpy.float64)
    return 2.0 * float((d.prod(axis=1) * k.prod(axis=1)).sum())


class SigmaOperator(object):
    """sigma = sum_p w_p R_p W_p[i+1] W_p[i] L_p psi for the dot (isite, isite+1)."""

    def __init__(self, ws, isite, psi_layout, L, R, Wi, Wj, qkey, opers, hpwts, precision="f64",
                 tensor_cores=None, use_fiber=False, fuse_w=True, panel1=True, panel4=True, live=None,
                 fg_budget=None):
        """fg_budget: (A, W) shared-memory budgets of the dense fiber-group GEMM (qc_fgemm), as
        chosen by qcmpodmrg_b200.autotune; None keeps the engine's defaults.
        live: optional mask over the wavefunction layout's flat blocks.  Blocks outside it
        are zero in every input vector and discarded in every output (the blocks that N
        symmetry adds to an (N, Sz) wavefunction under spin projection): block pairs that
        read them in the first contraction or write them in the last are not compiled."""
        self.ws, self.psi, self.precision = ws, psi_layout, precision
        # tcgen05 tiles for the two large contractions (L.psi and .R) in TF32 modes
        tc = (precision in ("tf32", "tf32x3")) if tensor_cores is None else tensor_cores
        # tf32x3: the .R panel GEMMs on the TMA-fed tcgen05 kernel (qc_tcpanel_f32); the older
        # gathered tensor-core tiles (qc_bgemm_tf32*) stay for plain tf32 and explicit requests
        want_tc4 = precision == "tf32x3" and tensor_cores is None and use_fiber and panel4
        want_tc1 = precision == "tf32x3" and tensor_cores is None and panel1
        if want_tc4 or want_tc1:
            tc = False
        self.L, self.R, self.Wi, self.Wj = L, R, Wi, Wj
        self._lays = (list(L.layouts), list(R.layouts))      # held: identity is the plan's key
        dev = ws.device
        groups = _groups(opers, isite, 2)
        nops = len(opers)
        ax = (([2], [0]), ([0, 2], [0, 3]), ([1, 3], [3, 0]), ([1, 3], [2, 0]))
        bases = [numpy.zeros(nops, dtype=numpy.int64) for _ in range(3)]
        tot = [0, 0, 0]
        wbase = numpy.zeros(nops, dtype=numpy.int64)
        wtot = 0
        plans = {}
        for key, ops in sorted(groups.items()):
            i0 = ops[0]
            Ll, W1, W2 = L.layouts[i0], Wi.layouts[i0], Wj.layouts[i0]
            Rl = flip_right(R.layouts[i0], qkey)
            for i in ops:
                if (L.layouts[i] is not Ll or Wi.layouts[i] is not W1 or Wj.layouts[i] is not W2
                        or flip_right(R.layouts[i], qkey) is not Rl):
                    raise ValueError("operators of one symmetry class must share their block structure")
            c1 = Contraction(Ll, psi_layout, ax[0])
            t1 = c1.triples if live is None else prune(c1.triples, live2=live)
            # L.psi as dense panel GEMMs (T1 blocks stored panel by panel)
            pan = panel_sigma1(Ll, psi_layout, t1, c1.out.nblks) if panel1 else None
            t1off = pan["t1off"] if pan is not None else None
            c2 = Contraction(c1.out, W1, ax[1])
            t2 = prune(c2.triples, live1=live_blocks(c1.out, t1))
            c3 = Contraction(c2.out, W2, ax[2])
            t3 = prune(c3.triples, live1=live_blocks(c2.out, t2))
            # .W_i and .W_{i+1} fused: T3 = T1 . (W_i W_{i+1}) with the two-site MPO
            # block Wij[a, n1', n1, c, n2', n2] = sum_b W_i[a, b, n1', n1] W_{i+1}[b, c, n2', n2]
            # made once per dot, so T2 is never written (fiber-group kernel only)
            c4 = Contraction(c3.out, Rl, ax[3])
            t4all = c4.triples if live is None else c4.triples[live[c4.triples[:, 0]]]
            # .R as dense panel GEMMs (T3 blocks written into sigma-block panels by the
            # fiber kernel, R blocks permuted into per-sector panels once per dot)
            pan4 = panel_sigma4(c3.out, Rl, psi_layout, t4all) if (use_fiber and panel4) else None
            o3 = {} if pan4 is None else {"out_off": pan4["t3off"], "out_fhs": pan4["t3fhs"],
                                          "out_flo": pan4["t3flo"], "extra_out": pan4["needed"]}
            fused = None
            fib2 = fib3 = None
            if use_fiber and fuse_w:
                cW = Contraction(W1, W2, ([1], [0]))
                cF = Contraction(c1.out, cW.out, ([0, 2, 3], [0, 2, 5]))
                if cF.out is c3.out:
                    tF = prune(cF.triples, live1=live_blocks(c1.out, t1), live2=live_blocks(cW.out, cW.triples))
                    fp = compile_fiber(cF, tF, 0, 0, in_off=t1off, **o3)
                    if fp is not None:
                        fused = (cW, cF, tF, fp)
            elif use_fiber:
                # .W_i and .W_{i+1} on the fiber kernel: T2 stored column by column (its
                # physical axes have extent 1, so a T2 block's columns are the next
                # contraction's rows and its fibers that contraction's fibers), read back
                # with contiguous fibers
                cm = bool(unit_phys_t2(c2.out))
                fib2 = compile_fiber(c2, t2, 0, 0, in_off=t1off, out_colmajor=cm)
                cm = cm and fib2 is not None
                if pan4 is not None:
                    fib3 = compile_fiber(c3, t3, 3, 0 if cm else 1, **o3)
                    if fib3 is None:
                        pan4 = None
                if fib3 is None:
                    fib3 = compile_fiber(c3, t3, 3, 0 if cm else 1)
                if fib3 is None and cm:
                    fib2 = compile_fiber(c2, t2, 0, 0, in_off=t1off)       # T2 packed for the grouped GEMM
            if pan4 is not None and fused is None and fib3 is None:
                pan4 = None                 # T3 comes from the grouped GEMM in the packed layout
            t4 = prune(t4all, live1=live_blocks(c3.out, fused[2] if fused else t3))
            if c4.out is not psi_layout:
                raise ValueError("sigma output layout differs from the wavefunction template")
            plans[key] = (ops, (c1, t1), (c2, t2), (c3, t3), (c4, t4), Rl, fused, pan, pan4, fib2, fib3)
            for s, c in enumerate((c1, c2, c3)):
                if s == 1 and fused is not None:
                    continue            # no T2 for fused classes
                size = pan["t1size"] if (s == 0 and pan is not None) else c.out.size
                if s == 2 and pan4 is not None:
                    size = pan4["t3size"]
                size = (int(size) + 31) // 32 * 32      # 128-byte aligned operator slices (TMA)
                for i in ops:
                    bases[s][i] = tot[s]
                    tot[s] += size
            if fused is not None:
                for i in ops:
                    wbase[i] = wtot
                    wtot += fused[0].out.size
        self.tot = tot
        self.nops = nops
        hp = numpy.asarray(hpwts, dtype=numpy.float64)
        # operator tables: operators ordered class by class; the last contraction
        # writes one partial sigma per operator (slot = position in that order)
        order = numpy.concatenate([numpy.array(plans[k][0]) for k in sorted(plans)])
        slot = numpy.arange(nops, dtype=numpy.int64) * psi_layout.size
        tabs = [op_table(L.offsets[order], 0, bases[0][order], 1.0),
                op_table(bases[0][order], Wi.offsets[order], bases[1][order], 1.0),
                op_table(bases[1][order], Wj.offsets[order], bases[2][order], 1.0),
                op_table(bases[2][order], R.offsets[order], slot, hp[order])]
        st = [{}, {}, {}, {}]
        fib = [[], [], [], []]
        fuse_parts, wij_parts = [], {}
        # how the W contractions of each symmetry class run: fused / fiber / grouped GEMM
        self.w_paths = {"fused": 0, "fiber": 0, "generic": 0}
        pos = 0
        # W contractions: fiber-group kernel (inputs staged once per fiber tile) where
        # every group fits in shared memory, generic grouped GEMM otherwise
        lperm = []
        pst, pst_tc = {}, {}            # panel GEMM parts of the L.psi contraction
        rperm = []
        p4st, p4st_tc = {}, {}          # panel GEMM parts of the .R contraction
        crow_all, crow_n = [], 0        # their row table (panel row -> sigma element offset)
        tc4_classes = []                # (operator range, pan4, row-table base) for the tensor-core .R
        tc1_classes = []                # (operator range, pan["tc"]) for the tensor-core L.psi
        any4 = any(v[8] is not None for v in plans.values())
        for key, (ops, *cs, Rl, fused, pan, pan4, fib2, fib3) in sorted(plans.items()):
            rng = (pos, pos + len(ops))
            pos += len(ops)
            t1off = pan["t1off"] if pan is not None else None
            if panel1:
                if pan is not None:
                    src, dst, n = pan["lperm"]
                else:                   # no panels for this class: L blocks copied in place
                    Ll = cs[0][0].l1
                    src = dst = Ll.ioff[Ll.idx_allowed]
                    n = Ll.ndim[Ll.idx_allowed]
                d = numpy.zeros(len(src), BPERM_DT)
                d["src_off"], d["dst_off"] = src, dst
                d["d0"], d["d1"], d["d2"] = 1, 1, n
                d["s2"] = 1
                d["op_b"], d["op_e"] = rng
                lperm.append(d)
            if any4:
                d = numpy.zeros(0, BPERM_DT)
                if pan4 is not None:
                    src, dst, dU = pan4["rperm"]
                    d = numpy.zeros(len(src), BPERM_DT)
                    d["src_off"], d["dst_off"] = src, dst
                    d["d0"], d["d1"], d["d2"] = dU[:, 0], dU[:, 1], dU[:, 2]
                    d["s0"], d["s1"], d["s2"] = dU[:, 1], 1, dU[:, 0] * dU[:, 1]
                else:                       # R blocks copied in place
                    src = dst = Rl.ioff[Rl.idx_allowed]
                    d = numpy.zeros(len(src), BPERM_DT)
                    d["src_off"], d["dst_off"] = src, dst
                    d["d0"], d["d1"], d["d2"] = 1, 1, Rl.ndim[Rl.idx_allowed]
                    d["s2"] = 1
                d["op_b"], d["op_e"] = rng
                rperm.append(d)
            if pan4 is not None:
                g4 = pan4["gemm"]
                g4 = g4[:6] + (g4[6] + crow_n,) + tuple(g4[7:])     # row-table indices into the stage's table
                if want_tc4:
                    tc4_classes.append((rng, pan4, crow_n))
                crow_all.append(pan4["crow"])
                crow_n += len(pan4["crow"])
                parts = compile_panels(g4, rng, tensor_cores=bool(tc))
                if tc:
                    parts, tcp = parts
                    add_parts(p4st_tc, tcp)
                for cfg, part in parts.items():
                    p4st.setdefault(cfg, []).append(part)
            if fib3 is not None:
                fib[2].append(fib3 + (rng,))
                self.w_paths["fiber"] += 1
            if fused is not None:
                cW, cF, tF, fp = fused
                fuse_parts.append(fp + (rng,))
                self.w_paths["fused"] += 1
                add_parts(wij_parts, compile_classes(cW, cW.triples, ([1], [0])), op_range=rng)
            for si, (c, t) in enumerate(cs):
                if fused is not None and si in (1, 2):
                    continue
                if (si == 2 and fib3 is not None) or (si == 3 and pan4 is not None):
                    continue
                if si == 0 and pan is not None:
                    if want_tc1:
                        tc1_classes.append((rng, pan["tc"]))
                    parts = compile_panels(pan["gemm"], rng, tensor_cores=bool(tc))
                    if tc:
                        parts, tcp = parts
                        add_parts(pst_tc, tcp)
                    for cfg, part in parts.items():
                        pst.setdefault(cfg, []).append(part)
                    continue
                off1 = t1off if si == 1 else None
                if si == 1 and fib2 is not None:
                    fib[1].append(fib2 + (rng,))
                    self.w_paths["fiber"] += 1
                    continue
                if si in (1, 2):
                    self.w_paths["generic"] += 1
                add_parts(st[si], compile_classes(c, t, ax[si], tensor_cores=tc if si in (0, 3) else False,
                                                  off1=off1), op_range=rng)
        self.stages = []
        for si in range(4):
            g = Stage(st[si], dev, "sigma%d" % (si + 1), tabs[si]) if st[si] else None
            f = fiber_stages(fib[si], dev, "sigma%d" % (si + 1), tabs[si], fg_budget) if fib[si] else []
            if si == 0:
                self._s0_generic = g
            if si == 0 and (pst or pst_tc):
                f = [PanelStage(pst, dev, "sigma1", tabs[0], pst_tc)]
            if si == 3 and (p4st or p4st_tc):
                f = [PanelStage(p4st, dev, "sigma4", tabs[3], p4st_tc,
                                crow=numpy.concatenate(crow_all) if crow_all else None)]
            if not f:
                self.stages.append(g if g is not None else Stage({}, dev, "sigma%d" % (si + 1), tabs[si]))
            else:
                self.stages.append(CompositeStage(f + [g], "sigma%d" % (si + 1)))
        # per-dot L panels (a block permutation of every operator's L), FP64 and FP32
        self.lperm = None
        if lperm:
            self._lperm_h = numpy.concatenate(lperm)
            self.lperm = upload(self._lperm_h, dev)
            self._lperm_ops = op_table(L.offsets[order], 0, L.offsets[order], 1.0)
            self._lperm_ops_d = upload(self._lperm_ops, dev)
            self._lperm_span = int(max(len(v[0]) for v in plans.values()))
            self._build_lpan()
        # per-dot R panels (every operator's R blocks permuted), FP64 and FP32
        self.rperm = None
        if rperm:
            self._rperm_h = numpy.concatenate(rperm)
            self.rperm = upload(self._rperm_h, dev)
            rops = op_table(R.offsets[order], 0, R.offsets[order], 1.0)
            self._rperm_ops_d = upload(rops, dev)
            self._rperm_span = int(max(len(v[0]) for v in plans.values()))
            self._build_rpan()
        # the .R contraction on the tensor cores: R panels transposed and split into TF32
        # hi / lo planes once per dot, T3 read raw by TMA and split in the kernel
        self.tc1 = None
        if tc1_classes:
            self._setup_tc1(tc1_classes, order, L, tabs[0])
        self.tc4 = None
        if tc4_classes:
            self._setup_tc4(tc4_classes, order, bases[2], R, st4_ops=tabs[3],
                            crow=numpy.concatenate(crow_all) if crow_all else numpy.zeros(1, numpy.int64))
        # fused W stage (T1 -> T3) and the per-dot two-site MPO blocks it reads
        self.fused = None
        self.wtot = wtot
        if fuse_parts:
            ftab = op_table(bases[0][order], wbase[order], bases[2][order], 1.0)
            self.fused = CompositeStage(fiber_stages(fuse_parts, dev, "sigma23", ftab, fg_budget), "sigma23")
            wst = Stage(wij_parts, dev, "wij", op_table(Wi.offsets[order], Wj.offsets[order], wbase[order], 1.0))
            self.Wij = torch.zeros(max(wtot, 1), dtype=torch.float64, device=dev)
            wst.run(Wi.values, Wj.values, self.Wij, "f64")
            self._Wij32 = None
        # algorithmic bytes per stage (FP64): every operand block read once, output written once
        def stage_bytes(c, t, nop, shared2):
            if len(t) == 0:
                return 0
            u1 = numpy.unique(t[:, 1])
            u2 = numpy.unique(t[:, 2])
            uo = numpy.unique(t[:, 0])
            b1 = c.l1.ndim[u1].sum() * nop
            b2 = c.l2.ndim[u2].sum() * (1 if shared2 else nop)
            bo = c.out.ndim[uo].sum() * nop
            return 8 * (b1 + b2 + bo)

        fb = 0
        for si in range(4 if LOG.enabled else 0):       # only the launch log reads the byte counts
            tot_b = 0
            for key, (ops, *cs, Rl, fused, pan, pan4, fib2, fib3) in sorted(plans.items()):
                if fused is not None and si in (1, 2):
                    continue
                c, t = cs[si]
                tot_b += stage_bytes(c, t, len(ops), si == 0)      # psi is read by every operator
            self.stages[si].bytes = float(tot_b)
        for key, (ops, *cs, Rl, fused, pan, pan4, fib2, fib3) in sorted(plans.items()):
            if fused is not None and LOG.enabled:
                fb += stage_bytes(fused[1], fused[2], len(ops), False)
        if self.fused is not None:
            self.fused.bytes = float(fb)
        if self.tc4 is not None:
            self.tc4.bytes = self.stages[3].bytes
        if self.tc1 is not None:
            self.tc1.bytes = self.stages[0].bytes
        # FLOPs of the reference's four-contraction chain (tensordotCAL pair GEMMs),
        # whatever the fusion used here
        self.flops = 0.0
        for key, (ops, *cs, Rl, fused, pan, pan4, fib2, fib3) in sorted(plans.items()):
            for (c, t) in cs:
                self.flops += pair_flops(c, t) * len(ops)
        self.ndim0 = psi_layout.size
        # W panels of the dense fiber-group stages, gathered now (per dot) rather than in
        # the first matrix-vector product
        if torch.device(dev).type == "cuda":
            s = torch.cuda.current_stream(dev).cuda_stream
            wsets = [(self.stages[1], self.Wi), (self.stages[2], self.Wj)]
            for st, wset in wsets:
                for sub in (st.subs if isinstance(st, CompositeStage) else [st]):
                    if isinstance(sub, FiberStage) and sub.ntasks and sub.fgemm:
                        sub.wpanel(wset.values, s)
                        if precision != "f64":
                            sub.wpanel(wset.f32(), s)

    def rebind(self, L, R):
        """Use new environment values with the same block layouts (cached plan)."""
        if (len(L.layouts) != len(self._lays[0]) or len(R.layouts) != len(self._lays[1])
                or any(a is not b for a, b in zip(L.layouts, self._lays[0]))
                or any(a is not b for a, b in zip(R.layouts, self._lays[1]))):
            raise ValueError("rebind: environment layouts differ from the compiled plan")
        self.L, self.R = L, R
        if self.lperm is not None:
            self._build_lpan()
        if self.rperm is not None:
            self._build_rpan()
        if self.tc4 is not None:
            self._build_rpan_tc()
        if self.tc1 is not None:
            self._build_lpan_tc()

    def _setup_tc4(self, tc4_classes, order, t3bases, R, st4_ops, crow):
        from .engine import TCPanelStage, tc_sigma4_units
        dev = self.ws.device
        classes, t3b, rtb, rts, descs = [], [], [], [], []
        rt_tot = 0
        flops = 0.0
        for (rng, pan4, crow_n) in tc4_classes:
            sec = dict(pan4["sectors"])
            sec["crow_base"] = sec["crow_base"] + crow_n
            ops_c = order[rng[0]:rng[1]]
            t3stride = int(t3bases[ops_c[1]] - t3bases[ops_c[0]]) if len(ops_c) > 1 else \
                (int(pan4["t3size"]) + 31) // 32 * 32
            opstride = (int(pan4["rtsize"]) + 31) // 32 * 32
            classes.append((list(range(rng[0], rng[1])), sec, t3stride))
            t3b.append(int(t3bases[ops_c[0]]))
            rtb.append(rt_tot)
            rts.append(opstride)
            src, dst, dU, kp = pan4["rperm_t"]
            d = numpy.zeros(len(src), BPERM_DT)
            d["src_off"], d["dst_off"] = src, dst
            d["d0"], d["d1"], d["d2"] = dU[:, 0], dU[:, 1], dU[:, 2]
            d["s0"], d["s1"], d["s2"] = 1, kp, dU[:, 0]
            d["op_b"], d["op_e"] = rng
            descs.append(d)
            rt_tot += opstride * len(ops_c)
            flops += 2.0 * float((sec["M"] * sec["N"] * sec["K"]).sum()) * len(ops_c)
        rt_tot = (rt_tot + 31) // 32 * 32
        units, maps = tc_sigma4_units(classes, None, t3b, rtb, rts, rt_tot)
        self.tc4 = TCPanelStage("sigma4", units, maps, st4_ops, crow, flops, dev)
        self._rt_total = rt_tot
        self._rt_descs = numpy.concatenate(descs)
        self._rt_descs_d = upload(self._rt_descs, dev)
        base = numpy.zeros(len(order), dtype=numpy.int64)
        for (poss, sec, _), b0, st in zip(classes, rtb, rts):
            base[poss] = b0 + st * numpy.arange(len(poss))
        self._rt_ops_d = upload(op_table(R.offsets[order], 0, base, 1.0), dev)
        self._rt_span = int(max(len(c[0]) for c in classes))
        self._build_rpan_tc()

    def _setup_tc1(self, tc1_classes, order, L, st1_ops):
        from .engine import TCPanelStage, tc_sigma1_units, psi_panels
        dev = self.ws.device
        gidx, info, cols = psi_panels(self.psi)
        self._psi_total = (len(gidx) + 31) // 32 * 32
        self._psi_gidx = torch.from_numpy(numpy.concatenate(
            [gidx, numpy.full(self._psi_total - len(gidx), -1, dtype=numpy.int64)])).to(dev)
        classes, lpb, lps, descs = [], [], [], []
        tot = 0
        base = numpy.zeros(len(order), dtype=numpy.int64)
        for (rng, tcd) in tc1_classes:
            poss = list(range(rng[0], rng[1]))
            stride = (int(tcd["lpsize"]) + 31) // 32 * 32
            classes.append((poss, tcd))
            lpb.append(tot)
            lps.append(stride)
            base[poss] = tot + stride * numpy.arange(len(poss))
            src, dst, dL, kp = tcd["lperm_t"]
            d = numpy.zeros(len(src), BPERM_DT)
            d["src_off"], d["dst_off"] = src, dst
            d["d0"], d["d1"], d["d2"] = dL[:, 0], dL[:, 1], dL[:, 2]
            d["s0"], d["s1"], d["s2"] = dL[:, 1] * kp, kp, 1
            d["op_b"], d["op_e"] = rng
            descs.append(d)
            tot += stride * len(poss)
        self._lp_total = (tot + 31) // 32 * 32
        units, maps, segs = tc_sigma1_units(classes, info, cols, lpb, lps, self._lp_total, self._psi_total)
        self.tc1 = TCPanelStage("sigma1", units, maps, st1_ops, None, self.stages[0].flops, dev, segs=segs)
        self._lp_descs = numpy.concatenate(descs)
        self._lp_descs_d = upload(self._lp_descs, dev)
        self._lp_ops_d = upload(op_table(L.offsets[order], 0, base, 1.0), dev)
        self._lp_span = int(max(len(c[0]) for c in classes))
        self._build_lpan_tc()

    def _build_lpan_tc(self):
        """L panels of the tensor-core L.psi kernel: [M x Kp] per sector, FP32 hi plane then lo plane."""
        n = self._lp_total
        self.lpan_tc = torch.zeros(2 * max(n, 1), dtype=torch.float32, device=self.ws.device)
        block_permute(self._lp_descs_d, len(self._lp_descs), self._lp_span, self._lp_ops_d, self.L.values,
                      self.lpan_tc)
        tf32_split(self.lpan_tc[:n], self.lpan_tc[n:2 * n])

    def _build_rpan_tc(self):
        """R panels of the tensor-core .R kernel: [D_r' x K_r'] per sector, FP32 hi plane then lo plane."""
        n = self._rt_total
        self.rpan_tc = torch.zeros(2 * max(n, 1), dtype=torch.float32, device=self.ws.device)
        block_permute(self._rt_descs_d, len(self._rt_descs), self._rt_span, self._rt_ops_d, self.R.values,
                      self.rpan_tc)
        tf32_split(self.rpan_tc[:n], self.rpan_tc[n:2 * n])

    def _build_rpan(self):
        self.Rpan = torch.empty(max(self.R.total, 1), dtype=torch.float64, device=self.ws.device)
        block_permute(self.rperm, len(self._rperm_h), self._rperm_span, self._rperm_ops_d, self.R.values,
                      self.Rpan)
        self._Rpan32 = None

    def b4(self, kind):
        """Second operand of the .R contraction (R panels, or R itself without panels)."""
        if self.rperm is not None:
            if kind == "f64":
                return self.Rpan
            if self._Rpan32 is None:
                self._Rpan32 = torch.empty(max(self.R.total, 1), dtype=torch.float32, device=self.ws.device)
                block_permute(self.rperm, len(self._rperm_h), self._rperm_span, self._rperm_ops_d,
                              self.R.values, self._Rpan32)
            return self._Rpan32
        return self.R.values if kind == "f64" else self.R.f32()

    def _build_lpan(self):
        self.Lpan = torch.empty(max(self.L.total, 1), dtype=torch.float64, device=self.ws.device)
        block_permute(self.lperm, len(self._lperm_h), self._lperm_span, self._lperm_ops_d, self.L.values,
                      self.Lpan)
        self._Lpan32 = None

    def lpan32(self):
        if self._Lpan32 is None:
            self._Lpan32 = torch.empty(max(self.L.total, 1), dtype=torch.float32, device=self.ws.device)
            block_permute(self.lperm, len(self._lperm_h), self._lperm_span, self._lperm_ops_d, self.L.values,
                          self._Lpan32)
        return self._Lpan32

    def a1(self, kind):
        """First operand of the L.psi contraction (L panels, or L itself without panels)."""
        if self.lperm is not None:
            return self.Lpan if kind == "f64" else self.lpan32()
        return self.L.values if kind == "f64" else self.L.f32()

    def release(self):
        """Drop the references to the environment values (the plan stays valid)."""
        self.L = self.R = None
        self.Lpan = self._Lpan32 = None
        self.Rpan = self._Rpan32 = None
        self.rpan_tc = None
        self.lpan_tc = None

    def wij32(self):
        if self._Wij32 is None:
            self._Wij32 = self.Wij.to(torch.float32)
        return self._Wij32

    def scratch_bytes(self):
        return 8 * sum(self.tot)

    def check_device_status(self):
        """Raise if a tensor-core launch of this plan gave up a bounded wait (its device
        error flag, qc_tcpanel_status): its output would be incomplete.  Reads one int."""
        if (self.tc1 is not None or self.tc4 is not None) and torch.device(self.ws.device).type == "cuda":
            st = native.lib().qc_tcpanel_status(1)
            if st != 0:
                raise RuntimeError("tensor-core panel kernel: a bounded wait expired (status %d); the sigma of "
                                   "this dot is incomplete" % st)

    def work_groups(self):
        """The plan's device work-item groups in stage order, as the C-ABI's
        qc_sigma_f64_noalloc takes them: (stage, kind, tasks, ntasks, opspan, contribs,
        tile_cfg), kind one of native.GROUP_BGEMM / GROUP_PANEL / GROUP_FIBER.  Groups
        that read the per-dot panels (the tensor-core tiles of a panel stage included)
        are GROUP_PANEL; the fused two-site W stage counts as a fiber group of stage 1."""
        out = []

        def walk(st, si, kind=None):
            if st is None:
                return
            if isinstance(st, CompositeStage):
                for x in st.subs:
                    walk(x, si, kind)
            elif isinstance(st, PanelStage):
                for (cfg, tk, dt, span) in st.groups:
                    out.append((si, native.GROUP_PANEL, dt.data_ptr(), len(tk), span, 0, cfg))
                walk(st.tc, si, native.GROUP_PANEL)
            elif isinstance(st, FiberStage):
                if st.ntasks:
                    out.append((si, native.GROUP_FIBER, st.d[0].data_ptr(), st.ntasks, st.span, 0, 0))
            else:
                for (cfg, tk, ct, dt, dc, span) in st.groups:
                    out.append((si, kind or native.GROUP_BGEMM, dt.data_ptr(), len(tk), span, dc.data_ptr(), cfg))

        for si, st in enumerate(self.stages):
            walk(st, si)
            if si == 1:
                walk(self.fused, 1, native.GROUP_FIBER)
            if si == 3 and self.tc4 is not None:
                out.append((3, native.GROUP_PANEL, self.tc4.d_units.data_ptr(), self.tc4.ntasks, 1, 0, 0))
            if si == 0 and self.tc1 is not None:
                out.append((0, native.GROUP_PANEL, self.tc1.d_units.data_ptr(), self.tc1.ntasks, 1, 0, 0))
        return out

    def __call__(self, x, y=None, precision=None):
        """x: device tensor (ndim0,) float64 -> y = H x (float64).

        precision overrides the operator's precision for this call ("f64" runs the
        same plan, tensor-core tiles included, on the FP64 engine)."""
        ws = self.ws
        prec = precision or self.precision
        if y is None:
            y = torch.empty(self.ndim0, dtype=torch.float64, device=ws.device)
        if prec == "f64":
            T1 = ws.get("t1", self.tot[0], torch.float64)
            T2 = ws.get("t2", self.tot[1], torch.float64)
            T3 = ws.get("t3", self.tot[2], torch.float64)
            P = ws.get("part", self.nops * self.ndim0, torch.float64)
            s = self.stages
            s[0].run(self.a1("f64"), x, T1, "f64")
            s[1].run(T1, self.Wi.values, T2, "f64")
            s[2].run(T2, self.Wj.values, T3, "f64")
            if self.fused is not None:
                self.fused.run(T1, self.Wij, T3, "f64")
            P[:self.nops * self.ndim0].zero_()
            s[3].run(T3, self.b4("f64"), P, "f64")
            return reduce_ops(P, self.nops, self.ndim0, y)
        kind = prec if prec in ("tf32", "tf32x3") else "f32"
        T1 = ws.get("t1", self.tot[0], torch.float32)
        T2 = ws.get("t2", self.tot[1], torch.float32)
        T3 = ws.get("t3", self.tot[2], torch.float32)
        x32 = ws.get("x32", self.ndim0, torch.float32)
        y32 = ws.get("y32", self.ndim0, torch.float32)
        convert(x, x32)
        P = ws.get("part32", self.nops * self.ndim0, torch.float32)
        s = self.stages
        if self.tc1 is not None and kind == "tf32x3":
            pt = ws.get("psiT", 2 * self._psi_total, torch.float32)
            gather_split(x, self._psi_gidx, pt[:self._psi_total], pt[self._psi_total:2 * self._psi_total])
            self.tc1.run(self.lpan_tc, pt, T1)
            if self._s0_generic is not None:
                self._s0_generic.run(self.a1("f32"), x32, T1, "f32")
        else:
            s[0].run(self.a1("f32"), x32, T1, kind)
        s[1].run(T1, self.Wi.f32(), T2, "f32")
        s[2].run(T2, self.Wj.f32(), T3, "f32")
        if self.fused is not None:
            self.fused.run(T1, self.wij32(), T3, "f32")
        P[:self.nops * self.ndim0].zero_()
        if self.tc4 is not None and kind == "tf32x3":
            self.tc4.run(T3, self.rpan_tc, P)
        else:
            s[3].run(T3, self.b4("f32"), P, kind)
        reduce_ops(P, self.nops, self.ndim0, y32)
        convert(y32, y)
        return y


def _dense_tasks(M, N, K, a_off, a_m, a_k, b_off, b_k, b_n, c_off, c_m, alpha, per_group, tile_cfg):
    """Work items for dense GEMMs C_g = sum_{j in group g} alpha_j A_j B_j (vectorised).

    a_off / b_off / alpha are per contribution, grouped consecutively: group g owns
    contributions [g*per_group, (g+1)*per_group) and writes at c_off[g].
    """
    from .engine import TILES
    tm, tn = TILES[tile_cfg]
    a_off = numpy.asarray(a_off, dtype=numpy.int64)
    ncontr = len(a_off)
    contribs = numpy.zeros(ncontr, dtype=CONTRIB_DT)
    contribs["a_off"] = a_off
    contribs["b_off"] = b_off
    contribs["alpha"] = alpha
    contribs["K"] = K
    contribs["klo"] = K
    contribs["a_ml"] = a_m
    contribs["a_kl"] = a_k
    contribs["b_kl"] = b_k
    contribs["b_nl"] = b_n
    contribs["op_b"] = 0
    contribs["op_e"] = 1
    c_off = numpy.asarray(c_off, dtype=numpy.int64)
    ng = len(c_off)
    m0 = numpy.arange(0, M, tm)
    n0 = numpy.arange(0, N, tn)
    nt = len(m0) * len(n0)
    t = numpy.zeros(ng * nt, dtype=TASK_DT)
    g = numpy.repeat(numpy.arange(ng), nt)
    t["c_off"] = c_off[g]
    t["M"], t["N"], t["mlo"], t["nlo"] = M, N, M, N
    t["m0"] = numpy.tile(numpy.repeat(m0, len(n0)), ng)
    t["n0"] = numpy.tile(numpy.tile(n0, len(m0)), ng)
    t["c_ml"], t["c_nl"] = c_m, 1
    t["cb"] = g * per_group
    t["ce"] = g * per_group + per_group
    t["op_b"], t["op_e"] = 0, 1
    return t, contribs, 2.0 * M * N * K * ncontr


_DENSE_STAGES = {}


def _diag_stages(dev, nops, A, Ab, Ac, ldim, rdim, hp):
    """The three dense stages of the diagonal; they depend only on the dimensions (and the
    operator weights), so dots of equal shape share one set of device work lists."""
    key = (str(dev), nops, A, Ab, Ac, ldim, rdim, hp.tobytes())
    hit = _DENSE_STAGES.get(key)
    if hit is not None:
        return hit
    p = numpy.repeat(numpy.arange(nops), 16)
    nm = numpy.tile(numpy.arange(16), nops)
    n, m = nm // 4, nm % 4
    # X[p, n, m, a, c] = sum_b W1[p, a, b, n] W2[p, b, c, m]
    sX = _dense_tasks(A, Ac, Ab, p * A * Ab * 4 + n, Ab * 4, 4, p * Ab * Ac * 4 + m, Ac * 4, 4,
                      (p * 16 + nm) * A * Ac, Ac, 1.0, 1, 0)
    # T[p, nm, c, l] = sum_a X[p, nm, a, c] Ld[p, a, l]
    sT = _dense_tasks(Ac, ldim, A, (p * 16 + nm) * A * Ac, 1, Ac, p * A * ldim, ldim, 1,
                      (p * 16 + nm) * Ac * ldim, ldim, 1.0, 1, 0)
    # D[nm, l, r] = sum_p w_p sum_c T[p, nm, c, l] Rd[p, c, r]   (contributions ordered nm-major)
    nm2 = numpy.repeat(numpy.arange(16), nops)
    p2 = numpy.tile(numpy.arange(nops), 16)
    sD = _dense_tasks(ldim, rdim, Ac, (p2 * 16 + nm2) * Ac * ldim, 1, ldim, p2 * Ac * rdim, rdim, 1,
                      numpy.arange(16) * ldim * rdim, rdim, hp[p2], nops, 0)
    out = (Stage({0: [sX]}, dev, "diagX"), Stage({0: [sT]}, dev, "diagT"), Stage({0: [sD]}, dev, "diagD"))
    if len(_DENSE_STAGES) > 256:
        _DENSE_STAGES.clear()
    _DENSE_STAGES[key] = out
    return out


_DIAG_CACHE = {}


def _cached(key, lay, build):
    hit = _DIAG_CACHE.get(key)
    if hit is not None and hit[0] is lay:
        return hit[1]
    if len(_DIAG_CACHE) > 4096:
        _DIAG_CACHE.clear()
    val = build()
    _DIAG_CACHE[key] = (lay, val)
    return val


def _ragged(n):
    """Block id and in-block position of every element of blocks with n elements each."""
    n = numpy.asarray(n, dtype=numpy.int64)
    b = numpy.repeat(numpy.arange(len(n)), n)
    e = numpy.arange(int(n.sum()), dtype=numpy.int64) - numpy.repeat(numpy.cumsum(n) - n, n)
    return b, e


def _env_diag_map(lay, ncol):
    """Environment E[a, l, l'] -> its diagonal E[a, l, l] as a dense [A x ncol] matrix (src, dst)."""
    def build():
        idx = lay.idx_allowed
        sa, s1, s2 = numpy.unravel_index(idx, tuple(lay.nsyms))
        keep = s1 == s2
        idx, sa, s1 = idx[keep], sa[keep], s1[keep]
        d = lay.block_dims(idx) if len(idx) else numpy.zeros((0, 3), dtype=numpy.int64)
        da, dl = d[:, 0], d[:, 1]
        b, e = _ragged(da * dl)
        w, u = e // dl[b], e % dl[b]
        src = lay.ioff[idx][b] + w * dl[b] * dl[b] + u * dl[b] + u
        dst = (lay.secoff[0][sa][b] + w) * ncol + lay.secoff[1][s1][b] + u
        return src.astype(numpy.int64), dst.astype(numpy.int64)
    return _cached(("e", id(lay), ncol), lay, build)


def _w_diag_map(lay, n2):
    """MPO site operator W[a, b, n, n'] -> its physical diagonal as a dense [A x n2 x 4] array (src, dst)."""
    def build():
        idx = lay.idx_allowed
        sa, sb, n, n_ = numpy.unravel_index(idx, tuple(lay.nsyms))
        keep = n == n_
        idx, sa, sb, n = idx[keep], sa[keep], sb[keep], n[keep]
        d = lay.block_dims(idx) if len(idx) else numpy.zeros((0, 4), dtype=numpy.int64)
        da, db = d[:, 0], d[:, 1]
        b, e = _ragged(da * db)
        w, v = e // db[b], e % db[b]
        src = lay.ioff[idx][b] + w * db[b] + v
        dst = ((lay.secoff[0][sa][b] + w) * n2 + lay.secoff[1][sb][b] + v) * 4 + n[b]
        return src.astype(numpy.int64), dst.astype(numpy.int64)
    return _cached(("w", id(lay), n2), lay, build)


def _psi_diag_gather(ql, ldim, rdim):
    """Packed wavefunction position -> index of the dense [16, ldim, rdim] diagonal
    (qc_psi_diag_gather, host code of the native library)."""
    def build():
        blocks = numpy.ascontiguousarray(ql.idx_allowed, dtype=numpy.int64)
        gat = numpy.empty(max(ql.size, 1), dtype=numpy.int64)
        check(native.lib().qc_psi_diag_gather(len(blocks), native.ptr(blocks), native.ptr(ql.nsyms),
                                              native.ptr(ql.ndims_cat), native.ptr(ql.ioff), ldim, rdim, ql.size,
                                              native.ptr(gat)), "qc_psi_diag_gather")
        return gat[:ql.size]
    return _cached(("p", id(ql), ldim, rdim), ql, build)


class DiagOperator(object):
    """Davidson diagonal in the packed wavefunction layout (HDiagQt, two-site)."""

    def __init__(self, ws, isite, psi_layout, L, R, Wi, Wj, qkey, opers, hpwts):
        dev = ws.device
        self.ws = ws
        nops = len(opers)
        ql = psi_layout
        ldim = int(ql.shape[0])
        rdim = int(ql.shape[3])
        A = int(L.layouts[0].shape[0])
        Ab = int(Wi.layouts[0].shape[1])
        Ac = int(R.layouts[0].shape[0])
        self.dims = (A, Ab, Ac, ldim, rdim)
        # ---- index maps for the diagonal elements (host; cached per interned layout) ----
        Lsrc, Ldst = [], []
        Rsrc, Rdst = [], []
        Wsrc1, Wdst1, Wsrc2, Wdst2 = [], [], [], []
        for i in range(nops):
            s_, d_ = _env_diag_map(L.layouts[i], ldim)
            Lsrc.append(s_ + L.offsets[i])
            Ldst.append(d_ + i * A * ldim)
            s_, d_ = _env_diag_map(R.layouts[i], rdim)
            Rsrc.append(s_ + R.offsets[i])
            Rdst.append(d_ + i * Ac * rdim)
            s_, d_ = _w_diag_map(Wi.layouts[i], Ab)
            Wsrc1.append(s_ + Wi.offsets[i])
            Wdst1.append(d_ + i * A * Ab * 4)
            s_, d_ = _w_diag_map(Wj.layouts[i], Ac)
            Wsrc2.append(s_ + Wj.offsets[i])
            Wdst2.append(d_ + i * Ab * Ac * 4)
        cat = lambda x: torch.from_numpy(numpy.concatenate(x).astype(numpy.int64)).to(dev)
        self.maps = [(cat(Lsrc), cat(Ldst), nops * A * ldim, "ld", L),
                     (cat(Rsrc), cat(Rdst), nops * Ac * rdim, "rd", R),
                     (cat(Wsrc1), cat(Wdst1), nops * A * Ab * 4, "w1", Wi),
                     (cat(Wsrc2), cat(Wdst2), nops * Ab * Ac * 4, "w2", Wj)]
        # ---- packed output gather: psi block (sl, n, m, sr), element (u, v) ----
        gat = _psi_diag_gather(ql, ldim, rdim)
        self.gather = torch.from_numpy(gat).to(dev)
        self.ndim0 = ql.size
        # ---- three dense GEMM stages (shared by dots of equal dimensions) ----
        hp = numpy.asarray(hpwts, dtype=numpy.float64)
        self.sX, self.sT, self.sD = _diag_stages(dev, nops, A, Ab, Ac, ldim, rdim, hp)
        self.nX = nops * 16 * A * Ac
        self.nT = nops * 16 * Ac * ldim
        self.nD = 16 * ldim * rdim
        self.flops = self.sX.flops + self.sT.flops + self.sD.flops

    def rebind(self, L, R):
        """Use new environment values with the same block layouts (cached plan)."""
        sub = {"ld": L, "rd": R}
        self.maps = [(src, dst, n, name, sub[name] if name in sub else tset)
                     for (src, dst, n, name, tset) in self.maps]

    def release(self):
        self.rebind(None, None)

    def __call__(self):
        ws = self.ws
        bufs = {}
        for (src, dst, n, name, tset) in self.maps:
            b = ws.get("diag_" + name, n, torch.float64)
            b[:n].zero_()
            if src.numel():
                b[dst] = tset.values[src]
            bufs[name] = b
        X = ws.get("diag_x", self.nX, torch.float64)
        T = ws.get("diag_t", self.nT, torch.float64)
        D = ws.get("diag_d", self.nD, torch.float64)
        self.sX.run(bufs["w1"], bufs["w2"], X, "f64")
        self.sT.run(X, bufs["ld"], T, "f64")
        self.sD.run(T, bufs["rd"], D, "f64")
        out = torch.empty(self.ndim0, dtype=torch.float64, device=ws.device)
        return gather(D, self.gather, out)


class Renormalizer(object):
    """New environments of every operator after a decimation (renormQt_H00).

    status 'L': L'[b, r, r'] = sum site*[l, n, r] L[a, l, l'] W[a, b, n, n'] site[l', n', r']
    status 'R': the mirror image with W's bond indices flipped (kernelQt.py:723-740).
    """

    def __init__(self, ws, isite, status, site_layout, E, W, opers):
        self.ws, self.status = ws, status
        dev = ws.device
        groups = _groups(opers, isite, 1)
        nops = len(opers)
        if status == "L":
            ax = (([0], [1]), ([0, 2], [2, 0]), ([1, 3], [1, 0]))
        else:
            ax = (([2], [1]), ([1, 2], [2, 1]), ([1, 3], [1, 2]))
        bases = [numpy.zeros(nops, dtype=numpy.int64) for _ in range(3)]
        tot = [0, 0, 0]
        wbase = numpy.zeros(nops, dtype=numpy.int64)
        wtot = 0
        plans = {}
        out_layouts = [None] * nops
        for key, ops in sorted(groups.items()):
            i0 = ops[0]
            El = E.layouts[i0]
            Wl = W.layouts[i0] if status == "L" else flip_horizontal(W.layouts[i0])
            for i in ops:
                if E.layouts[i] is not El or W.layouts[i] is not W.layouts[i0]:
                    raise ValueError("operators of one symmetry class must share their block structure")
            c1 = Contraction(site_layout, El, ax[0])
            t1 = c1.triples
            c2 = Contraction(Wl, c1.out, ax[1])
            t2 = prune(c2.triples, live2=live_blocks(c1.out, t1))
            c3 = Contraction(c2.out, site_layout, ax[2])
            t3 = prune(c3.triples, live1=live_blocks(c2.out, t2))
            plans[key] = (ops, (c1, t1), (c2, t2), (c3, t3))
            for s, c in enumerate((c1, c2, c3)):
                for i in ops:
                    bases[s][i] = tot[s]
                    tot[s] += c.out.size
                    if s == 2:
                        out_layouts[i] = c.out
        self.out_layouts = out_layouts
        self.out_offsets = bases[2].copy()
        self.tot = tot
        order = numpy.concatenate([numpy.array(plans[k][0]) for k in sorted(plans)])
        tabs = [op_table(0, E.offsets[order], bases[0][order], 1.0),
                op_table(W.offsets[order], bases[0][order], bases[1][order], 1.0),
                op_table(bases[1][order], 0, bases[2][order], 1.0)]
        st = [{}, {}, {}]
        pos = 0
        for key, (ops, *cs) in sorted(plans.items()):
            rng = (pos, pos + len(ops))
            pos += len(ops)
            for si, (c, t) in enumerate(cs):
                add_parts(st[si], compile_classes(c, t, ax[si]), op_range=rng)
        self.stages = [Stage(st[si], dev, "renorm%d" % (si + 1), tabs[si]) for si in range(3)]
        self.flops = sum(s.flops for s in self.stages)
        self.E, self.W = E, W

    def __call__(self, site_values):
        """site_values: packed site tensor (float64, device) -> new TensorSet."""
        ws = self.ws
        T1 = ws.get("r1", self.tot[0], torch.float64)
        T2 = ws.get("r2", self.tot[1], torch.float64)
        out = torch.zeros(max(self.tot[2], 1), dtype=torch.float64, device=ws.device)
        s = self.stages
        s[0].run(site_values, self.E.values, T1, "f64")
        s[1].run(self.W.values, T1, T2, "f64")
        s[2].run(T2, site_values, out, "f64")
        return TensorSet(self.out_layouts, out, self.out_offsets)


class NoiseRDM(object):
    """Noise term of the decimation's density matrix (pRDMQt with noise > 0).

    status 'L' (source/mpo_dmrg_kernelQt.py:488-531): with psi as [l, n1, X]
    (X = (n2, r) merged), T2_p[l, X, b, n1'] = sum W_p[a, b, n1', n1] L_p[a, l, l'] psi[l', n1, X]
    and rho[l n1', l' n1''] = sum_p sum_{X, b} T2_p T2_p.
    status 'R' (:568-611): with psi as [Y, n2, r] (Y = (l, n1) merged) and R_p flipped,
    T2_p[a, n2', Y, r'] and rho[n2' r', n2'' r''] = sum_p sum_{a, Y} T2_p T2_p.
    Three grouped-GEMM launches over all operators (per-operator Gram blocks), one
    fixed-order sum over operators, and a scatter into the dense matrix the
    decimation uses.  ``psi_layout`` is the rank-3 wavefunction layout (N-reduced
    with spin projection, with qkey[:1] then).
    """

    def __init__(self, ws, isite, status, psi_layout, E, W, opers, qkey, dense_idl):
        self.ws, self.status = ws, status
        dev = ws.device
        groups = _groups(opers, isite, 1)
        nops = len(opers)
        if status == "L":
            ax = (([2], [0]), ([0, 2], [0, 3]), ([1, 2], [1, 2]))
        else:
            ax = (([2], [2]), ([1, 3], [2, 1]), ([0, 2], [0, 2]))
        bases = [numpy.zeros(nops, dtype=numpy.int64) for _ in range(2)]
        tot = [0, 0]
        plans = {}
        out = None
        for key, ops in sorted(groups.items()):
            i0 = ops[0]
            El, Wl = E.layouts[i0], W.layouts[i0]
            for i in ops:
                if E.layouts[i] is not El or W.layouts[i] is not Wl:
                    raise ValueError("operators of one symmetry class must share their block structure")
            if status == "L":
                c1 = Contraction(El, psi_layout, ax[0])
                t1 = c1.triples
                c2 = Contraction(c1.out, Wl, ax[1])
                t2 = prune(c2.triples, live1=live_blocks(c1.out, t1))
            else:
                Rl = _flip_right_ket(El, qkey)
                c1 = Contraction(psi_layout, Rl, ax[0])
                t1 = c1.triples
                c2 = Contraction(Wl, c1.out, ax[1])
                t2 = prune(c2.triples, live2=live_blocks(c1.out, t1))
            c3 = Contraction(c2.out, c2.out, ax[2])
            live2 = live_blocks(c2.out, t2)
            t3 = prune(c3.triples, live1=live2, live2=live2)
            if out is None:
                out = c3.out
            elif c3.out is not out:
                raise ValueError("noise RDM blocks differ between operator classes")
            plans[key] = (ops, (c1, t1), (c2, t2), (c3, t3))
            for s, c in enumerate((c1, c2)):
                for i in ops:
                    bases[s][i] = tot[s]
                    tot[s] += c.out.size
        self.out_layout = out
        self.tot = tot
        self.nops = nops
        self.size = out.size if out is not None else 0
        order = numpy.concatenate([numpy.array(plans[k][0]) for k in sorted(plans)])
        slot = numpy.arange(nops, dtype=numpy.int64) * self.size
        if status == "L":
            t0 = op_table(E.offsets[order], 0, bases[0][order], 1.0)
            t1_ = op_table(bases[0][order], W.offsets[order], bases[1][order], 1.0)
        else:
            t0 = op_table(0, E.offsets[order], bases[0][order], 1.0)
            t1_ = op_table(W.offsets[order], bases[0][order], bases[1][order], 1.0)
        tabs = [t0, t1_, op_table(bases[1][order], bases[1][order], slot, 1.0)]
        st = [{}, {}, {}]
        pos = 0
        for key, (ops, *cs) in sorted(plans.items()):
            rng = (pos, pos + len(ops))
            pos += len(ops)
            for si, (c, t) in enumerate(cs):
                add_parts(st[si], compile_classes(c, t, ax[si]), op_range=rng)
        self.stages = [Stage(st[si], dev, "prdm%d" % (si + 1), tabs[si]) for si in range(3)]
        self.flops = sum(s.flops for s in self.stages)
        self.E, self.W = E, W
        n = int(numpy.prod(out.shape)) if out is not None else 0
        self.dense_shape = tuple(int(x) for x in out.shape) if out is not None else (0,)
        self.prj = torch.from_numpy(out.prjmap(dense_idl)).to(dev) if out is not None else None
        self.ndense = n

    def __call__(self, psi_values):
        """psi_values: packed rank-3 wavefunction (device FP64) -> dense noise RDM (d x d)."""
        ws = self.ws
        T1 = ws.get("n1", self.tot[0], torch.float64)
        T2 = ws.get("n2", self.tot[1], torch.float64)
        P = ws.get("npart", self.nops * self.size, torch.float64)
        s = self.stages
        if self.status == "L":
            s[0].run(self.E.values, psi_values, T1, "f64")
            s[1].run(T1, self.W.values, T2, "f64")
        else:
            s[0].run(psi_values, self.E.values, T1, "f64")
            s[1].run(self.W.values, T1, T2, "f64")
        P[:self.nops * self.size].zero_()
        s[2].run(T2, T2, P, "f64")
        vals = torch.empty(max(self.size, 1), dtype=torch.float64, device=ws.device)[:self.size]
        reduce_ops(P, self.nops, self.size, vals)
        dense = torch.empty(self.ndense, dtype=torch.float64, device=ws.device)
        scatter(vals, self.prj, dense)
        d = self.dense_shape
        return dense.reshape(d[0] * d[1], d[2] * d[3])


def _flip_right_ket(lay, qkey):
    """R environment as pRDMQt 'R' contracts it with the wavefunction's right index
    (kernelQt.py:592-598): qsyms [-q0, -(qkey - q1), qkey - q2], index 1 flipped in/out."""
    st = lay.status.copy()
    st[1] = not st[1]
    qkey = numpy.asarray(qkey, dtype=numpy.float64)
    return Layout(st, [-lay.qsyms[0], -(qkey - lay.qsyms[1]), qkey - lay.qsyms[2]], lay.ndims)
