"""Many independent DMRG calculations in lockstep (no counterpart in the reference,
which runs one Hamiltonian per process).

Every instance sweeps its own chain with its own Davidson; at each Davidson step
the pending matrix-vector products of all instances are executed together: one
launch per sigma contraction and tile configuration for all instances.  The
instances' work lists are concatenated and their operator tables rewritten to
absolute element addresses (every buffer is element-aligned), so the kernels run
with null base pointers.  The combined launch sequence is captured in a CUDA
graph and replayed while no instance changes dot.
"""
import numpy
import torch

from . import native
from .native import check
from .engine import OP_DT, TASK_DT, CONTRIB_DT, TC_CFG, LOG, FiberStage, CompositeStage, PanelStage


def _abs_ops(ops, a, b, c):
    """Operator table with bases turned into absolute element addresses."""
    t = ops.copy()
    el = a.element_size()
    for name, buf in (("a_base", a), ("b_base", b), ("c_base", c)):
        ptr = buf.data_ptr()
        assert ptr % el == 0
        t[name] += ptr // el
    return t


class BatchedSigma(object):
    """sigma for several (SigmaOperator, input, output) triples in one launch per stage group."""

    def __init__(self, items, device, kind="f64", ws=None):
        """ws: optional dict of grow-only scratch buffers shared by the batches of one run
        (one batch is live at a time); without it every batch allocates its own."""
        self.device = device
        self.kind = kind
        dt = torch.float64 if kind == "f64" else torch.float32

        def buf(name, n):
            if ws is None:
                return torch.zeros(n, dtype=dt, device=device)
            b = ws.get((name, dt))
            if b is None or b.numel() < n:
                ws.pop((name, dt), None)
                b = torch.empty(max(int(n), 1) + 64, dtype=dt, device=device)
                ws[(name, dt)] = b
            return b
        self.dtype = dt
        self.items = items
        n = len(items)
        # per-instance scratch regions in one buffer per intermediate
        tot = numpy.array([[s.tot[0], s.tot[1], s.tot[2], s.nops * s.ndim0] for s in items], dtype=numpy.int64)
        pad = lambda v: ((v + 63) // 64) * 64
        offs = numpy.zeros((n, 4), dtype=numpy.int64)
        sizes = []
        for k in range(4):
            o = 0
            for i in range(n):
                offs[i, k] = o
                o += pad(int(tot[i, k]) + 1)
            sizes.append(o)
        self.T = [buf("t%d" % k, sizes[k]) for k in range(4)]
        nd = [s.ndim0 for s in items]
        self.xoff = numpy.concatenate([[0], numpy.cumsum([pad(v + 1) for v in nd])])
        self.X = buf("x", int(self.xoff[-1]))
        self.Y = buf("y", int(self.xoff[-1]))
        self.offs = offs
        groups = {}
        fibers = {}
        panels = {}
        ops_all = [[], [], [], [], []]
        nops_acc = [0, 0, 0, 0, 0]
        for i, s in enumerate(items):
            L = s.a1("f64" if kind == "f64" else "f32")      # L panels of the L.psi contraction
            R = s.b4("f64" if kind == "f64" else "f32")      # R panels of the .R contraction
            Wi = s.Wi.values if kind == "f64" else s.Wi.f32()
            Wj = s.Wj.values if kind == "f64" else s.Wj.f32()
            T1 = self.T[0][int(offs[i, 0]):]
            T2 = self.T[1][int(offs[i, 1]):]
            T3 = self.T[2][int(offs[i, 2]):]
            P = self.T[3][int(offs[i, 3]):]
            x = self.X[int(self.xoff[i]):]
            abc = [(L, x, T1), (T1, Wi, T2), (T2, Wj, T3), (T3, R, P)]
            stages = list(s.stages)
            if s.fused is not None:         # slot 4: fused W stage, T1 -> T3
                abc.append((T1, s.Wij if kind == "f64" else s.wij32(), T3))
                stages.append(s.fused)
            for si, st in enumerate(stages):
                ops = _abs_ops(st.host_ops, *abc[si])
                base = nops_acc[si]
                nops_acc[si] += len(ops)
                ops_all[si].append(ops)
                for sub in (st.subs if isinstance(st, CompositeStage) else [st]):
                    if isinstance(sub, FiberStage):
                        if sub.ntasks:
                            fibers.setdefault((si, sub.tile), []).append((sub, base))
                        continue
                    if isinstance(sub, PanelStage):
                        if sub.tc is not None:      # tensor-core panel tiles: grouped-GEMM work items
                            for (cfg, tk, ct) in sub.tc.host_groups:
                                tk = tk.copy()
                                tk["op_b"] += base
                                tk["op_e"] += base
                                groups.setdefault((si, cfg), []).append((tk, ct))
                        for (cfg, tk, _, _) in sub.groups:
                            tk = tk.copy()
                            tk["op_b"] += base
                            tk["op_e"] += base
                            panels.setdefault((si, cfg), []).append((tk, sub.h_crow))
                        continue
                    for (cfg, tk, ct) in sub.host_groups:
                        tk = tk.copy()
                        tk["op_b"] += base
                        tk["op_e"] += base
                        groups.setdefault((si, cfg), []).append((tk, ct))
        self.d_ops = [torch.from_numpy(numpy.concatenate(o).view(numpy.uint8).copy()).to(device) if o else None
                      for o in ops_all]
        self.launches = []
        for (si, cfg), parts in sorted(groups.items()):
            nc = 0
            tks, cts = [], []
            for tk, ct in parts:
                tk = tk.copy()
                tk["cb"] += nc
                tk["ce"] += nc
                nc += len(ct)
                tks.append(tk)
                cts.append(ct)
            tk = numpy.concatenate(tks)
            ct = numpy.concatenate(cts)
            span = int(max(1, (tk["op_e"] - tk["op_b"]).max()))
            self.launches.append((si, cfg, len(tk), span, torch.from_numpy(tk.view(numpy.uint8).copy()).to(device),
                                  torch.from_numpy(ct.view(numpy.uint8).copy()).to(device)))
        # fiber-group work items of all instances, one launch per W contraction
        up = lambda a: torch.from_numpy(a.view(numpy.uint8).copy()).to(device)
        self.fiber_launches = []
        for (si, tile), parts in sorted(fibers.items()):
            tks, fis, fos, fps = [], [], [], []
            nin = nout = npair = 0
            mr = 1
            for sub, base in parts:
                tk = sub.h_tasks.copy()
                fo = sub.h_fout.copy()
                tk["in_b"] += nin
                tk["in_e"] += nin
                tk["out_b"] += nout
                tk["out_e"] += nout
                tk["op_b"] += base
                tk["op_e"] += base
                fo["pair_b"] += npair
                fo["pair_e"] += npair
                tks.append(tk)
                fis.append(sub.h_fin)
                fos.append(fo)
                fps.append(sub.h_fpair)
                nin += len(sub.h_fin)
                nout += len(fo)
                npair += len(sub.h_fpair)
                mr = max(mr, sub.max_rows)
            tk = numpy.concatenate(tks)
            span = int(max(1, (tk["op_e"] - tk["op_b"]).max()))
            self.fiber_launches.append((si, len(tk), span, mr, tile, up(tk), up(numpy.concatenate(fis)),
                                        up(numpy.concatenate(fos)), up(numpy.concatenate(fps))))
        self.panel_launches = []
        for (si, cfg), parts in sorted(panels.items()):
            tks, crows, nrow = [], [], 0
            for tk, crow in parts:          # row tables concatenated, task indices rebased
                tk = tk.copy()
                tk["crow"] = numpy.where(tk["crow"] >= 0, tk["crow"] + nrow, -1)
                tks.append(tk)
                crows.append(crow)
                nrow += len(crow)
            tk = numpy.concatenate(tks)
            span = int(max(1, (tk["op_e"] - tk["op_b"]).max()))
            crow = torch.from_numpy(numpy.concatenate(crows).astype(numpy.int64)).to(device)
            self.panel_launches.append((si, cfg, len(tk), span, up(tk), crow))
        self.graph = None

    def _launch_all(self):
        lib = native.lib()
        s = torch.cuda.current_stream(self.device).cuda_stream
        self.T[3].zero_()
        ffn = lib.qc_fiber_f64 if self.kind == "f64" else lib.qc_fiber_f32
        pfn = lib.qc_pgemm_f64 if self.kind == "f64" else lib.qc_pgemm_f32
        for stage in (0, 1, 2, 4, 3):       # contractions in dependency order (4: fused W stage)
            for (si, cfg, nt, span, dt, crow) in self.panel_launches:
                if si != stage:
                    continue
                check(pfn(dt.data_ptr(), nt, span, self.d_ops[si].data_ptr(), crow.data_ptr(), None, None, None, cfg,
                          s), "batched qc_pgemm")
                LOG.launches += 1
            for (si, nt, span, mr, tile, dt, dfi, dfo, dfp) in self.fiber_launches:
                if si != stage:
                    continue
                check(ffn(dt.data_ptr(), nt, span, dfi.data_ptr(), dfo.data_ptr(), dfp.data_ptr(),
                          self.d_ops[si].data_ptr(), mr, tile, None, None, None, s), "batched qc_fiber")
                LOG.launches += 1
            for (si, cfg, nt, span, dt, dc) in self.launches:
                if si != stage:
                    continue
                if self.kind == "f64":
                    fn = lib.qc_bgemm_f64
                elif self.kind == "tf32" and cfg == TC_CFG and si in (0, 3):
                    fn = lib.qc_bgemm_tf32
                else:
                    fn = lib.qc_bgemm_f32
                check(fn(dt.data_ptr(), nt, span, dc.data_ptr(), self.d_ops[si].data_ptr(), 0, None, None, None, cfg,
                         s), "batched qc_bgemm")
                LOG.launches += 1
        red = lib.qc_reduce_ops_f64 if self.kind == "f64" else lib.qc_reduce_ops_f32
        for i, it in enumerate(self.items):
            P = self.T[3][int(self.offs[i, 3]):]
            y = self.Y[int(self.xoff[i]):]
            check(red(P.data_ptr(), it.nops, it.ndim0, y.data_ptr(), s), "batched reduce")
            LOG.launches += 1

    def capture(self):
        """Capture the launch sequence in a CUDA graph (inputs/outputs are the static X / Y);
        the launches run once directly first (the warm-up capture needs)."""
        self._launch_all()
        torch.cuda.synchronize(self.device)
        self._capture()

    def _capture(self):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._launch_all()
        self.graph = g

    def __call__(self, xs, graph_after=None):
        """graph_after: capture the launch sequence once the batch has run this many times
        directly (the direct runs are the capture's warm-up), then replay it; None: never."""
        for i, x in enumerate(xs):
            if x is not None:
                self.X[int(self.xoff[i]):int(self.xoff[i]) + x.numel()].copy_(x)
        self.calls = getattr(self, "calls", 0) + 1
        if self.graph is None and graph_after is not None and self.calls > graph_after:
            torch.cuda.synchronize(self.device)
            self._capture()
            self.captured = True
        if self.graph is not None:
            self.graph.replay()
        else:
            self._launch_all()
        out = []
        for i, it in enumerate(self.items):
            y = self.Y[int(self.xoff[i]):int(self.xoff[i]) + it.ndim0]
            out.append(y.to(torch.float64).clone())
        return out


class BatchedDMRG(object):
    """Lockstep two-site sweeps of independent DMRG instances (FP64 Davidson each)."""

    def __init__(self, instances, kind="f64", use_graphs=True):
        self.inst = instances
        self.kind = kind
        self.use_graphs = use_graphs
        self.device = instances[0].device
        self.steps = 0
        self.captures = 0
        self.ws = {}              # scratch shared by the run's batches

    def sweep(self, status, dmax, crit_e):
        """One sweep of every instance; dmax is one bond dimension or one per instance."""
        n = len(self.inst)
        dmaxs = list(dmax) if isinstance(dmax, (list, tuple)) else [dmax] * n
        acts = []
        for d in self.inst:
            K = d.nsite
            acts.append(list(range(0, K - 1)) if status == "L" else list(range(K - 2, -1, -1)))
        pos = [0] * n
        ctx = [None] * n
        pend = [None] * n
        elst = [[] for _ in range(n)]
        dlst = [[] for _ in range(n)]
        last = [None] * n
        batch = None
        while True:
            changed = False
            for i, d in enumerate(self.inst):
                while ctx[i] is None and pos[i] < len(acts[i]):
                    ctx[i] = d.dot_begin(acts[i][pos[i]], crit_e)
                    pend[i] = next(ctx[i]["gen"])
                    changed = True
            active = [i for i in range(n) if ctx[i] is not None]
            if not active:
                break
            if changed or batch is None or active != batch_ids:
                items = [ctx[i]["sig"] for i in active]
                batch = None                      # the previous batch's graph goes before its buffers move
                batch = BatchedSigma(items, self.device, self.kind, self.ws)
                batch_ids = active
            xs = [pend[i] if ctx[i] is not None else None for i in batch_ids]
            # a batch runs directly the first time and is captured in a CUDA graph when it is
            # used again (most batches live one step: an instance moves to its next dot)
            had = batch.graph is not None
            ys = batch(xs, graph_after=1 if self.use_graphs else None)
            if batch.graph is not None and not had:
                self.captures += 1
            self.steps += 1
            for k, i in enumerate(batch_ids):
                if ctx[i] is None:
                    continue
                try:
                    pend[i] = ctx[i]["gen"].send(ys[k])
                except StopIteration as stop:
                    res = stop.value
                    last[i] = self.inst[i].dot_end(ctx[i], res, status, dmaxs[i], acts[i], elst[i], dlst[i])
                    ctx[i] = None
                    pos[i] += 1
        out = []
        for i, d in enumerate(self.inst):
            qred, srotR = last[i]
            d.boundary(status, qred, srotR)
            j = int(numpy.argmin(elst[i]))
            out.append((elst[i][j], dlst[i][j], elst[i], dlst[i]))
        return out
