"""Device execution of block-pair contraction stages.

A *stage* is one contraction (one tensordotSYM/tensordotCAL pair of the
reference) applied to every operator at once: its block-pair lists are
compiled into GPU work items (one task per output tile, one contribution per
block pair) by the native plan compiler and executed by one launch of the
grouped block GEMM (qc_bgemm_*).  Plans are built once per dot and reused for
every Davidson iteration.
"""
import numpy
import torch

from . import native
from .native import ptr, check
from .qtensor import Contraction

TASK_DT = numpy.dtype([("c_off", "<i8"), ("M", "<i4"), ("N", "<i4"), ("m0", "<i4"), ("n0", "<i4"),
                       ("mlo", "<i4"), ("nlo", "<i4"), ("c_mh", "<i4"), ("c_ml", "<i4"), ("c_nh", "<i4"),
                       ("c_nl", "<i4"), ("cb", "<i4"), ("ce", "<i4"), ("op_b", "<i4"), ("op_e", "<i4")])
CONTRIB_DT = numpy.dtype([("a_off", "<i8"), ("b_off", "<i8"), ("alpha", "<f8"), ("K", "<i4"), ("klo", "<i4"),
                          ("a_mh", "<i4"), ("a_ml", "<i4"), ("a_kh", "<i4"), ("a_kl", "<i4"), ("b_kh", "<i4"),
                          ("b_kl", "<i4"), ("b_nh", "<i4"), ("b_nl", "<i4"), ("op_b", "<i4"), ("op_e", "<i4"),
                          ("pad2", "<i4"), ("pad3", "<i4")])
OP_DT = numpy.dtype([("a_base", "<i8"), ("b_base", "<i8"), ("c_base", "<i8"), ("alpha", "<f8")])
assert TASK_DT.itemsize == native.TASK_BYTES and CONTRIB_DT.itemsize == native.CONTRIB_BYTES
assert OP_DT.itemsize == native.OP_BYTES

TILES = {0: (64, 64), 1: (128, 32), 2: (256, 16), 3: (32, 32), 4: (64, 16), 5: (128, 64)}
TC_CFG = 5      # output tile of the tensor-core kernel (qc_bgemm_tf32)


def tile_class(M, N):
    """Output-tile configuration for output blocks of extent M x N (vectorised)."""
    M = numpy.asarray(M)
    N = numpy.asarray(N)
    return numpy.where(N <= 16, numpy.where(M <= 64, 4, 2),
                       numpy.where(N <= 32, numpy.where(M <= 32, 3, 1), numpy.where(M <= 32, 3, 0)))


def tile_class_tc(M, N, K):
    """Tensor-core tiles for output blocks that fill a useful part of a 128 x 64 tile."""
    base = tile_class(M, N)
    return numpy.where((numpy.asarray(M) > 64) & (numpy.asarray(N) > 24) & (numpy.asarray(K) >= 16), TC_CFG, base)


def compile_classes(c, triples, axes, tensor_cores=False, off1=None):
    """Compile one contraction's pair list, binned by output-block shape into tile classes.

    Returns {tile_cfg: (tasks, contribs, flops)} for a single operator (template).
    tensor_cores: route large output blocks to the tcgen05 tile class (TC_CFG);
    tensor_cores == "all" routes every block there (tests).
    """
    out = {}
    if len(triples) == 0:
        return out
    ne1 = c.l1.rank - len(axes[0])
    d = c.out.block_dims(triples[:, 0])
    M = numpy.prod(d[:, :ne1], axis=1)
    N = numpy.prod(d[:, ne1:], axis=1)
    if tensor_cores == "all":
        cls = numpy.full(len(M), TC_CFG)
    elif tensor_cores:
        d1 = c.l1.block_dims(triples[:, 1])
        K = numpy.prod(d1[:, axes[0]], axis=1)
        # every pair of one output block must land in the same class
        cls = tile_class_tc(M, N, K)
        ob = triples[:, 0]
        first = numpy.unique(ob, return_index=True)[1]
        cmap = dict(zip(ob[first].tolist(), cls[first].tolist()))
        cls = numpy.array([cmap[x] for x in ob.tolist()])
    else:
        cls = tile_class(M, N)
    for k in numpy.unique(cls):
        sel = triples[cls == k]
        out[int(k)] = compile_template(c.l1, c.l2, c.out, axes, sel, int(k), off1=off1)
    return out


def panel_sigma1(Ll, psi, t1, nblks_out):
    """Panel form of the L.psi contraction (HVecQt top1, kernelQt.py:301).

    Every T1 block (a, l, n1, n2, r) is the product of exactly one L block
    (a, l, l') and one psi block (l', n1, n2, r).  For a fixed contracted sector l'
    the L blocks (a, l, l') are stacked into one panel [M_l' x D_l'] (a per-dot
    block permutation of L), so each psi block j gives one GEMM
    T1panel_j [M_l' x N_j] = Lpanel_l' . psi_j with a long M extent.  T1 blocks
    keep their row-major storage inside the panel rows.

    Returns None if the pair list is not the full product per sector, else a
    dict with the L permutation (src/dst offsets of L blocks), the T1 block
    offsets (by flat T1 block index, for the consumers of T1), the T1 size and
    the per-panel GEMM descriptions.
    """
    if len(t1) == 0:
        return None
    ob, iL, ip = t1[:, 0], t1[:, 1], t1[:, 2]
    if len(numpy.unique(ob)) != len(ob):
        return None
    uL = numpy.unique(iL)
    dL = Ll.block_dims(uL)
    lkL = Ll.block_sectors(uL)[2]
    oL = numpy.lexsort((uL, lkL))
    uL, dL, lkL = uL[oL], dL[oL], lkL[oL]
    Mb = dL[:, 0] * dL[:, 1]
    Dk = dL[:, 2]
    nsec = int(Ll.nsyms[2])
    M_lk = numpy.bincount(lkL, weights=Mb, minlength=nsec).astype(numpy.int64)
    cnt_lk = numpy.bincount(lkL, minlength=nsec)
    start = numpy.searchsorted(lkL, numpy.arange(nsec))
    cs = numpy.cumsum(Mb) - Mb
    rowoff = cs - cs[numpy.minimum(start[lkL], len(cs) - 1)]
    Dk_sec = numpy.zeros(nsec, dtype=numpy.int64)
    Dk_sec[lkL] = Dk
    pan_size = M_lk * Dk_sec
    pan_off = numpy.cumsum(pan_size) - pan_size
    lperm_src = Ll.ioff[uL]
    lperm_dst = pan_off[lkL] + rowoff * Dk
    lperm_n = Mb * Dk
    # psi blocks: every one pairs with all L blocks of its sector
    up = numpy.unique(ip)
    lkp = psi.block_sectors(up)[0]
    npair_expect = int(cnt_lk[lkp].sum())
    if npair_expect != len(t1):
        return None
    dp = psi.block_dims(up)
    Nj = numpy.prod(dp[:, 1:], axis=1)
    Mj = M_lk[lkp]
    Kj = Dk_sec[lkp]
    if numpy.any(Kj != dp[:, 0]):
        return None
    psz = Mj * Nj
    t1pan = numpy.cumsum(psz) - psz
    # T1 block offsets
    posL = numpy.empty(int(Ll.nblks), dtype=numpy.int64)
    posL[uL] = numpy.arange(len(uL))
    posP = numpy.empty(int(psi.nblks), dtype=numpy.int64)
    posP[up] = numpy.arange(len(up))
    t1off = numpy.zeros(int(nblks_out), dtype=numpy.int64)
    t1off[ob] = t1pan[posP[ip]] + rowoff[posL[iL]] * Nj[posP[ip]]
    # tensor-core form: the L panels with rows padded to Kp (16-byte stride), [M x Kp] per sector
    Kp_sec = (Dk_sec + 3) // 4 * 4
    tsz = M_lk * Kp_sec
    tpoff = numpy.cumsum(tsz) - tsz
    secs = numpy.unique(lkp)
    tc = {"sectors": secs, "M": M_lk[secs], "K": Dk_sec[secs], "Kp": Kp_sec[secs], "lpoff": tpoff[secs],
          "lpsize": int(tsz.sum()), "lperm_t": (lperm_src, tpoff[lkL] + rowoff * Kp_sec[lkL], dL, Kp_sec[lkL]),
          "blocks": up, "t1pan": t1pan, "Nj": Nj}
    return {"lperm": (lperm_src, lperm_dst, lperm_n), "t1off": t1off, "t1size": int(psz.sum()),
            "gemm": (pan_off[lkp], psi.ioff[up], t1pan, Mj, Nj, Kj), "tc": tc}


def panel_sigma4(t3lay, Rl, psi, t4):
    """Panel form of the .R contraction (HVecQt top4, kernelQt.py:306-316).

    sigma block s = (l, n1', n2', r') receives T3 blocks (l, r, n1', c, n2') times
    R blocks (c, r', r) over the MPO sectors c (r follows from c and r').  For one
    sector r' all sigma blocks use the same R blocks, so: the R blocks of r' form
    one row-major panel [K_r' x D_r'] (a per-dot permutation of R with the (c, r)
    rows transposed); the T3 blocks of every sigma block of r' are written (by the
    fiber kernel) as row block x column slab of one row-major panel
    [M_r' x K_r'] (rows: the sigma blocks stacked, D_l rows each; columns: the
    (c, r, c) slabs in R-panel order); and one dense GEMM per sector and operator
    writes its rows straight into the sigma blocks through a row table.  Returns
    None unless every sigma block pairs with all R blocks of its sector.
    """
    if len(t4) == 0:
        return None
    so, i3, iR = t4[:, 0], t4[:, 1], t4[:, 2]
    if len(numpy.unique(i3)) != len(i3):
        return None
    secR = Rl.block_sectors(iR)
    cR, rbR = secR[0], secR[1]
    o = numpy.lexsort((cR, so))
    so, i3, iR, cR, rbR = so[o], i3[o], iR[o], cR[o], rbR[o]
    dR = Rl.block_dims(iR)                   # (Dc, Drb, Dr)
    kb = dR[:, 0] * dR[:, 2]                 # K extent of the pair
    # R panels per r' sector: all R blocks of the sector, ordered by c
    uR = numpy.unique(iR)
    sR = Rl.block_sectors(uR)
    oR = numpy.lexsort((sR[0], sR[1]))
    uR = uR[oR]
    rbU = sR[1][oR]
    dU = Rl.block_dims(uR)
    kU = dU[:, 0] * dU[:, 2]
    nrb = int(Rl.nsyms[1])
    Krb = numpy.bincount(rbU, weights=kU, minlength=nrb).astype(numpy.int64)
    Drb_sec = numpy.zeros(nrb, dtype=numpy.int64)
    Drb_sec[rbU] = dU[:, 1]
    start = numpy.searchsorted(rbU, numpy.arange(nrb))
    ck = numpy.cumsum(kU) - kU
    koffU = ck - ck[numpy.minimum(start[rbU], len(ck) - 1)]
    psz = Krb * Drb_sec
    poff = numpy.cumsum(psz) - psz
    # every sigma block uses all R blocks of its sector, in the same order
    us, first = numpy.unique(so, return_index=True)
    rb_s = rbR[first]
    cnt = numpy.diff(numpy.r_[first, len(so)])
    if not numpy.array_equal(cnt, numpy.bincount(rbU, minlength=nrb)[rb_s]):
        return None
    posU = numpy.empty(int(Rl.nblks), dtype=numpy.int64)
    posU[uR] = numpy.arange(len(uR))
    ckb = numpy.cumsum(kb) - kb
    if numpy.any(koffU[posU[iR]] != ckb - numpy.repeat(ckb[first], cnt)):
        return None
    # sigma blocks stacked per r' sector
    dS = psi.block_dims(us)
    Dl = dS[:, 0] * dS[:, 1] * dS[:, 2]
    if numpy.any(dS[:, 3] != Drb_sec[rb_s]):
        return None
    os_ = numpy.lexsort((us, rb_s))
    us, Dl, rb_s = us[os_], Dl[os_], rb_s[os_]
    crs = numpy.cumsum(Dl) - Dl
    sstart = numpy.searchsorted(rb_s, numpy.arange(nrb))
    rowoff = crs - crs[numpy.minimum(sstart[rb_s], len(crs) - 1)]
    Mrb = numpy.bincount(rb_s, weights=Dl, minlength=nrb).astype(numpy.int64)
    used = numpy.flatnonzero(Mrb > 0)
    # T3 panel rows padded to a multiple of 4 elements: 16-byte row stride (tensor-map rule)
    Kp = (Krb + 3) // 4 * 4
    tsz = Mrb * Kp
    t3pan = numpy.cumsum(tsz) - tsz
    # T3 block -> (panel of its r', row block of its sigma block, column slab of its c)
    spos_by_blk = dict(zip(us.tolist(), range(len(us))))
    sidx = numpy.array([spos_by_blk[x] for x in so.tolist()], dtype=numpy.int64)
    t3off = numpy.zeros(int(t3lay.nblks), dtype=numpy.int64)
    t3fhs = numpy.zeros(int(t3lay.nblks), dtype=numpy.int64)
    t3flo = numpy.ones(int(t3lay.nblks), dtype=numpy.int64)
    t3off[i3] = t3pan[rbR] + rowoff[sidx] * Kp[rbR] + koffU[posU[iR]]
    t3fhs[i3] = Kp[rbR]
    t3flo[i3] = dR[:, 2]                     # fibers (l, r): r is the fast fiber index
    # row table: panel row -> element offset of that row in its sigma block
    crow = numpy.concatenate([psi.ioff[us] [k] + numpy.arange(Dl[k]) * Drb_sec[rb_s[k]] for k in range(len(us))]) \
        if len(us) else numpy.zeros(0, dtype=numpy.int64)
    crow_base = numpy.zeros(nrb, dtype=numpy.int64)
    crow_base[used] = (numpy.cumsum(Mrb) - Mrb)[used]
    rperm = (Rl.ioff[uR], poff[rbU] + koffU * dU[:, 1], dU)
    gemm = (t3pan[used], poff[used], numpy.zeros(len(used), dtype=numpy.int64), Mrb[used], Drb_sec[used],
            Krb[used], crow_base[used], Kp[used])
    # the R panels transposed ([D_r' x K_r'], k contiguous, row stride Kp) for the tensor-core
    # kernel: R block (c, r', r) element -> rtoff[r'] + r' * Kp + koff + r * D_c + c
    rtsz = Drb_sec * Kp
    rtoff = numpy.cumsum(rtsz) - rtsz
    rperm_t = (Rl.ioff[uR], rtoff[rbU] + koffU, dU, Kp[rbU])
    return {"t3off": t3off, "t3fhs": t3fhs, "t3flo": t3flo, "t3size": int(tsz.sum()), "needed": i3,
            "rperm": rperm, "gemm": gemm, "crow": crow.astype(numpy.int64),
            "sectors": {"used": used, "M": Mrb[used], "N": Drb_sec[used], "K": Krb[used], "Kp": Kp[used],
                        "t3pan": t3pan[used], "rtoff": rtoff[used], "crow_base": crow_base[used]},
            "rperm_t": rperm_t, "rtsize": int(rtsz.sum())}


PTASK_DT = numpy.dtype([("a_off", "<i8"), ("b_off", "<i8"), ("c_off", "<i8"), ("M", "<i4"), ("N", "<i4"),
                        ("K", "<i4"), ("m0", "<i4"), ("n0", "<i4"), ("op_b", "<i4"), ("op_e", "<i4"),
                        ("crow", "<i4"), ("lda", "<i4"), ("pad", "<i4")])
assert PTASK_DT.itemsize == 64
PANEL_TILES = {0: (128, 64), 1: (128, 32), 2: (128, 16)}


def panel_class(N):
    N = numpy.asarray(N)
    return numpy.where(N > 32, 0, numpy.where(N > 16, 1, 2))


def compile_panels(gemm, op_range, tensor_cores=False):
    """Work items {cfg: (ptasks, flops)} of dense panel GEMMs
    C_j[M_j x N_j] = A_j[M_j x K_j] . B_j[K_j x N_j], all operands row-major (qc_pgemm_*).
    With tensor_cores, panels that fill a useful part of a 128 x 64 tile are
    returned separately as grouped-GEMM work items {TC_CFG: (tasks, contribs, flops)}."""
    a_off, b_off, c_off, M, N, K = (numpy.asarray(x, dtype=numpy.int64) for x in gemm[:6])
    crow = numpy.asarray(gemm[6], dtype=numpy.int64) if len(gemm) > 6 else numpy.full(len(M), -1, dtype=numpy.int64)
    lda = numpy.asarray(gemm[7], dtype=numpy.int64) if len(gemm) > 7 else K.copy()
    # rows scattered through a row table run on the CUDA-core panel kernel
    tcsel = (M >= 64) & (N > 24) & (K >= 8) & (crow < 0) if tensor_cores else numpy.zeros(len(M), dtype=bool)
    tc = {}
    if tcsel.any():
        sel = numpy.flatnonzero(tcsel)
        tm, tn = TILES[TC_CFG]
        nm = (M[sel] + tm - 1) // tm
        nn = (N[sel] + tn - 1) // tn
        nt = nm * nn
        pid = numpy.repeat(numpy.arange(len(sel)), nt)
        loc = numpy.arange(int(nt.sum())) - numpy.repeat(numpy.cumsum(nt) - nt, nt)
        g = sel[pid]
        tasks = numpy.zeros(len(g), TASK_DT)
        tasks["c_off"] = c_off[g]
        tasks["M"], tasks["N"] = M[g], N[g]
        tasks["m0"] = (loc // nn[pid]) * tm
        tasks["n0"] = (loc % nn[pid]) * tn
        tasks["mlo"], tasks["nlo"] = M[g], N[g]
        tasks["c_ml"] = N[g]
        tasks["c_nl"] = 1
        tasks["cb"], tasks["ce"] = pid, pid + 1
        tasks["op_b"], tasks["op_e"] = op_range
        contribs = numpy.zeros(len(sel), CONTRIB_DT)
        contribs["a_off"], contribs["b_off"] = a_off[sel], b_off[sel]
        contribs["alpha"] = 1.0
        contribs["K"] = contribs["klo"] = K[sel]
        contribs["a_ml"] = K[sel]
        contribs["a_kl"] = 1
        contribs["b_kl"] = N[sel]
        contribs["b_nl"] = 1
        contribs["op_b"], contribs["op_e"] = 0, 1
        nop = op_range[1] - op_range[0]
        tc[TC_CFG] = (tasks, contribs, 2.0 * float((M[sel] * N[sel] * K[sel]).sum()) * nop)
        keep = numpy.flatnonzero(~tcsel)
        a_off, b_off, c_off, M, N, K, crow, lda = (x[keep] for x in (a_off, b_off, c_off, M, N, K, crow, lda))
    cls = panel_class(N)
    out = {}
    for k in numpy.unique(cls):
        sel = numpy.flatnonzero(cls == k)
        tm, tn = PANEL_TILES[int(k)]
        nm = (M[sel] + tm - 1) // tm
        nn = (N[sel] + tn - 1) // tn
        nt = nm * nn
        pid = numpy.repeat(numpy.arange(len(sel)), nt)
        loc = numpy.arange(int(nt.sum())) - numpy.repeat(numpy.cumsum(nt) - nt, nt)
        g = sel[pid]
        tasks = numpy.zeros(len(g), PTASK_DT)
        tasks["a_off"], tasks["b_off"], tasks["c_off"] = a_off[g], b_off[g], c_off[g]
        tasks["M"], tasks["N"], tasks["K"] = M[g], N[g], K[g]
        tasks["m0"] = (loc // nn[pid]) * tm
        tasks["n0"] = (loc % nn[pid]) * tn
        tasks["op_b"], tasks["op_e"] = op_range
        tasks["crow"] = crow[g]
        tasks["lda"] = lda[g]
        nop = op_range[1] - op_range[0]
        out[int(k)] = (tasks, 2.0 * float((M[sel] * N[sel] * K[sel]).sum()) * nop)
    if tensor_cores:
        return out, tc
    return out


class PanelStage(object):
    """Dense panel GEMMs of one contraction (qc_pgemm_*), one launch per tile class."""

    def __init__(self, parts, device, name, ops, tc_parts=None, crow=None):
        """parts: {cfg: [(ptasks, flops), ...]}; tc_parts: {TC_CFG: [(tasks, contribs, flops)]} run by the
        tensor-core grouped GEMM in TF32 modes (by the CUDA-core grouped GEMM otherwise); crow: the row
        table the tasks' crow indices point into."""
        self.name = name
        self.h_crow = crow if crow is not None and len(crow) else numpy.zeros(1, dtype=numpy.int64)
        self.d_crow = torch.from_numpy(self.h_crow.astype(numpy.int64)).to(device)
        self.tc = Stage(tc_parts, device, name, ops) if tc_parts else None
        self.host_ops = ops
        self.d_ops = upload(ops, device)
        self.groups = []
        self.flops = self.tc.flops if self.tc is not None else 0.0
        self.bytes = 0.0
        self.ntasks = self.tc.ntasks if self.tc is not None else 0
        for cfg in sorted(parts):
            tk = numpy.concatenate([p[0] for p in parts[cfg]])
            self.flops += sum(p[1] for p in parts[cfg])
            if not len(tk):
                continue
            span = int(max(1, (tk["op_e"] - tk["op_b"]).max()))
            self.groups.append((cfg, tk, upload(tk, device), span))
            self.ntasks += len(tk)

    def run(self, A, B, C, kind="f64", stream=None):
        lib = native.lib()
        s = stream if stream is not None else torch.cuda.current_stream(C.device).cuda_stream
        fn = lib.qc_pgemm_f64 if kind == "f64" else lib.qc_pgemm_f32
        if LOG.enabled:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
        for (cfg, tk, dt, span) in self.groups:
            check(fn(dt.data_ptr(), len(tk), span, self.d_ops.data_ptr(), self.d_crow.data_ptr(), A.data_ptr(),
                     B.data_ptr(), C.data_ptr(), cfg, s), "qc_pgemm_" + kind)
            LOG.launches += 1
        if self.tc is not None:
            en = LOG.enabled
            LOG.enabled = False
            self.tc.run(A, B, C, kind, stream)
            LOG.enabled = en
        if LOG.enabled:
            e1.record()
            LOG.records.append((self.name, e0, e1, self.flops, self.bytes * (A.element_size() / 8.0)))


def compile_template(l1, l2, lo, axes, triples, tile_cfg, off1=None):
    """Work items of one contraction for a single operator with zero base offsets.

    The operator loop is added afterwards through op ranges into an operator table.
    off1 replaces the packed block offsets of operand 1 (a permuted storage order).
    """
    return compile_pairs(l1, l2, lo, axes, triples, [0], [0], [0], [1.0], 0, tile_cfg, off1=off1)


def compile_pairs(l1, l2, lo, axes, triples, base1, base2, baseo, alpha, group_ops, tile_cfg, off1=None):
    """Native plan compiler wrapper -> (tasks, contribs, flops)."""
    o1 = l1.ioff if off1 is None else numpy.ascontiguousarray(off1, dtype=numpy.int64)
    assert len(o1) == l1.nblks
    lib = native.lib()
    tm, tn = TILES[tile_cfg]
    ax1 = numpy.array(axes[0], dtype=numpy.int32)
    ax2 = numpy.array(axes[1], dtype=numpy.int32)
    tri = numpy.ascontiguousarray(triples, dtype=numpy.int64)
    b1 = numpy.ascontiguousarray(base1, dtype=numpy.int64)
    b2 = numpy.ascontiguousarray(base2, dtype=numpy.int64)
    bo = numpy.ascontiguousarray(baseo, dtype=numpy.int64)
    al = numpy.ascontiguousarray(alpha, dtype=numpy.float64)
    nt = numpy.zeros(1, dtype=numpy.int64)
    fl = numpy.zeros(1, dtype=numpy.float64)
    head = (l1.rank, ptr(l1.nsyms), ptr(l1.ndims_cat), ptr(o1), l2.rank, ptr(l2.nsyms), ptr(l2.ndims_cat),
            ptr(l2.ioff), lo.rank, ptr(lo.nsyms), ptr(lo.ndims_cat), ptr(lo.ioff), len(axes[0]), ptr(ax1), ptr(ax2), len(tri), ptr(tri), len(b1), ptr(b1), ptr(b2), ptr(bo),
            ptr(al), int(group_ops), tm, tn)
    nc = check(lib.qc_compile_pairs(*(head + (None, 0, None, 0, ptr(nt), ptr(fl)))), "qc_compile_pairs")
    ntask = int(nt[0])
    tasks = numpy.zeros(max(ntask, 1), dtype=TASK_DT)
    contribs = numpy.zeros(max(nc, 1), dtype=CONTRIB_DT)
    nc2 = check(lib.qc_compile_pairs(*(head + (ptr(tasks), ntask, ptr(contribs), nc, ptr(nt), ptr(fl)))),
                "qc_compile_pairs")
    assert nc2 == nc and int(nt[0]) == ntask
    return tasks[:ntask], contribs[:nc], float(fl[0])


def merge_grouped(parts):
    """Merge per-class task lists that write the same output blocks (sigma's sum over operators).

    Tasks of one output block (same c_off) share one contribution range within a
    part.  The merged list has, per output block, the contributions of all parts
    (in part order) and the tiles of that block once.
    """
    parts = [p for p in parts if len(p[0])]
    flops = sum(p[2] for p in parts)
    if not parts:
        return numpy.zeros(0, TASK_DT), numpy.zeros(0, CONTRIB_DT), flops
    cbase = numpy.cumsum([0] + [len(p[1]) for p in parts])
    tbase = numpy.cumsum([0] + [len(p[0]) for p in parts])
    all_t = numpy.concatenate([p[0] for p in parts])
    all_c = numpy.concatenate([p[1] for p in parts])
    part_of = numpy.repeat(numpy.arange(len(parts)), [len(p[0]) for p in parts])
    coff = all_t["c_off"]
    first = numpy.ones(len(all_t), dtype=bool)
    first[1:] = (coff[1:] != coff[:-1]) | (part_of[1:] != part_of[:-1])
    fidx = numpy.flatnonzero(first)
    # records: one per (part, output block)
    r_coff = coff[fidx]
    r_part = part_of[fidx]
    r_cb = all_t["cb"][fidx] + cbase[r_part]
    r_ce = all_t["ce"][fidx] + cbase[r_part]
    r_ntile = numpy.diff(numpy.append(fidx, len(all_t)))
    order = numpy.lexsort((r_part, r_coff))
    r_coff, r_part, r_cb, r_ce, r_ntile, fidx = (x[order] for x in (r_coff, r_part, r_cb, r_ce, r_ntile, fidx))
    lens = r_ce - r_cb
    # contribution gather index: concatenation of [cb, ce) in record order
    starts = numpy.repeat(r_cb - numpy.cumsum(numpy.append(0, lens[:-1])), lens)
    gidx = starts + numpy.arange(lens.sum())
    new_c = all_c[gidx]
    # one group per output block
    gfirst = numpy.ones(len(r_coff), dtype=bool)
    gfirst[1:] = r_coff[1:] != r_coff[:-1]
    gstart = numpy.flatnonzero(gfirst)
    cum = numpy.append(0, numpy.cumsum(lens))
    g_cb = cum[gstart]
    g_ce = cum[numpy.append(gstart[1:], len(r_coff))]
    # tiles: those of the first record of each group
    g_t0 = fidx[gstart]
    g_nt = r_ntile[gstart]
    tix = numpy.repeat(g_t0 - numpy.cumsum(numpy.append(0, g_nt[:-1])), g_nt) + numpy.arange(g_nt.sum())
    new_t = all_t[tix].copy()
    new_t["cb"] = numpy.repeat(g_cb, g_nt)
    new_t["ce"] = numpy.repeat(g_ce, g_nt)
    return new_t, new_c, flops


class LaunchLog(object):
    """Optional per-launch CUDA-event log (bench instrumentation) and launch counter."""

    def __init__(self):
        self.enabled = False
        self.records = []
        self.launches = 0

    def reset(self):
        self.records = []
        self.launches = 0


LOG = LaunchLog()


class Stage(object):
    """A compiled stage resident on the device: one launch per tile configuration.

    parts: {tile_cfg: [(tasks, contribs, flops), ...]} whose op ranges index
    ``ops`` (OP_DT).  summed: tasks accumulate over the operators of each
    contribution instead of writing one tile per operator.
    """

    def __init__(self, parts, device, name="", ops=None, summed=False):
        if ops is None:
            ops = numpy.zeros(1, dtype=OP_DT)
            ops["alpha"] = 1.0
        self.name = name
        self.summed = bool(summed)
        self.host_ops = ops
        self.d_ops = upload(ops, device)
        self.groups = []
        self.bytes = 0.0          # algorithmic bytes (operands read once, output written once)
        self.flops = 0.0
        self.ntasks = 0
        self.ncontribs = 0
        for cfg in sorted(parts):
            tasks, contribs = [], []
            nc = 0
            for (t, c, f) in parts[cfg]:
                self.flops += f
                if len(t):
                    t = t.copy()
                    t["cb"] += nc
                    t["ce"] += nc
                    tasks.append(t)
                    contribs.append(c)
                    nc += len(c)
            if not tasks:
                continue
            tk = numpy.concatenate(tasks)
            ct = numpy.concatenate(contribs)
            span = 1 if self.summed else int(max(1, (tk["op_e"] - tk["op_b"]).max()))
            self.groups.append((cfg, tk, ct, upload(tk, device), upload(ct, device), span))
            self.ntasks += len(tk)
            self.ncontribs += len(ct)

    @property
    def host_groups(self):
        return [(cfg, tk, ct) for (cfg, tk, ct, _, _, _) in self.groups]

    def run(self, A, B, C, kind="f64", stream=None):
        lib = native.lib()
        s = stream if stream is not None else torch.cuda.current_stream(C.device).cuda_stream
        fn = {"f64": lib.qc_bgemm_f64, "f32": lib.qc_bgemm_f32, "tf32": lib.qc_bgemm_f32,
              "tf32x3": lib.qc_bgemm_f32}[kind]
        tcfn = lib.qc_bgemm_tf32x3 if kind == "tf32x3" else lib.qc_bgemm_tf32
        if LOG.enabled:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
        for (cfg, tk, ct, dt, dc, span) in self.groups:
            f = tcfn if (kind in ("tf32", "tf32x3") and cfg == TC_CFG) else fn
            check(f(dt.data_ptr(), len(tk), span, dc.data_ptr(), self.d_ops.data_ptr(), int(self.summed),
                    A.data_ptr(), B.data_ptr(), C.data_ptr(), cfg, s), "qc_bgemm_" + kind)
            LOG.launches += 1
        if LOG.enabled:
            e1.record()
            LOG.records.append((self.name, e0, e1, self.flops, self.bytes * (A.element_size() / 8.0)))


def add_parts(dst, parts, op_range=None, contrib_range=None):
    """Append compiled class parts to {cfg: [...]}, stamping operator ranges."""
    for cfg, (tk, ct, fl) in parts.items():
        if op_range is not None:
            tk["op_b"], tk["op_e"] = op_range
        if contrib_range is not None:
            ct["op_b"], ct["op_e"] = contrib_range
        nops = (op_range or contrib_range)
        mult = (nops[1] - nops[0]) if nops else 1
        dst.setdefault(cfg, []).append((tk, ct, fl * mult))


# ---------------------------------------------------------------- fiber-group stages
FTASK_DT = numpy.dtype([("f0", "<i4"), ("F", "<i4"), ("in_b", "<i4"), ("in_e", "<i4"), ("out_b", "<i4"),
                        ("out_e", "<i4"), ("op_b", "<i4"), ("op_e", "<i4")])
FIN_DT = numpy.dtype([("a_off", "<i8"), ("rows", "<i4"), ("fiber_major", "<i4"), ("srow", "<i4"), ("pad", "<i4"),
                      ("pad2", "<i8")])
FOUT_DT = numpy.dtype([("c_off", "<i8"), ("fhs", "<i4"), ("colmajor", "<i4"), ("ncols", "<i4"), ("pair_b", "<i4"),
                       ("pair_e", "<i4"), ("flo", "<i4")])
BPERM_DT = numpy.dtype([("src_off", "<i8"), ("dst_off", "<i8"), ("d0", "<i4"), ("d1", "<i4"), ("d2", "<i4"),
                        ("s0", "<i4"), ("s1", "<i4"), ("s2", "<i4"), ("op_b", "<i4"), ("op_e", "<i4"),
                        ("pad", "<i4", (4,))])
assert BPERM_DT.itemsize == 64
FPAIR_DT = numpy.dtype([("w_off", "<i8"), ("srow", "<i4"), ("rows", "<i4")])
assert FTASK_DT.itemsize == 32 and FIN_DT.itemsize == 32 and FOUT_DT.itemsize == 32 and FPAIR_DT.itemsize == 16
FIBER_TILE = 32
FIBER_FGEMM = True        # fiber groups as dense GEMMs (qc_fgemm_*); False: one CTA per fiber tile (qc_fiber_*)
FGITEM_DT = numpy.dtype([("wpan", "<i8"), ("group", "<i4"), ("f0", "<i4"), ("nf", "<i4"), ("op_b", "<i4"),
                         ("op_e", "<i4"), ("wstride", "<i4")])
FGGRP_DT = numpy.dtype([("row_b", "<i8"), ("col_b", "<i8"), ("F", "<i4"), ("R", "<i4"), ("CT", "<i4"), ("CTs", "<i4"),
                        ("FT", "<i4"), ("mc", "<i4"), ("flo", "<i4"), ("pad", "<i4")])
FGROW_DT = numpy.dtype([("off", "<i8"), ("fs", "<i8")])
FGCOL_DT = numpy.dtype([("off", "<i8"), ("fhs", "<i8"), ("fs", "<i8"), ("pad", "<i8")])
# one W block of a W panel (qc_wpanel_pairs_*): for each operator o of [op_b, op_b + nops),
# rows r < nr and columns j < ncol, panel element dst + o * opstride + (r0 + r) * width +
# perm(j0 + j) takes W[b_base(op_b + o) + src + r * src_ld + j] (perm: fg_col_perm)
WPAIR_DT = numpy.dtype([("dst", "<i8"), ("opstride", "<i8"), ("src", "<i8"), ("width", "<i4"), ("mc", "<i4"),
                        ("r0", "<i4"), ("nr", "<i4"), ("j0", "<i4"), ("ncol", "<i4"), ("src_ld", "<i4"),
                        ("op_b", "<i4"), ("nops", "<i4"), ("pad", "<i4")])
assert FGITEM_DT.itemsize == 32 and FGGRP_DT.itemsize == 48 and FGROW_DT.itemsize == 16 and FGCOL_DT.itemsize == 32
FG_THREADS = 128          # threads per CTA of qc_fgemm (one thread tile = 4 fibers x mc columns)
FG_A_BUDGET = 4096        # staged A elements (rows x tile fibers) per buffer
FG_W_BUDGET = 4096        # W panel elements (rows x padded columns) per buffer: wider groups are cut into column slices
FIBER_ROWS_WIDE = 128     # staged rows up to which a tile holds 64 fibers (two per lane)
FIBER_MAX_ROWS = 256


def fg_col_perm(col, width, mc):
    """Place of panel column col in a W panel row of the dense fiber-group GEMM: with
    8-column thread tiles the row is stored as two halves, column 8k + 4q + j at
    q * width/2 + 4k + j (each load instruction then reads contiguous 16-byte chunks)."""
    col = numpy.asarray(col, dtype=numpy.int64)
    width = numpy.asarray(width, dtype=numpy.int64)
    mc = numpy.asarray(mc, dtype=numpy.int64)
    half = (col % 8) // 4
    perm = half * (width // 2) + (col // 8) * 4 + col % 4
    return numpy.where(mc == 8, perm, col)


def compile_fiber(c, triples, rows_axis, fiber_major, extra_out=None, in_off=None, out_off=None, out_fhs=None,
                  out_flo=None, out_colmajor=False):
    """Fiber-group work items of a W contraction (template for one operator).

    The first three output axes form the fiber group (their block dims multiply
    to the fiber count F), the last two the column block.  Returns None when a
    group needs more than FIBER_MAX_ROWS staged rows.  Optional overrides:
    in_off / out_off (block offsets by flat block index, instead of the packed
    layouts' ioff), out_fhs / out_flo (two-level fiber strides of output blocks),
    extra_out (output blocks that must be written: those without pairs are
    written as zeros; with out_off, pairs into any other output block are dropped),
    out_colmajor (output blocks stored column by column, [ncols][F]: the next W
    contraction then reads them with contiguous fibers, fiber_major=0).
    """
    empty = (numpy.zeros(0, FTASK_DT), numpy.zeros(0, FIN_DT), numpy.zeros(0, FOUT_DT), numpy.zeros(0, FPAIR_DT), 1,
             0.0, FIBER_TILE)
    out, l1, l2 = c.out, c.l1, c.l2
    if out.rank != 5:
        return None
    tri = numpy.asarray(triples, dtype=numpy.int64).reshape(-1, 3)
    if out_off is not None and extra_out is not None:
        # output blocks with a remapped location: only the listed ones exist
        need = numpy.zeros(out.nblks, dtype=bool)
        need[numpy.asarray(extra_out, dtype=numpy.int64)] = True
        tri = tri[need[tri[:, 0]]]
    if extra_out is not None and len(extra_out):
        have = numpy.zeros(out.nblks, dtype=bool)
        have[tri[:, 0]] = True
        extra = numpy.unique(numpy.asarray(extra_out, dtype=numpy.int64))
        extra = extra[~have[extra]]
    else:
        extra = numpy.zeros(0, dtype=numpy.int64)
    if len(tri) == 0 and len(extra) == 0:
        return empty
    srt = numpy.argsort(tri[:, 0], kind="stable")      # pairs of one output block contiguous
    ob, i1, i2 = tri[srt, 0], tri[srt, 1], tri[srt, 2]
    d1 = l1.block_dims(i1) if len(i1) else numpy.zeros((0, l1.rank), dtype=numpy.int64)
    rows = d1[:, rows_axis]
    if not numpy.array_equal(rows, numpy.prod(d1[:, list(c.axes[0])], axis=1)):
        return None                  # contracted extent is not a single axis
    ns = out.nsyms.astype(numpy.int64)
    # output blocks (with pairs, plus zero-filled extras), sorted by block index
    uo, firsto = numpy.unique(ob, return_index=True)
    ends = numpy.r_[firsto[1:], len(ob)] if len(ob) else numpy.zeros(0, dtype=numpy.int64)
    allo = numpy.concatenate([uo, extra])
    pb = numpy.concatenate([firsto, numpy.zeros(len(extra), dtype=numpy.int64)])
    pe = numpy.concatenate([ends, numpy.zeros(len(extra), dtype=numpy.int64)])
    oo = numpy.argsort(allo, kind="stable")
    allo, pb, pe = allo[oo], pb[oo], pe[oo]
    dO = out.block_dims(allo)
    Fo = dO[:, 0] * dO[:, 1] * dO[:, 2]
    gko = allo // (ns[3] * ns[4])
    gstart = numpy.flatnonzero(numpy.r_[True, gko[1:] != gko[:-1]])
    ng = len(gstart)
    gid_o = numpy.cumsum(numpy.r_[False, gko[1:] != gko[:-1]]) if len(gko) else gko
    gout_b = gstart
    gout_e = numpy.r_[gstart[1:], len(allo)]
    gF = Fo[gstart]
    # staged input blocks: unique (group, input block) in (group, block) order
    gk_pair = ob // (ns[3] * ns[4])
    gid_pair = numpy.searchsorted(gko[gstart], gk_pair)
    key = gid_pair * int(l1.nblks) + i1
    uk, first_k, inv_k = numpy.unique(key, return_index=True, return_inverse=True)
    inv_k = inv_k.ravel()
    u_gid = uk // int(l1.nblks)
    u_blk = uk % int(l1.nblks)
    u_rows = rows[first_k]
    cs = numpy.cumsum(u_rows) - u_rows
    gin_b = numpy.searchsorted(u_gid, numpy.arange(ng), side="left")
    gin_e = numpy.searchsorted(u_gid, numpy.arange(ng), side="right")
    grow0 = numpy.where(gin_b < len(cs), cs[numpy.minimum(gin_b, max(len(cs) - 1, 0))], 0) if len(cs) else \
        numpy.zeros(ng, dtype=numpy.int64)
    u_srow = cs - grow0[u_gid] if len(cs) else cs
    R = numpy.zeros(ng, dtype=numpy.int64)
    if len(u_rows):
        numpy.add.at(R, u_gid, u_rows)
    if len(R) and R.max() > FIBER_MAX_ROWS:
        return None
    fins = numpy.zeros(len(uk), FIN_DT)
    fins["a_off"] = (l1.ioff if in_off is None else in_off)[u_blk]
    fins["rows"] = u_rows
    fins["fiber_major"] = fiber_major
    fins["srow"] = u_srow
    fouts = numpy.zeros(len(allo), FOUT_DT)
    fouts["c_off"] = (out.ioff if out_off is None else out_off)[allo]
    fouts["ncols"] = dO[:, 3] * dO[:, 4]
    fouts["flo"] = Fo if out_flo is None else out_flo[allo]
    fouts["fhs"] = 0 if out_fhs is None else out_fhs[allo]
    if out_fhs is not None and len(allo) and int(out_fhs[allo].max()) >= 2 ** 31:
        return None
    fouts["colmajor"] = 1 if out_colmajor else 0
    fouts["pair_b"] = pb
    fouts["pair_e"] = pe
    pairs = numpy.zeros(len(ob), FPAIR_DT)
    pairs["w_off"] = l2.ioff[i2]
    pairs["srow"] = u_srow[inv_k] if len(inv_k) else 0
    pairs["rows"] = rows
    mr = int(max(1, R.max() if len(R) else 1))
    tile = 64 if mr <= FIBER_ROWS_WIDE else FIBER_TILE      # two fibers per lane where rows allow
    nt = (gF + tile - 1) // tile
    gt = numpy.repeat(numpy.arange(ng), nt)
    tasks = numpy.zeros(len(gt), FTASK_DT)
    tasks["f0"] = (numpy.arange(len(gt)) - numpy.repeat(numpy.cumsum(nt) - nt, nt)) * tile
    tasks["F"] = gF[gt]
    tasks["in_b"], tasks["in_e"] = gin_b[gt], gin_e[gt]
    tasks["out_b"], tasks["out_e"] = gout_b[gt], gout_e[gt]
    dO_p = out.block_dims(ob) if len(ob) else numpy.zeros((0, 5), dtype=numpy.int64)
    flops = 2.0 * float((dO_p[:, 0] * dO_p[:, 1] * dO_p[:, 2] * dO_p[:, 3] * dO_p[:, 4] * rows).sum())
    return tasks, fins, fouts, pairs, mr, flops, tile


class FiberStage(object):
    """Fiber-group work items of several symmetry classes, resident on the device."""

    def __init__(self, parts, device, name, ops, budget=None):
        """parts: list of (tasks, fin, fout, fpair, max_rows, flops, fiber_tile, op_range), one fiber tile.
        budget: (A, W) elements staged per shared-memory buffer by qc_fgemm (fibers per tile and
        the width of W panel slices follow from it)."""
        self.a_budget, self.w_budget = (FG_A_BUDGET, FG_W_BUDGET) if budget is None else (int(budget[0]),
                                                                                          int(budget[1]))
        tks, fis, fos, fps = [], [], [], []
        nin = nout = npair = 0
        self.max_rows = 1
        self.flops = 0.0
        tiles = set(p[6] for p in parts)
        assert len(tiles) <= 1, "one fiber tile per stage"
        self.tile = tiles.pop() if tiles else FIBER_TILE
        for (tk, fi, fo, fp, mr, fl, _, rng) in parts:
            tk = tk.copy()
            fo = fo.copy()
            tk["in_b"] += nin
            tk["in_e"] += nin
            tk["out_b"] += nout
            tk["out_e"] += nout
            tk["op_b"], tk["op_e"] = rng
            fo["pair_b"] += npair
            fo["pair_e"] += npair
            tks.append(tk)
            fis.append(fi)
            fos.append(fo)
            fps.append(fp)
            nin += len(fi)
            nout += len(fo)
            npair += len(fp)
            self.max_rows = max(self.max_rows, mr)
            self.flops += fl * (rng[1] - rng[0])
        cat = lambda xs, dt: numpy.concatenate(xs) if xs else numpy.zeros(0, dt)
        self.h_tasks, self.h_fin = cat(tks, FTASK_DT), cat(fis, FIN_DT)
        self.h_fout, self.h_fpair = cat(fos, FOUT_DT), cat(fps, FPAIR_DT)
        self.host_ops = ops
        self.d = [upload(a, device) for a in (self.h_tasks, self.h_fin, self.h_fout, self.h_fpair, ops)]
        self.ntasks = len(self.h_tasks)
        self.span = int(max(1, (self.h_tasks["op_e"] - self.h_tasks["op_b"]).max())) if self.ntasks else 1
        self.name = name
        self.bytes = 0.0
        # dense fiber-group GEMM: per group a row table, a column table and a W panel map
        self.fgemm = FIBER_FGEMM
        self._wpan = {}
        if self.ntasks and self.fgemm:
            self._build_fgemm(device)

    def _build_fgemm(self, device):
        """Tables of qc_fgemm_* from the fiber-group records (vectorised over groups).

        Group g (the tasks sharing their first output) is the product
        C_g[F x CT] = A_g[F x R] . W_g[R x CT]: row srow + r of A_g is row r of an input
        block, column col0_j + c of C_g column c of output block j, and W_g[srow_p + r,
        col0_j + c] = W[w_off_p + r * ncols_j + c] for the pairs p of output j (zero where a
        pair is absent).  W panel maps are shared by the groups of an operator range that
        have the same one; the panels are gathered once per W tensor (qc_wpanel_*).
        """
        fo, fi, fp, ops = self.h_fout, self.h_fin, self.h_fpair, self.host_ops
        i64 = numpy.int64
        ht = self.h_tasks
        live = numpy.flatnonzero(ht["out_e"] > ht["out_b"])
        gs, first = numpy.unique(ht["out_b"][live].astype(i64), return_index=True)
        t0 = ht[live[first]]
        ng = len(gs)
        F = t0["F"].astype(i64)
        in_b, in_e = t0["in_b"].astype(i64), t0["in_e"].astype(i64)
        out_b, out_e = gs, t0["out_e"].astype(i64)

        def ranges(n):
            n = numpy.asarray(n, dtype=i64)
            own = numpy.repeat(numpy.arange(len(n)), n)
            return own, numpy.arange(int(n.sum()), dtype=i64) - numpy.repeat(numpy.cumsum(n) - n, n)

        # rows: the contracted rows of every input block, in staging order
        gi, li = ranges(in_e - in_b)
        fidx = in_b[gi] + li
        frows = fi["rows"][fidx].astype(i64)
        R = numpy.bincount(gi, weights=frows, minlength=ng).astype(i64)
        e, r_in = ranges(frows)
        fin_e, g_r = fidx[e], gi[e]
        fm = fi["fiber_major"][fin_e] != 0
        row_pos = (numpy.cumsum(R) - R)[g_r] + fi["srow"][fin_e].astype(i64) + r_in
        rows_rec = numpy.zeros(int(R.sum()), FGROW_DT)
        rows_rec["off"][row_pos] = fi["a_off"][fin_e] + numpy.where(fm, r_in, r_in * F[g_r])
        rows_rec["fs"][row_pos] = numpy.where(fm, fi["rows"][fin_e].astype(i64), 1)
        row_b = numpy.cumsum(R) - R
        # columns: every output block's columns, output by output
        go, lo = ranges(out_e - out_b)
        oidx = out_b[go] + lo
        nco = fo["ncols"][oidx].astype(i64)
        CT = numpy.bincount(go, weights=nco, minlength=ng).astype(i64)
        col_b = numpy.cumsum(CT) - CT
        c0o = numpy.cumsum(nco) - nco - col_b[go]           # first column of each output in its group
        e, c_in = ranges(nco)
        o_e, g_c = oidx[e], go[e]
        cm = fo["colmajor"][o_e] != 0
        nc_e = nco[e]
        cols_rec = numpy.zeros(int(CT.sum()), FGCOL_DT)
        cols_rec["off"] = fo["c_off"][o_e] + numpy.where(cm, c_in * F[g_c], c_in)
        cols_rec["fhs"] = numpy.where(cm, 0, fo["fhs"][o_e].astype(i64))
        cols_rec["fs"] = numpy.where(cm, 1, nc_e)
        cmo = fo["colmajor"][oidx] != 0
        flo_o = numpy.where(cmo | (fo["flo"][oidx].astype(i64) >= F[go]), F[go], fo["flo"][oidx].astype(i64))
        flo = numpy.full(ng, numpy.iinfo(i64).max, dtype=i64)
        numpy.minimum.at(flo, go, flo_o)
        flo_hi = numpy.zeros(ng, dtype=i64)
        numpy.maximum.at(flo_hi, go, flo_o)
        if numpy.any(flo != flo_hi):
            raise ValueError("fiber group with outputs of different fiber splits")
        flo = numpy.where(flo == numpy.iinfo(i64).max, F, flo)
        # column tile width and padded panel rows
        p4, p8 = (CT + 3) // 4 * 4, (CT + 7) // 8 * 8
        mc = numpy.where((CT > 12) & (p8 * 10 <= p4 * 11), 8, 4).astype(i64)
        CTs = (CT + mc - 1) // mc * mc
        # the pairs of every group (in group order): W block, its rows and columns in the panel
        npo = numpy.maximum((fo["pair_e"][oidx] - fo["pair_b"][oidx]).astype(i64), 0)
        e, lp = ranges(npo)
        pidx = fo["pair_b"][oidx][e].astype(i64) + lp
        PA = numpy.stack([fp["srow"][pidx].astype(i64), c0o[e], fp["rows"][pidx].astype(i64), nco[e],
                          fp["w_off"][pidx].astype(i64)], axis=1)
        p_g = go[e]
        gp_n = numpy.bincount(p_g, minlength=ng).astype(i64) if len(p_g) else numpy.zeros(ng, dtype=i64)
        gp_b = numpy.cumsum(gp_n) - gp_n

        # group records: whole groups, and column slices of groups wider than the W budget;
        # records of one operator range with the same panel content share one panel
        op_b, op_e = t0["op_b"].astype(i64), t0["op_e"].astype(i64)
        wide = R * CTs > self.w_budget
        width = numpy.maximum(mc, self.w_budget // numpy.maximum(R, 1) // mc * mc)
        nsl = numpy.where(wide, (CT + width - 1) // width, 1)
        rg, sl = ranges(nsl)
        rc0 = numpy.where(wide[rg], sl * width[rg], 0)
        rct = numpy.where(wide[rg], numpy.minimum(width[rg], CT[rg] - rc0), CT[rg])
        rcts = (rct + mc[rg] - 1) // mc[rg] * mc[rg]
        nrec = len(rg)
        seen, panels = {}, []           # key -> panel id; per panel (operator range, size, representative record)
        pan_id = numpy.zeros(nrec, dtype=i64)
        # the loop reads plain Python values: the pair rows of group g are the bytes
        # [gp_b[g], gp_b[g] + gp_n[g]) x 40 of PA (five int64 columns, row-major)
        pab = numpy.ascontiguousarray(PA, dtype=i64).tobytes()
        opb_l, ope_l, R_l, CTs_l, CT_l = op_b.tolist(), op_e.tolist(), R.tolist(), CTs.tolist(), CT.tolist()
        wide_l, gpb_l, gpn_l, rg_l, rcts_l = wide.tolist(), gp_b.tolist(), gp_n.tolist(), rg.tolist(), rcts.tolist()
        for k in range(nrec):
            g = rg_l[k]
            if not wide_l[g]:
                key = (opb_l[g], R_l[g], CTs_l[g], CT_l[g], pab[40 * gpb_l[g]:40 * (gpb_l[g] + gpn_l[g])])
            else:
                pa = PA[gp_b[g]:gp_b[g] + gp_n[g]]
                # the W blocks of the slice, clipped to its columns [rc0, rc0 + rct)
                lo = numpy.maximum(pa[:, 1], rc0[k])
                hi = numpy.minimum(pa[:, 1] + pa[:, 3], rc0[k] + rct[k])
                ok = hi > lo
                clip = numpy.stack([pa[ok, 0], pa[ok, 2], lo[ok] - rc0[k], hi[ok] - lo[ok],
                                    pa[ok, 4] + lo[ok] - pa[ok, 1], pa[ok, 3]], axis=1)
                key = (int(op_b[g]), "slice", int(R[g]), int(rcts[k]), int(mc[g]), clip.tobytes())
            pid = seen.get(key)
            if pid is None:
                pid = seen[key] = len(panels)
                panels.append((opb_l[g], ope_l[g], R_l[g] * rcts_l[k], k))
            pan_id[k] = pid
        # panels stored [operator][panel] per operator range
        npan = len(panels)
        p_ob = numpy.array([x[0] for x in panels], dtype=i64)
        p_oe = numpy.array([x[1] for x in panels], dtype=i64)
        p_sz = numpy.array([x[2] for x in panels], dtype=i64)
        p_rec = numpy.array([x[3] for x in panels], dtype=i64)
        cls_ob, cls_first, cls_of_p = numpy.unique(p_ob, return_index=True, return_inverse=True)
        cls_of_p = cls_of_p.ravel()
        order = numpy.argsort(cls_of_p, kind="stable")
        p_off = numpy.zeros(npan, dtype=i64)
        stride_c = numpy.zeros(len(cls_ob), dtype=i64)
        for pid in order:
            c = cls_of_p[pid]
            p_off[pid] = stride_c[c]
            stride_c[c] += p_sz[pid]
        nops_c = p_oe[cls_first] - cls_ob
        base_c = numpy.cumsum(stride_c * nops_c) - stride_c * nops_c
        panel_of = (base_c[cls_of_p] + p_off)[pan_id]
        stride_of = stride_c[cls_of_p][pan_id]
        if nrec and int(stride_of.max()) >= 2 ** 31:
            raise ValueError("W panel stride exceeds the work-item field")
        # the W blocks of every distinct panel (its representative record's group, clipped to
        # the record's columns): qc_wpanel_pairs_* copies each block of every operator of the
        # panel's range into the zero-filled panels, columns permuted as the kernel reads them
        if npan:
            pg = rg[p_rec]
            q, lp_ = ranges(gp_n[pg])
            pp = gp_b[pg][q] + lp_                       # pair row in PA
            c0_ = rc0[p_rec][q]
            lo = numpy.maximum(PA[pp, 1], c0_)
            hi = numpy.minimum(PA[pp, 1] + PA[pp, 3], c0_ + rct[p_rec][q])
            ok = hi > lo
            q, pp, c0_, lo, hi = q[ok], pp[ok], c0_[ok], lo[ok], hi[ok]
            wp = numpy.zeros(len(q), WPAIR_DT)
            wp["dst"] = (base_c[cls_of_p] + p_off)[q]
            wp["opstride"] = stride_c[cls_of_p][q]
            wp["src"] = PA[pp, 4] + (lo - PA[pp, 1])
            wp["width"] = rcts[p_rec][q]
            wp["mc"] = mc[pg][q]
            wp["r0"], wp["nr"] = PA[pp, 0], PA[pp, 2]
            wp["j0"], wp["ncol"] = lo - c0_, hi - lo
            wp["src_ld"] = PA[pp, 3]
            wp["op_b"] = p_ob[q]
            wp["nops"] = (p_oe - p_ob)[q]
        else:
            wp = numpy.zeros(0, WPAIR_DT)
        self.h_wpairs = wp
        self.wpanel_size = int((stride_c * nops_c).sum())
        # fibers per tile: a multiple of 4 that fills the CTA's threads with thread tiles
        # (decided once per distinct (column chunks, rows, fiber quads) of the records)
        chunks = rcts // mc[rg]
        combo = numpy.stack([chunks, numpy.maximum(R[rg], 1), numpy.maximum((F[rg] + 3) // 4, 1)], axis=1)
        if len(combo) and int(combo.max()) < (1 << 20):
            ck = (combo[:, 0] << 40) | (combo[:, 1] << 20) | combo[:, 2]       # one int64 key per record
            uk, cinv = numpy.unique(ck, return_inverse=True)
            ucombo = numpy.stack([uk >> 40, (uk >> 20) & ((1 << 20) - 1), uk & ((1 << 20) - 1)], axis=1)
        else:
            ucombo, cinv = numpy.unique(combo, axis=0, return_inverse=True)
        nn = numpy.arange(1, 65, dtype=i64)
        tot = nn[None, :] * ucombo[:, 0:1]
        util = tot / (FG_THREADS * ((tot + FG_THREADS - 1) // FG_THREADS))
        valid = (4 * nn[None, :] * ucombo[:, 1:2] <= self.a_budget)
        valid &= nn[None, :] <= ucombo[:, 2:3]
        valid[:, 0] = True
        util = numpy.where(valid, util, -1.0)
        good = util >= 0.97 * util.max(axis=1)[:, None]
        FT = (4 * (nn.size - numpy.argmax(good[:, ::-1], axis=1)))[cinv.ravel()]
        grp = numpy.zeros(nrec, FGGRP_DT)
        grp["row_b"] = row_b[rg]
        grp["col_b"] = col_b[rg] + rc0
        grp["F"], grp["R"], grp["CT"], grp["CTs"] = F[rg], R[rg], rct, rcts
        grp["FT"], grp["mc"], grp["flo"] = FT, mc[rg], flo[rg]
        # items: tiles of fibers, operator ranges kept whole (the kernel walks them in order)
        nt = (F[rg] + FT - 1) // FT
        it_r, t = ranges(nt)
        items = numpy.zeros(len(it_r), FGITEM_DT)
        items["group"] = it_r
        items["f0"] = t * FT[it_r]
        items["nf"] = numpy.minimum(FT[it_r], F[rg][it_r] - t * FT[it_r])
        items["op_b"], items["op_e"] = op_b[rg][it_r], op_e[rg][it_r]
        items["wpan"] = panel_of[it_r]
        items["wstride"] = stride_of[it_r]
        self.h_items, self.h_groups, self.h_rows, self.h_cols = items, grp, rows_rec, cols_rec
        self.max_a = int(max(4, ((R[rg] * FT).max() + 3) // 4 * 4)) if nrec else 4
        self.max_w = int((R[rg] * rcts).max()) if nrec else 0
        self.max_ct = int(rct.max()) if nrec else 0
        self.d_items = upload(items, device)
        self.d_groups = upload(grp, device)
        self.d_rows = upload(rows_rec if len(rows_rec) else numpy.zeros(1, FGROW_DT), device)
        self.d_cols = upload(cols_rec if len(cols_rec) else numpy.zeros(1, FGCOL_DT), device)
        self.d_wpairs = upload(self.h_wpairs if len(self.h_wpairs) else numpy.zeros(1, WPAIR_DT), device)

    def wpanel(self, B, stream):
        """The stage's W panels for the W values B (assembled on the first call for B)."""
        key = (B.data_ptr(), B.dtype, B.numel())
        P = self._wpan.get(key)
        if P is None:
            n = self.wpanel_size
            P = torch.zeros(max(n, 4), dtype=B.dtype, device=B.device)
            if len(self.h_wpairs):
                fn = native.lib().qc_wpanel_pairs_f64 if B.dtype == torch.float64 else \
                    native.lib().qc_wpanel_pairs_f32
                nmax = int(self.h_wpairs["nops"].max())
                check(fn(B.data_ptr(), B.numel(), self.d_wpairs.data_ptr(), len(self.h_wpairs), nmax,
                         self.d[4].data_ptr(), P.data_ptr(), P.numel(), stream), "qc_wpanel_pairs")
                LOG.launches += 1
            self._wpan[key] = P
        return P

    def run(self, A, B, C, kind="f64", stream=None):
        if self.ntasks == 0:
            return
        lib = native.lib()
        s = stream if stream is not None else torch.cuda.current_stream(C.device).cuda_stream
        if self.fgemm:
            P = self.wpanel(B, s)
        if LOG.enabled:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
        if self.fgemm:
            fn = lib.qc_fgemm_f64 if kind == "f64" else lib.qc_fgemm_f32
            check(fn(self.d_items.data_ptr(), len(self.h_items), self.d_groups.data_ptr(), self.d_rows.data_ptr(),
                     self.d_cols.data_ptr(), self.d[4].data_ptr(), self.max_a, self.max_w, self.max_ct,
                     A.data_ptr(), P.data_ptr(), C.data_ptr(), s), "qc_fgemm_" + kind)
        else:
            fn = lib.qc_fiber_f64 if kind == "f64" else lib.qc_fiber_f32
            check(fn(self.d[0].data_ptr(), self.ntasks, self.span, self.d[1].data_ptr(), self.d[2].data_ptr(),
                     self.d[3].data_ptr(), self.d[4].data_ptr(), self.max_rows, self.tile, A.data_ptr(), B.data_ptr(),
                     C.data_ptr(), s), "qc_fiber_" + kind)
        LOG.launches += 1
        if LOG.enabled:
            e1.record()
            LOG.records.append((self.name, e0, e1, self.flops, self.bytes * (A.element_size() / 8.0)))


class CompositeStage(object):
    """Sub-stages (fiber-group and generic) that together perform one contraction."""

    def __init__(self, subs, name):
        self.subs = [x for x in subs if x is not None]
        self.name = name
        self.flops = sum(x.flops for x in self.subs)
        self._bytes = 0.0

    @property
    def bytes(self):
        return self._bytes

    @bytes.setter
    def bytes(self, v):
        self._bytes = v
        tot = sum(x.flops for x in self.subs) or 1.0
        for x in self.subs:
            x.bytes = v * x.flops / tot

    @property
    def ntasks(self):
        return sum(x.ntasks for x in self.subs)

    @property
    def host_ops(self):
        return self.subs[0].host_ops

    def run(self, A, B, C, kind="f64", stream=None):
        for x in self.subs:
            x.run(A, B, C, kind, stream)


def upload(a, device):
    """Bytes of a host work list as a device tensor (no intermediate host copy for a GPU; a
    private copy on the CPU so that the tensor never aliases the host array)."""
    b = numpy.ascontiguousarray(a).view(numpy.uint8)
    t = torch.from_numpy(b)
    return t.clone() if torch.device(device).type == "cpu" else t.to(device)


def op_table(a_base, b_base, c_base, alpha):
    n = max(numpy.size(x) for x in (a_base, b_base, c_base, alpha))
    t = numpy.zeros(n, dtype=OP_DT)
    t["a_base"] = a_base
    t["b_base"] = b_base
    t["c_base"] = c_base
    t["alpha"] = alpha
    return t


def live_blocks(layout, triples):
    live = numpy.zeros(layout.nblks, dtype=bool)
    if len(triples):
        live[triples[:, 0]] = True
    return live


def prune(triples, live1=None, live2=None):
    keep = numpy.ones(len(triples), dtype=bool)
    if live1 is not None and len(triples):
        keep &= live1[triples[:, 1]]
    if live2 is not None and len(triples):
        keep &= live2[triples[:, 2]]
    return triples[keep]


def fiber_stages(parts, device, name, ops, budget=None):
    """FiberStage per fiber tile (parts compiled with 32- and 64-fiber tiles); budget: the
    dense fiber-group GEMM's (A, W) shared-memory budgets, default (FG_A_BUDGET, FG_W_BUDGET)."""
    by = {}
    for p in parts:
        by.setdefault(p[6], []).append(p)
    return [FiberStage(v, device, name, ops, budget) for k, v in sorted(by.items())]


# ---------------------------------------------------------------- tensor-core panel GEMM (qc_tcpanel_f32)
TCUNIT_DT = numpy.dtype([("a_map", "<i4"), ("b_map", "<i4"), ("a_c1", "<i4"), ("b_c1", "<i4"), ("a_c2", "<i4"),
                         ("b_c2", "<i4"), ("nk", "<i4"), ("m_valid", "<i4"), ("n_valid", "<i4"), ("op", "<i4"),
                         ("nseg", "<i4"), ("pad1", "<i4"), ("c_off", "<i8"), ("pad2", "<i8")])
TMDESC_DT = numpy.dtype([("addr", "<i8"), ("rank", "<i4"), ("swizzle", "<i4"), ("dims", "<i8", (5,)),
                         ("strides", "<i8", (4,)), ("box", "<i4", (5,)), ("pad", "<i4")])
TCSEG_DT = numpy.dtype([("off", "<i8"), ("col0", "<i4"), ("ncol", "<i4"), ("ldc", "<i4"), ("pad", "<i4", (3,))])
assert TCUNIT_DT.itemsize == 64 and TMDESC_DT.itemsize == 112 and TCSEG_DT.itemsize == 32
TC_BM, TC_BN, TC_BK = 128, 128, 32
SWIZZLE_128B = 3


class TCPanelStage(object):
    """Panel GEMMs C[rows] = A . B^T on the tensor cores (split TF32), A and B read by TMA.

    maps: list of (operand, element offset, dims, element strides of dims 1.., box) with
    operand "A" (the raw FP32 buffer passed to run) or "B" (the pre-split hi/lo buffer);
    units: TCUNIT_DT records indexing those maps, the stage's operator table and row table.
    The tensor maps embed buffer addresses: they are encoded on the host whenever run sees
    buffers other than the last ones."""

    def __init__(self, name, units, maps, ops, crow, flops, device, segs=None):
        """crow: row table (row form); segs: TCSEG_DT column segments (segment form, crow unused)."""
        self.name = name
        self.h_units = units
        self.d_units = upload(units, device)
        self.map_specs = maps
        self.d_ops = upload(ops, device)
        self.host_ops = ops
        self.h_segs = segs
        self.d_segs = upload(segs, device) if segs is not None else None
        if crow is None:
            crow = numpy.zeros(1, dtype=numpy.int64)
        self.d_crow = torch.from_numpy(numpy.ascontiguousarray(crow, dtype=numpy.int64)).to(device)
        self.flops = flops
        self.bytes = 0.0
        self.ntasks = len(units)
        self.device = device
        self._key = None
        self._maps = None

    def maps(self, A, B):
        key = (A.data_ptr(), B.data_ptr())
        if key != self._key:
            d = numpy.zeros(len(self.map_specs), TMDESC_DT)
            for i, (which, off, dims, strides, box) in enumerate(self.map_specs):
                base = A if which == "A" else B
                d[i]["addr"] = base.data_ptr() + 4 * int(off)
                d[i]["rank"] = len(dims)
                d[i]["swizzle"] = SWIZZLE_128B
                d[i]["dims"][:len(dims)] = dims
                d[i]["strides"][:len(strides)] = [4 * int(x) for x in strides]
                d[i]["box"][:len(box)] = box
            out = numpy.zeros(max(len(d), 1) * 128, dtype=numpy.uint8)
            check(native.lib().qc_tmap_encode(len(d), d.ctypes.data, out.ctypes.data), "qc_tmap_encode")
            self._maps = torch.from_numpy(out).to(self.device)
            self._key = key
        return self._maps

    def run(self, A, B, C, kind="tf32x3", stream=None):
        if self.ntasks == 0:
            return
        lib = native.lib()
        s = stream if stream is not None else torch.cuda.current_stream(C.device).cuda_stream
        maps = self.maps(A, B)
        if LOG.enabled:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
        if self.d_segs is not None:
            check(lib.qc_tcpanel_seg_f32(self.d_units.data_ptr(), self.ntasks, maps.data_ptr(), self.d_ops.data_ptr(),
                                         self.d_segs.data_ptr(), C.data_ptr(), s), "qc_tcpanel_seg_f32")
        else:
            check(lib.qc_tcpanel_f32(self.d_units.data_ptr(), self.ntasks, maps.data_ptr(), self.d_ops.data_ptr(),
                                     self.d_crow.data_ptr(), C.data_ptr(), s), "qc_tcpanel_f32")
        LOG.launches += 1
        if LOG.enabled:
            e1.record()
            LOG.records.append((self.name, e0, e1, self.flops, self.bytes * 0.5))


def _replicate_units(tiles, poss):
    """tiles: TCUNIT_DT records of one operator (op slot q = 0); one copy per operator of a
    class, the tiles of an operator back to back (consecutive units share its operands)."""
    n, k = len(tiles), len(poss)
    u = numpy.tile(tiles, k)
    q = numpy.repeat(numpy.arange(k, dtype=numpy.int32), n)
    u["op"] = numpy.repeat(numpy.asarray(poss, dtype=numpy.int32), n)
    return u, q


def tc_sigma4_units(classes, order_pos, t3_base_of_class, rt_base_of_class, rt_opstride, rt_total):
    """Work units and tensor maps of the .R contraction on the tensor cores.

    classes: list of (op positions in the stage's operator table, pan4 sectors dict, T3 op stride).
    Unit order: per operator and sector all row tiles back to back (they share the R panel)."""
    units, maps = [], []
    for ci, (poss, sec, t3stride) in enumerate(classes):
        nops = len(poss)
        amap0 = len(maps)
        tl = []
        for j in range(len(sec["used"])):
            K, M, N, Kp = int(sec["K"][j]), int(sec["M"][j]), int(sec["N"][j]), int(sec["Kp"][j])
            maps.append(("A", t3_base_of_class[ci] + int(sec["t3pan"][j]), (K, M, nops), (Kp, t3stride),
                         (TC_BK, TC_BM, 1)))
            maps.append(("B", rt_base_of_class[ci] + int(sec["rtoff"][j]), (K, N, nops, 2),
                         (Kp, rt_opstride[ci], rt_total), (TC_BK, TC_BN, 1, 2)))
            n0 = numpy.arange(0, N, TC_BN)
            m0 = numpy.arange(0, M, TC_BM)
            t = numpy.zeros(len(n0) * len(m0), TCUNIT_DT)
            t["a_map"], t["b_map"] = amap0 + 2 * j, amap0 + 2 * j + 1
            t["a_c1"] = numpy.tile(m0, len(n0))
            t["b_c1"] = numpy.repeat(n0, len(m0))
            t["nk"] = (K + TC_BK - 1) // TC_BK
            t["m_valid"] = numpy.minimum(TC_BM, M - t["a_c1"])
            t["n_valid"] = numpy.minimum(TC_BN, N - t["b_c1"])
            t["c_off"] = int(sec["crow_base"][j]) + t["a_c1"]
            tl.append(t)
        if tl:
            u, q = _replicate_units(numpy.concatenate(tl), poss)
            u["a_c2"] = u["b_c2"] = q
            units.append(u)
    u = numpy.concatenate(units) if units else numpy.zeros(0, TCUNIT_DT)
    return u, maps


def _ranges(n):
    """(owner, local index) of the concatenation of arange(n[i]) (vectorised)."""
    n = numpy.asarray(n, dtype=numpy.int64)
    own = numpy.repeat(numpy.arange(len(n)), n)
    return own, numpy.arange(int(n.sum()), dtype=numpy.int64) - numpy.repeat(numpy.cumsum(n) - n, n)


def psi_panels(psi):
    """The wavefunction as the B operand of the tensor-core L.psi GEMMs: per first-index
    sector l' the psi blocks (l', n1, n2, r) of that sector side by side as columns,
    transposed to [sum_j N_j x Kp] (k = l' index contiguous, rows padded to Kp = D_l'
    rounded up to 4).  Returns (gather index into the packed vector, -1 for padding),
    {sector: (offset, N total, K, Kp)} and {block: (sector, first column)}."""
    blocks = numpy.asarray(psi.idx_allowed, dtype=numpy.int64)
    if len(blocks) == 0:
        return numpy.zeros(0, dtype=numpy.int64), {}, {}
    sec = psi.block_sectors(blocks)[0].astype(numpy.int64)
    d = psi.block_dims(blocks)
    K = d[:, 0].astype(numpy.int64)
    N = numpy.prod(d[:, 1:], axis=1).astype(numpy.int64)
    o = numpy.argsort(sec, kind="stable")                 # blocks grouped by sector, in block order
    blocks, sec, K, N = blocks[o], sec[o], K[o], N[o]
    us, first = numpy.unique(sec, return_index=True)
    cnt = numpy.diff(numpy.r_[first, len(sec)])
    ks = K[first]
    kps = (ks + 3) // 4 * 4
    ntot = numpy.add.reduceat(N, first)
    size = ntot * kps
    soff = numpy.cumsum(size) - size
    col = numpy.cumsum(N) - N - numpy.repeat((numpy.cumsum(N) - N)[first], cnt)    # first column in its sector
    sidx = numpy.repeat(numpy.arange(len(us)), cnt)                                   # sector position per block
    # gather index: panel element (column c, k) of sector s at soff + c * Kp + k
    gidx = numpy.full(int(size.sum()), -1, dtype=numpy.int64)
    b, e = _ranges(N * K[...])                       # (block, local element) over each block's N x K values
    nb, kb = N[b], K[b]
    cc, kk = e % nb, e // nb                         # element (k, column) of the block: psi offset k * N + c
    gidx[soff[sidx[b]] + (col[b] + cc) * kps[sidx[b]] + kk] = psi.ioff[blocks[b]] + kk * nb + cc
    info = {int(s_): (int(a), int(n), int(k), int(kp)) for s_, a, n, k, kp in zip(us, soff, ntot, ks, kps)}
    cols = {int(bb): (int(s_), int(c)) for bb, s_, c in zip(blocks, sec, col)}
    return gidx, info, cols


def tc_sigma1_units(classes, psi_info, psi_cols, lp_base, lp_opstride, lp_total, psi_total):
    """Work units, column segments and tensor maps of L.psi on the tensor cores.

    classes: list of (op positions, pan["tc"] dict).  A: the class's TC L panels (pre-split
    planes, lp_total apart); B: the psi panels of the sector (psi_info, planes psi_total apart).
    The T1 destination of psi block j is its panel [M x N_j] at t1pan_j (rows = L panel rows).
    A unit is one 128-row tile of one 128-column tile of a sector's psi panel; its segments
    are the pieces of the psi blocks that column tile holds (vectorised over blocks)."""
    units, maps, segs = [], [], []
    bmap = {}
    for s_, (off, ntot, k, kp) in sorted(psi_info.items()):
        bmap[s_] = len(maps)
        maps.append(("B", off, (k, ntot, 1, 2), (kp, ntot * kp, psi_total), (TC_BK, TC_BN, 1, 2)))
    nseg = 0
    for ci, (poss, tc) in enumerate(classes):
        nops = len(poss)
        secs = numpy.asarray(tc["sectors"], dtype=numpy.int64)
        amap = len(maps) + numpy.arange(len(secs))
        for j in range(len(secs)):
            K, M, Kp = int(tc["K"][j]), int(tc["M"][j]), int(tc["Kp"][j])
            maps.append(("A", lp_base[ci] + int(tc["lpoff"][j]), (K, M, nops, 2), (Kp, lp_opstride[ci], lp_total),
                         (TC_BK, TC_BM, 1, 2)))
        if len(secs) == 0:
            continue
        jpos = {int(s_): j for j, s_ in enumerate(secs.tolist())}
        # the class's blocks: sector position j, first column c, width nj, T1 panel offset
        bl = tc["blocks"].tolist()
        bj = numpy.array([jpos.get(psi_cols[b][0], -1) for b in bl], dtype=numpy.int64)
        bc = numpy.array([psi_cols[b][1] for b in bl], dtype=numpy.int64)
        nj = numpy.asarray(tc["Nj"], dtype=numpy.int64)
        t1p = numpy.asarray(tc["t1pan"], dtype=numpy.int64)
        keep = bj >= 0
        bj, bc, nj, t1p = bj[keep], bc[keep], nj[keep], t1p[keep]
        # (block, column tile) pairs: tiles first .. last that the block's columns touch
        t0 = bc // TC_BN
        t1 = (bc + nj - 1) // TC_BN
        pb, pl = _ranges(numpy.maximum(t1 - t0 + 1, 0))
        tile = t0[pb] + pl
        o = numpy.lexsort((bc[pb], tile, bj[pb]))            # by sector, column tile, first column
        pb, tile = pb[o], tile[o]
        n0 = tile * TC_BN
        ntot_j = numpy.array([psi_info[int(s_)][1] for s_ in secs], dtype=numpy.int64)
        w = numpy.minimum(TC_BN, ntot_j[bj[pb]] - n0)
        lo = numpy.maximum(bc[pb], n0)
        hi = numpy.minimum(bc[pb] + nj[pb], n0 + w)
        ok = hi > lo
        pb, tile, n0, lo, hi, w = pb[ok], tile[ok], n0[ok], lo[ok], hi[ok], w[ok]
        sg = numpy.zeros(len(pb), TCSEG_DT)
        sg["off"] = t1p[pb] + (lo - bc[pb])
        sg["col0"] = lo - n0
        sg["ncol"] = hi - lo
        sg["ldc"] = nj[pb]
        segs.append(sg)
        # one unit group per (sector, column tile) that holds a segment
        key = bj[pb] * (1 << 32) + tile
        gstart = numpy.flatnonzero(numpy.r_[True, key[1:] != key[:-1]]) if len(key) else numpy.zeros(0, numpy.int64)
        gn = numpy.diff(numpy.r_[gstart, len(key)])
        gj, gn0, gw = bj[pb][gstart], n0[gstart], w[gstart]
        Mj = numpy.asarray(tc["M"], dtype=numpy.int64)[gj]
        nm = (Mj + TC_BM - 1) // TC_BM
        ug, um = _ranges(nm)
        t = numpy.zeros(len(ug), TCUNIT_DT)
        t["a_map"] = amap[gj[ug]]
        t["b_map"] = numpy.array([bmap[int(s_)] for s_ in secs], dtype=numpy.int64)[gj[ug]]
        t["a_c1"] = um * TC_BM
        t["b_c1"] = gn0[ug]
        Kj = numpy.asarray(tc["K"], dtype=numpy.int64)[gj]
        t["nk"] = ((Kj + TC_BK - 1) // TC_BK)[ug]
        t["m_valid"] = numpy.minimum(TC_BM, Mj[ug] - um * TC_BM)
        t["n_valid"] = gw[ug]
        t["nseg"] = gn[ug]
        t["c_off"] = nseg + gstart[ug]
        nseg += len(pb)
        if len(t):
            u, q = _replicate_units(t, poss)
            u["a_c2"] = q
            units.append(u)
    u = numpy.concatenate(units) if units else numpy.zeros(0, TCUNIT_DT)
    sg = numpy.concatenate(segs) if segs and sum(len(x) for x in segs) else numpy.zeros(1, TCSEG_DT)
    return u, maps, sg

