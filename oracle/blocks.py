"""ORACLE (test infrastructure only): symmetry-blocked tensors, restated in NumPy.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import
this package; the product never does.  It restates the reference's block-sparse
tensor ("qtensor") semantics:

* sector classification by first occurrence   -- source/qtensor/qtensor_util.py:34-51
* allowed-block mask (symAllowed)              -- ctypes/qsym.c:5-480, qtensor_util.py:70-90
  restated in integer arithmetic: every quantum number is a multiple of 1/2,
  so 2q is an exact integer and "|sum| < 1e-10" becomes "sum == 0".
* packed layout (iblks/idx/ioff/ndim)          -- source/qtensor/qtensor.py:272-346
* contraction pair lists + execution           -- source/qtensor/qtensor.py:563-659
* dense <-> packed conversions, diagonal       -- source/qtensor/qtensor.py:356-411
* projection maps                              -- source/qtensor/qtensor.py:442-453, 528-560
"""
import numpy


def qint(q):
    """Quantum numbers (float, multiples of 1/2) -> exact int32 2q."""
    q = numpy.asarray(q, dtype=numpy.float64)
    t = numpy.rint(2.0 * q)
    if numpy.any(numpy.abs(2.0 * q - t) > 1e-8):
        raise ValueError("quantum numbers must be multiples of 1/2")
    return t.astype(numpy.int64)


def classification(qnums, collect=True):
    """qtensor_util.classification: sectors in order of first occurrence."""
    qnums = numpy.asarray(qnums, dtype=numpy.float64)
    if qnums.ndim == 1:
        qnums = qnums.reshape(-1, 1)
    if not collect:
        return qnums.copy(), numpy.ones(len(qnums), dtype=numpy.int64), [[i] for i in range(len(qnums))]
    keys = {}
    order = []
    for idx, val in enumerate(map(tuple, qint(qnums))):
        if val not in keys:
            keys[val] = []
            order.append(val)
        keys[val].append(idx)
    qsyms = numpy.array([numpy.array(k) / 2.0 for k in order], dtype=numpy.float64)
    idlst = [keys[k] for k in order]
    ndims = numpy.array([len(x) for x in idlst], dtype=numpy.int64)
    return qsyms, ndims, idlst


def sym_allowed(nsyms, status, qsyms):
    """Row-major mask over the Cartesian product of sectors (int32 0/1).

    sum over status==False indices of q  minus  sum over status==True == 0.
    """
    rank = len(nsyms)
    acc = numpy.zeros(tuple(nsyms) + (qsyms[0].shape[1],), dtype=numpy.int64)
    for i in range(rank):
        qi = qint(qsyms[i])
        shape = [1] * rank + [qi.shape[1]]
        shape[i] = nsyms[i]
        acc = acc + (-1 if status[i] else 1) * qi.reshape(shape)
    return numpy.all(acc == 0, axis=-1).astype(numpy.int32).ravel()


class QTensor(object):
    """Block-sparse tensor with the reference's packed layout."""

    def __init__(self, status=None):
        self.status = None if status is None else numpy.array(status, dtype=bool)
        self.value = None
        self.idlst = None

    # qtensor.fromQsyms (qtensor.py:272-346)
    def from_qsyms(self, rank, qsyms, ndims, allocate=True, idlst=None):
        self.rank = rank
        self.qsyms = [numpy.array(q, dtype=numpy.float64).reshape(len(q), -1) for q in qsyms]
        self.ndims = [numpy.array(n, dtype=numpy.int64) for n in ndims]
        if idlst is not None:
            self.idlst = idlst
        self.nqnum = self.qsyms[0].shape[1]
        self.shape = numpy.array([int(n.sum()) for n in self.ndims])
        self.nsyms = numpy.array([len(q) for q in self.qsyms], dtype=numpy.int64)
        self.nblks = int(numpy.prod(self.nsyms))
        mask = sym_allowed(self.nsyms, self.status, self.qsyms)
        self.idx_allowed = numpy.flatnonzero(mask)
        self.nblks_allowed = len(self.idx_allowed)
        iblks = numpy.zeros(self.nblks, dtype=numpy.int64)
        iblks[self.idx_allowed] = self.idx_allowed + 1
        self.iblks = iblks.reshape(self.nsyms)
        grids = numpy.meshgrid(*self.ndims, indexing="ij") if rank > 0 else []
        self.dims_allowed = numpy.stack([g.ravel() for g in grids], axis=1)
        self.ndim_allowed = numpy.prod(self.dims_allowed, axis=1)
        self.ioff_allowed = numpy.zeros(self.nblks, dtype=numpy.int64)
        sizes = self.ndim_allowed[self.idx_allowed]
        offs = numpy.concatenate([[0], numpy.cumsum(sizes)[:-1]]) if len(sizes) else numpy.zeros(0, numpy.int64)
        self.ioff_allowed[self.idx_allowed] = offs
        self.size_allowed = int(sizes.sum())
        self.value = numpy.zeros(self.size_allowed) if allocate else None
        return self

    def blocks(self):
        """Iterate (idx, isyms, ioff, dims) over allowed blocks in packed order."""
        for idx in self.idx_allowed:
            isyms = numpy.unravel_index(idx, self.nsyms)
            yield idx, isyms, int(self.ioff_allowed[idx]), self.dims_allowed[idx]

    def block(self, idx):
        off = int(self.ioff_allowed[idx])
        return self.value[off:off + int(self.ndim_allowed[idx])].reshape(self.dims_allowed[idx])

    # qtensor.fromDenseTensor (qtensor.py:356-380)
    def from_dense(self, val, qnums, collect=None):
        rank = len(qnums)
        collect = collect or [True] * rank
        cls = [classification(q, c) for q, c in zip(qnums, collect)]
        self.from_qsyms(rank, [c[0] for c in cls], [c[1] for c in cls])
        self.idlst = [c[2] for c in cls]
        for idx, isyms, off, dims in self.blocks():
            ix = numpy.ix_(*[self.idlst[i][isyms[i]] for i in range(rank)])
            self.value[off:off + int(numpy.prod(dims))] = val[ix].ravel()
        return self

    def to_dense(self, idlst=None):
        idlst = idlst or self.idlst
        val = numpy.zeros(self.shape)
        for idx, isyms, off, dims in self.blocks():
            ix = numpy.ix_(*[idlst[i][isyms[i]] for i in range(self.rank)])
            val[ix] = self.value[off:off + int(numpy.prod(dims))].reshape(dims)
        return val

    # qtensor.toDenseDiag (qtensor.py:401-411): diagonal of the last two indices
    def to_dense_diag(self, idlst=None):
        idlst = idlst or self.idlst
        val = numpy.zeros(self.shape[:-1])
        for idx, isyms, off, dims in self.blocks():
            if isyms[-1] != isyms[-2]:
                continue
            ix = numpy.ix_(*[idlst[i][isyms[i]] for i in range(self.rank - 1)])
            blk = self.value[off:off + int(numpy.prod(dims))].reshape(dims)
            val[ix] = numpy.einsum("...ii->...i", blk)
        return val

    # qtensor.prjmap (qtensor.py:442-453): packed position -> dense flat index
    def prjmap(self, idlst):
        out = []
        for idx, isyms, off, dims in self.blocks():
            grids = numpy.meshgrid(*[numpy.array(idlst[i][isyms[i]]) for i in range(self.rank)], indexing="ij")
            out.append(numpy.ravel_multi_index([g.ravel() for g in grids], self.shape))
        return numpy.concatenate(out) if out else numpy.zeros(0, numpy.int64)

    def copy_structure(self):
        q = QTensor(self.status)
        q.from_qsyms(self.rank, self.qsyms, self.ndims, allocate=False)
        q.idlst = self.idlst
        return q

    # qtensor.reduceQsymsToN (qtensor.py:528-543)
    def reduce_to_n(self):
        q = QTensor(self.status)
        q.from_qsyms(self.rank, [x[:, 0:1] for x in self.qsyms], self.ndims, idlst=self.idlst)
        for idx, isyms, off, dims in self.blocks():
            j = q.iblks[isyms] - 1
            o = int(q.ioff_allowed[j])
            n = int(self.ndim_allowed[idx])
            q.value[o:o + n] = self.value[off:off + n]
        return q

    # qtensor.projectionNMs (qtensor.py:546-560)
    def projection_nms(self, qsyms0):
        q = QTensor(self.status)
        q.from_qsyms(self.rank, qsyms0, self.ndims)
        for idx, isyms, off, dims in q.blocks():
            j = self.iblks[isyms] - 1
            o = int(self.ioff_allowed[j])
            n = int(q.ndim_allowed[idx])
            q.value[off:off + n] = self.value[o:o + n]
        return q


def from_dict(d):
    """Rebuild a QTensor from the essential fields (rank, qsyms*, ndims*, status, value)."""
    rank = int(d["rank"])
    q = QTensor(numpy.array(d["status"], dtype=bool))
    q.from_qsyms(rank, [d["qsyms%d" % i] for i in range(rank)], [d["ndims%d" % i] for i in range(rank)])
    if "idlst0" in d:
        q.idlst = []
        for i in range(rank):
            flat = list(numpy.asarray(d["idlst%d" % i]).tolist())
            parts, o = [], 0
            for n in q.ndims[i]:
                parts.append(flat[o:o + int(n)])
                o += int(n)
            q.idlst.append(parts)
    q.value = numpy.array(d["value"], dtype=numpy.float64).copy()
    return q


class Contraction(object):
    """tensordotSYM + tensordotCAL (qtensor.py:563-659) as one object.

    ``plan(qt1, qt2, axes)`` builds the output structure and the pair list
    ``clst`` (one entry per allowed output block x matching internal sectors,
    internal sectors in row-major order); ``run`` executes it.
    """

    def plan(self, qt1, qt2, axes):
        i1, i2 = list(axes[0]), list(axes[1])
        e1 = [i for i in range(qt1.rank) if i not in i1]
        e2 = [i for i in range(qt2.rank) if i not in i2]
        for a, b in zip(i1, i2):
            assert numpy.array_equal(qt1.qsyms[a], qt2.qsyms[b]), "contracted sectors differ"
        ints1 = [qt1.status[i] for i in i1]
        ints2 = [qt2.status[i] for i in i2]
        exts1 = [qt1.status[i] for i in e1]
        exts2 = [qt2.status[i] for i in e2]
        if len(i1) != 0 and ints1[0] == ints2[0]:
            ints2 = [not x for x in ints2]
            exts2 = [not x for x in exts2]
        for s1, s2 in zip(ints1, ints2):
            assert s1 != s2
        out = QTensor(exts1 + exts2)
        out.from_qsyms(len(e1) + len(e2), [qt1.qsyms[i] for i in e1] + [qt2.qsyms[i] for i in e2],
                       [qt1.ndims[i] for i in e1] + [qt2.ndims[i] for i in e2], allocate=False)
        ib1 = qt1.iblks.transpose(e1 + i1)
        ib2 = qt2.iblks.transpose(e2 + i2)
        ne1 = len(e1)
        clst = []
        for idx, isyms, off, dims in out.blocks():
            n1 = ib1[tuple(isyms[:ne1])]
            n2 = ib2[tuple(isyms[ne1:])]
            for inz in zip(*numpy.nonzero(numpy.logical_and(n1, n2))):
                clst.append((idx, int(n1[inz]) - 1, int(n2[inz]) - 1))
        self.out, self.clst, self.axes = out, clst, (i1, i2)
        self.e1, self.e2 = e1, e2
        return self

    def run(self, qt1, qt2, conj1=False):
        out = self.out
        val = numpy.zeros(out.size_allowed)
        for idx, j1, j2 in self.clst:
            t1 = qt1.block(j1)
            t2 = qt2.block(j2)
            o = int(out.ioff_allowed[idx])
            val[o:o + int(out.ndim_allowed[idx])] += numpy.tensordot(t1, t2, self.axes).ravel()
        res = out.copy_structure()
        res.value = val
        return res

    def flops(self, qt1, qt2):
        """Algorithmic FLOPs: 2 * prod(out block dims) * prod(contracted dims) per pair."""
        tot = 0
        i1 = self.axes[0]
        for idx, j1, j2 in self.clst:
            d1 = qt1.dims_allowed[j1]
            tot += 2 * int(numpy.prod(self.out.dims_allowed[idx])) * int(numpy.prod([d1[a] for a in i1]))
        return tot


def contract(qt1, qt2, axes, conj1=False):
    c = Contraction().plan(qt1, qt2, axes)
    return c.run(qt1, qt2)
