"""Symmetry-blocked tensor layouts, computed by the native block-map library.

Mirrors the structure fields of the reference's ``qtensor`` class
(source/qtensor/qtensor.py:108-149): rank, qsyms, ndims, status, nsyms,
iblks_allowed (1-based inverse of idx_allowed), idx_allowed, ioff_allowed,
dims_allowed, ndim_allowed, size_allowed.  Values live elsewhere (device
buffers); a ``Layout`` is immutable and cached by its defining data.

Quantum numbers are multiples of 1/2 and are handed to the native code as
exact int32 values of 2q, so every block map is built in integer arithmetic.
"""
import collections
import weakref

import numpy

from . import native
from .native import ptr, check

# layouts are interned by content while alive: equal layouts are the same object, and
# no entry outlives its layout (a weak map never hands out a recycled object); the most
# recently used ones are also held strongly so that dots with the same sectors share them
_CACHE = weakref.WeakValueDictionary()
_RECENT = collections.OrderedDict()
_RECENT_MAX = 8192


def _hold(key, obj):
    _RECENT[key] = obj
    _RECENT.move_to_end(key)
    while len(_RECENT) > _RECENT_MAX:
        _RECENT.popitem(last=False)


def qint(q):
    q = numpy.asarray(q, dtype=numpy.float64)
    t = numpy.rint(2.0 * q)
    if q.size and numpy.max(numpy.abs(2.0 * q - t)) > 1e-8:
        raise ValueError("quantum numbers must be multiples of 1/2")
    return t.astype(numpy.int32)


def classification(qnums, collect=True):
    """Sectors in order of first occurrence (qtensor_util.py:34-51)."""
    qnums = numpy.asarray(qnums, dtype=numpy.float64)
    if qnums.ndim == 1:
        qnums = qnums.reshape(-1, 1)
    n = len(qnums)
    if not collect:
        return qnums.copy(), numpy.ones(n, dtype=numpy.int64), [numpy.array([i]) for i in range(n)]
    q2 = qint(qnums)
    uniq, first, inv = numpy.unique(q2, axis=0, return_index=True, return_inverse=True)
    inv = inv.ravel()
    order = numpy.argsort(first, kind="stable")          # sectors by first occurrence
    rank_of = numpy.empty(len(order), dtype=numpy.int64)
    rank_of[order] = numpy.arange(len(order))
    sec = rank_of[inv]
    idl = [numpy.flatnonzero(sec == s) for s in range(len(order))]
    qsyms = uniq[order].astype(numpy.float64) / 2.0
    ndims = numpy.array([len(x) for x in idl], dtype=numpy.int64)
    return qsyms, ndims, idl


class Layout(object):
    """Packed block layout of a block-sparse tensor (qtensor.fromQsyms)."""

    def __new__(cls, status, qsyms, ndims):
        status = numpy.asarray(status, dtype=bool)
        qs = [numpy.asarray(q, dtype=numpy.float64).reshape(len(q), -1) for q in qsyms]
        nd = [numpy.asarray(n, dtype=numpy.int64).ravel() for n in ndims]
        key = (status.tobytes(), tuple(qint(q).tobytes() + bytes([q.shape[1]]) for q in qs),
               tuple(n.tobytes() for n in nd))
        obj = _CACHE.get(key)
        if obj is not None:
            _hold(key, obj)
            return obj
        obj = super(Layout, cls).__new__(cls)
        obj._init(status, qs, nd)
        _CACHE[key] = obj
        _hold(key, obj)
        return obj

    def _init(self, status, qsyms, ndims):
        lib = native.lib()
        self.status = status
        self.rank = len(qsyms)
        self.qsyms = qsyms
        self.ndims = ndims
        self.nqnum = qsyms[0].shape[1]
        self.nsyms = numpy.array([len(q) for q in qsyms], dtype=numpy.int32)
        self.nblks = int(numpy.prod(self.nsyms.astype(numpy.int64)))
        self.shape = numpy.array([int(n.sum()) for n in ndims], dtype=numpy.int64)
        q2 = numpy.ascontiguousarray(numpy.concatenate([qint(q) for q in qsyms]).ravel(), dtype=numpy.int32)
        st = numpy.ascontiguousarray(status.astype(numpy.int32))
        allowed = numpy.empty(self.nblks, dtype=numpy.int32)
        check(lib.qc_sym_allowed(self.rank, self.nqnum, ptr(self.nsyms), ptr(st), ptr(q2), ptr(allowed)),
              "qc_sym_allowed")
        nd = numpy.ascontiguousarray(numpy.concatenate(ndims), dtype=numpy.int64)
        iblks = numpy.empty(self.nblks, dtype=numpy.int32)
        ioff = numpy.empty(self.nblks, dtype=numpy.int64)
        ndim = numpy.empty(self.nblks, dtype=numpy.int64)
        size = numpy.zeros(1, dtype=numpy.int64)
        nall = numpy.zeros(1, dtype=numpy.int64)
        check(lib.qc_block_layout(self.rank, ptr(self.nsyms), ptr(nd), ptr(allowed), ptr(iblks), ptr(ioff),
                                  ptr(ndim), ptr(size), ptr(nall)), "qc_block_layout")
        self.allowed = allowed
        self.iblks_flat = iblks
        self.iblks = iblks.reshape(tuple(self.nsyms))
        self.ioff = ioff
        self.ndim = ndim
        self.size = int(size[0])
        self.idx_allowed = numpy.flatnonzero(allowed)
        self.ndims_cat = nd
        # per-index packed-sector offsets (position of sector s within the index)
        self.secoff = [numpy.concatenate([[0], numpy.cumsum(n)[:-1]]).astype(numpy.int64) for n in ndims]

    def block_dims(self, idx):
        """Dimensions [len(idx), rank] of the blocks with flat indices idx."""
        idx = numpy.atleast_1d(numpy.asarray(idx, dtype=numpy.int64))
        sec = numpy.unravel_index(idx, tuple(self.nsyms))
        return numpy.stack([self.ndims[i][sec[i]] for i in range(self.rank)], axis=1)

    def block_sectors(self, idx):
        return numpy.unravel_index(idx, tuple(self.nsyms))

    def prjmap(self, idlst):
        """Packed position -> row-major dense flat index (qtensor.prjmap, qtensor.py:442-453)."""
        out = numpy.empty(self.size, dtype=numpy.int64)
        strides = numpy.ones(self.rank, dtype=numpy.int64)
        for i in range(self.rank - 2, -1, -1):
            strides[i] = strides[i + 1] * self.shape[i + 1]
        for idx in self.idx_allowed:
            isyms = numpy.unravel_index(idx, tuple(self.nsyms))
            lin = numpy.zeros(1, dtype=numpy.int64)
            for i in range(self.rank):
                pos = numpy.asarray(idlst[i][isyms[i]], dtype=numpy.int64) * strides[i]
                lin = (lin[:, None] + pos[None, :]).ravel()
            o = int(self.ioff[idx])
            out[o:o + len(lin)] = lin
        return out

    def sector_map(self):
        """Packed position -> flat index in the 'sector-packed' dense order.

        Like prjmap with idlst[i][s] = secoff[i][s] + arange(ndims[i][s]); used where
        only a consistent enumeration of every index is needed.
        """
        idl = [[numpy.arange(int(self.secoff[i][s]), int(self.secoff[i][s] + self.ndims[i][s]))
                for s in range(len(self.ndims[i]))] for i in range(self.rank)]
        return self.prjmap(idl)


def flip_right(lay, qkey):
    """R environment seen from the left (source/mpo_dmrg_kernelQt.py:297-300)."""
    return Layout(lay.status, [-lay.qsyms[0], qkey - lay.qsyms[1], qkey - lay.qsyms[2]], lay.ndims)


def flip_horizontal(lay):
    """W seen from the right: bond indices negated and flipped (kernelQt.py:723-727)."""
    st = lay.status.copy()
    st[0] = not st[0]
    st[1] = not st[1]
    return Layout(st, [-lay.qsyms[0], -lay.qsyms[1], lay.qsyms[2], lay.qsyms[3]], lay.ndims)


class Contraction(object):
    """tensordotSYM (source/qtensor/qtensor.py:563-637): output layout + block-pair list."""

    def __init__(self, l1, l2, axes):
        i1, i2 = list(axes[0]), list(axes[1])
        e1 = [i for i in range(l1.rank) if i not in i1]
        e2 = [i for i in range(l2.rank) if i not in i2]
        for a, b in zip(i1, i2):
            if not numpy.array_equal(qint(l1.qsyms[a]), qint(l2.qsyms[b])) or \
                    not numpy.array_equal(l1.ndims[a], l2.ndims[b]):
                raise ValueError("contracted indices have different sectors")
        ints1 = [bool(l1.status[i]) for i in i1]
        ints2 = [bool(l2.status[i]) for i in i2]
        exts1 = [bool(l1.status[i]) for i in e1]
        exts2 = [bool(l2.status[i]) for i in e2]
        if len(i1) and ints1[0] == ints2[0]:
            ints2 = [not x for x in ints2]
            exts2 = [not x for x in exts2]
        if any(a == b for a, b in zip(ints1, ints2)):
            raise ValueError("contracted indices must pair in/out")
        self.out = Layout(exts1 + exts2, [l1.qsyms[i] for i in e1] + [l2.qsyms[i] for i in e2],
                          [l1.ndims[i] for i in e1] + [l2.ndims[i] for i in e2])
        self.l1, self.l2, self.axes = l1, l2, (i1, i2)
        lib = native.lib()
        ax1 = numpy.array(i1, dtype=numpy.int32)
        ax2 = numpy.array(i2, dtype=numpy.int32)
        args = (l1.rank, ptr(l1.nsyms), ptr(l1.iblks_flat), l2.rank, ptr(l2.nsyms), ptr(l2.iblks_flat),
                len(i1), ptr(ax1), ptr(ax2), ptr(self.out.iblks_flat))
        n = check(lib.qc_contract_pairs(*(args + (None, 0))), "qc_contract_pairs")
        tri = numpy.empty((max(n, 1), 3), dtype=numpy.int64)
        n2 = check(lib.qc_contract_pairs(*(args + (ptr(tri), n))), "qc_contract_pairs")
        assert n2 == n
        self.triples = tri[:n]

    def prune(self, live_in1):
        """Drop pairs whose first operand block is structurally zero (never written)."""
        if live_in1 is None:
            return self.triples
        keep = live_in1[self.triples[:, 1]]
        return self.triples[keep]
