"""The C-ABI libraries load, export what include/*.h declares, and their host-side
block maps equal the oracle's (no GPU needed)."""
import ctypes
import os
import re

import numpy
import pytest

from helpers import load, layout_of
from oracle.blocks import QTensor, Contraction as OContraction, from_dict
from qcmpodmrg_b200 import native
from qcmpodmrg_b200.qtensor import Layout, Contraction, classification

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "qcmpodmrg_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.findall(r"\b(\w+)\s*\(", src)


def test_libraries_export_every_declared_symbol():
    names = [n for n in declared_symbols() if n not in ("defined",)]
    qc = native.lib()
    qs = native.qsym_lib()
    for n in names:
        if n == "symAllowed":
            assert hasattr(qs, n)
        else:
            assert hasattr(qc, n), n


def test_dropin_symallowed_matches_reference_golden():
    q = native.qsym_lib()
    for c in load("qsym_cases.npz")["cases"]:
        rank = int(c["rank"])
        ndims = numpy.ascontiguousarray(c["ndims"], dtype=numpy.int32)
        status = numpy.ascontiguousarray(c["status"], dtype=numpy.int32)
        qs = [numpy.ascontiguousarray(x, dtype=numpy.float64).reshape(int(n), -1) for x, n in zip(c["qsyms"], ndims)]
        out = numpy.full(int(numpy.prod(ndims)), -7, dtype=numpy.int32)
        args = [x.ctypes.data for x in qs] + [None] * (8 - rank)
        rc = q.symAllowed(rank, int(c["nqnum"]), ndims.ctypes.data, status.ctypes.data, out.ctypes.data, *args)
        assert rc == 0
        assert numpy.array_equal(out, c["allowed"])


def test_dropin_symallowed_rejects_non_half_integers():
    q = native.qsym_lib()
    nd = numpy.array([2, 2], dtype=numpy.int32)
    st = numpy.array([0, 1], dtype=numpy.int32)
    a = numpy.array([[0.3], [1.0]])
    out = numpy.zeros(4, dtype=numpy.int32)
    rc = q.symAllowed(2, 1, nd.ctypes.data, st.ctypes.data, out.ctypes.data, a.ctypes.data, a.ctypes.data,
                      *([None] * 6))
    assert rc == -5  # QC_ERR_HALFINT


def _rand_tensor(rng, rank, status):
    qs, nd = [], []
    for _ in range(rank):
        n = int(rng.integers(1, 5))
        qs.append(rng.integers(-3, 4, size=(n, 2)) / 2.0)
        nd.append(rng.integers(1, 4, size=n))
    return qs, nd


def test_layout_matches_oracle_random():
    rng = numpy.random.default_rng(3)
    for _ in range(40):
        rank = int(rng.integers(1, 6))
        status = rng.integers(0, 2, size=rank).astype(bool)
        qs, nd = _rand_tensor(rng, rank, status)
        lay = Layout(status, qs, nd)
        o = QTensor(status).from_qsyms(rank, qs, nd, allocate=False)
        assert numpy.array_equal(lay.idx_allowed, o.idx_allowed)
        assert numpy.array_equal(lay.iblks.ravel(), o.iblks.ravel())
        assert numpy.array_equal(lay.ioff, o.ioff_allowed)
        assert numpy.array_equal(lay.block_dims(numpy.arange(lay.nblks)), o.dims_allowed)
        assert lay.size == o.size_allowed


@pytest.mark.parametrize("tag", ["K4", "K6"])
def test_contraction_pairs_match_oracle_on_reference_tensors(tag):
    """Pair lists (tensordotSYM clst) for all four sigma contractions, bit-exact and in order."""
    from oracle.kernels import flip_right
    from qcmpodmrg_b200.qtensor import flip_right as pflip
    for r in load("kernels_%s.npz" % tag)["records"]:
        qtmp = from_dict(r["qtmp"])
        for iop in range(len(r["envL"])):
            L, R = from_dict(r["envL"][iop]), from_dict(r["envR"][iop])
            Wi, Wj = from_dict(r["mpo_i"][iop]), from_dict(r["mpo_j"][iop])
            Rf = flip_right(R, numpy.asarray(r["qkey"]))
            o1 = OContraction().plan(L, qtmp, ([2], [0]))
            o2 = OContraction().plan(o1.out, Wi, ([0, 2], [0, 3]))
            o3 = OContraction().plan(o2.out, Wj, ([1, 3], [3, 0]))
            o4 = OContraction().plan(o3.out, Rf, ([1, 3], [2, 0]))
            pL, pR = layout_of(r["envL"][iop]), layout_of(r["envR"][iop])
            pWi, pWj = layout_of(r["mpo_i"][iop]), layout_of(r["mpo_j"][iop])
            p1 = Contraction(pL, layout_of(r["qtmp"]), ([2], [0]))
            p2 = Contraction(p1.out, pWi, ([0, 2], [0, 3]))
            p3 = Contraction(p2.out, pWj, ([1, 3], [3, 0]))
            p4 = Contraction(p3.out, pflip(pR, numpy.asarray(r["qkey"])), ([1, 3], [2, 0]))
            for o, p in ((o1, p1), (o2, p2), (o3, p3), (o4, p4)):
                assert numpy.array_equal(numpy.array(o.clst, dtype=numpy.int64).reshape(-1, 3), p.triples)
                assert numpy.array_equal(o.out.ioff_allowed, p.out.ioff)
            assert p4.out is layout_of(r["qtmp"])


def test_classification_first_occurrence():
    q = numpy.array([[1, .5], [0, 0], [1, .5], [2, 0], [0, 0]])
    qs, nd, idl = classification(q)
    assert numpy.array_equal(qs, [[1, .5], [0, 0], [2, 0]])
    assert list(nd) == [2, 2, 1]
    assert [list(x) for x in idl] == [[0, 2], [1, 4], [3]]
