"""The grouped block-GEMM engine on random block-sparse contractions (CPU interpreter of the
work items): random ranks, sectors, quantum numbers (N only or (N, Sz), half-integers),
ragged block sizes, one or two contracted indices in any order and either in/out status,
including contractions with no allowed output block.  Every result equals the oracle's
tensordotSYM + tensordotCAL (source/qtensor/qtensor.py:563-659) on the same tensors.
The work-item format indexes at most two axes of size > 1 in each of M, N and K; a
contraction beyond that is refused with an error, never computed wrongly."""
import numpy
import pytest
import torch

from emulate import patch_stage_run
from oracle.blocks import QTensor, Contraction as OContraction


def _random_pair(rng):
    nq = int(rng.integers(1, 3))
    k = int(rng.integers(1, 3))                  # the work items index at most two axes per
    r1, r2 = k + int(rng.integers(1, 3)), k + int(rng.integers(1, 3))     # GEMM dimension
    ax1 = [int(x) for x in rng.permutation(r1)[:k]]
    ax2 = [int(x) for x in rng.permutation(r2)[:k]]

    def sectors():
        n = int(rng.integers(1, 5))
        return rng.integers(-2, 3, size=(n, nq)) / 2.0, rng.integers(1, 4, size=n)

    q1 = [sectors() for _ in range(r1)]
    q2 = [sectors() for _ in range(r2)]
    for a, b in zip(ax1, ax2):
        q2[b] = q1[a]                            # contracted indices share their sectors
    st1 = rng.integers(0, 2, size=r1).astype(bool)
    st2 = rng.integers(0, 2, size=r2).astype(bool)
    flip = bool(rng.integers(0, 2))              # contracted pairs in/out, or all flipped
    for a, b in zip(ax1, ax2):
        st2[b] = (not st1[a]) if not flip else st1[a]
    if flip:                                     # the rule needs one consistent flip for all pairs
        for a, b in zip(ax1, ax2):
            st2[b] = st1[a]
    return (st1, q1), (st2, q2), (ax1, ax2)


def _tensors(rng, spec):
    st, q = spec
    o = QTensor(st).from_qsyms(len(q), [x[0] for x in q], [x[1] for x in q])
    o.value = rng.standard_normal(o.size_allowed)
    return o


@pytest.mark.parametrize("seed", range(6))
def test_random_contractions_match_oracle(seed, monkeypatch):
    patch_stage_run(monkeypatch)
    from qcmpodmrg_b200.qtensor import Layout, Contraction
    from qcmpodmrg_b200.engine import compile_classes, Stage, add_parts
    rng = numpy.random.default_rng(100 + seed)
    done = 0
    for _ in range(25):
        s1, s2, axes = _random_pair(rng)
        t1, t2 = _tensors(rng, s1), _tensors(rng, s2)
        oc = OContraction().plan(t1, t2, axes)
        want = oc.run(t1, t2).value
        l1 = Layout(s1[0], [x[0] for x in s1[1]], [x[1] for x in s1[1]])
        l2 = Layout(s2[0], [x[0] for x in s2[1]], [x[1] for x in s2[1]])
        c = Contraction(l1, l2, axes)
        assert c.out.size == oc.out.size_allowed
        assert numpy.array_equal(c.out.idx_allowed, oc.out.idx_allowed)
        parts = {}
        add_parts(parts, compile_classes(c, c.triples, axes), op_range=(0, 1))
        st = Stage(parts, "cpu")
        out = torch.zeros(max(c.out.size, 1), dtype=torch.float64)
        st.run(torch.from_numpy(t1.value), torch.from_numpy(t2.value), out)
        assert numpy.abs(out.numpy()[:c.out.size] - want).max(initial=0.0) <= 1e-12 * max(1.0, numpy.abs(want).max(initial=0.0))
        done += 1
    assert done == 25


def test_more_than_two_axes_per_gemm_dimension_is_refused():
    from qcmpodmrg_b200.qtensor import Layout, Contraction
    from qcmpodmrg_b200.engine import compile_classes
    from qcmpodmrg_b200.native import NativeError
    z = numpy.zeros((1, 1))
    two = numpy.array([2])
    l1 = Layout([False, False, False, True], [z] * 4, [two] * 4)       # three external axes of size 2
    l2 = Layout([False, True], [z] * 2, [two] * 2)
    c = Contraction(l1, l2, ([3], [0]))
    with pytest.raises(NativeError):
        compile_classes(c, c.triples, ([3], [0]))
