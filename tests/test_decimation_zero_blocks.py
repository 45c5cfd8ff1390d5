"""Decimation with RDM classes the wavefunction has no weight in (exactly zero blocks):
the blocks get LAPACK's eigenpairs of a zero matrix (zero eigenvalues, unit vectors) without
the device eigensolver, and the kept states follow the reference's rdm_blkdiag
(source/mpo_dmrg_qparser.py:106-183): the weighted states first, then zero-weight states up
to the bond dimension, sorted by quantum number.  On the B200 the device eigensolver
returned NaN eigenvalues for an all-zero 41 x 41 block, which emptied the next dot."""
import numpy
import torch

from qcmpodmrg_b200.dmrg import DMRG


class _Probe(DMRG):
    def __init__(self):          # only the decimation attributes are needed
        self.thresh = -1.e-14


def test_zero_class_blocks_give_unit_vectors_and_finite_weights(monkeypatch):
    rng = numpy.random.default_rng(5)
    # three classes: (1, 0.5) x 3 rows with weight, (2, 0) x 41 rows without, (0, 0) x 2 with
    classes = numpy.array([[1, 0.5]] * 3 + [[2, 0.0]] * 41 + [[0, 0.0]] * 2)
    n = len(classes)
    c = numpy.zeros((n, 5))
    w = numpy.r_[numpy.arange(3), numpy.arange(44, 46)]
    c[w] = rng.standard_normal((len(w), 5))
    rho = torch.from_numpy(c @ c.T)
    rho = rho / torch.trace(rho)
    calls = []
    real_eigh = torch.linalg.eigh

    def eigh(a, *args, **kw):
        calls.append(tuple(a.shape))
        assert float(a.abs().max()) > 0, "the eigensolver is not called on a zero block"
        return real_eigh(a, *args, **kw)

    monkeypatch.setattr(torch.linalg, "eigh", eigh)
    dwts, qred, rot, s = _Probe().rdm_blkdiag(rho, classes, 10)
    assert sorted(calls) == [(2, 2), (3, 3)]
    assert numpy.isfinite(s).all() and abs(dwts) < 1e-12
    assert len(qred) == 10
    # the five weighted states are kept; the rest are zero-weight states of class (2, 0)
    assert int((s > 1e-12).sum()) == 5
    zero_cols = rot[:, torch.from_numpy(numpy.flatnonzero(s <= 1e-12))]
    # unit vectors supported on the rows of the zero class
    assert torch.allclose(zero_cols.abs().sum(dim=0), torch.ones(zero_cols.shape[1], dtype=rot.dtype))
    assert set(numpy.flatnonzero(zero_cols.abs().sum(dim=1).numpy() > 0)) <= set(range(3, 44))
    # kept states sorted by quantum number (reference order)
    assert all(tuple(qred[i]) <= tuple(qred[i + 1]) for i in range(len(qred) - 1))
