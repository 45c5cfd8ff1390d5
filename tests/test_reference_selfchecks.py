"""The reference's own consistency checks, run on the product (CPU, kernels interpreted):

* checkDiagQt (source/mpo_dmrg_kernelQt.py:129-150): the effective Hamiltonian built
  column by column from HVec is symmetric and its diagonal is HDiag (1e-10);
* pdvdson's self-test (source/tools/pdvdson.py:396-424): Davidson on a random
  symmetric matrix returns the lowest eigenpairs of a dense eigensolver (two states,
  crit_vec 1e-7 with the energy criterion tightened so that the residuals decide, no
  start-vector noise), on the device solver.
"""
import numpy
import pytest
import torch

from helpers import load, record_operators
from emulate import patch_stage_run


@pytest.mark.parametrize("tag", ["K4"])
def test_check_diag_qt(tag, monkeypatch):
    patch_stage_run(monkeypatch)
    recs = load("kernels_%s.npz" % tag)["records"]
    for r in [max(recs, key=lambda x: len(x["hvec_x"]))]:      # the largest recorded dot
        sig, dg, ws = record_operators(r, "cpu", use_fiber=True)
        n = sig.ndim0
        h = numpy.array([sig(torch.from_numpy(e)).numpy() for e in numpy.identity(n)]).T
        assert numpy.linalg.norm(h - h.T) <= 1e-10
        assert numpy.linalg.norm(numpy.diag(h) - dg().numpy()) <= 1e-10


def test_davidson_self_test():
    import scipy.linalg
    from qcmpodmrg_b200.davidson import davidson
    rng = numpy.random.RandomState(0)
    ndim, neig = 100, 2
    mat = rng.uniform(-1, 1, size=(ndim, ndim))
    mat = 0.5 * (mat + mat.T)
    efull, v = scipy.linalg.eigh(mat)
    m = torch.from_numpy(mat)
    res = davidson(lambda x: m @ x, torch.from_numpy(numpy.diag(mat).copy()), neig, crit_e=1e-14, crit_vec=1e-7,
                   maxcycle=200)
    assert max(res.rnorms[-1]) <= 1e-6          # a state stops on its residual or on |de| <= crit_e
    assert numpy.abs(res.eigs - efull[:neig]).max() <= 1e-12
    ova = numpy.abs(v[:, :neig].T @ res.vecs.numpy().T)
    assert numpy.linalg.norm(ova - numpy.identity(neig)) <= 1e-6
