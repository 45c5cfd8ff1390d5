"""Batched multi-instance sweeps (one launch per sigma stage for all instances,
CUDA-graph replay) give the same energies as running each instance alone."""
import numpy
import pytest
import torch

pytestmark = pytest.mark.gpu


def _instances(cuda, kind_prec="f64"):
    from qcmpodmrg_b200.hamiltonian import make_hamiltonian
    from qcmpodmrg_b200.synthetic import product_mps
    from qcmpodmrg_b200.dmrg import DMRG
    out = []
    for (K, seed) in ((6, 1001), (8, 1002), (8, 1003)):
        ham = make_hamiltonian(K, K, seed, 3.0)
        d = DMRG(ham, device=cuda, precision=kind_prec)
        d.load_mps(product_mps(ham))
        out.append(d)
    return out


def test_batched_matches_sequential(cuda):
    from qcmpodmrg_b200.batched import BatchedDMRG
    seq = _instances(cuda)
    bat = _instances(cuda)
    b = BatchedDMRG(bat, kind="f64", use_graphs=True)
    for D in (16, 24):
        for st in ("R", "L"):
            ref = [d.sweep(st, D, 1e-8) for d in seq]
            got = b.sweep(st, D, 1e-8)
            for (n, e, dw, el, dl), (e2, dw2, el2, dl2) in zip(ref, got):
                assert abs(e - e2) <= 1e-9
                assert numpy.abs(numpy.array(el) - numpy.array(el2)).max() <= 1e-8
    assert b.captures > 0 and b.steps > 0
