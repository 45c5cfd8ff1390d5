"""MPS files in the reference's HDF5 layout (qcmpodmrg_b200.mps_io, source/mpo_dmrg_io.py):
a swept state written and read back exactly (symmetry-blocked and dense sites), read by the
reference's own loadMPS / qtensor.load, and a tensor dumped by the reference's qtensor read
back.  The file objects are the in-memory h5py stand-in of tests/golden/shims (h5py is not
installed here); the module only uses the h5py interface."""
import os

import numpy
import pytest
import torch

from helpers import load
from emulate import patch_stage_run
from qcmpodmrg_b200.hamiltonian import make_hamiltonian

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "baseline", "_ref", "qcmpodmrg")
needs_ref = pytest.mark.skipif(not os.path.isdir(REF), reason="converted reference not present (baseline/_ref)")


def _swept(monkeypatch):
    patch_stage_run(monkeypatch)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    from qcmpodmrg_b200.dmrg import DMRG
    fx = load("sweep_K5.npz")
    ham = make_hamiltonian(int(fx["K"]), int(fx["N"]), int(fx["seed"]), None if fx["decay"] < 0 else fx["decay"])
    d = DMRG(ham, device="cpu")
    d.load_mps(fx["init_mps"])
    d.sweep("R", int(fx["D"]), 1e-8)
    d.sweep("L", int(fx["D"]), 1e-8)
    return d


def _h5(tmp_path, name):
    import sys
    shims = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "shims")
    if shims not in sys.path:
        sys.path.insert(0, shims)
    import h5py      # the in-memory stand-in
    return h5py.File(str(tmp_path / name), "w")


@pytest.mark.parametrize("qt", [True, False])
def test_save_load_round_trip(monkeypatch, tmp_path, qt):
    from qcmpodmrg_b200.mps_io import save_mps, load_mps
    d = _swept(monkeypatch)
    f = _h5(tmp_path, "mps_%d" % qt)
    save_mps(f, d, qt=qt)
    got = load_mps(f)
    for i in range(d.nsite):
        assert numpy.array_equal(got["site%d" % i], d.lmps[i].dense.numpy())
    for i in range(d.nsite + 1):
        assert numpy.array_equal(got["qnum%d" % i], d.qnuml[i])
    # the loaded state restarts the sweep where it was: the same energy as the original
    e0 = d.sweep("R", 16, 1e-8)[1]
    from qcmpodmrg_b200.dmrg import DMRG
    d2 = DMRG(d.ham, device="cpu")
    d2.load_mps(got)
    assert abs(d2.sweep("R", 16, 1e-8)[1] - e0) <= 1e-10


@needs_ref
def test_reference_reads_our_files_and_we_read_its_tensors(monkeypatch, tmp_path):
    import reference_runner  # noqa: F401  (puts the converted reference and the shims on sys.path)
    from qcmpodmrg.source import mpo_dmrg_io
    from qcmpodmrg.source.qtensor import qtensor
    from qcmpodmrg_b200.mps_io import save_mps, load_qtensor
    d = _swept(monkeypatch)
    f = _h5(tmp_path, "mps_ref")
    save_mps(f, d, qt=True)
    sites, qnums = mpo_dmrg_io.loadMPS(f, icase=2)
    for i in range(d.nsite):
        st, q = d.lmps[i], sites[i]
        assert numpy.array_equal(numpy.asarray(q.value), st.values.numpy())
        assert numpy.array_equal(numpy.asarray(q.idx_allowed), st.layout.idx_allowed)
        assert numpy.array_equal(numpy.asarray(q.ioff_allowed)[q.idx_allowed], st.layout.ioff[st.layout.idx_allowed])
        for k in range(st.layout.rank):
            assert numpy.array_equal(numpy.asarray(q.qsyms[k]), st.layout.qsyms[k])
            assert numpy.array_equal(numpy.asarray(q.ndims[k]), st.layout.ndims[k])
        assert numpy.array_equal(numpy.asarray(qnums[i]), d.qnuml[i])
    # a tensor of the reference's own making, dumped by its qtensor.dump
    rng = numpy.random.default_rng(2)
    ql = numpy.array([[0.0, 0.0], [1.0, 0.5], [1.0, -0.5], [2.0, 0.0]])
    qp = numpy.array([[0.0, 0.0], [1.0, -0.5], [1.0, 0.5], [2.0, 0.0]])
    qr = (ql[:, None, :] + qp[None, :, :]).reshape(-1, 2)
    t = qtensor.qtensor(numpy.array([False, False, True]))
    t.fromDenseTensor(rng.standard_normal((4, 4, 16)), [ql, qp, qr])
    t.dump(f, "refsite")
    lay, values, idlst = load_qtensor(f, "refsite")
    assert numpy.array_equal(values, numpy.asarray(t.value))
    assert numpy.array_equal(lay.idx_allowed, numpy.asarray(t.idx_allowed))
    assert numpy.array_equal(lay.ioff[lay.idx_allowed], numpy.asarray(t.ioff_allowed)[t.idx_allowed])
    dense = numpy.zeros(int(numpy.prod(lay.shape)))
    dense[lay.prjmap(idlst)] = values
    assert numpy.array_equal(dense.reshape(lay.shape), t.toDenseTensor(t.idlst))


@needs_ref
def test_we_read_files_the_reference_writes(monkeypatch, tmp_path):
    """An MPS written by the reference's own saveSite / saveQnum (dense and qtensor sites)
    loads into the same start state."""
    import reference_runner  # noqa: F401
    from qcmpodmrg.source import mpo_dmrg_io
    from qcmpodmrg.source.qtensor import qtensor
    from qcmpodmrg_b200.mps_io import load_mps
    d = _swept(monkeypatch)
    for qt in (False, True):
        f = _h5(tmp_path, "mps_written_by_ref_%d" % qt)
        f["nsite"] = d.nsite
        for i in range(d.nsite + 1):
            mpo_dmrg_io.saveQnum(f, i, numpy.asarray(d.qnuml[i]))
        for i in range(d.nsite):
            dense = d.lmps[i].dense.numpy()
            if qt:
                t = qtensor.qtensor(numpy.array([False, False, True]))
                t.fromDenseTensor(dense, [d.qnuml[i], numpy.array([[0., 0.], [1., -0.5], [1., 0.5], [2., 0.]]),
                                          d.qnuml[i + 1]])
                mpo_dmrg_io.saveSite(f, i, t)
            else:
                mpo_dmrg_io.saveSite(f, i, dense)
        got = load_mps(f)
        for i in range(d.nsite):
            assert numpy.array_equal(got["site%d" % i], d.lmps[i].dense.numpy())
            assert numpy.array_equal(got["qnum%d" % i], d.qnuml[i])
