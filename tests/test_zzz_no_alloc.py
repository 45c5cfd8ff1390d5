"""The allocation-free sigma entry point (qc_sigma_f64_noalloc), called through the
C-ABI, gives the same sigma as the regular path (qc_bgemm_f64 stages with
caller-provided scratch), on two calls in a row, on a stream of its own, without
allocating device memory.

Host codes that keep the whole GPU memory budget to themselves (a parent
application that reserves device memory for its own pool up front, or a solver
that must not trigger cudaMalloc's device-wide synchronisation between
iterations) cannot provide the intermediate buffers the regular path needs; this
entry point uses a fixed device array inside the library instead.  Only plans of
packed-layout grouped-GEMM groups are accepted; the default plan (dense panels,
fiber groups) is refused.  This file is collected last.
"""
import ctypes

import numpy
import pytest
import torch

from helpers import load, record_operators
from qcmpodmrg_b200 import native

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-12   # same tolerance as the other FP64 sigma tests
QC_ERR_ARG, QC_ERR_CAPACITY = -1, -2


def _ops_ptr(st):
    """Device operator table of a stage (of its first sub-stage for composite stages)."""
    if hasattr(st, "d_ops"):
        return st.d_ops.data_ptr()
    sub = st.subs[0]
    return sub.d_ops.data_ptr() if hasattr(sub, "d_ops") else sub.d[4].data_ptr()


def _call(sig, x, y, stream=None, tot=None):
    groups = sig.work_groups()
    n = len(groups)
    col = lambda k, ct: (ct * n)(*[g[k] for g in groups])
    stage, kind, tasks = col(0, ctypes.c_int), col(1, ctypes.c_int), col(2, ctypes.c_void_p)
    ntasks, span = col(3, ctypes.c_longlong), col(4, ctypes.c_int)
    contribs, cfg = col(5, ctypes.c_void_p), col(6, ctypes.c_int)
    ops = (ctypes.c_void_p * 4)(*[_ops_ptr(st) for st in sig.stages])
    t1, t2, t3 = tot or sig.tot
    s = (stream or torch.cuda.current_stream()).cuda_stream
    return native.lib().qc_sigma_f64_noalloc(
        n, ctypes.addressof(stage), ctypes.addressof(tasks), ctypes.addressof(ntasks), ctypes.addressof(span),
        ctypes.addressof(contribs), ctypes.addressof(cfg), ctypes.addressof(kind), ctypes.addressof(ops),
        sig.L.values.data_ptr(), sig.Wi.values.data_ptr(), sig.Wj.values.data_ptr(), sig.R.values.data_ptr(),
        x.data_ptr(), y.data_ptr(), sig.nops, sig.ndim0, t1, t2, t3, s)


def _alloc_count():
    st = torch.cuda.memory_stats()
    return st.get("allocation.all.allocated", 0), torch.cuda.mem_get_info()[0]


def test_noalloc_sigma_matches_regular_path(cuda):
    r = load("kernels_K6.npz")["records"][0]
    sig, dg, ws = record_operators(r, cuda, use_fiber=False, panel1=False)   # packed-layout stages
    assert all(g[1] == native.GROUP_BGEMM for g in sig.work_groups())
    gen = torch.Generator(device="cpu").manual_seed(7)
    side = torch.cuda.Stream()
    for call in range(2):
        x = torch.randn(sig.ndim0, dtype=torch.float64, generator=gen).to(cuda)
        ref = sig(x).cpu().numpy()
        y = torch.full((sig.ndim0,), float("nan"), dtype=torch.float64, device=cuda)
        torch.cuda.synchronize()
        before = _alloc_count()
        side.wait_stream(torch.cuda.current_stream())
        assert _call(sig, x, y, stream=side) == 0           # a stream of its own
        side.synchronize()
        after = _alloc_count()
        if call == 1:      # the first call may load the library's kernels; the second allocates nothing
            assert after == before, (before, after)
        got = y.cpu().numpy()
        assert numpy.abs(got - ref).max() <= TOL_F64 * max(1.0, numpy.abs(ref).max()), call
    # the reference's own sigma for the recorded vector, through the allocation-free path
    x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64)).to(cuda)
    y = torch.empty(sig.ndim0, dtype=torch.float64, device=cuda)
    assert _call(sig, x, y) == 0
    ref = numpy.asarray(r["hvec_y"])
    assert numpy.abs(y.cpu().numpy() - ref).max() <= TOL_F64 * max(1.0, numpy.abs(ref).max())


def test_noalloc_rejects_oversized_dot(cuda):
    r = load("kernels_K4.npz")["records"][0]
    sig, dg, ws = record_operators(r, cuda, use_fiber=False, panel1=False)   # packed-layout stages
    x = torch.zeros(sig.ndim0, dtype=torch.float64, device=cuda)
    y = torch.zeros(sig.ndim0, dtype=torch.float64, device=cuda)
    # pretend the first intermediate needs 8 GiB: refused, nothing queued
    assert _call(sig, x, y, tot=[1 << 30, sig.tot[1], sig.tot[2]]) == QC_ERR_CAPACITY


def test_noalloc_refuses_panel_and_fiber_plans(cuda):
    """The default sigma plan (dense panels for L.psi and .R, fiber groups for the MPO
    sites) reads other operands through other work-item records: refused before any launch."""
    r = load("kernels_K6.npz")["records"][0]
    sig, dg, ws = record_operators(r, cuda, use_fiber=True, fuse_w=False, panel1=True)
    kinds = set(g[1] for g in sig.work_groups())
    assert native.GROUP_PANEL in kinds and native.GROUP_FIBER in kinds
    x = torch.zeros(sig.ndim0, dtype=torch.float64, device=cuda)
    y = torch.full((sig.ndim0,), 3.0, dtype=torch.float64, device=cuda)
    torch.cuda.synchronize()
    assert _call(sig, x, y) == QC_ERR_ARG
    torch.cuda.synchronize()
    assert bool((y == 3.0).all())                          # nothing ran
