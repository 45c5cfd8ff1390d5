"""The allocation-free sigma entry point (qc_sigma_f64_noalloc), called through the
C-ABI, gives the same sigma as the regular path (qc_bgemm_f64 stages with
caller-provided scratch), on two calls in a row.

Host codes that keep the whole GPU memory budget to themselves cannot provide
the intermediate buffers the regular path needs; this entry point uses a fixed
device array inside the library instead.  This file is collected last.
"""
import ctypes

import numpy
import pytest
import torch

from helpers import load, record_operators
from qcmpodmrg_b200 import native

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-12   # same tolerance as the other FP64 sigma tests


def _call(sig, x, y):
    groups = []
    for si, st in enumerate(sig.stages):
        for (cfg, tk, ct, dt, dc, span) in st.groups:
            groups.append((si, dt.data_ptr(), len(tk), span, dc.data_ptr(), cfg))
    n = len(groups)
    stage = (ctypes.c_int * n)(*[g[0] for g in groups])
    tasks = (ctypes.c_void_p * n)(*[g[1] for g in groups])
    ntasks = (ctypes.c_longlong * n)(*[g[2] for g in groups])
    span = (ctypes.c_int * n)(*[g[3] for g in groups])
    contribs = (ctypes.c_void_p * n)(*[g[4] for g in groups])
    cfg = (ctypes.c_int * n)(*[g[5] for g in groups])
    ops = (ctypes.c_void_p * 4)(*[st.d_ops.data_ptr() for st in sig.stages])
    lib = native.lib()
    return lib.qc_sigma_f64_noalloc(n, ctypes.addressof(stage), ctypes.addressof(tasks), ctypes.addressof(ntasks),
                                    ctypes.addressof(span), ctypes.addressof(contribs), ctypes.addressof(cfg),
                                    ctypes.addressof(ops), sig.L.values.data_ptr(), sig.Wi.values.data_ptr(),
                                    sig.Wj.values.data_ptr(), sig.R.values.data_ptr(), x.data_ptr(), y.data_ptr(),
                                    sig.nops, sig.ndim0, sig.tot[0], sig.tot[1], sig.tot[2],
                                    torch.cuda.current_stream().cuda_stream)


def test_noalloc_sigma_matches_regular_path(cuda):
    r = load("kernels_K6.npz")["records"][0]
    sig, dg, ws = record_operators(r, cuda, use_fiber=False, panel1=False)   # packed-layout stages
    gen = torch.Generator(device="cpu").manual_seed(7)
    for call in range(2):
        x = torch.randn(sig.ndim0, dtype=torch.float64, generator=gen).to(cuda)
        ref = sig(x).cpu().numpy()
        y = torch.full((sig.ndim0,), float("nan"), dtype=torch.float64, device=cuda)
        assert _call(sig, x, y) == 0
        torch.cuda.synchronize()
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
    tot = sig.tot
    sig.tot = [1 << 30, tot[1], tot[2]]      # pretend the first intermediate needs 8 GiB
    try:
        assert _call(sig, x, y) == -2         # QC_ERR_CAPACITY, nothing queued
    finally:
        sig.tot = tot
