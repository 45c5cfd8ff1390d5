"""GPU parity of the fiber-group kernel (qc_fiber_f64 / qc_fiber_f32) used for the
two MPO-site contractions of sigma: against the reference's own sigma and against
the grouped-GEMM stages on the same plan."""
import numpy
import pytest
import torch

from helpers import load, record_operators
from qcmpodmrg_b200.engine import CompositeStage, FiberStage

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-12      # relative to max|sigma|: FP64, different summation order
TOL_F32 = 2e-5       # relative 2-norm: FP32 operands and accumulation


@pytest.mark.parametrize("tag", ["K4", "K5", "K6"])
def test_fiber_sigma_f64_matches_reference_and_generic(tag, cuda):
    gen = torch.Generator(device="cpu").manual_seed(3)
    for r in load("kernels_%s.npz" % tag)["records"]:
        ref_sig, _, _ = record_operators(r, cuda, use_fiber=False)
        xr = torch.randn(ref_sig.ndim0, dtype=torch.float64, generator=gen).to(cuda)
        b = ref_sig(xr).cpu().numpy()
        for fuse in (True, False):
            sig, _, _ = record_operators(r, cuda, use_fiber=True, fuse_w=fuse)
            subs = [x for s in sig.stages if isinstance(s, CompositeStage) for x in s.subs]
            assert sig.fused is not None or any(isinstance(x, FiberStage) for x in subs)
            x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64)).to(cuda)
            y = sig(x).cpu().numpy()
            ref = numpy.asarray(r["hvec_y"])
            assert numpy.abs(y - ref).max() <= TOL_F64 * max(1.0, numpy.abs(ref).max())
            assert numpy.array_equal(y, sig(x).cpu().numpy()), "bitwise reproducible"
            a = sig(xr).cpu().numpy()
            assert numpy.abs(a - b).max() <= TOL_F64 * max(1.0, numpy.abs(b).max())


@pytest.mark.parametrize("tag", ["K5", "K6"])
def test_fiber_sigma_f32(tag, cuda):
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, _, _ = record_operators(r, cuda, precision="f32", use_fiber=True)
        x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64)).to(cuda)
        y = sig(x).cpu().numpy()
        ref = numpy.asarray(r["hvec_y"])
        assert numpy.linalg.norm(y - ref) <= TOL_F32 * numpy.linalg.norm(ref)
