"""GPU parity: the sm_100a kernels, called through the C-ABI, against the reference's
own outputs (tests/golden) and the oracle."""
import numpy
import pytest
import torch

from helpers import load, record_operators, record_renormalizer
from qcmpodmrg_b200 import native

pytestmark = pytest.mark.gpu

# FP64 tolerance: sums of O(100) products of O(1) numbers, different summation order
TOL_F64 = 1e-12
# FP32 operands and accumulation: relative error of the sigma vector
TOL_F32 = 2e-5


@pytest.mark.parametrize("tag", ["K4", "K5", "K6", "K5N2", "K5N8"])
def test_sigma_diag_renorm_f64(tag, cuda):
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, dg, ws = record_operators(r, cuda)
        x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64)).to(cuda)
        y = sig(x).cpu().numpy()
        ref = numpy.asarray(r["hvec_y"])
        assert numpy.abs(y - ref).max() <= TOL_F64 * max(1.0, numpy.abs(ref).max())
        y2 = sig(x).cpu().numpy()
        assert numpy.array_equal(y, y2), "sigma must be bitwise reproducible"
        d = dg().cpu().numpy()
        assert numpy.abs(d - numpy.asarray(r["hdiag"])).max() <= TOL_F64
        rn, site = record_renormalizer(r, cuda)
        out = rn(torch.from_numpy(site).to(cuda))
        for i, b in enumerate(r["renorm_out"]):
            got = out.op_values(i).cpu().numpy()
            assert numpy.abs(got - b["value"]).max() <= TOL_F64


@pytest.mark.parametrize("tag", ["K4", "K6"])
def test_sigma_f32(tag, cuda):
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, dg, ws = record_operators(r, cuda, precision="f32")
        x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64)).to(cuda)
        y = sig(x).cpu().numpy()
        ref = numpy.asarray(r["hvec_y"])
        assert numpy.linalg.norm(y - ref) <= TOL_F32 * numpy.linalg.norm(ref)


def test_sym_allowed_gpu_matches_reference(cuda):
    lib = native.lib()
    from qcmpodmrg_b200.qtensor import qint
    for c in load("qsym_cases.npz")["cases"]:
        rank = int(c["rank"])
        nd = numpy.ascontiguousarray(c["ndims"], dtype=numpy.int32)
        st = numpy.ascontiguousarray(c["status"], dtype=numpy.int32)
        q2 = numpy.concatenate([qint(numpy.asarray(x).reshape(int(n), -1)) for x, n in zip(c["qsyms"], nd)]).ravel()
        dq = torch.from_numpy(q2.astype(numpy.int32)).to(cuda)
        out = torch.full((int(numpy.prod(nd)),), -1, dtype=torch.int32, device=cuda)
        rc = lib.qc_sym_allowed_gpu(rank, int(c["nqnum"]), nd.ctypes.data, st.ctypes.data, dq.data_ptr(),
                                    out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        assert rc == 0
        assert numpy.array_equal(out.cpu().numpy(), c["allowed"])
