"""tcgen05 (kind::tf32) grouped block GEMM: dense known answers first, then the
sigma contraction with every block routed to the tensor-core tiles."""
import numpy
import pytest
import torch

from helpers import load, record_operators
from qcmpodmrg_b200 import native
from qcmpodmrg_b200.engine import TASK_DT, CONTRIB_DT, OP_DT, TC_CFG, TILES

pytestmark = pytest.mark.gpu

TOL_TF32 = 3e-3     # relative Frobenius error: TF32 operands (10-bit mantissa), FP32 accumulation


def _run(tasks, contribs, ops, A, B, C, opspan=1):
    dev = A.device
    t = torch.from_numpy(tasks.view(numpy.uint8).copy()).to(dev)
    c = torch.from_numpy(contribs.view(numpy.uint8).copy()).to(dev)
    o = torch.from_numpy(ops.view(numpy.uint8).copy()).to(dev)
    rc = native.lib().qc_bgemm_tf32(t.data_ptr(), len(tasks), opspan, c.data_ptr(), o.data_ptr(), 0,
                                    A.data_ptr(), B.data_ptr(), C.data_ptr(), TC_CFG,
                                    torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    assert native.lib().qc_tc_status() == 0


def _tiles(M, N, c_off, ldc, cb, ce, op_b=0, op_e=1):
    tm, tn = TILES[TC_CFG]
    out = []
    for m0 in range(0, M, tm):
        for n0 in range(0, N, tn):
            out.append((c_off, M, N, m0, n0, M, N, 0, ldc, 0, 1, cb, ce, op_b, op_e))
    return numpy.array(out, dtype=TASK_DT)


def test_tc_dense_single_tile(cuda):
    rng = numpy.random.default_rng(1)
    M, N, K = 100, 50, 40
    A = rng.standard_normal((M, K)).astype(numpy.float32)
    B = rng.standard_normal((K, N)).astype(numpy.float32)
    c = numpy.zeros(1, dtype=CONTRIB_DT)
    c["alpha"], c["K"], c["klo"] = 0.5, K, K
    c["a_ml"], c["a_kl"], c["b_kl"], c["b_nl"] = K, 1, N, 1
    ops = numpy.zeros(1, dtype=OP_DT)
    ops["alpha"] = 1.0
    dA = torch.from_numpy(A.ravel()).to(cuda)
    dB = torch.from_numpy(B.ravel()).to(cuda)
    dC = torch.full((M * N,), float("nan"), dtype=torch.float32, device=cuda)
    _run(_tiles(M, N, 0, N, 0, 1), c, ops, dA, dB, dC)
    ref = 0.5 * A.astype(numpy.float64) @ B.astype(numpy.float64)
    got = dC.cpu().numpy().reshape(M, N)
    assert numpy.linalg.norm(got - ref) <= TOL_TF32 * numpy.linalg.norm(ref)


def test_tc_dense_two_level_two_ops(cuda):
    """Two contributions (one with a two-level K map), two operators with their own bases."""
    rng = numpy.random.default_rng(2)
    M, N, K1, Kh, Kl = 130, 70, 24, 3, 12
    A1 = rng.standard_normal((M, K1)).astype(numpy.float32)
    B1 = rng.standard_normal((K1, N)).astype(numpy.float32)
    # second pair: K = (kh, kl) with A stored [kh][m][kl] and B stored [kh][kl][n]
    A2 = rng.standard_normal((Kh, M, Kl)).astype(numpy.float32)
    B2 = rng.standard_normal((Kh, Kl, N)).astype(numpy.float32)
    blob_a = numpy.concatenate([A1.ravel(), A2.ravel()])
    blob_b = numpy.concatenate([B1.ravel(), B2.ravel()])
    nops = 2
    A = numpy.concatenate([blob_a, 2.0 * blob_a])           # operator 1 sees doubled A
    B = numpy.concatenate([blob_b, blob_b])
    c = numpy.zeros(2, dtype=CONTRIB_DT)
    c["alpha"] = 1.0
    c[0]["K"], c[0]["klo"], c[0]["a_ml"], c[0]["a_kl"], c[0]["b_kl"], c[0]["b_nl"] = K1, K1, K1, 1, N, 1
    c[1]["a_off"], c[1]["b_off"] = A1.size, B1.size
    c[1]["K"], c[1]["klo"] = Kh * Kl, Kl
    c[1]["a_ml"], c[1]["a_kh"], c[1]["a_kl"] = Kl, M * Kl, 1
    c[1]["b_kh"], c[1]["b_kl"], c[1]["b_nl"] = Kl * N, N, 1
    ops = numpy.zeros(nops, dtype=OP_DT)
    ops["a_base"] = [0, blob_a.size]
    ops["b_base"] = [0, blob_b.size]
    ops["c_base"] = [0, M * N]
    ops["alpha"] = [1.0, -0.25]
    dA = torch.from_numpy(A).to(cuda)
    dB = torch.from_numpy(B).to(cuda)
    dC = torch.full((nops * M * N,), float("nan"), dtype=torch.float32, device=cuda)
    _run(_tiles(M, N, 0, N, 0, 2, 0, nops), c, ops, dA, dB, dC, opspan=nops)
    r0 = A1.astype(numpy.float64) @ B1 + numpy.einsum("hmk,hkn->mn", A2.astype(numpy.float64), B2)
    got = dC.cpu().numpy().reshape(nops, M, N)
    for o, ref in ((0, r0), (1, -0.25 * 2.0 * r0)):
        assert numpy.linalg.norm(got[o] - ref) <= TOL_TF32 * numpy.linalg.norm(ref)


@pytest.mark.parametrize("tag", ["K4", "K6"])
def test_sigma_tf32_all_blocks_on_tensor_cores(tag, cuda):
    from qcmpodmrg_b200.kernels import SigmaOperator
    import helpers
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, dg, ws = record_operators(r, cuda, precision="tf32")
        # rebuild with every block of the L.psi and .R contractions on tcgen05 tiles
        sig = SigmaOperator(ws, int(r["key"][2]), helpers.layout_of(r["qtmp"]), sig.L, sig.R, sig.Wi, sig.Wj,
                            numpy.asarray(r["qkey"], dtype=numpy.float64),
                            [int(x) for x in numpy.atleast_1d(r["opers"])],
                            numpy.atleast_1d(r["hpwts"]).astype(numpy.float64), "tf32", tensor_cores="all",
                            panel1=False)
        x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64)).to(cuda)
        y = sig(x).cpu().numpy()
        ref = numpy.asarray(r["hvec_y"])
        assert numpy.linalg.norm(y - ref) <= TOL_TF32 * numpy.linalg.norm(ref)
    assert native.lib().qc_tc_status() == 0


TOL_TF32X3 = 2e-5   # split TF32 (hi*hi + hi*lo + lo*hi): FP32-level relative error of sigma


@pytest.mark.parametrize("tag", ["K5", "K6"])
def test_sigma_tf32x3_panels(tag, cuda):
    """L.psi and .R panel GEMMs on the tensor cores with split operands reach FP32 accuracy."""
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, _, _ = record_operators(r, cuda, precision="tf32x3", use_fiber=True)
        x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64)).to(cuda)
        y = sig(x).cpu().numpy()
        ref = numpy.asarray(r["hvec_y"])
        assert numpy.linalg.norm(y - ref) <= TOL_TF32X3 * numpy.linalg.norm(ref)
        assert native.lib().qc_tc_status() == 0
