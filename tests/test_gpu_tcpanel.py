"""The TMA-fed tcgen05 panel GEMM (qc_tcpanel_f32): dense known answers against an FP64
product of the same operands (several row tiles, a partial K stage, two column tiles,
two operators with their own weights), then sigma of reference dots with the .R
contraction on it (split TF32: FP32-level accuracy)."""
import numpy
import pytest
import torch

from helpers import load, record_operators
from qcmpodmrg_b200 import native
from qcmpodmrg_b200.engine import TCPanelStage, tc_sigma4_units, op_table

pytestmark = pytest.mark.gpu

TOL_TF32X3 = 2e-5   # split TF32 (hi*hi + hi*lo + lo*hi): relative Frobenius error


def _pad(n, q=32):
    return (n + q - 1) // q * q


@pytest.mark.parametrize("shape", [(300, 150, 100), (128, 32, 16), (77, 5, 9), (130, 301, 150)])
def test_tcpanel_dense_known_answer(cuda, shape):
    M, N, K = shape
    nops = 2
    rng = numpy.random.default_rng(M + N + K)
    Kp = (K + 3) // 4 * 4
    sa, sb = _pad(M * Kp), _pad(N * Kp)
    A = numpy.zeros(nops * sa, dtype=numpy.float32)
    Bh = numpy.zeros(nops * sb, dtype=numpy.float32)
    a = rng.standard_normal((nops, M, K)).astype(numpy.float32)
    b = rng.standard_normal((nops, N, K)).astype(numpy.float32)
    for o in range(nops):
        A[o * sa:o * sa + M * Kp].reshape(M, Kp)[:, :K] = a[o]
        Bh[o * sb:o * sb + N * Kp].reshape(N, Kp)[:, :K] = b[o]
    tot = nops * sb
    dA = torch.from_numpy(A).to(cuda)
    dB = torch.zeros(2 * tot, dtype=torch.float32, device=cuda)
    dB[:tot] = torch.from_numpy(Bh).to(cuda)
    assert native.lib().qc_tf32_split(dB.data_ptr(), dB[tot:].data_ptr(), tot,
                                      torch.cuda.current_stream().cuda_stream) == 0
    sec = {"used": numpy.array([0]), "K": numpy.array([K]), "M": numpy.array([M]), "N": numpy.array([N]),
           "Kp": numpy.array([Kp]), "t3pan": numpy.array([0]), "rtoff": numpy.array([0]),
           "crow_base": numpy.array([0])}
    units, maps = tc_sigma4_units([([0, 1], sec, sa)], None, [0], [0], [sb], tot)
    alpha = numpy.array([0.5, -1.25])
    ops = op_table(0, 0, numpy.arange(nops) * M * N, alpha)
    crow = numpy.arange(M, dtype=numpy.int64) * N
    st = TCPanelStage("dense", units, maps, ops, crow, 2.0 * M * N * K * nops, cuda)
    C = torch.full((nops * M * N,), float("nan"), dtype=torch.float32, device=cuda)
    native.lib().qc_tcpanel_status(1)
    st.run(dA, dB, C)
    torch.cuda.synchronize()
    assert native.lib().qc_tcpanel_status(1) == 0
    got = C.cpu().numpy().astype(numpy.float64).reshape(nops, M, N)
    for o in range(nops):
        ref = alpha[o] * a[o].astype(numpy.float64) @ b[o].astype(numpy.float64).T
        assert numpy.isfinite(got[o]).all()
        assert numpy.linalg.norm(got[o] - ref) <= TOL_TF32X3 * numpy.linalg.norm(ref), o


@pytest.mark.parametrize("tag", ["K5", "K6", "K5N8"])
def test_sigma_with_tensor_core_panels(tag, cuda):
    """L.psi and .R both on the TMA-fed tensor-core kernel (column segments into the T1
    panels, row table into sigma)."""
    for r in load("kernels_%s.npz" % tag)["records"]:
        sig, _, _ = record_operators(r, cuda, precision="tf32x3", use_fiber=True, fuse_w=False)
        assert sig.tc4 is not None and sig.tc1 is not None
        x = torch.from_numpy(numpy.asarray(r["hvec_x"], dtype=numpy.float64)).to(cuda)
        native.lib().qc_tcpanel_status(1)
        y = sig(x).cpu().numpy()
        assert native.lib().qc_tcpanel_status(1) == 0
        ref = numpy.asarray(r["hvec_y"])
        assert numpy.linalg.norm(y - ref) <= TOL_TF32X3 * numpy.linalg.norm(ref)
        # the same plan in FP64 (CUDA cores, padded T3 rows) stays exact
        y64 = sig(x, precision="f64").cpu().numpy()
        assert numpy.abs(y64 - ref).max() <= 1e-12 * max(1.0, numpy.abs(ref).max())
