"""Every sigma evaluation path gives the same H_eff . x at every dot of a real sweep
state (K=12, N=12, D=64): the grouped GEMM in the packed layout (reference order),
the panel GEMMs with the fiber kernel for the two MPO-site contractions, and the
fused two-site-W fiber kernel; FP64, and FP32 / split-TF32 within FP32 tolerance."""
import numpy
import pytest
import torch

from qcmpodmrg_b200.hamiltonian import make_hamiltonian
from qcmpodmrg_b200.synthetic import product_mps

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-12     # relative to max|sigma|
TOL_F32 = 2e-5      # relative 2-norm


def test_sigma_paths_agree_on_sweep_state(cuda):
    from qcmpodmrg_b200.dmrg import DMRG
    from qcmpodmrg_b200.kernels import SigmaOperator
    ham = make_hamiltonian(12, 12, 21, 3.0)
    d = DMRG(ham, device=cuda)
    d.load_mps(product_mps(ham))
    for D in (24, 64):
        d.sweep("R", D, 1e-7)
        d.sweep("L", D, 1e-7)
    d.sweep("R", 64, 1e-7)          # left environments of every dot are now current
    gen = torch.Generator(device="cpu").manual_seed(5)
    checked = 0
    for isite in range(0, d.nsite - 1):
        if (isite - 1) not in d.lenv or (isite + 2) not in d.renv:
            continue
        lay, idl, ref_sig, _ = d.dot_operators(isite)
        L, R = d.lenv[isite - 1], d.renv[isite + 2]
        Wi, Wj = d.mpo[isite], d.mpo[isite + 1]
        x = torch.randn(lay.size, dtype=torch.float64, generator=gen).to(cuda)
        y0 = ref_sig(x).cpu().numpy()
        scale = max(1.0, numpy.abs(y0).max())
        for opts in ({"use_fiber": False}, {"use_fiber": True, "fuse_w": False}, {"use_fiber": True, "fuse_w": True}):
            for prec in ("f64", "f32", "tf32x3"):
                s = SigmaOperator(d.ws, isite, lay, L, R, Wi, Wj, d.qkey, d.opers, d.hpwts, prec, **opts)
                y = s(x).cpu().numpy()
                if prec == "f64":
                    assert numpy.abs(y - y0).max() <= TOL_F64 * scale, (isite, opts)
                else:
                    assert numpy.linalg.norm(y - y0) <= TOL_F32 * numpy.linalg.norm(y0), (isite, opts, prec)
        checked += 1
    assert checked >= 5
