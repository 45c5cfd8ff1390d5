"""Mixed precision: FP32 (CUDA cores) and TF32 (tensor cores) sigma inside the
Davidson, FP64 Rayleigh quotient / residual check / decimation, converge to the
FP64 energy within 1e-6 Eh on the same seeded inputs."""
import numpy
import pytest

from qcmpodmrg_b200.hamiltonian import make_hamiltonian
from qcmpodmrg_b200.synthetic import product_mps

pytestmark = pytest.mark.gpu

TOL_E = 1e-6        # |E_mixed - E_FP64| at convergence (Eh)


def _converged(cuda, precision, w_path, K=10, D=48, nsweeps=12):
    from qcmpodmrg_b200.dmrg import DMRG
    ham = make_hamiltonian(K, K, 11, 3.0)
    d = DMRG(ham, device=cuda, precision=precision, w_path=w_path)
    out = d.run(product_mps(ham), D, nsweeps, tol=1e-8)
    return out, d.stats


@pytest.mark.parametrize("precision", ["f32", "tf32", "tf32x3"])
def test_mixed_converges_to_fp64(cuda, precision):
    ref, _ = _converged(cuda, "f64", "fiber")
    got, st = _converged(cuda, precision, "fiber")
    print(precision, "E64 %.10f  Emixed %.10f  matvecs f64/low %s/%s" % (
        ref["eav"][-1], got["eav"][-1], st.get("nmvp_f64"), st.get("nmvp_low")))
    assert abs(got["eav"][-1] - ref["eav"][-1]) <= TOL_E
    assert st.get("nmvp_low", 0) > st.get("nmvp_f64", 0)      # most matvecs in low precision


def test_mixed_converges_to_fp64_k14_d128(cuda):
    """A larger converged pair (K=14, D=128, decay 3): FP32 sigma inside the Davidson, one
    FP64 product per dot for the energy, against the plain FP64 run."""
    ref, st64 = _converged(cuda, "f64", "fiber", K=14, D=128, nsweeps=16)
    got, st = _converged(cuda, "f32", "fiber", K=14, D=128, nsweeps=16)
    print("K=14 D=128: E64 %.10f (%d sweeps, %d matvecs)  Emixed %.10f (%d sweeps, matvecs f64/low %s/%s)" % (
        ref["eav"][-1], len(ref["eav"]), st64["nmvp"], got["eav"][-1], len(got["eav"]), st.get("nmvp_f64"),
        st.get("nmvp_low")))
    assert abs(got["eav"][-1] - ref["eav"][-1]) <= TOL_E
    assert st.get("nmvp_low", 0) > 2 * st.get("nmvp_f64", 0)
