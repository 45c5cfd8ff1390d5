"""ORACLE -- test infrastructure, not product.

A CPU (NumPy/SciPy, FP64) restatement of the reference's two-site Qt DMRG hot
path: block layout and pair lists (blocks.py), the H_p site operators (mpo.py),
sigma/diagonal/renormalisation and the pRDM noise term (kernels.py), Davidson
and RDM decimation (solver.py), the sweep driver (dmrg.py) and spin projection
(spin.py: quadrature, H_p R(theta) operators, SVecQt/SDiagQt/renormQt_S00, the
generalised Davidson and the projected sweep).  Each function cites the reference
file:line it follows.  It is pinned against outputs of the reference itself,
run here through tests/golden/convert_reference.py, stored as fixtures under
tests/golden/.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm may import this package.  The product (qcmpodmrg_b200) never imports it.
"""
