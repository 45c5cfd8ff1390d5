"""Generate the golden fixtures under tests/golden/ from the reference itself.

Requires the converted reference (python tests/golden/convert_reference.py)
and the reference's sources (environment QCMPODMRG_REFERENCE); run where they are present:

    python tests/golden/make_golden.py            # small fixtures (seconds)
    python tests/golden/make_golden.py --config1  # K=12, N=12, D=100, 6 sweeps (~30 min CPU)
    python tests/golden/make_golden.py --config1-converged   # the same to convergence (hours of CPU)
    python tests/golden/make_golden.py --spin     # spin-projected K=4 / K=5 runs (minutes)
    python tests/golden/make_golden.py --noise    # K=5 / K=6 runs with the pRDM noise term
    python tests/golden/make_golden.py --sliced   # K=5 run with the MPO bond in 3 slices (maxslc=3)
    python tests/golden/make_golden.py --filling  # K=5 runs with N=2 and N=8 electrons

Outputs:
  qsym_cases.npz       symAllowed masks from the reference's own libqsym.so
  kernels_<tag>.npz    HVecQt/HDiagQt/renormQt_H00 inputs and outputs at chosen dots
  sweep_<tag>.npz      sweep energies/discarded weights/matvec counts + initial Qt L-MPS
"""
import argparse
import ctypes
import os
import sys

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import reference_runner as rr  # noqa: E402
import fixtures  # noqa: E402

REPO = os.path.dirname(os.path.dirname(HERE))


def qsym_cases(seed=7):
    lib = ctypes.CDLL(os.path.join(REPO, "baseline", "_ref", "qcmpodmrg", "libs", "libqsym.so"))
    rng = numpy.random.default_rng(seed)
    cases = []
    for rank in [2, 3, 3, 4, 4, 5, 6, 7, 8]:
        nqnum = int(rng.integers(1, 3))
        ndims = rng.integers(1, 6, size=rank).astype(numpy.int32)
        if rank == 8:   # the reference's rank-8 loop runs its last index over ndims[6] (qsym.c:436)
            ndims[7] = ndims[6]
        status = rng.integers(0, 2, size=rank).astype(numpy.int32)
        qs = [(rng.integers(-4, 5, size=(int(n), nqnum)) / 2.0).astype(numpy.float64) for n in ndims]
        nblks = int(numpy.prod(ndims))
        allowed = numpy.zeros(nblks, dtype=numpy.int32)
        args = [q.ctypes.data_as(ctypes.c_void_p) for q in qs] + [None] * (8 - rank)
        lib.symAllowed(ctypes.c_int(rank), ctypes.c_int(nqnum), ndims.ctypes.data_as(ctypes.c_void_p),
                       status.ctypes.data_as(ctypes.c_void_p), allowed.ctypes.data_as(ctypes.c_void_p), *args)
        cases.append({"rank": rank, "nqnum": nqnum, "ndims": ndims, "status": status,
                      "qsyms": qs, "allowed": allowed.copy()})
    fixtures.save(os.path.join(HERE, "qsym_cases.npz"), {"cases": cases})
    print("qsym cases:", len(cases), "allowed counts", [int(c["allowed"].sum()) for c in cases])


def run_case(tag, K, N, D, nsweeps, seed, decay, targets, record_envs=True, npts=None, noise=0.0,
             quad="GaussLegendre", maxslc=1, tol=1.e-7):
    res, rec = rr.run_reference(K=K, N=N, D=D, nsweeps=nsweeps, seed=seed, decay=decay, targets=targets,
                                record_envs=record_envs, npts=npts, noise=noise, quad=quad, maxslc=maxslc,
                                tol=tol)
    sweep = {"K": K, "N": N, "D": D, "seed": seed, "decay": -1.0 if decay is None else float(decay),
             "nsweeps": nsweeps, "eav": res["eav"], "dwt": res["dwt"], "esweeps": res["esweeps"],
             "nmvp": res["nmvp"], "init_mps": {k: v for k, v in res["init_mps"].items() if k != "nsite"},
             "npts": 0 if npts is None else int(npts), "noise": float(noise), "quad": quad, "maxslc": maxslc,
             "tol": float(tol)}
    fixtures.save(os.path.join(HERE, "sweep_%s.npz" % tag), sweep)
    if targets:
        recs = []
        for k in targets:
            r = rec.records.get(k)
            if r and "hvec_x" in r:
                d = dict(r)
                d["key"] = numpy.array([k[0], 0 if k[1] == "L" else 1, k[2]])
                recs.append(d)
        fixtures.save(os.path.join(HERE, "kernels_%s.npz" % tag),
                      {"K": K, "N": N, "seed": seed, "decay": -1.0 if decay is None else float(decay),
                       "records": recs})
    print(tag, "eav", res["eav"], "nmvp", res["nmvp"])


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--config1", action="store_true")
    ap.add_argument("--config1-converged", action="store_true",
                    help="K=12, N=12, D=100 to convergence (Davidson and sweep tolerance 1e-9, up to 16 sweeps)")
    ap.add_argument("--spin", action="store_true", help="only the spin-projected (SP-MPS) fixtures")
    ap.add_argument("--noise", action="store_true", help="only the fixtures with the pRDM noise term")
    ap.add_argument("--sliced", action="store_true", help="only the run with the MPO bond cut into slices")
    ap.add_argument("--filling", action="store_true", help="only the runs away from half filling")
    a = ap.parse_args()
    if a.filling:
        run_case("K5N2", 5, 2, 16, 2, 4, None, [(0, "L", 2)])
        run_case("K5N8", 5, 8, 16, 2, 5, 2.0, [(0, "R", 1)])
        sys.exit(0)
    if a.sliced:
        run_case("SL_K5", 5, 4, 12, 3, 2, 2.0, [], record_envs=False, maxslc=3)
        sys.exit(0)
    if a.noise:
        run_case("NZ_K5", 5, 4, 12, 3, 2, 2.0, [(0, "R", 2), (0, "L", 1), (1, "L", 2)], noise=1e-4)
        run_case("NZ_K6", 6, 6, 14, 3, 3, None, [(0, "R", 3), (1, "L", 2)], noise=1e-3)
        run_case("NZSP_K5", 5, 4, 12, 1, 2, 2.0, [(0, "R", 2), (0, "L", 1)], npts=3, noise=1e-4)
        sys.exit(0)
    if a.spin:
        run_case("SP_K4", 4, 4, 16, 2, 1, None, [(0, "R", 1), (0, "L", 1), (1, "L", 2)], npts=3)
        run_case("SP_K5", 5, 4, 12, 3, 2, 2.0, [(0, "R", 2), (1, "L", 1)], npts=4)
        run_case("SPS_K4", 4, 4, 16, 1, 1, None, [(0, "L", 1)], npts=5, quad="Simpson")
        sys.exit(0)
    if a.config1:
        run_case("C1", 12, 12, 100, 6, 1, None, [], record_envs=False)
        sys.exit(0)
    if a.config1_converged:
        run_case("C1C", 12, 12, 100, 16, 1, None, [], record_envs=False, tol=1.e-9)
        sys.exit(0)
    qsym_cases()
    run_case("K4", 4, 4, 16, 2, 1, None, [(0, "R", 1), (0, "L", 1), (0, "R", 0), (0, "L", 2), (1, "R", 2)])
    run_case("K5", 5, 4, 12, 6, 2, 2.0, [(0, "R", 2), (0, "L", 1), (1, "L", 3)])
    run_case("K6", 6, 6, 20, 3, 3, None, [(0, "R", 3), (1, "L", 2)])
