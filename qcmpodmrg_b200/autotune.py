"""Measured choice of the sigma kernels' schedule parameters.

The dense fiber-group GEMM (qc_fgemm, the .W_i and .W_{i+1} contractions of HVecQt,
source/mpo_dmrg_kernelQt.py:301-306) stages, per (work item, operator) step, an A tile of
FT fibers x R contracted rows and the operator's W panel [R x CT] in shared memory, twice
(double buffer).  The two element budgets of those buffers set

  * FT, the fibers of a work item (the largest multiple of 4 whose tile fits the A budget
    and fills the CTA's threads),
  * the width of the column slices wide W panels are cut into, and
  * the dynamic shared memory of the launch, hence how many CTAs share an SM.

Larger budgets stage more work per step; smaller ones let more CTAs hide each other's
latency.  Which wins depends on the block-size histogram of the dot (bond dimension,
sector structure, MPO bond) and on the precision (FP64 needs twice the bytes).  The tuner
compiles the sigma plan of one representative dot for each candidate, checks that every
candidate gives the same sigma (each output element is still one sum over the same
contracted rows in the same order; the check allows rounding, 1e-12 relative in FP64 and
1e-5 otherwise), times the matrix-vector products with CUDA events and keeps the
fastest.  The choice is cached per (precision, bond dimension) and applied to every later
plan of the run (DMRG.sigma_opts).
"""
import time

import numpy
import torch

from .engine import FG_A_BUDGET, FG_W_BUDGET

# (A elements, W elements) per shared-memory buffer.  FP32 shared memory per CTA is about
# 8 (A + W) bytes plus 64 bytes per panel column: 4096/4096 gives three CTAs per SM,
# 3072/3072 four, 2304/2304 five.
CANDIDATES = ((FG_A_BUDGET, FG_W_BUDGET), (3072, 3072), (2304, 2304), (1792, 1792), (3072, 1536), (1536, 3072))

_CACHE = {}


def _time_sigma(sig, x, precision, repeats):
    """Mean CUDA-event time (ms) of one sigma application on the current stream."""
    y = sig(x, precision=precision)           # warm-up (W panels, tensor maps, workspace)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(repeats):
        sig(x, precision=precision)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / repeats, y


def tune_fiber_budget(d, isite=None, candidates=CANDIDATES, repeats=4, precision=None):
    """Pick the fiber-GEMM budgets for DMRG ``d`` at dot ``isite`` (default: the middle of
    the chain) in ``precision`` (default: the run's); stores the choice in d.sigma_opts and
    returns a report {"choice", "table": [(budget, ms)], "dot", "ndim0", "s"}."""
    if not d.sigma_opts.get("use_fiber", False):
        return {"choice": None, "reason": "the fiber-group kernels are not used by this sigma path"}
    prec = precision or d.precision
    dmax = int(max(len(q) for q in d.qnuml if q is not None))
    key = (prec, dmax, str(torch.cuda.get_device_name(d.device)))
    if key in _CACHE:
        d.sigma_opts["fg_budget"] = _CACHE[key]["choice"]
        return dict(_CACHE[key], cached=True)
    isite = d.nsite // 2 if isite is None else int(isite)
    t0 = time.time()
    saved = d.sigma_opts.get("fg_budget")
    cache_size, d.plan_cache_size = d.plan_cache_size, 0       # every candidate compiles its own plan
    d.plan_cache.clear()
    table, ref, ndim0 = [], None, 0
    x = None
    for cand in candidates:
        d.sigma_opts["fg_budget"] = tuple(int(v) for v in cand)
        lay, idl, sig, dg = d.dot_operators(isite)
        if x is None:
            ndim0 = int(sig.ndim0)
            x = torch.from_numpy(numpy.random.default_rng(7).standard_normal(ndim0)).to(d.device)
        ms, y = _time_sigma(sig, x, prec, repeats)
        if ref is None:
            ref = y
            tol = (1e-12 if prec == "f64" else 1e-5) * max(float(ref.abs().max()), 1e-300)
        elif not float((y - ref).abs().max()) <= tol:
            raise RuntimeError("autotune: fiber-GEMM budget %s changed the sigma (max |diff| %.3e)"
                               % (cand, float((y - ref).abs().max())))
        table.append((tuple(int(v) for v in cand), round(ms, 4)))
        del sig, dg
    best = min(table, key=lambda t: t[1])[0]
    d.sigma_opts["fg_budget"] = best if best != (FG_A_BUDGET, FG_W_BUDGET) else saved
    d.plan_cache_size = cache_size
    d.plan_cache.clear()
    rep = {"choice": best, "table": table, "dot": isite, "ndim0": ndim0, "precision": prec, "bond": dmax,
           "s": round(time.time() - t0, 2)}
    _CACHE[key] = rep
    return rep
