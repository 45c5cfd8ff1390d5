"""Benchmark: two-site MPO-DMRG sweeps at K=24, N=24, Sz=0, D=500 on one B200.

Workload (the reference's config quoted by the metric): seeded synthetic
integrals (K=24 spatial orbitals, N=24 electrons, locality decay 3, seed 1),
the occupation-number product state as start, a bond-dimension ramp
D = 50, 100, 200 (set-up, untimed), then W warm-up and K timed steps.  One
step = one full two-site sweep (right-to-left then left-to-right) at D=500:
per dot the sigma/diagonal plans, Davidson (FP64 Rayleigh-Ritz), RDM
decimation and renormalisation of every operator's environment.

  python bench.py [--steps K] [--warmup W] [--precision mixed-tc|mixed|f64|tf32] [--gpus N]
                  [--w-path fiber|generic|fused] [--no-plan-cache] [--sites K] [--dmax D]
  python bench.py --impl reference      # the reference algorithm (oracle port) on the host CPU
  python bench.py --workload batched    # 64 independent instances in lockstep vs one after another
  python bench.py --workload sp --sites 12 --dmax 100 --npts 4   # spin-projected (S=0) sweeps, FP64
  python bench.py --workload dot --sites 24 --dmax 200   # one mid-chain dot's sigma (kernel profiles)
  python bench.py --workload converge --dmax 200 --steps 30   # mixed and FP64 to convergence, same start

Prints one JSON line.  value = seconds per sweep (lower is better).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sweep sec & sigma TFLOP/s @K=24,D=500: mixed+learned vs FP64, |ΔE|≤1e-6 Eh"
METRIC_SP = "spin-projected sweep sec (S=0 projector)"
K_SITES, N_ELEC, DECAY, SEED, DMAX = 24, 24, 3.0, 1, 500
RAMP = (50, 100, 200)
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return PEAKS_FALLBACK, "fallback"


class ClockSampler(object):
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(numpy.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(backend="nccl"):
    """One process per GPU (torchrun environment); replicas only: the process group
    carries the barrier and the max-over-ranks of the timings, no data."""
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        if backend == "nccl":
            torch.cuda.set_device(local)
        return dist, rank, ws, local
    return None, 0, 1, 0


def barrier(dist, cuda=True):
    import torch
    if dist is not None:
        dist.barrier()
    if cuda:
        torch.cuda.synchronize()


def max_over_ranks(dist, value, device="cuda"):
    """The largest value over all ranks (the job's time is that of its slowest replica)."""
    import torch
    if dist is None:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _make_dmrg(args, prec, dev, seed_rank=0):
    from qcmpodmrg_b200.hamiltonian import make_hamiltonian
    from qcmpodmrg_b200.synthetic import product_mps
    from qcmpodmrg_b200.dmrg import DMRG
    ham = make_hamiltonian(args.sites, args.sites, SEED + seed_rank * 0, DECAY)
    if args.workload == "sp":
        from qcmpodmrg_b200.spin import SPDMRG
        if prec not in ("f64", "f32"):
            raise SystemExit("--workload sp runs with --precision f64 or mixed")
        d = SPDMRG(ham, args.npts, 0.0, 0.0, device=dev, w_path=args.w_path, precision=prec)
    else:
        d = DMRG(ham, device=dev, precision=prec, w_path=args.w_path, plan_cache=args.plan_cache)
    if args.precond == "learned" and prec != "f64":
        from qcmpodmrg_b200.precond import LearnedPreconditioner
        d.preconditioner = LearnedPreconditioner(dev, train_sweeps=args.precond_train)
    d.load_mps(product_mps(ham))
    for D in RAMP:
        if D < args.dmax:
            d.sweep("R", D, 1e-7)
            d.sweep("L", D, 1e-7)
    return d


def _step(d, args):
    """One sweep (R then L) at D = dmax; returns (energy, discarded weight, matvecs)."""
    f0, n0 = d.stats["sigma_flops"], d.stats["nmvp"]
    d.sweep("R", args.dmax, 1e-7)
    n, e, dw, el, dl = d.sweep("L", args.dmax, 1e-7)
    d.sweep_sigma_flops = d.stats["sigma_flops"] - f0
    if hasattr(d.preconditioner, "end_sweep"):
        d.preconditioner.end_sweep()
    return e, dw, d.stats["nmvp"] - n0


def _timed_sweeps(d, args, nsteps, dist):
    """nsteps sweeps bracketed by barrier + synchronize, CUDA events on the launching
    stream before every sweep and after the last; returns (total ms, per-sweep ms, results)."""
    import torch
    barrier(dist)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(nsteps + 1)]
    res = []
    evs[0].record()
    for k in range(nsteps):
        res.append(_step(d, args))
        evs[k + 1].record()
    barrier(dist)
    per = [evs[k].elapsed_time(evs[k + 1]) for k in range(nsteps)]
    return evs[0].elapsed_time(evs[-1]), per, res


def run_ours(args):
    import gc
    import torch
    from qcmpodmrg_b200.engine import LOG

    dist, rank, world, local = dist_init()
    dev = torch.device("cuda:%d" % local)
    torch.cuda.set_device(dev)
    prec = {"mixed": "f32", "f64": "f64", "tf32": "tf32", "mixed-tc": "tf32x3"}[args.precision]
    sp = args.workload == "sp"
    d = _make_dmrg(args, prec, dev, rank)
    tuned = {}
    if args.autotune and not sp:
        # measured choice of the fiber-GEMM schedule at the mid-chain dot, for this arm's
        # precision and for the FP64 arm (both applied to every later plan of their run)
        from qcmpodmrg_b200.autotune import tune_fiber_budget
        tuned[prec] = tune_fiber_budget(d)
        if prec != "f64" and args.f64_steps > 0:
            tuned["f64"] = tune_fiber_budget(d, precision="f64")
            d.sigma_opts["fg_budget"] = tuned[prec]["choice"]
    warm = [_step(d, args) for _ in range(args.warmup)]
    snap = d.snapshot()          # the state the timed sweeps start from (e2e, accuracy and FP64 legs)
    # ---- timed region (device events on the launching stream, barrier + sync both sides)
    s0 = {k: v for k, v in d.stats.items() if not isinstance(v, dict)}
    LOG.reset()
    LOG.enabled = True
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.nvtx.range_push("timed")
    ms_local, per_sweep, energies = _timed_sweeps(d, args, args.steps, dist)
    torch.cuda.nvtx.range_pop()
    ck = clocks.stop()
    LOG.enabled = False
    ms = max_over_ranks(dist, ms_local, dev)
    ms_per_step = ms / args.steps
    stats = {k: d.stats[k] - s0[k] for k in s0}
    # per-stage device time from the launch log
    per = {}
    for (name, e0, e1, fl, by) in LOG.records:
        t = e0.elapsed_time(e1)
        a = per.setdefault(name, [0, 0.0, 0.0, 0.0])
        a[0] += 1
        a[1] += t
        a[2] += fl
        a[3] += by
    sig_ms = sum(v[1] for k, v in per.items() if k.startswith("sigma"))
    sig_fl = stats["sigma_flops"]     # the reference chain's algorithmic FLOPs, whatever the fusion
    top = max(per.items(), key=lambda kv: kv[1][1])
    pk, src = peaks()
    n_l, t_l, f_l, b_l = top[1]
    gbs = b_l / (t_l / 1e3) / 1e9
    kname = stage_kernel(top[0], args.w_path, prec)
    roof = {"kernel": "%s (%s)" % (kname, top[0]), "bound": "hbm", "achieved": round(gbs, 1),
            "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": round(gbs / pk["hbm_gbs"], 4),
            "peak_source": src, "traffic": traffic_per_launch(top[0], prec, b_l / max(n_l, 1)),
            "traffic_source": "ncu DRAM bytes per algorithmic byte of this stage at K=24 D=200, times this "
                              "launch's algorithmic bytes", "launches": n_l,
            "achieved_tflops": round(f_l / (t_l / 1e3) / 1e12, 3)}
    # whole job: world replicas each did args.steps sweeps in ms (slowest rank)
    line = {
        "metric": METRIC_SP if sp else METRIC, "value": round(ms_per_step / 1e3 / world, 3), "unit": "s/sweep",
        "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 1),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": {"f64": "f64", "f32": "f32 (sigma), f64 (Davidson, decimation)",
                  "tf32": "tf32 (sigma), f64 (Davidson, decimation)",
                  "tf32x3": "3xtf32 split on tensor cores + f32 (sigma), f64 (Davidson, decimation)"}[prec],
        "data": "synthetic: seeded integrals (K=%d, N=%d, decay 3, seed 1), product-state start, D ramp %s"
                % (args.sites, args.sites, "/".join(str(x) for x in RAMP if x < args.dmax)),
        "config": {"workload": ("spin-projected (S=0, %d Gauss-Legendre points) two-site Qt DMRG sweep, K=%d "
                                "N=%d Sz=0 D=%d, %d operators H_p R(theta_g) + %d projector terms"
                                % (args.npts, args.sites, args.sites, args.dmax, 2 * args.sites * args.npts,
                                   args.npts)) if sp else
                               "two-site Qt DMRG sweep, K=%d N=%d Sz=0 D=%d, %d operators H_p"
                               % (args.sites, args.sites, args.dmax, 2 * args.sites), "K": args.sites,
                   "N": args.sites, "D": args.dmax, "precision": args.precision,
                   "w_path": args.w_path, "precond": args.precond,
                   "l2": "inputs larger than L2: environments and sigma scratch are tens of GB per sweep",
                   "parallelism": "replicas" if world > 1 else "1 GPU",
                   "value_definition": "slowest rank's seconds for its sweeps / sweeps done by all ranks"},
        "energy": energies[-1][0], "dwt": energies[-1][1],
        "sweep_ms": [round(x, 1) for x in per_sweep],
        "sigma_tflops": round(sig_fl / (sig_ms / 1e3) / 1e12, 3) if sig_ms else None,
        "sigma_share": round(sig_ms / ms_local, 3) if ms_local else None,
        "matvecs_per_step": stats["nmvp"] / args.steps,
        "matvecs_f64_low_per_step": [stats.get("nmvp_f64", stats["nmvp"] if prec == "f64" else 0) / args.steps,
                                     stats.get("nmvp_low", 0) / args.steps],
        "stage_ms_per_step": {k: round(v[1] / args.steps, 1) for k, v in sorted(per.items())},
        "stage_gbs": {k: round(v[3] / (v[1] / 1e3) / 1e9, 1) for k, v in sorted(per.items()) if v[1] > 0},
        "stage_tflops": {k: round(v[2] / (v[1] / 1e3) / 1e12, 2) for k, v in sorted(per.items()) if v[1] > 0},
        "roofline": roof, "clocks": ck, "gpu_launches": LOG.launches,
        "w_contraction_paths": d.stats.get("w_paths"),
        "phase_s_per_step": {k: round(stats[k] / args.steps, 2) for k in ("plan_s", "hvec_s", "hdiag_s", "renorm_s",
                                                                         "decim_s") if k in stats},
    }
    if "plan_hits" in d.stats or "plan_misses" in d.stats:
        line["plan_cache"] = {"hits": stats.get("plan_hits", 0), "misses": stats.get("plan_misses", 0)}
    if args.e2e:
        e2e = e2e_leg(d, args, snap, per_sweep[0], energies[0][2])
        e2e["value"] = round(max_over_ranks(dist, e2e["value"], dev) / world, 3)
        line["e2e"] = e2e
    if args.shadow and prec != "f64" and not sp:
        line["same_input_dots"] = shadow_leg(d, args, snap)
    if rank == 0:
        acc = accuracy_leg(d, prec, args.cpu_baseline, sp)
        if args.cpu_baseline:
            line["cpu_baseline"] = acc.pop("cpu_baseline")
        line["accuracy"] = acc
    if tuned:
        line["autotune"] = tuned
    if hasattr(d.preconditioner, "summary"):
        line["precond_stats"] = d.preconditioner.summary()
    if args.f64_steps > 0 and prec != "f64" and not sp:
        # the FP64 GPU arm: the same sweeps from the same state (the snapshot the timed
        # sweeps started from), timed the same way
        del d
        gc.collect()
        torch.cuda.empty_cache()
        line["f64_arm"] = f64_arm(args, dev, dist, rank, snap, [e[0] for e in energies], per_sweep,
                                  tuned.get("f64", {}).get("choice"))
    del snap
    if dist is not None:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def stage_kernel(stage, w_path, prec):
    panel = w_path in ("fiber", "fused")
    from qcmpodmrg_b200.engine import FIBER_FGEMM
    fk = "k_fgemm" if FIBER_FGEMM else "k_fiber"
    tc = "k_tcpanel" if prec == "tf32x3" else "k_pgemm"
    return {"sigma1": tc if panel else "k_bgemm", "sigma2": fk if panel else "k_bgemm",
            "sigma3": fk if panel else "k_bgemm", "sigma23": fk,
            "sigma4": tc if panel else "k_bgemm"}.get(stage, "k_bgemm")


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum, ncu) per algorithmic byte of a
# stage's launches, measured on the mid-chain dot of K=24, D=200 (bench.py --workload dot;
# profiles/ holds the captures and the commands); the traffic of a D=500 launch is its
# algorithmic bytes times this ratio (the kernels stream their operands once, so the
# traffic grows in proportion to the blocks processed)
TRAFFIC_RATIO = {("sigma1", "f32"): 0.987, ("sigma2", "f32"): 1.024, ("sigma3", "f32"): 1.007,
                 ("sigma4", "f32"): 1.010,
                 ("sigma1", "tf32x3"): 1.035, ("sigma2", "tf32x3"): 1.024, ("sigma3", "tf32x3"): 1.007,
                 ("sigma4", "tf32x3"): 1.146,
                 ("sigma1", "f64"): 1.083, ("sigma2", "f64"): 1.041, ("sigma3", "f64"): 1.029,
                 ("sigma4", "f64"): 1.008}


def traffic_per_launch(stage, prec, algo_bytes):
    r = TRAFFIC_RATIO.get((stage, prec))
    return None if r is None else round(r * algo_bytes)


def e2e_leg(d, args, snap, device_ms_first, matvecs_first):
    """The first timed sweep again, from the same state (restored from the snapshot taken
    before the timed region), through the reference-facing API: mpo_dmrg_kernel.HVec/HDiag
    with host NumPy vectors and the Davidson on the host, as the reference's pdvdson calls
    them; host<->device copies are inside the timed region."""
    import torch
    d.restore(snap)
    d.host_api = True
    d.h2d_bytes = d.d2h_bytes = 0
    n0 = d.stats["nmvp"]
    torch.cuda.synchronize()
    t0 = time.time()
    d.sweep("R", args.dmax, 1e-7)
    d.sweep("L", args.dmax, 1e-7)
    torch.cuda.synchronize()
    dt = time.time() - t0
    d.host_api = False
    return {"value": round(dt, 3), "unit": "s/sweep", "h2d_bytes_per_step": int(d.h2d_bytes),
            "d2h_bytes_per_step": int(d.d2h_bytes), "matvecs": int(d.stats["nmvp"] - n0),
            "same_sweep_device_s": round(device_ms_first / 1e3, 3), "same_sweep_device_matvecs": int(matvecs_first),
            "path": "qcmpodmrg_b200.mpo_dmrg_kernel.HVec/HDiag%s with host buffers, host Davidson; the first "
                    "timed sweep re-run from the same state" % ("/SVec" if getattr(d, "ifs2proj", False) else "")}


def accuracy_leg(d, prec, with_oracle, sp):
    """Sigma at the mid-chain dot of the final state, on a seeded vector: the FP64 GPU path
    and the timed precision against the oracle (the NumPy restatement of HVecQt, timed on
    this host's cores, which also gives cpu_baseline)."""
    import torch
    isite = d.nsite // 2
    lay, idl, s, dg = d.dot_operators(isite)
    out = {"dot": isite, "ndim0": int(s.ndim0)}
    x = numpy.random.default_rng(0).standard_normal(s.ndim0)
    xd = torch.from_numpy(x).to(d.device)
    y64 = s(xd, precision="f64").cpu().numpy()
    ylo = s(xd).cpu().numpy() if prec != "f64" else y64
    if with_oracle:
        from oracle.bench_cpu import oracle_dot, oracle_sp_dot
        ora, xo, flops_dot = (oracle_sp_dot if sp else oracle_dot)(d, isite)
        t0 = time.time()
        yo = ora(x)
        t = time.time() - t0
        if sp:
            yo = yo[0]
        nrm = numpy.linalg.norm(yo)
        out["sigma_relerr_vs_oracle"] = {"f64": float(numpy.linalg.norm(y64 - yo) / nrm),
                                         prec: float(numpy.linalg.norm(ylo - yo) / nrm)}
        rate = flops_dot / t
        out["cpu_baseline"] = {"value": round(d.sweep_sigma_flops / rate, 1), "unit": "s/sweep",
                               "cores": os.cpu_count(), "kind": "port",
                               "sample": "one oracle sigma matvec at the mid-chain dot (%.1f s, %.2f GFLOP/s), "
                                         "scaled to the last timed sweep's sigma FLOPs" % (t, rate / 1e9)}
    out["sigma_relerr_vs_f64_gpu"] = float(numpy.linalg.norm(ylo - y64) / numpy.linalg.norm(y64))
    return out


def shadow_leg(d, args, snap):
    """The first timed sweep again from the same state, with every dot's low-precision
    solve repeated in plain FP64 from the same start vector on the same operators: the
    largest |E_mixed - E_FP64| over the dots (same inputs), and the matvec counts."""
    d.restore(snap)
    d.shadow = []
    d.sweep("R", args.dmax, 1e-7)
    d.sweep("L", args.dmax, 1e-7)
    sh, d.shadow = d.shadow, None
    de = [abs(r["e_mixed"] - r["e_f64"]) for r in sh]
    # a solve that ends at the iteration cap (19 Rayleigh-Ritz steps) is unconverged in
    # either precision; |dE| is then the two solvers' distance from convergence
    conv = [abs(r["e_mixed"] - r["e_f64"]) for r in sh if r["niter_f64"] < 19 and r["niter_mixed"] < 19]
    worst = max(sh, key=lambda r: abs(r["e_mixed"] - r["e_f64"])) if sh else None
    return {"dots": len(sh), "max_abs_dE": max(de) if de else None,
            "mean_abs_dE": float(numpy.mean(de)) if de else None,
            "dots_both_converged": len(conv), "max_abs_dE_converged": max(conv) if conv else None,
            "median_abs_dE": float(numpy.median(de)) if de else None, "worst_dot": worst,
            "matvecs_mixed": sum(r["nmvp_mixed"] for r in sh), "matvecs_f64": sum(r["nmvp_f64"] for r in sh),
            "definition": "one sweep from the timed sweeps' start state; at every dot the mixed-precision "
                          "Davidson and the plain FP64 Davidson from the same start vector on the same "
                          "operators; |dE| between their energies (converged: neither solve at the "
                          "iteration cap)"}


def f64_arm(args, dev, dist, rank, snap, e_mixed, ms_mixed, fg_budget=None):
    """The plain FP64 GPU path from the same state as the timed sweeps (the snapshot they
    started from), timing the first f64_steps of the same sweeps; compared with the mixed
    arm's energy after the same number of sweeps and its time for those sweeps."""
    from qcmpodmrg_b200.hamiltonian import make_hamiltonian
    from qcmpodmrg_b200.dmrg import DMRG
    n = min(args.f64_steps, args.steps)
    ham = make_hamiltonian(args.sites, args.sites, SEED, DECAY)
    d = DMRG(ham, device=dev, precision="f64", w_path=args.w_path, plan_cache=args.plan_cache)
    if fg_budget is not None and d.sigma_opts.get("use_fiber"):
        d.sigma_opts["fg_budget"] = tuple(fg_budget)
    d.restore(snap)
    ms, per, res = _timed_sweeps(d, args, n, dist)
    ms = max_over_ranks(dist, ms, dev)
    e64 = res[-1][0]
    em = e_mixed[n - 1]
    t_mixed = max_over_ranks(dist, sum(ms_mixed[:n]), dev)
    out = {"sweeps_timed": n, "s_per_sweep": round(ms / n / 1e3, 3), "sweep_ms": [round(x, 1) for x in per],
           "energy_f64": e64, "energy_mixed_same_sweep": em, "abs_dE_vs_f64": abs(em - e64),
           "energy_mixed_final": e_mixed[-1], "matvecs_per_sweep": sum(r[2] for r in res) / n,
           "speedup_vs_f64": round(ms / t_mixed, 3),
           "definition": "both arms start from the same state (after the ramp and %d warm-up sweeps of the "
                         "mixed arm) and run the same %d sweep(s): FP64 GPU time / mixed time for those "
                         "sweeps; |dE| between the two arms' energies after them" % (args.warmup, n)}
    del d
    return out


def run_reference(args):
    """The reference algorithm (oracle port of HVecQt/HDiagQt/renormQt_H00) on the host cores."""
    dist, rank, world, local = None, int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), 0
    if rank != 0:
        return
    from oracle.bench_cpu import reference_step
    for _ in range(args.warmup):
        reference_step(args, warm=True)
    t0 = time.time()
    res = [reference_step(args, step=k) for k in range(args.steps)]
    wall = time.time() - t0
    v = float(res[-1]["sweep_s_est"])          # from every dot sampled
    line = {"metric": METRIC, "impl": "reference", "value": round(v, 1), "unit": "s/sweep", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * wall / args.steps, 1),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded integrals (K=%d, N=%d, decay 3, seed 1), synthetic D=%d state"
                    % (args.sites, args.sites, args.dmax),
            "config": {"workload": "two-site Qt DMRG sweep, K=%d N=%d Sz=0 D=%d, %d operators H_p"
                                   % (args.sites, args.sites, args.dmax, 2 * args.sites),
                       "K": args.sites, "N": args.sites, "D": args.dmax},
            "cpu_baseline": {"value": round(v, 1), "unit": "s/sweep", "cores": res[0]["cores"], "kind": "port",
                             "sample": res[-1]["sample"]},
            "dots_sampled": {str(r["dot"]): round(r["dot_cost_s"], 2) for r in res},
            "e2e": {"value": round(v, 1), "unit": "s/sweep", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_dot(args):
    """One mid-chain dot, for kernel profiles: the ramp up to D = dmax (one sweep pair per
    bond dimension of RAMP below dmax, then one at dmax), then the sigma of the middle dot
    applied once to warm up and --steps times under the NVTX range "dot" (the range an
    ncu capture selects with --nvtx --nvtx-include "dot/"), in the bench's precision and
    in FP64.  Prints one JSON line: per launch the stage, kernel, algorithmic bytes and
    FLOPs and the CUDA-event time."""
    import torch
    from qcmpodmrg_b200.engine import LOG
    dev = torch.device("cuda:0")
    prec = {"mixed": "f32", "f64": "f64", "tf32": "tf32", "mixed-tc": "tf32x3"}[args.precision]
    # the state is prepared by FP64 sweeps for --precision f64 and by FP32-sigma sweeps
    # otherwise; the profiled dot's plan is then compiled for the requested precision
    d = _make_dmrg(args, "f64" if prec == "f64" else "f32", dev)
    d.sweep("R", args.dmax, 1e-7)
    n, e, dw, el, dl = d.sweep("L", args.dmax, 1e-7)
    d.precision = prec
    isite = d.nsite // 2
    tune = None
    if args.autotune:
        from qcmpodmrg_b200.autotune import tune_fiber_budget
        tune = {p: tune_fiber_budget(d, isite, precision=p) for p in ([prec] if prec == "f64" else [prec, "f64"])}
        d.sigma_opts["fg_budget"] = tune[prec]["choice"]
    LOG.enabled = True            # the plan records its algorithmic byte counts for the launch log
    lay, idl, s, dg = d.dot_operators(isite)
    LOG.enabled = False
    x = torch.from_numpy(numpy.random.default_rng(0).standard_normal(s.ndim0)).to(dev)
    precs = [prec] if prec == "f64" else [prec, "f64"]
    for p in precs:
        s(x, precision=p)
    torch.cuda.synchronize()
    LOG.reset()
    LOG.enabled = True
    torch.cuda.nvtx.range_push("dot")
    marks = []
    for _ in range(args.steps):
        for p in precs:
            marks.append((len(LOG.records), p))
            s(x, precision=p)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    LOG.enabled = False
    recs = []
    prec_of = {}
    for i0, p in marks:
        for i in range(i0, len(LOG.records)):
            prec_of[i] = p
    for i, (name, e0, e1, fl, by) in enumerate(LOG.records):
        ms = e0.elapsed_time(e1)
        p = prec_of.get(i, prec)
        recs.append({"stage": name, "precision": p, "kernel": stage_kernel(name, args.w_path, p), "ms": round(ms, 4),
                     "algo_bytes": int(by), "flops": float(fl), "gbs": round(by / (ms / 1e3) / 1e9, 1) if ms else None})
    line = {"workload": "mid-chain dot sigma, K=%d N=%d D=%d" % (args.sites, args.sites, args.dmax),
            "set_up_energy": e, "set_up_matvecs": int(d.stats["nmvp"]), "dot": isite, "ndim0": int(s.ndim0), "precisions": precs, "repeats": args.steps,
            "launches_logged": len(recs), "gpu_launches": LOG.launches, "autotune": tune, "launches": recs}
    print(json.dumps(line), flush=True)


def run_converge(args):
    """Time to convergence, both arms from the same state: the ramp (RAMP below dmax) in the
    mixed precision, then sweeps (R then L) at dmax until the sweep energy changes by less
    than --tol, at most --steps sweeps, first in the mixed precision and then, from the same
    state, in plain FP64.  Prints one JSON line with both arms' sweeps, seconds (CUDA events)
    and energies, |E_mixed - E_FP64| and the speed-up."""
    import torch
    from qcmpodmrg_b200.hamiltonian import make_hamiltonian
    from qcmpodmrg_b200.dmrg import DMRG
    dev = torch.device("cuda:0")
    prec = {"mixed": "f32", "f64": "f64", "tf32": "tf32", "mixed-tc": "tf32x3"}[args.precision]
    d = _make_dmrg(args, prec, dev)
    if args.autotune:
        from qcmpodmrg_b200.autotune import tune_fiber_budget
        budgets = {prec: tune_fiber_budget(d)["choice"], "f64": tune_fiber_budget(d, precision="f64")["choice"]}
        d.sigma_opts["fg_budget"] = tuple(budgets[prec])
    snap = d.snapshot()

    def converge(dm):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        hist, eold = [], None
        for k in range(args.steps):
            e, dw, nmv = _step(dm, args)
            hist.append((e, dw, nmv))
            if eold is not None and abs(e - eold) < args.tol:
                break
            eold = e
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3, hist

    t_mix, h_mix = converge(d)
    st_mix = {k: d.stats.get(k, 0) for k in ("nmvp_f64", "nmvp_low")}
    del d
    torch.cuda.empty_cache()
    ham = make_hamiltonian(args.sites, args.sites, SEED, DECAY)
    d64 = DMRG(ham, device=dev, precision="f64", w_path=args.w_path, plan_cache=args.plan_cache)
    if args.autotune and d64.sigma_opts.get("use_fiber"):
        d64.sigma_opts["fg_budget"] = tuple(budgets["f64"])
    d64.restore(snap)
    t64, h64 = converge(d64)
    line = {"metric": "time to convergence (sweep energy change < %g Eh), mixed vs FP64" % args.tol,
            "value": round(t_mix, 2), "unit": "s", "higher_is_better": False, "n_gpus": 1,
            "config": {"workload": "two-site Qt DMRG, K=%d N=%d Sz=0 D=%d, decay 3, seed 1, from the same "
                                   "ramped state (D %s)" % (args.sites, args.sites, args.dmax,
                                                            "/".join(str(x) for x in RAMP if x < args.dmax)),
                       "precision": args.precision, "tol": args.tol, "max_sweeps": args.steps},
            "mixed": {"s": round(t_mix, 2), "sweeps": len(h_mix), "energy": h_mix[-1][0], "dwt": h_mix[-1][1],
                      "matvecs": sum(h[2] for h in h_mix), "energies": [h[0] for h in h_mix],
                      "matvecs_f64_low": [st_mix["nmvp_f64"], st_mix["nmvp_low"]]},
            "f64": {"s": round(t64, 2), "sweeps": len(h64), "energy": h64[-1][0], "dwt": h64[-1][1],
                    "matvecs": sum(h[2] for h in h64), "energies": [h[0] for h in h64]},
            "abs_dE_vs_f64": abs(h_mix[-1][0] - h64[-1][0]),
            "speedup_vs_f64": round(t64 / t_mix, 3) if t_mix > 0 else None}
    print(json.dumps(line), flush=True)


def run_batched(args):
    """Independent instances (the batched configuration: K uniform in 8..20 with N = K, Sz = 0
    or 1/2, D uniform in 64..256, seeded decayed integrals; --instances of them) swept in
    lockstep: one launch per sigma contraction for all instances per Davidson step, replayed
    from CUDA graphs (or launched directly with --no-graphs), against the same instances swept
    one after another.  Prints one JSON line."""
    import torch
    from qcmpodmrg_b200.hamiltonian import make_hamiltonian
    from qcmpodmrg_b200.synthetic import product_mps
    from qcmpodmrg_b200.dmrg import DMRG
    from qcmpodmrg_b200.batched import BatchedDMRG
    dev = torch.device("cuda:0")
    rng = numpy.random.default_rng(1000)
    shapes = [(int(rng.integers(8, 21)), int(rng.integers(64, 257))) for _ in range(args.instances)]

    def make():
        out = []
        for i, (K, D) in enumerate(shapes):
            ham = make_hamiltonian(K, K, 1000 + i, 3.0)
            d = DMRG(ham, device=dev, precision="f64", sz=0.5 * (K % 2), plan_cache=False)
            d.load_mps(product_mps(ham))
            for st in ("R", "L"):          # set-up sweep at a small bond dimension
                d.sweep(st, 16, 1e-7)
            out.append(d)
        return out

    seq = make()
    torch.cuda.synchronize()
    t0 = time.time()
    e_seq = []
    for d, (K, D) in zip(seq, shapes):
        for st in ("R", "L"):
            n, e, dw, el, dl = d.sweep(st, D, 1e-7)
        e_seq.append(e)
    torch.cuda.synchronize()
    t_seq = time.time() - t0
    del seq
    torch.cuda.empty_cache()
    bat = make()
    b = BatchedDMRG(bat, kind="f64", use_graphs=args.graphs)
    torch.cuda.synchronize()
    t0 = time.time()
    for st in ("R", "L"):
        got = b.sweep(st, [D for _, D in shapes], 1e-7)
    torch.cuda.synchronize()
    t_bat = time.time() - t0
    line = {"metric": "instance-sweeps per second, lockstep batched vs sequential", "value":
            round(len(shapes) / t_bat, 3), "unit": "instance-sweeps/s", "n_gpus": 1, "steps": 1, "warmup": 0,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic: seeded integrals per instance",
            "config": {"workload": "%d independent two-site DMRG instances, K in [8, 20] (N = K), D in [64, 256], "
                                   "one sweep each after a D=16 set-up sweep" % len(shapes), "shapes": shapes},
            "sequential_instance_sweeps_per_s": round(len(shapes) / t_seq, 3),
            "batched_s": round(t_bat, 2), "sequential_s": round(t_seq, 2),
            "graphs": args.graphs, "graph_captures": b.captures, "lockstep_steps": b.steps}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None, choices=["mixed", "f64", "tf32", "mixed-tc"],
                    help="mixed-tc (default): L.psi and .R on the tensor cores in split TF32, the MPO-site "
                         "contractions in FP32, FP64 Rayleigh-Ritz / residual check / decimation; mixed: FP32 "
                         "CUDA cores for all of sigma; f64: everything FP64 (the parity path); tf32: plain TF32 "
                         "(default for --workload sp: mixed)")
    ap.add_argument("--sites", type=int, default=K_SITES)
    ap.add_argument("--dmax", type=int, default=DMAX)
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu", dest="cpu_baseline", action="store_false")
    ap.add_argument("--w-path", default="fiber", choices=["generic", "fiber", "fused"],
                    help="kernels of the two MPO-site contractions of sigma")
    ap.add_argument("--no-plan-cache", dest="plan_cache", action="store_false",
                    help="compile every dot's plans afresh instead of reusing those of dots whose sectors "
                         "did not change")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default fiber-GEMM schedule instead of the measured choice")
    ap.add_argument("--no-shadow", dest="shadow", action="store_false",
                    help="skip the same-input leg (each dot of one sweep also solved in plain FP64)")
    ap.add_argument("--f64-steps", type=int, default=3,
                    help="sweeps timed on the plain FP64 GPU arm from the timed sweeps' start state (0: no FP64 arm)")
    ap.add_argument("--precond", default="jacobi", choices=["jacobi", "learned"],
                    help="Davidson preconditioner of the mixed-precision arm")
    ap.add_argument("--precond-train", type=int, default=2, help="sweeps whose solver pairs train the network")
    ap.add_argument("--tol", type=float, default=1e-8, help="--workload converge: sweep energy change")
    ap.add_argument("--workload", default="sweep", choices=["sweep", "batched", "sp", "dot", "converge"],
                    help="sp: spin-projected sweeps (SP-MPS, S=0) with --npts quadrature points; dot: the "
                         "mid-chain dot's sigma under the NVTX range 'dot' (kernel profiles)")
    ap.add_argument("--npts", type=int, default=4)
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--no-graphs", dest="graphs", action="store_false",
                    help="batched workload: plain lockstep launches instead of CUDA-graph replay")
    args = ap.parse_args()
    if args.precision is None:
        args.precision = "mixed" if args.workload == "sp" else "mixed-tc"
    world = os.environ.get("WORLD_SIZE")
    if args.gpus > 1 and world is None:
        # one process per GPU: relaunch under torch.distributed.run (replicas, see dist_init)
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
               "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
        sys.exit(subprocess.call(cmd))
    if world is not None and int(world) != args.gpus:
        sys.exit("bench.py: --gpus %d but WORLD_SIZE=%s" % (args.gpus, world))
    if args.workload == "batched":
        # 64 instances hold ~90 GB of environments next to the batches' scratch: let the
        # caching allocator grow segments instead of fragmenting (set before CUDA starts)
        os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "expandable_segments:True")
        run_batched(args)
    elif args.workload == "dot":
        run_dot(args)
    elif args.workload == "converge":
        run_converge(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
