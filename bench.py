#!/usr/bin/env python3
"""Benchmark of the fused PDHG iteration on the large power-law LP.

Workload (one GPU): LP with m = 1,000,000 rows, n = 2,000,000 columns and about
20,000,000 nonzeros, column degrees Zipf(1.5) capped at 1,000, rows uniform,
|a| log-uniform in [1e-3, 1e3] with random signs, bounds [0, 10], rows centred on
A x0 (the-solver_b200/instances.py: lp_config1, seed 1). FP64 throughout.

A step is one call of the reference C entry point
sankhya_cuda_qp_pdhg_preconditioned (the LP case: no Hessian, per-row and
per-column steps 0.9 / (1 + |row|_1) and 0.9 / (1 + |column|_1), as sk_solve
chooses them) with max_iterations = check_every = ITERS_PER_STEP:
ITERS_PER_STEP fused PDHG iterations plus one checkpoint evaluation, host
arrays in and out.

  value   GB/s of algorithmic bytes, timed on the engine's stream with CUDA
          events around the iteration kernels and checkpoints (inputs resident)
  e2e     the same metric over host wall time of whole C-ABI calls from pinned
          host buffers (uploads of c and bounds, solution download included)
Algorithmic bytes of one iteration (each vector element and nonzero once):
  A-side launch : 12 nnz + 4 (m+1) + 8 n (x_bar gather) + 32 m (y, rl, ru, y_new)
  A'-side launch: 12 nnz + 4 (n+1) + 8 m (y_new gather) + 48 n (x, c, cl, cu, x_new, x_bar)

--impl reference runs the reference's own CPU PDHG (sk_solve with
lp_engine = SK_LP_FIRST_ORDER from its C sources, oracle/_ref, the OpenMP build on
every core this process may use) on the same instance and reports the same metric
over its loop time.
Multi-GPU: replicas only (one independent instance per rank, no exchange).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
ITERS_PER_STEP = 100
SEED = 1
M, N, NNZ = 1_000_000, 2_000_000, 20_000_000
WORKLOAD = "lp_config1: m=1e6, n=2e6, nnz~2e7, Zipf(1.5) columns, |a| log-U[1e-3,1e3], FP64"
METRIC = "PDHG fused-iteration throughput (algorithmic HBM bytes), power-law LP 1Mx2M, 20M nnz"


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def dual_bytes(m, n, nnz):
    return 12 * nnz + 4 * (m + 1) + 8 * n + 32 * m


def primal_bytes(m, n, nnz):
    return 12 * nnz + 4 * (n + 1) + 8 * m + 48 * n


def iteration_bytes(m, n, nnz):
    return dual_bytes(m, n, nnz) + primal_bytes(m, n, nnz)


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                self.out = ""

    def summary(self):
        rows = [r.split(",") for r in getattr(self, "out", "").strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(n_gpus, backend="nccl"):
    """One process per GPU (torchrun env). Replicas only: the process group is
    used for the barrier and the max-over-ranks of the timed region, never for
    data."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def _reduce_device():
    import torch
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def barrier_max(value, world):
    """Max of a per-rank scalar over all ranks (the job's time is the slowest rank's)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def job_throughput(world, bytes_per_unit, units_per_rank, seconds_max):
    """Whole-job rate: every rank processed units_per_rank units of bytes_per_unit
    bytes; the job took the slowest rank's time."""
    return world * bytes_per_unit * units_per_rank / seconds_max / 1e9


def reference_core():
    """(library, threads) for the timed runs of the reference's C core: its OpenMP build
    (threaded csc_tmv, the same bits) on every core this process may use, or, where
    that build or its OpenMP runtime is missing, the serial build on one."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    try:
        O.load("ref_omp")
        return "ref_omp", len(os.sched_getaffinity(0))
    except OSError:
        return "ref", 1


def reference_loop_gbs(inst, iterations, core=("ref", 1)):
    """The reference's sk_solve (SK_LP_FIRST_ORDER) for `iterations` iterations;
    returns (GB/s over its loop time, loop seconds, iterations)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    lib_name, threads = core
    st, out = O.ref_sk_solve(inst, lib_name=lib_name, threads=threads, primal_tol=1e-300, dual_tol=1e-300,
                             iteration_limit=iterations)
    if st != 0:
        raise RuntimeError(f"reference sk_solve failed with status {st}")
    secs = out["solve_seconds"]
    nnz = int(inst["ptr"][-1])
    return iteration_bytes(inst["m"], inst["n"], nnz) * out["iterations"] / secs / 1e9, secs, out["iterations"]


def _core_text(core):
    lib_name, threads = core
    return (f"{threads} threads, the reference's c/src built with OpenMP" if lib_name == "ref_omp"
            else "1 thread, the reference's c/src built without OpenMP")


# Iterations of the reference loop per sk_solve call in both CPU legs (the cpu_baseline
# sample and each step of --impl reference). sk_solve's loop time includes one extra
# product at the last iteration (its final checkpoint), so short calls understate the
# loop's rate: at 64 iterations that extra product is under 1 % of the call.
REFERENCE_ITERS_PER_CALL = 64


def cpu_baseline(inst, calls=2):
    """Bounded sample of the reference CPU PDHG on this instance (rank 0, N=1):
    `calls` sk_solve calls of REFERENCE_ITERS_PER_CALL iterations after one
    warm-up call of one iteration."""
    core = reference_core()
    reference_loop_gbs(inst, 1, core)
    secs, its = 0.0, 0
    for _ in range(calls):
        _, s, i = reference_loop_gbs(inst, REFERENCE_ITERS_PER_CALL, core)
        secs += s
        its += i
    nnz = int(inst["ptr"][-1])
    gbs = iteration_bytes(inst["m"], inst["n"], nnz) * its / secs / 1e9
    return {"value": round(gbs, 4), "unit": "GB/s", "cores": core[1], "kind": "reference",
            "sample": f"{its} iterations of sk_solve (SK_LP_FIRST_ORDER, {_core_text(core)}) on the same "
                      f"instance, {secs:.2f} s of loop time"}


def _marginal_ms(call, reps=3):
    """Wall-time cost of one more iteration: (best of reps at 200 iterations - best of
    reps at 100) / 100; both calls pay the same setup, uploads, one checkpoint and the
    download, which the difference cancels."""
    best = {}
    for its in (100, 200):
        call(its)                                  # warm-up (allocations, graphs)
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            call(its)
            ts.append(time.perf_counter() - t0)
        best[its] = min(ts)
    return 1e3 * (best[200] - best[100]) / 100.0


def reference_gpu_baseline(E, A, inst, ps, ds, limit_s=120.0):
    """The reference's own GPU code on the same instance and GPU: a baseline leg, like
    cpu_baseline (oracle/_ref holds test infrastructure and is never on the engine's
    path).
      cuda_prototype: the reference's CUDA prototype (cuda/src/sankhya_cuda_lp.cu:101-437,
        thread-per-row SpMV and an atomicAdd transpose, recompiled for sm_100a) through
        the same entry point with the same steps, host arrays; the marginal wall time of
        one iteration and its algorithmic GB/s, beside the engine's measured the same way;
      gpupdlp: the reference C++ core's GPU PDLP (src/cuda/GpuPdlp.cpp over cuSPARSE
        CSR SpMV, with its first-order driver's Ruiz + Pock-Chambolle scaling) to 1e-6
        relative KKT, beside the engine's FP64 PDLP to the same tolerance."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    m, n, nnz = inst["m"], inst["n"], int(inst["ptr"][-1])
    byt = iteration_bytes(m, n, nnz)
    out = {}
    settings = lambda its: dict(max_iterations=its, check_every=its, tau=0.0, sigma=0.0, theta=1.0, tolerance=1e-12,
                                time_limit=0.0)
    host = {k: np.ascontiguousarray(inst[k]) for k in ("c", "rl", "ru", "cl", "cu")}

    def engine_call(its):
        rc, _, _, _ = E.pdhg(A, host, E.settings(**settings(its)), primal_steps=ps, dual_steps=ds,
                             entry="preconditioned")
        if rc != 0:
            raise RuntimeError(E.last_error())

    eng_ms = _marginal_ms(engine_call)
    try:
        R = O.RefCudaPrototype(inst)
        try:
            def ref_call(its):
                rc, _, _ = R.pdhg(settings(its), ps, ds)
                if rc != 0:
                    raise RuntimeError(f"reference prototype returned {rc}")
            ref_ms = _marginal_ms(ref_call)
        finally:
            R.close()
        out["cuda_prototype"] = {"ms_per_iteration": round(ref_ms, 4), "gbs": round(byt / ref_ms / 1e6, 1),
                                 "engine_ms_per_iteration": round(eng_ms, 4),
                                 "engine_gbs": round(byt / eng_ms / 1e6, 1),
                                 "engine_speedup": round(ref_ms / eng_ms, 2),
                                 "method": "marginal wall time per iteration, 200- vs 100-iteration calls"}
    except (OSError, FileNotFoundError, RuntimeError) as exc:
        out["cuda_prototype"] = {"unavailable": str(exc)}
    try:
        t0 = time.perf_counter()
        x, st = O.ref_gpupdlp(inst, eps=1e-6, max_iterations=20_000_000, time_limit=limit_s, scale=True)
        wall = time.perf_counter() - t0
        out["gpupdlp"] = {"seconds": round(wall, 3), "converged": st["converged"], "iterations": st["iterations"],
                          "solver_seconds": round(st["seconds"], 3), "objective": _finite(np.dot(inst["c"], x)),
                          "kkt": [_finite(st[k]) for k in ("relative_primal_residual", "relative_dual_residual",
                                                           "relative_gap")], "eps": 1e-6, "time_limit_s": limit_s}
    except (OSError, FileNotFoundError, RuntimeError) as exc:
        out["gpupdlp"] = {"unavailable": str(exc)}
    return out


ORACLE_OBJECTIVE = os.path.join(ROOT, "tests", "golden", "objective_lp_config1.json")


def oracle_objective():
    """The FP64 objective of the bench instance solved to 1e-9 relative KKT (tests/golden,
    written by tests/golden/make_config1_objective.py), or None where it is absent."""
    try:
        with open(ORACLE_OBJECTIVE) as f:
            return float(json.load(f)["objective"])
    except (OSError, KeyError, ValueError):
        return None


def _pdlp_run(E, A, inst, eps, precision, algorithm, limit_s, oracle):
    s = E.pdlp_default_settings()
    s.eps_optimal, s.precision, s.time_limit, s.max_iterations = eps, precision, limit_s, 20_000_000
    s.algorithm = algorithm
    t0 = time.perf_counter()
    rc, x, y, r = E.pdlp_solve(A, inst, s)
    wall = time.perf_counter() - t0
    obj = _finite(np.dot(inst["c"], x))
    out = {"seconds": round(wall, 3), "status": r["status"], "iterations": r["iterations"],
           "restarts": r["restarts"], "refinements": r["refinements"], "objective": obj,
           "kkt": [_finite(r[k]) for k in ("relative_primal_residual", "relative_dual_residual", "relative_gap")]}
    if oracle is not None and obj is not None:
        out["objective_rel_err_vs_oracle"] = _finite(abs(obj - oracle) / (1.0 + abs(oracle)))
    return out


def time_to_kkt(E, A, inst, eps_list=(1e-4, 1e-6, 1e-8), limit_s=120.0, halpern=False, limit_1e8_s=60.0):
    """Wall time of sankhya_b200_pdlp_solve to each relative-KKT tolerance on the same
    instance: plain FP64 PDLP (GpuPdlp's restarted adaptive loop) versus FP32 inner
    iterations refined in FP64 at every restart, with FP32 and with bf16 matrix values
    (FP32 products). Host arrays in and out, scaling
    included. Each run's objective is compared with the FP64 oracle value of the
    instance (the tightest FP64 solves of two independent codes) where it is present.
    With halpern, the reflected restarted Halpern loop runs at the middle tolerance.
    Tolerances below 1e-7 get limit_1e8_s: the restarted loop stalls near a 2e-6 gap on
    the bench instance, so those runs report where they stopped."""
    oracle = oracle_objective()
    out = {"relative_kkt": "max(primal, dual, gap) as in GpuPdlp", "oracle_objective": oracle,
           "oracle": "tests/golden/objective_lp_config1.json (the reference's GpuPdlp and the engine, FP64, tightest)"}
    for eps in eps_list:
        key = f"eps_{eps:.0e}"
        lim = limit_1e8_s if eps < 1e-7 else limit_s
        row = {"fp64": _pdlp_run(E, A, inst, eps, E.FP64, E.PDLP_ADAPTIVE, lim, oracle),
               "fp32_refined": _pdlp_run(E, A, inst, eps, E.FP32_REFINE, E.PDLP_ADAPTIVE, lim, oracle),
               "bf16_values_refined": _pdlp_run(E, A, inst, eps, E.BF16_REFINE, E.PDLP_ADAPTIVE, lim, oracle)}
        if halpern and eps == eps_list[len(eps_list) // 2]:
            row["halpern_fp64"] = _pdlp_run(E, A, inst, eps, E.FP64, E.PDLP_HALPERN, limit_s, oracle)
        for name in [k for k in row if k != "fp64"]:
            if row["fp64"]["status"] == 0 and row[name]["status"] == 0 and row[name]["seconds"] > 0:
                row[f"speedup_{name}_vs_fp64"] = round(row["fp64"]["seconds"] / row[name]["seconds"], 3)
        out[key] = row
    return out


def config0_to_1e8(E, I, reps=3):
    """Config 0 (2,000 x 5,000, the metric's 1e-8 tolerance): wall time of
    sankhya_b200_pdlp_solve to 1e-8 relative KKT, host arrays in and out, for FP64 and
    the two refined modes (best of `reps` after an untimed solve), each objective
    against the reference simplex's (tests/golden/simplex_lp_config0.json, certified
    by its sk_verify); and the reference's own GPU PDLP to the same tolerance on the
    same GPU, as in reference_gpu."""
    inst = I.lp_config0(0)
    golden = None
    try:
        with open(os.path.join(ROOT, "tests", "golden", "simplex_lp_config0.json")) as f:
            golden = float(json.load(f)["objective"])
    except (OSError, KeyError, ValueError):
        pass
    A = E.Matrix.from_instance(inst)
    out = {"workload": "lp_config0: m=2000, n=5000, 5 per column, seed 0", "eps": 1e-8,
           "oracle": "tests/golden/simplex_lp_config0.json (the reference's simplex)", "oracle_objective": golden}
    for name, prec in (("fp64", E.FP64), ("fp32_refined", E.FP32_REFINE), ("bf16_values_refined", E.BF16_REFINE)):
        _pdlp_run(E, A, inst, 1e-8, prec, E.PDLP_ADAPTIVE, 60.0, golden)
        runs = [_pdlp_run(E, A, inst, 1e-8, prec, E.PDLP_ADAPTIVE, 60.0, golden) for _ in range(reps)]
        out[name] = min(runs, key=lambda r: r["seconds"])
    A.close()
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        O.ref_gpupdlp(inst, eps=1e-8, time_limit=60.0, scale=True)
        best = None
        for _ in range(reps):
            t0 = time.perf_counter()
            x, st = O.ref_gpupdlp(inst, eps=1e-8, time_limit=60.0, scale=True)
            wall = time.perf_counter() - t0
            if best is None or wall < best[0]:
                best = (wall, x, st)
        wall, x, st = best
        obj = _finite(np.dot(inst["c"], x))
        g = {"seconds": round(wall, 3), "converged": st["converged"], "iterations": st["iterations"],
             "objective": obj}
        if golden is not None and obj is not None:
            g["objective_rel_err_vs_oracle"] = _finite(abs(obj - golden) / (1.0 + abs(golden)))
        out["reference_gpupdlp"] = g
        if st["converged"] == 1 and out["fp64"]["status"] == 0:
            out["engine_fp64_speedup_vs_reference_gpupdlp"] = round(wall / out["fp64"]["seconds"], 2)
    except (OSError, FileNotFoundError, RuntimeError) as exc:
        out["reference_gpupdlp"] = {"unavailable": str(exc)}
    return out


def run_plain_pdhg(args):
    """Config 1: the plain fixed-step FP64 PDHG the reference's GPU code runs
    (sankhya_cuda_qp_pdhg_preconditioned, steps 0.9 / (1 + |A| mass), no restarts or
    adaptive step; this engine's kernels) from zero for growing iteration budgets, each
    point's objective error against the oracle value and its largest row violation
    (relative to 1 + max |row bound|), beside the restarted PDLP with FP32 iterations
    refined in FP64 stopped at 1e-6 relative KKT. Prints one JSON line."""
    E = _load("sankhya_b200", os.path.join(ROOT, "the-solver_b200", "__init__.py"))
    I = _load("sankhya_b200_instances", os.path.join(ROOT, "the-solver_b200", "instances.py"))
    import scipy.sparse as sp
    inst = I.lp_config1(SEED)
    m, n = inst["m"], inst["n"]
    A = E.Matrix.from_instance(inst)
    Ah = sp.csr_matrix((inst["val"], inst["idx"], inst["ptr"]), shape=(m, n))
    rows = np.repeat(np.arange(m), np.diff(inst["ptr"]))
    rmass = np.bincount(rows, weights=np.abs(inst["val"]), minlength=m)
    cmass = np.bincount(inst["idx"], weights=np.abs(inst["val"]), minlength=n)
    ps, ds = 0.9 / (1 + cmass), 0.9 / (1 + rmass)
    oracle = oracle_objective()
    bscale = 1.0 + max(np.abs(inst["rl"]).max(), np.abs(inst["ru"]).max())

    def quality(x):
        act = Ah @ x
        viol = max(0.0, float(np.max(inst["rl"] - act)), float(np.max(act - inst["ru"])))
        obj = float(np.dot(inst["c"], x))
        q = {"objective": obj, "row_violation_rel": viol / bscale}
        if oracle is not None:
            q["objective_rel_err_vs_oracle"] = abs(obj - oracle) / (1.0 + abs(oracle))
        return q

    out = {"metric": "plain fixed-step FP64 PDHG vs restarted PDLP (FP32 refined), config 1", "unit": "s",
           "higher_is_better": False, "data": "synthetic", "dtype": "f64",
           "workload": "lp_config1: m=1,000,000, n=2,000,000, 20M nnz", "oracle_objective": oracle, "plain": []}
    host = {k: np.ascontiguousarray(inst[k]) for k in ("c", "rl", "ru", "cl", "cu")}
    for its in (20_000, 60_000, 180_000):
        s = E.settings(its, its, 0.0, 0.0, 1.0, 1e-12)
        t0 = time.perf_counter()
        rc, x, _, r = E.pdhg(A, host, s, primal_steps=ps, dual_steps=ds, entry="preconditioned")
        wall = time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError(E.last_error())
        out["plain"].append({"iterations": its, "seconds": round(wall, 2), **quality(x)})
    p = E.pdlp_default_settings()
    p.eps_optimal, p.precision, p.time_limit, p.max_iterations = 1e-6, E.FP32_REFINE, 120.0, 20_000_000
    t0 = time.perf_counter()
    rc, x, _, r = E.pdlp_solve(A, inst, p)
    wall = time.perf_counter() - t0
    out["pdlp_fp32_refined_1e-6"] = {"seconds": round(wall, 2), "status": r["status"], "iterations": r["iterations"],
                                     **quality(x)}
    print(json.dumps(out), flush=True)
    return 0


def run_crossover(args):
    """Config 0 to a certified vertex: the engine's FP64 restarted PDLP to 1e-8 (config
    0's target; host arrays, on the GPU), then the crossover sources run on the host with the
    reference's own simplex codes (the C++ core's warm-started basis, and the C core's
    held columns), each answer checked against the reference simplex's certified
    optimum. The cold simplex times are the recorded ones of the same LP. Prints one
    JSON line."""
    E = _load("sankhya_b200", os.path.join(ROOT, "the-solver_b200", "__init__.py"))
    I = _load("sankhya_b200_instances", os.path.join(ROOT, "the-solver_b200", "instances.py"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    print(json.dumps(crossover_legs(E, I, O)), flush=True)
    return 0


def crossover_legs(E, I, O, with_c_core=True):
    """The legs of run_crossover for engine, instance and oracle modules."""
    golden = json.load(open(os.path.join(ROOT, "tests", "golden", "simplex_lp_config0.json")))
    opt = golden["objective"]
    inst = I.lp_config0(0)
    out = {"metric": "config 0 to a certified vertex: engine PDLP 1e-8, then crossover", "unit": "s",
           "higher_is_better": False, "data": "synthetic", "dtype": "f64",
           "workload": "lp_config0: m=2,000, n=5,000, 25,000 nnz",
           "cold_simplex_recorded_s": {"c_core": golden.get("seconds"), "cpp_core": 312.6},
           "oracle_objective": opt}
    A = E.Matrix.from_instance(inst)
    s = E.pdlp_default_settings()
    s.eps_optimal, s.max_iterations, s.time_limit = 1e-8, 400000, 60.0
    t0 = time.perf_counter()
    rc, x, y, r = E.pdlp_solve(A, inst, s)
    out["engine_pdlp"] = {"seconds": round(time.perf_counter() - t0, 4), "status": r["status"],
                          "iterations": r["iterations"], "rc": rc}
    A.close()
    if rc != 0:
        raise RuntimeError(E.last_error())
    rel = lambda v: abs(v - opt) / (1.0 + abs(opt))
    t0 = time.perf_counter()
    xrc, xo = O.ref_sihps_crossover(inst, x, y, time_budget=600.0)
    out["cpp_core_crossover"] = {"seconds": round(time.perf_counter() - t0, 3), "rc": xrc, "status": xo["status"],
                                 "used_warm_start": xo["used_warm_start"], "dual_pivots": xo["dual_iterations"],
                                 "cold_pivots": xo["cold_iterations"],
                                 "objective_rel_err_vs_oracle": rel(xo["objective"])}
    if with_c_core:
        t0 = time.perf_counter()
        src, so = O.ref_crossover(inst, x, y)
        out["c_core_crossover"] = {"seconds": round(time.perf_counter() - t0, 3), "rc": src, "result": so["result"],
                                   "direct": so["direct"], "pivots": so["simplex_iterations"],
                                   "held_columns": so["fixed_columns"],
                                   "full_fallback": so["full_fallback"],
                                   "objective_rel_err_vs_oracle": rel(so["objective"])}
    return out


def run_polish(args):
    """Feasibility polishing on config 1 (and config 0): the restarted FP64 PDLP
    stopped at 1e-4 relative KKT beside the polished solve (gap 1e-4, then 1e-6;
    primal and dual residual 1e-8), with wall time, the rounds and iterations of each
    part, and each answer's objective error against the oracle value and largest row
    violation (relative to 1 + max |row bound|). Prints one JSON line."""
    E = _load("sankhya_b200", os.path.join(ROOT, "the-solver_b200", "__init__.py"))
    I = _load("sankhya_b200_instances", os.path.join(ROOT, "the-solver_b200", "instances.py"))
    print(json.dumps(polish_legs(E, I)), flush=True)
    return 0


def polish_legs(E, I, time_limit=60.0):
    """The legs of run_polish for an engine module E and an instance module I."""
    import scipy.sparse as sp
    out = {"metric": "restarted FP64 PDLP with feasibility polishing (primal and dual residual 1e-8)", "unit": "s",
           "higher_is_better": False, "data": "synthetic", "dtype": "f64"}
    golden0 = os.path.join(ROOT, "tests", "golden", "simplex_lp_config0.json")
    cases = [("lp_config1", I.lp_config1(SEED), oracle_objective(), (1e-4, 1e-6)),
             ("lp_config0", I.lp_config0(0), json.load(open(golden0))["objective"], (1e-4, 1e-8))]
    for name, inst, oracle, gaps in cases:
        m, n = inst["m"], inst["n"]
        A = E.Matrix.from_instance(inst)
        Ah = sp.csr_matrix((inst["val"], inst["idx"], inst["ptr"]), shape=(m, n))
        bscale = 1.0 + max(np.abs(inst["rl"]).max(), np.abs(inst["ru"]).max())

        def quality(x, r):
            act = Ah @ x
            viol = max(0.0, float(np.max(inst["rl"] - act)), float(np.max(act - inst["ru"])))
            obj = float(np.dot(inst["c"], x))
            q = {"status": r["status"], "iterations": r["iterations"], "objective": obj,
                 "row_violation_rel": viol / bscale, "relative_primal_residual": _finite(r["relative_primal_residual"]),
                 "relative_dual_residual": _finite(r["relative_dual_residual"]),
                 "relative_gap": _finite(r["relative_gap"])}
            if oracle is not None:
                q["objective_rel_err_vs_oracle"] = abs(obj - oracle) / (1.0 + abs(oracle))
            return q

        def settings(eps):
            p = E.pdlp_default_settings()
            p.eps_optimal, p.time_limit, p.max_iterations = eps, time_limit, 20_000_000
            return p

        leg = {"workload": f"{name}: m={m:,}, n={n:,}, {int(inst['ptr'][-1]):,} nnz", "oracle_objective": oracle}
        t0 = time.perf_counter()
        rc, x, _, r = E.pdlp_solve(A, inst, settings(1e-4))
        if rc != 0:
            raise RuntimeError(E.last_error())
        leg["plain_1e-4"] = {"seconds": round(time.perf_counter() - t0, 2), **quality(x, r)}
        for gap in gaps:
            t0 = time.perf_counter()
            rc, x, _, r, pr = E.pdlp_solve_polished(A, inst, settings(gap))
            if rc != 0:
                raise RuntimeError(E.last_error())
            leg[f"polished_gap_{gap:.0e}"] = {
                "seconds": round(time.perf_counter() - t0, 2), **quality(x, r),
                "rounds": pr["rounds"], "main_iterations": pr["main_iterations"],
                "primal_polish_iterations": pr["primal_iterations"], "dual_polish_iterations": pr["dual_iterations"],
                "main_seconds": round(pr["main_seconds"], 2), "polish_seconds": round(pr["polish_seconds"], 2),
                "last_pair": {"relative_primal_residual": _finite(pr["pair_relative_primal_residual"]),
                              "relative_gap": _finite(pr["pair_relative_gap"]),
                              "primal_objective": _finite(pr["pair_primal_objective"])},
                "main_at_last_handover": {"relative_primal_residual": _finite(pr["main_relative_primal_residual"]),
                                          "relative_gap": _finite(pr["main_relative_gap"])}}
        out[name] = leg
        A.close()
    return out


def _finite(v):
    """A float for the JSON line, or None where it is not finite (NaN is not JSON)."""
    v = float(v)
    return v if np.isfinite(v) else None


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    I = _load("sankhya_b200_instances", os.path.join(ROOT, "the-solver_b200", "instances.py"))
    inst = I.lp_config1(SEED)
    nnz = int(inst["ptr"][-1])
    per_step = REFERENCE_ITERS_PER_CALL  # the same calls as the engine line's cpu_baseline sample
    core = reference_core()
    for _ in range(args.warmup):
        reference_loop_gbs(inst, 1, core)
    total_secs, total_iters = 0.0, 0
    for _ in range(args.steps):
        gbs, secs, its = reference_loop_gbs(inst, per_step, core)
        total_secs += secs
        total_iters += its
    value = iteration_bytes(M if inst["m"] == M else inst["m"], inst["n"], nnz) * total_iters / total_secs / 1e9
    line = {"metric": METRIC, "value": round(value, 4), "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * total_secs / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "m": inst["m"], "n": inst["n"], "nnz": nnz,
                       "iterations_per_step": per_step, "seed": SEED},
            "cpu_baseline": {"value": round(value, 4), "unit": "GB/s", "cores": core[1], "kind": "reference",
                             "sample": f"{per_step} iterations of the reference sk_solve first-order loop per step "
                                       f"({_core_text(core)})"},
            "e2e": {"value": round(value, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_engine(args, world, rank, local):
    import torch
    E = _load("sankhya_b200", os.path.join(ROOT, "the-solver_b200", "__init__.py"))
    I = _load("sankhya_b200_instances", os.path.join(ROOT, "the-solver_b200", "instances.py"))
    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    t0 = time.time()
    inst = I.lp_config1(SEED + rank)
    m, n, nnz = inst["m"], inst["n"], int(inst["ptr"][-1])
    gen_s = time.time() - t0
    t0 = time.time()
    A = E.Matrix.from_instance(inst)
    create_s = time.time() - t0
    # pinned host copies of the per-call inputs and the solution
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).pin_memory().numpy()
    host = {k: pin(inst[k]) for k in ("c", "rl", "ru", "cl", "cu")}
    x_out = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    # steps: 0.9 / (1 + mass) per row / column (the reference CPU path's diagonal steps)
    rows = np.repeat(np.arange(m), np.diff(inst["ptr"]))
    rmass = np.bincount(rows, weights=np.abs(inst["val"]), minlength=m)
    cmass = np.bincount(inst["idx"], weights=np.abs(inst["val"]), minlength=n)
    ps, ds = pin(0.9 / (1 + cmass)), pin(0.9 / (1 + rmass))
    s = E.settings(ITERS_PER_STEP, ITERS_PER_STEP, 0.0, 0.0, 1.0, 1e-12)

    def step():
        rc, x, y, r = E.pdhg(A, host, s, primal_steps=ps, dual_steps=ds, entry="preconditioned", x_out=x_out)
        if rc not in (0,):
            raise RuntimeError(f"sankhya_cuda_qp_pdhg_preconditioned returned {rc}: {E.last_error()}")
        return r

    # per-kernel durations (timing level 2: events around every launch), untimed
    E.set_timing(2)
    step()
    t_kern = E.last_timing()
    E.set_timing(1)
    for _ in range(max(3, args.warmup)):
        step()
    barrier(world)
    torch.cuda.synchronize()
    dev_ms, launches, iters, h2d_ms, d2h_ms = 0.0, 0, 0, 0.0, 0.0
    with ClockSampler(local) as clk:
        t_start = time.perf_counter()
        for _ in range(args.steps):
            step()
            t = E.last_timing()
            dev_ms += t["loop_ms"] + t["checkpoint_ms"]
            h2d_ms += t["h2d_ms"]
            d2h_ms += t["d2h_ms"]
            launches += t["kernel_launches"]
            iters += t["iterations"]
        torch.cuda.synchronize()
        wall = time.perf_counter() - t_start
    barrier(world)
    wall = barrier_max(wall, world)
    dev_ms = barrier_max(dev_ms, world)
    bytes_iter = iteration_bytes(m, n, nnz)
    value = job_throughput(world, bytes_iter, iters, dev_ms / 1e3)
    e2e = job_throughput(world, bytes_iter, iters, wall)
    if rank != 0:
        return 0
    peak, peak_kind = measured_peak()
    d_ms, p_ms = t_kern["dual_kernel_ms"], t_kern["primal_kernel_ms"]
    dom_ms, dom_bytes, dom_name = (p_ms, primal_bytes(m, n, nnz), "A'-side (primal) launch") if p_ms >= d_ms else \
        (d_ms, dual_bytes(m, n, nnz), "A-side (dual) launch")
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_lp_config1.txt")
    if os.path.exists(tpath):
        figures = dict(line.strip().split("=", 1) for line in open(tpath)
                       if "=" in line and not line.lstrip().startswith("#"))
        key = "primal" if p_ms >= d_ms else "dual"
        traffic = int(figures[key]) if key in figures else None
    line = {"metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * wall / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "m": m, "n": n, "nnz": nnz, "iterations_per_step": ITERS_PER_STEP,
                       "seed": SEED, "entry_point": "sankhya_cuda_qp_pdhg_preconditioned (LP, diagonal steps)",
                       "l2": f"inputs larger than L2: {(12 * nnz * 2) / 1e6:.0f} MB of A and A^T streamed per "
                             f"iteration", "parallelism": "replicas" if world > 1 else "single"},
            "iterations_per_s": round(world * iters / (dev_ms / 1e3), 1),
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": round(achieved, 1) if achieved else None,
                         "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4) if achieved else None,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": dom_bytes, "avg_launch_ms": round(dom_ms, 4),
                         "other_launch_ms": round(d_ms if p_ms >= d_ms else p_ms, 4)},
            "e2e": {"value": round(e2e, 2), "unit": "GB/s",
                    "h2d_bytes_per_step": 8 * (4 * n + 3 * m), "d2h_bytes_per_step": 8 * n,
                    "wall_ms_per_step": round(1e3 * wall / max(1, args.steps), 3),
                    "h2d_ms_per_step": round(h2d_ms / max(1, args.steps), 3),
                    "d2h_ms_per_step": round(d2h_ms / max(1, args.steps), 3)},
            "gpu_launches": launches, "clocks": clk.summary(), "setup_s": {"generate": round(gen_s, 1),
                                                                                  "matrix_create": round(create_s, 3)}}
    if world == 1 and not args.no_time_to_kkt:
        line["time_to_kkt"] = time_to_kkt(E, A, inst)
        line["config0_time_to_1e8"] = config0_to_1e8(E, I)
    if world == 1 and not args.no_reference_gpu:
        line["reference_gpu"] = reference_gpu_baseline(E, A, inst, ps, ds)
        ttk = line.get("time_to_kkt", {}).get("eps_1e-06", {}).get("fp64", {})
        g = line["reference_gpu"].get("gpupdlp", {})
        if ttk.get("status") == 0 and g.get("converged") == 1:
            g["engine_fp64_seconds"] = ttk["seconds"]
            g["engine_speedup"] = round(g["seconds"] / ttk["seconds"], 2)
    if world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(inst)
        except Exception as exc:  # the reference core is test infrastructure; report why it is missing
            line["cpu_baseline"] = {"value": None, "unit": "GB/s", "cores": 1, "kind": "reference",
                                    "sample": f"unavailable: {exc}"}
    print(json.dumps(line), flush=True)
    A.close()
    return 0


def _device_us(E, run, settings, iterations, reps=3):
    """Device time per iteration of a batched solve: CUDA events around its
    iteration loop (windows and per-LP checks), best of reps, after one warm-up."""
    E.set_timing(1)
    try:
        run(settings(iterations))
        best = None
        for _ in range(reps):
            if run(settings(iterations)) != 0:
                raise RuntimeError(f"batched solve failed: {E.last_error()}")
            t = E.last_timing()
            per = 1e3 * t["loop_ms"] / t["iterations"]
            best = per if best is None else min(best, per)
        return best
    finally:
        E.set_timing(0)


def run_batches(args):
    """Batched workloads (not the headline line): 256 node relaxations of one
    binary MILP sharing A (m=5,000, n=10,000, 6 per column), as a shared-matrix
    batch and as a block-diagonal batch, and 4,096 uneven LPs (m log-U[50, 5,000],
    n = 2m, 4-8 per column) as a block-diagonal batch. --small: 64 nodes and 256
    LPs. Prints one JSON line."""
    E = _load("sankhya_b200", os.path.join(ROOT, "the-solver_b200", "__init__.py"))
    I = _load("sankhya_b200_instances", os.path.join(ROOT, "the-solver_b200", "instances.py"))
    nodes_n, lps_n = (64, 256) if args.small else (256, 4096)

    def settings(its):
        s = E.batch_default_settings()
        s.max_iterations, s.primal_tol, s.dual_tol = its, 1e-14, 1e-14   # fixed work: no LP stops early
        return s

    nodes = I.milp_nodes(3, nodes_n)
    base = nodes[0]
    A = E.Matrix.from_instance(base)
    cl = np.stack([nd["cl"] for nd in nodes])
    cu = np.stack([nd["cu"] for nd in nodes])
    shared = _device_us(E, lambda s: E.shared_batch_pdhg(A, nodes_n, base["c"], base["rl"], base["ru"], cl, cu, s)[0],
                        settings, 2000)
    m, n, nnz = base["m"], base["n"], int(base["ptr"][-1])
    bp = (nodes_n + 31) // 32 * 32
    shared_bytes = (2 * 12 * nnz + 4 * (m + 1) + 4 * (n + 1) + 8 * bp * (n + 2 * m) + 8 * bp * (m + 5 * n)
                    + 16 * (m + n))
    if args.nodes_only:
        print(json.dumps({"metric": "batched PDHG, device time per iteration (CUDA events around the iteration loop)",
                          "unit": "us", "higher_is_better": False, "data": "synthetic", "dtype": "f64",
                          "node_relaxations": {"workload": f"{nodes_n} node relaxations sharing A",
                                               "shared_matrix_us": round(shared, 2)}}))
        return 0
    blk, rseg, cseg = E.block_diagonal(nodes)
    B = E.Matrix.from_instance(blk)
    blockdiag = _device_us(E, lambda s: E.batch_pdhg(B, blk, rseg, cseg, s)[0], settings, 2000)
    lps = I.lp_batch_uneven(7, lps_n, 50, 5000)
    blk3, rseg3, cseg3 = E.block_diagonal(lps)
    B3 = E.Matrix.from_instance(blk3)
    uneven = _device_us(E, lambda s: E.batch_pdhg(B3, blk3, rseg3, cseg3, s)[0], settings, 400)
    M3, N3, NNZ3 = blk3["m"], blk3["n"], int(blk3["ptr"][-1])
    uneven_bytes = iteration_bytes(M3, N3, NNZ3)
    peak, peak_kind = measured_peak()
    out = {"metric": "batched PDHG, device time per iteration (CUDA events around the iteration loop)", "unit": "us",
           "higher_is_better": False, "data": "synthetic", "dtype": "f64",
           "node_relaxations": {"workload": f"{nodes_n} node relaxations sharing A, m={m}, n={n}, nnz={nnz}",
                                "shared_matrix_us": round(shared, 2), "block_diagonal_us": round(blockdiag, 2),
                                "shared_speedup": round(blockdiag / shared, 2),
                                "shared_algorithmic_gbs": round(shared_bytes / shared / 1e3, 1),
                                "shared_frac_of_hbm": round(shared_bytes / shared / 1e3 / peak, 3)},
           "uneven_lps": {"workload": f"{lps_n} uneven LPs, m={M3}, n={N3}, nnz={NNZ3}", "block_diagonal_us":
                          round(uneven, 2), "algorithmic_gbs": round(uneven_bytes / uneven / 1e3, 1),
                          "frac_of_hbm": round(uneven_bytes / uneven / 1e3 / peak, 3)},
           "peak_kind": peak_kind}

    # time to the gates: each LP runs sk_solve's loop until its own gates pass (row
    # violation, step and dual-step tests at 1e-4, checked every 20 iterations), the
    # reference's stopping rule for that loop; wall time of the whole batch call
    def to_gates(run, cap):
        s = E.batch_default_settings()
        s.max_iterations, s.primal_tol, s.dual_tol = cap, 1e-4, 1e-4
        run(s)
        t0 = time.perf_counter()
        rc, res = run(s)
        wall = time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError(E.last_error())
        its = np.array([r["iterations"] for r in res])
        return {"seconds": round(wall, 3), "tolerance": 1e-4, "iteration_cap": cap,
                "converged": int(sum(r["status"] == 0 for r in res)), "lps": len(res),
                "iterations_median": int(np.median(its)), "iterations_max": int(its.max())}

    def shared_run(s):
        rc, _, _, res = E.shared_batch_pdhg(A, nodes_n, base["c"], base["rl"], base["ru"], cl, cu, s)
        return rc, res

    def uneven_run(s):
        rc, _, _, res = E.batch_pdhg(B3, blk3, rseg3, cseg3, s)
        return rc, res

    out["node_relaxations"]["to_gates"] = to_gates(shared_run, 50_000)
    out["uneven_lps"]["to_gates"] = to_gates(uneven_run, 50_000)
    print(json.dumps(out))
    return 0


def run_qp(args):
    """Convex QP workload (not the headline line): n = 200,000, m = 100,000, A with 10
    N(0,1) entries per column, Q = diag(log-U[1e-2, 1e2]) + L L^T (L: 3 N(0, 0.1)
    entries per column), bounds [-5, 5], rows x0 -/+ U(0,1). Device time per PDHG
    iteration of the diagonal-proximal path (sankhya_cuda_diagonal_qp_pdhg, Q's
    diagonal D) and of the general sparse-Hessian path (sankhya_cuda_sparse_qp_pdhg,
    explicit Q = D + L L^T: one more fused product per iteration), then the restarted
    PDLP QP solve (sankhya_b200_pdlp_solve_qp) to 1e-6 relative KKT on both paths, FP64
    and FP32 iterations refined in FP64. Prints one JSON line."""
    E = _load("sankhya_b200", os.path.join(ROOT, "the-solver_b200", "__init__.py"))
    I = _load("sankhya_b200_instances", os.path.join(ROOT, "the-solver_b200", "instances.py"))
    inst = I.qp_config2(2)
    m, n, nnz = inst["m"], inst["n"], int(inst["ptr"][-1])
    qnnz = int(inst["q_ptr"][-1])
    A = E.Matrix.from_instance(inst)
    Q = E.Matrix.from_instance(inst, hessian=True)
    its = 400
    s = E.settings(its, its, 0.005, 0.5, 1.0, 1e-300)   # tau |Q| < 1, tau sigma |A|^2 < 1
    paths = {"diagonal": dict(qdiag=inst["qdiag"]), "sparse_hessian": dict(hessian=Q)}
    extra = {"diagonal": 8 * n, "sparse_hessian": 12 * qnnz + 4 * (n + 1) + 8 * n + 16 * n}
    out = {"metric": "QP PDHG device time per iteration", "unit": "us", "higher_is_better": False,
           "data": "synthetic", "dtype": "f64",
           "workload": f"qp_config2: n={n}, m={m}, nnz(A)={nnz}, nnz(Q)={qnnz}, Q = D + L L^T"}
    peak, _ = measured_peak()
    for name, kw in paths.items():
        E.set_timing(1)
        E.pdhg(A, inst, s, **kw)
        best = None
        for _ in range(3):
            rc, x, y, r = E.pdhg(A, inst, s, **kw)
            if rc != 0:
                raise RuntimeError(f"{name}: {E.last_error()}")
            t = E.last_timing()
            per = 1e3 * (t["loop_ms"] + t["checkpoint_ms"]) / t["iterations"]
            best = per if best is None else min(best, per)
        E.set_timing(0)
        byt = iteration_bytes(m, n, nnz) + extra[name]
        out[name] = {"us_per_iteration": round(best, 2), "algorithmic_bytes": byt,
                     "algorithmic_gbs": round(byt / best / 1e3, 1), "frac_of_hbm": round(byt / best / 1e3 / peak, 3),
                     "objective_after": r["objective"]}
    # restarted PDLP with the quadratic term to 1e-6 relative KKT: the diagonal Hessian
    # (exact prox; the QP with Q's diagonal D) and the general Hessian (Q = D + L L^T,
    # one more fused product per iteration), FP64 and FP32 iterations refined in FP64
    ttk = {"eps": 1e-6, "relative_kkt": "max(primal, dual, gap), reduced cost c + Qx + A'y"}
    for name, kw in (("diagonal", dict(qdiag=inst["qdiag"])), ("sparse_hessian", dict(hessian=Q))):
        for label, prec in (("fp64", E.FP64), ("fp32_refined", E.FP32_REFINE)):
            ps_ = E.pdlp_default_settings()
            ps_.eps_optimal, ps_.precision, ps_.time_limit, ps_.max_iterations = 1e-6, prec, 120.0, 20_000_000
            E.pdlp_solve_qp(A, inst, ps_, **kw)       # warm-up: plans, graphs, attributes
            t0 = time.perf_counter()
            rc, x, y, r = E.pdlp_solve_qp(A, inst, ps_, **kw)
            wall = time.perf_counter() - t0
            ttk[f"{name}_{label}"] = {"seconds": round(wall, 3), "status": r["status"], "iterations": r["iterations"],
                                      "restarts": r["restarts"], "refinements": r["refinements"],
                                      "primal_objective": _finite(r["primal_objective"]),
                                      "kkt": [_finite(r[k]) for k in ("relative_primal_residual",
                                                                      "relative_dual_residual", "relative_gap")]}
        a, b_ = ttk[f"{name}_fp64"], ttk[f"{name}_fp32_refined"]
        if a["status"] == 0 and b_["status"] == 0 and b_["seconds"] > 0:
            ttk[f"{name}_speedup_fp32_refined_vs_fp64"] = round(a["seconds"] / b_["seconds"], 3)
    out["time_to_kkt"] = ttk
    print(json.dumps(out))
    return 0


def run_pdlp_compare(args):
    """Restarted PDLP to 1e-6 relative KKT, GpuPdlp's adaptive loop versus the
    reflected restarted Halpern loop (FP64, default scaling), on four seeded
    instances of the engine's recipes. Prints one JSON line."""
    E = _load("sankhya_b200", os.path.join(ROOT, "the-solver_b200", "__init__.py"))
    I = _load("sankhya_b200_instances", os.path.join(ROOT, "the-solver_b200", "instances.py"))
    cases = (("lp_uniform(3, 20000, 40000, 5)", lambda: I.lp_uniform(3, 20000, 40000, 5)),
             ("lp_powerlaw(5, 200000, 400000, 4000000)", lambda: I.lp_powerlaw(5, 200000, 400000, 4000000)),
             ("milp_nodes(3, 1)[0]", lambda: I.milp_nodes(3, 1)[0]),
             ("lp_family_base(4, 50000, 100000, 10)", lambda: I.lp_family_base(4, 50000, 100000, 10)))
    rows = []
    for name, make in cases:
        inst = make()
        A = E.Matrix.from_instance(inst)
        row = {"instance": name}
        for label, alg in (("adaptive", E.PDLP_ADAPTIVE), ("halpern", E.PDLP_HALPERN)):
            s = E.pdlp_default_settings()
            s.eps_optimal, s.time_limit, s.algorithm = 1e-6, 120.0, alg
            E.pdlp_solve(A, inst, s)                     # warm-up: graphs, allocations
            t = time.perf_counter()
            rc, x, y, r = E.pdlp_solve(A, inst, s)
            row[label] = {"seconds": round(time.perf_counter() - t, 4), "status": r["status"],
                          "iterations": r["iterations"], "restarts": r["restarts"],
                          "objective": float(np.dot(inst["c"], x))}
        if row["adaptive"]["status"] == 0 and row["halpern"]["status"] == 0:
            row["speedup_halpern"] = round(row["adaptive"]["seconds"] / row["halpern"]["seconds"], 3)
        rows.append(row)
    print(json.dumps({"metric": "PDLP wall time to 1e-6 relative KKT", "unit": "s", "higher_is_better": False,
                      "data": "synthetic", "dtype": "f64", "cases": rows}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-time-to-kkt", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true", help="skip the reference GPU baseline legs")
    ap.add_argument("--batches", action="store_true", help="batched workloads instead of the headline line")
    ap.add_argument("--small", action="store_true", help="with --batches: 64 nodes and 256 LPs")
    ap.add_argument("--nodes-only", action="store_true", help="with --batches: the shared-matrix node batch only")
    ap.add_argument("--qp", action="store_true", help="convex QP workload instead of the headline line")
    ap.add_argument("--pdlp-compare", action="store_true", help="adaptive versus Halpern PDLP on four instances")
    ap.add_argument("--crossover", action="store_true",
                    help="config 0 to a certified vertex: engine PDLP, then the crossover sources")
    ap.add_argument("--polish", action="store_true",
                    help="feasibility polishing on configs 1 and 0 beside the plain restarted solve")
    ap.add_argument("--plain-pdhg", action="store_true",
                    help="plain fixed-step FP64 PDHG against the restarted refined PDLP on config 1")
    args = ap.parse_args()
    if args.plain_pdhg:
        return run_plain_pdhg(args)
    if args.polish:
        return run_polish(args)
    if args.crossover:
        return run_crossover(args)
    if args.pdlp_compare:
        return run_pdlp_compare(args)
    if args.batches:
        return run_batches(args)
    if args.qp:
        return run_qp(args)
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            return run_reference(args, world, rank)
        return run_engine(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
