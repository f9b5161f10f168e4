"""Writes objective_lp_config1.json: the FP64 objective of the 1,000,000 x 2,000,000
power-law LP (instances.lp_config1, seed 1, about 20,000,000 nonzeros), the value
the timed PDLP runs are compared with.

No simplex finishes on this LP in reasonable time, and the restarted PDLP loop stalls
near a 2e-6 relative gap on it (both implementations below share that algorithm), so
the value comes from two independent FP64 first-order solves on a GPU run to the
tightest tolerance they reach (--eps, default 1e-7):
  - the reference's own GPU PDLP (src/cuda/GpuPdlp.cpp over cuSPARSE, with the scaling
    of its run_first_order driver), built into oracle/_ref by `make -C oracle ref`,
  - this repository's engine (sankhya_b200_pdlp_solve, FP64, Ruiz + Pock-Chambolle).
Both objectives, their relative KKT triples, dual objectives, iterations and times are
written. The file's `objective` is the reference's primal objective when it converged
(else the engine's), so the engine's runs are measured against an independent code;
`rel_diff_engine_vs_reference` says how far apart the two landed. Every column of
this LP is boxed, so each dual objective is a valid lower bound on the optimum;
`lower_bound` is the larger one. Run on a machine with a GPU:

    python tests/golden/make_config1_objective.py [--out PATH]
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "objective_lp_config1.json")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=OUT)
    ap.add_argument("--eps", type=float, default=1e-7)
    ap.add_argument("--limit", type=float, default=300.0, help="seconds per solve")
    a = ap.parse_args()
    E = _load("sankhya_b200", os.path.join(ROOT, "the-solver_b200", "__init__.py"))
    I = _load("sankhya_b200_instances", os.path.join(ROOT, "the-solver_b200", "instances.py"))
    import oracle as O
    import torch
    torch.cuda.set_device(0)
    inst = I.lp_config1(1)
    A = E.Matrix.from_instance(inst)
    s = E.pdlp_default_settings()
    s.eps_optimal, s.time_limit, s.max_iterations = a.eps, a.limit, 20_000_000
    t = time.perf_counter()
    rc, x, y, r = E.pdlp_solve(A, inst, s)
    engine = dict(seconds=round(time.perf_counter() - t, 2), status=r["status"], iterations=r["iterations"],
                  objective=float(np.dot(inst["c"], x)), dual_objective=r["dual_objective"],
                  kkt=[r["relative_primal_residual"], r["relative_dual_residual"], r["relative_gap"]])
    A.close()
    print("engine", engine, flush=True)
    reference = None
    if O.available("ref_pdlp"):
        t = time.perf_counter()
        xr, st = O.ref_gpupdlp(inst, eps=a.eps, max_iterations=20_000_000, time_limit=a.limit, scale=True)
        reference = dict(seconds=round(time.perf_counter() - t, 2), converged=st["converged"],
                         iterations=st["iterations"], objective=float(np.dot(inst["c"], xr)),
                         dual_objective=st["dual_objective"],
                         kkt=[st["relative_primal_residual"], st["relative_dual_residual"], st["relative_gap"]])
        print("reference", reference, flush=True)
    use_ref = reference is not None and reference["converged"] == 1
    out = dict(instance="lp_config1(1): m=1,000,000, n=2,000,000, Zipf(1.5) column degrees, |a| log-U[1e-3,1e3]",
               eps=a.eps, objective=reference["objective"] if use_ref else engine["objective"],
               objective_from="reference GpuPdlp" if use_ref else "engine", engine=engine,
               reference_gpupdlp=reference)
    bounds = [engine["dual_objective"]] + ([reference["dual_objective"]] if reference is not None else [])
    out["lower_bound"] = max(b for b in bounds if np.isfinite(b))
    if reference is not None:
        out["rel_diff_engine_vs_reference"] = abs(engine["objective"] - reference["objective"]) / (
            1.0 + abs(reference["objective"]))
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
