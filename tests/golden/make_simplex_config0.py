"""Writes simplex_lp_config0.json: the optimal objective of the 2,000 x 5,000 LP
(instances.lp_config0, seed 0) from the reference's own simplex.

Run from the repository root after `make -C oracle ref` (which compiles the
reference's c/src/*.c into oracle/_ref/libsankhya_ref.so):

    python tests/golden/make_simplex_config0.py

sk_solve with lp_engine = SK_LP_SIMPLEX (1) sends a continuous LP to sk_simplex_solve
(c/src/sk_solve.c:1009-1046 -> c/src/sk_simplex.c), whose result sk_verify
certifies (c/src/sk_core.c:394-510). It runs for several minutes on one core.
The same LP is also solved by scipy's HiGHS (an independent third-party simplex /
interior-point code) as a cross-check; both objectives are written, and the
script fails if they differ by more than 1e-9 relative.
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
OUT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

spec = importlib.util.spec_from_file_location("instances", os.path.join(ROOT, "the-solver_b200", "instances.py"))
I = importlib.util.module_from_spec(spec)
spec.loader.exec_module(I)


def highs_objective(inst):
    import scipy.sparse as sp
    from scipy.optimize import linprog
    A = sp.csr_matrix((inst["val"], inst["idx"], inst["ptr"]), shape=(inst["m"], inst["n"]))
    A2 = sp.vstack([A, -A]).tocsr()
    b2 = np.concatenate([inst["ru"], -inst["rl"]])
    res = linprog(inst["c"], A_ub=A2, b_ub=b2, bounds=list(zip(inst["cl"], inst["cu"])), method="highs-ds",
                  options=dict(primal_feasibility_tolerance=1e-10, dual_feasibility_tolerance=1e-10))
    if res.status != 0:
        raise RuntimeError(f"HiGHS failed: {res.message}")
    return float(res.fun)


def main():
    inst = I.lp_config0(0)
    t0 = time.time()
    highs = highs_objective(inst)
    t_highs = time.time() - t0
    t0 = time.time()
    st, r = O.ref_sk_solve(inst, lp_engine=1, primal_tol=1e-9, dual_tol=1e-9)
    t_ref = time.time() - t0
    if st != 0 or r["result"] != 0:
        raise RuntimeError(f"reference simplex did not reach optimality: status {st}, result {r['result']}")
    vs, cert = O.ref_sk_verify(inst, r["x"], r["y"])
    obj = float(r["objective"])
    rel = abs(obj - highs) / (1.0 + abs(highs))
    if rel > 1e-9:
        raise RuntimeError(f"reference simplex {obj!r} and HiGHS {highs!r} differ by {rel:.3e}")
    with open(os.path.join(OUT, "simplex_lp_config0.json"), "w") as f:
        json.dump(dict(instance="lp_config0(0): m=2000, n=5000, 5 per column", status=st, result=r["result"],
                       objective=obj, iterations=r["iterations"], seconds=round(t_ref, 1),
                       sk_verify={k: float(v) for k, v in cert.items()},
                       highs_objective=highs, highs_seconds=round(t_highs, 1), rel_diff_vs_highs=rel), f, indent=1)


if __name__ == "__main__":
    main()
