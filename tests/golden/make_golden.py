"""Generates the golden fixtures in this folder from the reference's own C core.

Run from the repository root after `make -C oracle ref` (which compiles the
reference's c/src/*.c into oracle/_ref/libsankhya_ref.so):

    python tests/golden/make_golden.py

Every fixture is an output of a reference routine on a seeded synthetic
instance built by the-solver_b200/instances.py:
  sk_loop_*.npz     sk_solve with lp_engine = SK_LP_FIRST_ORDER (c/src/sk_solve.c:801-1046)
                    stopped by iteration_limit: x, y, rowact, iterations, objective
  sk_qp_*.npz       the same for a convex QP (Q = D + L L^T) through sk_solve
  sk_verify_*.npz   sk_verify (c/src/sk_core.c:394-510) on the sk_loop points
  sk_scale_*.npz    sk_scale_model (c/src/sk_scale.c:20-72) row / column factors
  simplex_*.json    sk_simplex_solve's optimal objective for small LPs (the objective oracle)
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
OUT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

spec = importlib.util.spec_from_file_location("instances", os.path.join(ROOT, "the-solver_b200", "instances.py"))
I = importlib.util.module_from_spec(spec)
spec.loader.exec_module(I)

LP_CASES = [  # (name, seed, m, n, per_col, iteration limits)
    ("lp300", 11, 300, 700, 5, (1, 20, 137, 400)),
    ("lp60", 12, 60, 150, 4, (7, 40)),
]
QP_CASES = [("qp700", 13, 600, 700, (20, 160))]  # both sizes > 512: no post-loop polish


def main():
    manifest = {}
    for name, seed, m, n, per_col, limits in LP_CASES:
        inst = I.lp_uniform(seed, m, n, per_col)
        for lim in limits:
            st, r = O.ref_sk_solve(inst, primal_tol=1e-300, dual_tol=1e-300, iteration_limit=lim)
            assert st == 0
            path = os.path.join(OUT, f"sk_loop_{name}_it{lim}.npz")
            np.savez_compressed(path, x=r["x"], y=r["y"], rowact=r["rowact"],
                                iterations=np.int64(r["iterations"]), objective=np.float64(r["objective"]),
                                result=np.int64(r["result"]))
            vs, v = O.ref_sk_verify(inst, r["x"], r["y"])
            np.savez_compressed(os.path.join(OUT, f"sk_verify_{name}_it{lim}.npz"),
                                **{k: np.float64(val) for k, val in v.items()})
            manifest[f"sk_loop_{name}_it{lim}"] = dict(seed=seed, m=m, n=n, per_col=per_col, limit=lim)
        R, Cs = O.ref_sk_scale_model(inst, 4)
        np.savez_compressed(os.path.join(OUT, f"sk_scale_{name}.npz"), R=R, C=Cs)
        st, simplex = O.ref_sk_solve(inst, lp_engine=1, primal_tol=1e-9, dual_tol=1e-9)
        with open(os.path.join(OUT, f"simplex_{name}.json"), "w") as f:
            json.dump(dict(status=st, result=simplex["result"], objective=simplex["objective"],
                           iterations=simplex["iterations"]), f, indent=1)
    for name, seed, m, n, limits in QP_CASES:
        inst = I.qp_diag_plus_lowrank(seed, m, n, a_per_col=4, l_per_col=2)
        for lim in limits:
            st, r = O.ref_sk_solve(inst, quadratic=True, primal_tol=1e-300, dual_tol=1e-300, iteration_limit=lim)
            assert st == 0, st
            np.savez_compressed(os.path.join(OUT, f"sk_qp_{name}_it{lim}.npz"), x=r["x"], y=r["y"],
                                iterations=np.int64(r["iterations"]), objective=np.float64(r["objective"]),
                                result=np.int64(r["result"]))
            manifest[f"sk_qp_{name}_it{lim}"] = dict(seed=seed, m=m, n=n, limit=lim)
    with open(os.path.join(OUT, "manifest.json"), "w") as f:
        json.dump(dict(cases=manifest, lp=LP_CASES, qp=QP_CASES), f, indent=1)


if __name__ == "__main__":
    main()
