"""Crossover from a first-order point to a vertex (include/integration/sk_crossover.c),
built against the reference's C core and run on the CPU: from the points of the
oracle's PDLP restatement (the engine's algorithm), of the reference's own first-order
loop, and from deliberately wrong points, the answer must be the optimum the reference
simplex certifies, with sk_verify's residuals at simplex accuracy."""
import json
import os

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


@pytest.fixture(scope="module")
def oracle():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not (O.available("ref_crossover") and O.available("oracle")):
        pytest.skip("reference C core not built (make -C oracle ref)")
    return O


CASES = {"lp60": (12, 60, 150, 4), "lp300": (11, 300, 700, 5)}


def golden(name):
    return json.load(open(os.path.join(ROOT, "tests", "golden", f"simplex_{name}.json")))


def certified(out, objective):
    assert out["result"] == 0, out
    assert out["primal_infeasibility"] <= 1e-9 and out["dual_infeasibility"] <= 1e-9, out
    assert abs(out["objective"] - objective) <= 1e-9 * (1.0 + abs(objective)), (out["objective"], objective)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("eps", [1e-4, 1e-6, 1e-8])
def test_from_pdlp_points(oracle, instances, name, eps):
    """From the PDLP restatement's point at 1e-4, 1e-6 and 1e-8: the certified simplex
    optimum, with columns fixed and fewer simplex iterations than the cold solve."""
    inst = instances.lp_uniform(*CASES[name])
    g = golden(name)
    x, y, _ = oracle.pdlp(inst, eps=eps, max_iterations=400000)
    rc, out = oracle.ref_crossover(inst, x, y)
    assert rc == 0
    certified(out, g["objective"])
    assert out["full_fallback"] == 0 and out["fixed_columns"] > 0, out
    assert out["simplex_iterations"] < g["iterations"], (out["simplex_iterations"], g["iterations"])
    assert out["iterations"] == out["simplex_iterations"]


def test_from_the_reference_first_order_loop(oracle, instances):
    """The point of the reference's own first-order loop (sk_solve, SK_LP_FIRST_ORDER)."""
    inst = instances.lp_uniform(*CASES["lp300"])
    st, fo = oracle.ref_sk_solve(inst, primal_tol=1e-6, dual_tol=1e-6, iteration_limit=100000)
    assert st == 0
    rc, out = oracle.ref_crossover(inst, fo["x"], fo["y"])
    assert rc == 0
    certified(out, golden("lp300")["objective"])


def test_wrong_duals_are_repaired_or_fall_back(oracle, instances):
    """A point whose duals point the wrong way fixes columns at the wrong bounds: the
    crossover releases them (or solves the whole model) and still certifies the optimum."""
    inst = instances.lp_uniform(*CASES["lp60"])
    g = golden("lp60")
    x, y, _ = oracle.pdlp(inst, eps=1e-6, max_iterations=400000)
    for bad_y in (-y, 3.0 * y, np.zeros_like(y)):
        rc, out = oracle.ref_crossover(inst, x, bad_y, max_rounds=3)
        assert rc == 0
        certified(out, g["objective"])
    # x mirrored in its box and the duals negated agree on the wrong bounds, so columns
    # are fixed there and must be released (with -y alone, x keeps them from fixing)
    mirrored = inst["cl"] + inst["cu"] - x
    rc, out = oracle.ref_crossover(inst, mirrored, -y, max_rounds=3)
    assert rc == 0 and out["fixed_columns"] >= 0
    certified(out, g["objective"])
    assert out["released_columns"] > 0 or out["full_fallback"] == 1, out


def test_one_sided_columns(oracle, instances):
    """x >= 0 without upper bounds: only the lower bound can be selected."""
    from scipy.optimize import linprog
    import scipy.sparse as sp
    inst = instances.lp_uniform(5, 80, 200, 4)
    inst["cu"] = np.full(inst["n"], 1e30)
    inst["cl"] = np.zeros(inst["n"])
    inst["c"] = np.abs(inst["c"]) + 0.1
    A = sp.csr_matrix((inst["val"], inst["idx"], inst["ptr"]), shape=(inst["m"], inst["n"]))
    ref = linprog(inst["c"], A_ub=sp.vstack([A, -A]), b_ub=np.concatenate([inst["ru"], -inst["rl"]]),
                  bounds=[(0, None)] * inst["n"], method="highs")
    assert ref.status == 0
    x, y, _ = oracle.pdlp(inst, eps=1e-6, max_iterations=400000)
    rc, out = oracle.ref_crossover(inst, x, y)
    assert rc == 0
    certified(out, float(ref.fun))
    assert out["full_fallback"] == 0


def test_argument_checks(oracle, instances):
    inst = instances.lp_uniform(*CASES["lp60"])
    x, y = np.zeros(inst["n"]), np.zeros(inst["m"])
    assert oracle.ref_crossover(inst, x, y, fix_tolerance=0.0)[0] == 1   # SK_ERR_ARG
    assert oracle.ref_crossover(inst, x, y, max_rounds=0)[0] == 1
