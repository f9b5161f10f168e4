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
    optimum, either from the identified basis as it stands (no simplex; always from the
    1e-8 point) or with columns held and fewer simplex iterations than the cold solve."""
    inst = instances.lp_uniform(*CASES[name])
    g = golden(name)
    x, y, _ = oracle.pdlp(inst, eps=eps, max_iterations=400000)
    rc, out = oracle.ref_crossover(inst, x, y)
    assert rc == 0
    certified(out, g["objective"])
    if out["direct"]:
        assert out["simplex_iterations"] == 0 and out["rounds"] == 0, out
    else:
        assert out["full_fallback"] == 0 and out["fixed_columns"] > 0, out
    if eps <= 1e-8:
        assert out["direct"] == 1, out
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


# ---------------------------------------------------------------- the C++ core's simplex

@pytest.fixture(scope="module")
def sihps(oracle):
    if not oracle.available("ref_sihps_crossover"):
        pytest.skip("reference C++ core not built (make -C oracle ref)")
    return oracle


def gate(out, objective):
    """OPTIMAL through the core's original-space gate (1e-6), at the simplex optimum."""
    assert out["status"] == 0, out
    assert out["primal_residual"] <= 1e-6 and out["dual_residual"] <= 1e-6, out
    assert abs(out["objective"] - objective) <= 1e-9 * (1.0 + abs(objective)), (out["objective"], objective)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("eps", [1e-4, 1e-6, 1e-8])
def test_seated_basis_from_pdlp_points(sihps, instances, name, eps):
    """A basis identified from the PDLP restatement's point, seated in the core's simplex:
    its warm path finishes it in a handful of dual pivots (the cold solve of lp300 takes
    3,785 primal pivots)."""
    inst = instances.lp_uniform(*CASES[name])
    x, y, _ = sihps.pdlp(inst, eps=eps, max_iterations=400000)
    rc, out = sihps.ref_sihps_crossover(inst, x, y)
    assert rc == 0
    gate(out, golden(name)["objective"])
    assert out["used_warm_start"] == 1 and out["cold_iterations"] == 0, out
    assert out["dual_iterations"] <= 50, out


def test_seated_basis_config0(sihps, instances):
    """Config 0 (2,000 x 5,000): from the 1e-6 point the warm dual simplex needs a few
    pivots, where the core's cold simplex takes minutes (312.6 s measured on this LP)."""
    inst = instances.lp_config0(0)
    x, y, _ = sihps.pdlp(inst, eps=1e-6, max_iterations=400000)
    rc, out = sihps.ref_sihps_crossover(inst, x, y)
    assert rc == 0
    gate(out, golden("lp_config0")["objective"])
    assert out["used_warm_start"] == 1 and out["dual_iterations"] <= 50, out
    assert out["seconds"] < 30.0, out


def test_seated_basis_wrong_point_falls_back(sihps, instances):
    """A point that names the wrong bounds: the core's gate refuses the warm answer or the
    repair takes longer, and the answer is still the optimum."""
    inst = instances.lp_uniform(*CASES["lp60"])
    x, y, _ = sihps.pdlp(inst, eps=1e-6, max_iterations=400000)
    rc, out = sihps.ref_sihps_crossover(inst, inst["cl"] + inst["cu"] - x, -y)
    assert rc == 0
    gate(out, golden("lp60")["objective"])


def test_seated_basis_one_sided_columns(sihps, instances):
    from scipy.optimize import linprog
    import scipy.sparse as sp
    inst = instances.lp_uniform(5, 80, 200, 4)
    inst["cu"] = np.full(inst["n"], np.inf)
    inst["cl"] = np.zeros(inst["n"])
    inst["c"] = np.abs(inst["c"]) + 0.1
    A = sp.csr_matrix((inst["val"], inst["idx"], inst["ptr"]), shape=(inst["m"], inst["n"]))
    ref = linprog(inst["c"], A_ub=sp.vstack([A, -A]), b_ub=np.concatenate([inst["ru"], -inst["rl"]]),
                  bounds=[(0, None)] * inst["n"], method="highs")
    x, y, _ = sihps.pdlp(inst, eps=1e-6, max_iterations=400000)
    rc, out = sihps.ref_sihps_crossover(inst, x, y)
    assert rc == 0
    gate(out, float(ref.fun))
    assert out["used_warm_start"] == 1, out


def test_seated_basis_time_budget(sihps, instances):
    """A budget the simplex cannot meet ends it with ITERATION_LIMIT (3), as HYBRID's
    budgeted simplex does, instead of a cold solve without end."""
    inst = instances.lp_uniform(*CASES["lp300"])
    x, y, _ = sihps.pdlp(inst, eps=1e-6, max_iterations=400000)
    rc, out = sihps.ref_sihps_crossover(inst, inst["cl"] + inst["cu"] - x, -y, time_budget=1e-9)
    assert rc == 0 and out["status"] == 3, out
    rc, out = sihps.ref_sihps_crossover(inst, x, y, time_budget=60.0)
    assert rc == 0 and out["status"] == 0 and out["used_warm_start"] == 1, out


@pytest.mark.parametrize("seed", [7, 8, 9, 10, 11])
@pytest.mark.parametrize("shape", [(10, 14), (30, 45)])
def test_mixed_row_and_column_types(sihps, seed, shape):
    """E, G, L and ranged rows; free, upper-only, boxed and fixed columns (the LPs the
    MPS tests write): both crossovers reach HiGHS's optimum, the C++ core's warm start
    without a fallback."""
    import sys
    import scipy.sparse as sp
    from scipy.optimize import linprog
    sys.path.insert(0, os.path.dirname(__file__))
    import mps_files
    m, n = shape
    inst = mps_files.lp_instance(seed, m, n)
    A = sp.csr_matrix((inst["val"], inst["idx"], inst["ptr"]), shape=(m, n)).toarray()
    eq = inst["rl"] == inst["ru"]
    up, lo = ~eq & np.isfinite(inst["ru"]), ~eq & np.isfinite(inst["rl"])
    G = np.vstack([A[up], -A[lo]])
    h = np.concatenate([inst["ru"][up], -inst["rl"][lo]])
    bounds = [(l if np.isfinite(l) else None, u if np.isfinite(u) else None) for l, u in zip(inst["cl"], inst["cu"])]
    ref = linprog(inst["c"], A_ub=G, b_ub=h, A_eq=A[eq], b_eq=inst["rl"][eq], bounds=bounds, method="highs")
    assert ref.status == 0
    x, y, st = sihps.pdlp(inst, eps=1e-6, max_iterations=200000)
    assert st["converged"]
    rc, out = sihps.ref_crossover(inst, x, y)
    assert rc == 0
    certified(out, float(ref.fun))
    rc, out = sihps.ref_sihps_crossover(inst, x, y)
    assert rc == 0
    gate(out, float(ref.fun))
    assert out["used_warm_start"] == 1, out


def test_config0_identified_basis_is_certified(oracle, instances):
    """Config 0 from its target tolerance (1e-8): the basis the point identifies is the
    optimal vertex as it stands; sk_verify certifies it with no simplex solve, where the
    cold simplex of the C core takes 876.8 s and 74,059 pivots."""
    inst = instances.lp_config0(0)
    x, y, _ = oracle.pdlp(inst, eps=1e-8, max_iterations=400000)
    rc, out = oracle.ref_crossover(inst, x, y)
    assert rc == 0
    certified(out, golden("lp_config0")["objective"])
    assert out["direct"] == 1 and out["simplex_iterations"] == 0, out


# the reference's PDLP known-answer LPs (tests/lp/test_pdlp.cpp:53-150), whose optimal
# vertices are stated there
INF = float("inf")
HAND = [
    (dict(rows=3, cols=2, dense=[1, 0, 0, 2, 3, 2], c=[-3, -5], rl=[-INF] * 3, ru=[4, 12, 18], cl=[0, 0],
          cu=[INF, INF]), [2.0, 6.0], -36.0),
    (dict(rows=1, cols=1, dense=[1], c=[-1], rl=[2], ru=[7], cl=[0], cu=[100]), [7.0], -7.0),
    (dict(rows=1, cols=2, dense=[1, 1], c=[-1, -1], rl=[-INF], ru=[100], cl=[0, 0], cu=[3, 4]), [3.0, 4.0], -7.0),
]


@pytest.mark.parametrize("case", range(len(HAND)))
def test_known_answer_vertices(sihps, instances, case):
    """The reference's own known answers: both crossovers return the stated vertex exactly
    (to the simplex's accuracy) from the PDLP restatement's 1e-6 point."""
    spec, vertex, objective = HAND[case]
    inst = instances.small_dense_lp(**spec)
    x, y, _ = sihps.pdlp(inst, eps=1e-6, max_iterations=100000)
    rc, out = sihps.ref_crossover(inst, x, y)
    assert rc == 0
    certified(out, objective)
    assert np.allclose(out["x"], vertex, atol=1e-9), out["x"]
    rc, out = sihps.ref_sihps_crossover(inst, x, y)
    assert rc == 0
    gate(out, objective)
    assert np.allclose(out["x"], vertex, atol=1e-9), out["x"]


@pytest.mark.parametrize("name", ["lp300", "lp_config0"])
def test_from_x_alone(sihps, instances, name):
    """A caller that kept only x (run_first_order returns x alone) passes y = 0: the basis
    is ranked by interiority, and both crossovers still reach the certified optimum, the
    C++ core through its warm start, the C core from the 1e-8 point with no simplex."""
    inst = instances.lp_uniform(*CASES[name]) if name in CASES else instances.lp_config0(0)
    g = golden(name)
    x, y, _ = sihps.pdlp(inst, eps=1e-8, max_iterations=400000)
    zero = np.zeros_like(y)
    rc, out = sihps.ref_sihps_crossover(inst, x, zero, time_budget=120.0)
    assert rc == 0
    gate(out, g["objective"])
    assert out["used_warm_start"] == 1 and out["dual_iterations"] <= 50, out
    rc, out = sihps.ref_crossover(inst, x, zero)
    assert rc == 0
    certified(out, g["objective"])
    assert out["direct"] == 1, out


# ------------------------------------------- HYBRID's simplex step through the crossover

@pytest.fixture(scope="module")
def stand_in(oracle):
    if not (oracle.available("ref_lp_cpu") and oracle.available("ref_lp_hybrid_cpu")):
        pytest.skip("LP driver builds over the CPU stand-in engine absent (make -C oracle ref-tests)")
    return oracle


def test_hybrid_fallback_through_the_crossover(stand_in, instances):
    """The reference's own LP driver, run_first_order spliced in (the engine's entry points
    answered on the CPU by the oracle's PDLP): its first-order answer converges but does not
    pass the driver's 1e-6 original-space gate, so HYBRID hands the model to the simplex.
    Without the crossover block that simplex starts cold (thousands of pivots); with it
    (include/integration/lpsolver_hybrid_crossover.inc) it starts from the basis the
    first-order x identifies and needs none. Same certified optimum either way."""
    inst = instances.lp_uniform(*CASES["lp300"])
    g = golden("lp300")["objective"]
    opts = dict(method=stand_in.LP_HYBRID, hybrid_row_threshold=1, pdlp_max_iterations=200000,
                hybrid_first_order_eps=1e-6)
    _, cold = stand_in.ref_solve_lp(inst, lib_name="ref_lp_cpu", **opts)
    _, warm = stand_in.ref_solve_lp(inst, lib_name="ref_lp_hybrid_cpu", **opts)
    for r in (cold, warm):
        assert r["status_name"] == "OPTIMAL" and r["pdlp_converged"] == 1 and r["used_first_order"] == 0, r
        assert abs(r["objective"] - g) <= 1e-9 * (1.0 + abs(g)) and r["primal_residual"] <= 1e-6, r
    assert cold["iterations"] > 1000 and warm["iterations"] <= 50, (cold, warm)


def test_hybrid_simplex_leading_is_unchanged(stand_in, instances):
    """When the simplex leads (row count below the threshold) nothing has iterated before
    it, so the crossover block leaves it cold: the same pivots as without the block."""
    inst = instances.lp_uniform(*CASES["lp60"])
    opts = dict(method=stand_in.LP_HYBRID, hybrid_row_threshold=10 ** 9)
    x0, a = stand_in.ref_solve_lp(inst, lib_name="ref_lp_cpu", **opts)
    x1, b = stand_in.ref_solve_lp(inst, lib_name="ref_lp_hybrid_cpu", **opts)
    assert a["status_name"] == b["status_name"] == "OPTIMAL"
    assert a["iterations"] == b["iterations"] and a["pdlp_iterations"] == b["pdlp_iterations"] == 0
    assert np.array_equal(x0, x1)


def test_infeasible_lp_is_reported_not_certified(sihps, instances):
    """x0 + x1 in [5, 6] with x in [0, 2]^2 has no solution: no basis is certified; the
    C core's fallback simplex and the C++ core's warm dual simplex both prove infeasibility."""
    inst = instances.small_dense_lp(rows=1, cols=2, dense=[1, 1], c=[1, 1], rl=[5], ru=[6], cl=[0, 0], cu=[2, 2])
    x, y = np.array([2.0, 2.0]), np.array([-1.0])
    rc, out = sihps.ref_crossover(inst, x, y)
    assert rc == 0 and out["result"] == 1 and out["direct"] == 0 and out["full_fallback"] == 1, out   # INFEASIBLE
    rc, out = sihps.ref_sihps_crossover(inst, x, y)
    assert rc == 0 and out["status"] == 1, out                                                          # INFEASIBLE


def test_unbounded_lp_is_reported_not_certified(sihps, instances):
    """min -x0 with x0 - x1 <= 1, x >= 0 is unbounded: no basis is certified, and both
    cores' fallbacks report UNBOUNDED (the C++ core's warm start is refused, no dual
    feasible basis existing)."""
    inf = float("inf")
    inst = instances.small_dense_lp(rows=1, cols=2, dense=[1, -1], c=[-1, 0], rl=[-inf], ru=[1], cl=[0, 0],
                                    cu=[inf, inf])
    x, y = np.array([5.0, 4.0]), np.array([0.5])
    rc, out = sihps.ref_crossover(inst, x, y)
    assert rc == 0 and out["result"] == 2 and out["full_fallback"] == 1, out    # UNBOUNDED
    rc, out = sihps.ref_sihps_crossover(inst, x, y)
    assert rc == 0 and out["status"] == 2 and out["used_warm_start"] == 0, out  # UNBOUNDED
