"""Feasibility polishing (sankhya_b200_pdlp_solve_polished). The reference has no
counterpart (its docs list crossover and polishing as not implemented), so the
answers are checked by their properties: the polished x meets the row bounds far
tighter than the main loop's own point, the polished y is dual feasible, and the
objective sits within the reported gap of an exact optimum (the reference simplex's
certified config-0 objective, or HiGHS through scipy)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def csr_matvec(inst, x):
    import scipy.sparse as sp
    A = sp.csr_matrix((inst["val"], inst["idx"], inst["ptr"]), shape=(inst["m"], inst["n"]))
    return A @ x, A


def row_violation(inst, x):
    """Relative 2-norm distance of A x from the row box (unscaled)."""
    ax, _ = csr_matvec(inst, x)
    lo = np.where(np.abs(inst["rl"]) >= 1e30, -np.inf, inst["rl"])
    hi = np.where(np.abs(inst["ru"]) >= 1e30, np.inf, inst["ru"])
    v = ax - np.clip(ax, lo, hi)
    b = np.concatenate([lo[np.isfinite(lo)], hi[np.isfinite(hi)]])
    return np.linalg.norm(v) / (1.0 + np.linalg.norm(b))


def settings(engine, eps, **kw):
    s = engine.pdlp_default_settings()
    s.eps_optimal = eps
    s.max_iterations = 400000
    s.time_limit = 60.0
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def test_boxed_config0_primal_polish(engine, instances, golden_dir):
    """Config 0 (every bound finite): the dual residual is zero by construction, so
    only the primal polish runs. With a 1e-4 gap and 1e-8 feasibility the pair is
    feasible two orders of magnitude beyond the main loop's point and its objective
    lies within the gap of the certified simplex optimum."""
    inst = instances.lp_config0(0)
    A = engine.Matrix.from_instance(inst)
    g = json.load(open(os.path.join(golden_dir, "simplex_lp_config0.json")))
    rc, x_plain, _, r_plain = engine.pdlp_solve(A, inst, settings(engine, 1e-4))
    assert rc == 0 and r_plain["status"] == 0, r_plain
    rc, x, y, r, p = engine.pdlp_solve_polished(A, inst, settings(engine, 1e-4))
    assert rc == 0 and r["status"] == 0, (r, p)
    assert r["relative_primal_residual"] <= 1e-8 and r["relative_dual_residual"] <= 1e-8, r
    assert r["relative_gap"] <= 1e-4, r
    assert p["rounds"] >= 1 and p["main_iterations"] > 0 and p["primal_iterations"] > 0, p
    assert p["dual_iterations"] == 0, p
    assert r_plain["relative_primal_residual"] > 1e-8, r_plain
    # x is projected onto the box in the scaled space, then unscaled: within a rounding
    assert np.all(x >= inst["cl"] - 1e-12) and np.all(x <= inst["cu"] * (1 + 1e-15))
    obj = float(inst["c"] @ x)
    assert abs(r["primal_objective"] - obj) <= 1e-9 * (1.0 + abs(obj)), (r["primal_objective"], obj)
    # the answer is the last pair scored
    assert (p["pair_relative_primal_residual"], p["pair_relative_gap"], p["pair_primal_objective"]) == \
        (r["relative_primal_residual"], r["relative_gap"], r["primal_objective"])
    v_plain, v_pol = row_violation(inst, x_plain), row_violation(inst, x)
    assert v_pol <= 1e-6 and v_pol < v_plain, (v_pol, v_plain)
    assert abs(obj - g["objective"]) / (1.0 + abs(g["objective"])) <= 1e-3, (obj, g["objective"])
    # the same call again gives the same bits
    rc2, x2, y2, r2, p2 = engine.pdlp_solve_polished(A, inst, settings(engine, 1e-4))
    counts = ("rounds", "main_iterations", "primal_iterations", "dual_iterations")
    assert rc2 == 0 and np.array_equal(x, x2) and np.array_equal(y, y2)
    assert [p2[k] for k in counts] == [p[k] for k in counts]


def one_sided(instances, seed=5, m=300, n=700):
    """x >= 0 with no upper bound and nonnegative costs (bounded below by 0), rows
    two-sided around A x0: the dual residual is live, so the dual polish runs."""
    inst = instances.lp_uniform(seed, m, n, 4)
    inst["cu"] = np.full(n, 1e30)
    inst["cl"] = np.zeros(n)
    inst["c"] = np.abs(inst["c"]) + 0.1
    return inst


def highs_objective(inst):
    from scipy.optimize import linprog
    _, A = csr_matvec(inst, np.zeros(inst["n"]))
    import scipy.sparse as sp
    G = sp.vstack([A, -A]).tocsr()
    h = np.concatenate([inst["ru"], -inst["rl"]])
    out = linprog(inst["c"], A_ub=G, b_ub=h, bounds=[(0, None)] * inst["n"], method="highs")
    assert out.status == 0, out.message
    return float(out.fun)


def test_one_sided_dual_polish(engine, instances):
    inst = one_sided(instances)
    A = engine.Matrix.from_instance(inst)
    opt = highs_objective(inst)
    rc, x, y, r, p = engine.pdlp_solve_polished(A, inst, settings(engine, 1e-4))
    assert rc == 0 and r["status"] == 0, (r, p)
    assert r["relative_primal_residual"] <= 1e-8 and r["relative_dual_residual"] <= 1e-8, r
    assert p["dual_iterations"] > 0, p
    assert np.all(x >= 0.0)
    # reduced costs c + A'y of x >= 0 columns must be >= 0 (the engine's sign convention)
    _, Am = csr_matvec(inst, x)
    rcost = inst["c"] + Am.T @ y
    dviol = np.linalg.norm(np.minimum(rcost, 0.0)) / (1.0 + np.linalg.norm(inst["c"]))
    assert dviol <= 1e-6, dviol
    assert row_violation(inst, x) <= 1e-6
    obj = float(inst["c"] @ x)
    assert abs(obj - opt) / (1.0 + abs(opt)) <= 1e-3, (obj, opt)
    # the pair's dual objective bounds the optimum from below (weak duality), up to
    # the dual residual the pair still has
    assert r["dual_objective"] <= opt + 1e-5 * (1.0 + abs(opt)), (r["dual_objective"], opt)


def test_rounds_tighten_to_the_gap(engine, instances, golden_dir):
    """A gap target below the hand-over tolerance resumes the main loop at 10x tighter
    tolerances until the polished pair meets it."""
    inst = instances.lp_config0(0)
    A = engine.Matrix.from_instance(inst)
    g = json.load(open(os.path.join(golden_dir, "simplex_lp_config0.json")))
    pol = engine.polish_default_settings()
    pol.start_tolerance = 1e-3
    rc, x, y, r, p = engine.pdlp_solve_polished(A, inst, settings(engine, 1e-6), pol)
    assert rc == 0 and r["status"] == 0, (r, p)
    assert r["relative_gap"] <= 1e-6 and r["relative_primal_residual"] <= 1e-8, r
    assert p["rounds"] >= 2, p
    obj = float(inst["c"] @ x)
    assert abs(obj - g["objective"]) / (1.0 + abs(g["objective"])) <= 1e-5, (obj, g["objective"])


def test_already_feasible_point_skips_polishing(engine, instances):
    """When the main loop's point already meets the polishing tolerance on both
    measures (a tight main solve), no polishing solve runs and the answer is that
    point, with the plain solve's bits."""
    inst = instances.lp_uniform(3, 60, 150, 4)
    A = engine.Matrix.from_instance(inst)
    pol = engine.polish_default_settings()
    pol.start_tolerance = 1e-9
    pol.polish_tolerance = 1e-6
    s = settings(engine, 1e-9)
    rc, x0, y0, r0 = engine.pdlp_solve(A, inst, s)
    assert rc == 0 and r0["status"] == 0
    rc, x, y, r, p = engine.pdlp_solve_polished(A, inst, s, pol)
    assert rc == 0 and r["status"] == 0, (r, p)
    assert p["primal_iterations"] == 0 and p["dual_iterations"] == 0 and p["rounds"] == 1, p
    assert np.array_equal(x, x0) and np.array_equal(y, y0)
    assert r["iterations"] == r0["iterations"]
