"""The sihps caller run for real: the reference C++ core's solve_lp (src/lp/LpSolver.cpp:
126-334: presolve, method dispatch, HYBRID fallback, postsolve, the 1e-6 original-space
gate) built from its own sources with run_first_order replaced by the integration block
(include/integration/lpsolver_run_first_order.inc, one sankhya_b200_pdlp_solve call), so
FIRST_ORDER and HYBRID go through the engine (oracle/_ref/libsihps_lp_hooked.so).

On a 400 x 1,000 LP (the config-0 recipe, 5 per column), against the same driver's
SIMPLEX answer (CPU):
  - FIRST_ORDER through the engine is OPTIMAL, passes the gate, and its objective is
    within 1e-6 relative of the simplex's; the unmodified core (the reference's own
    GpuPdlp) agrees as well;
  - HYBRID with the first-order method leading uses the engine's answer;
  - HYBRID with the first-order method leading but stopped after 32 iterations falls
    back to the simplex (src/lp/LpSolver.cpp:233-239) and returns the simplex optimum;
  - HYBRID with the simplex leading under a budget it cannot meet falls back to the
    engine (first_order_fallback_used)."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(oracle, instances):
    for name in ("ref_lp", "ref_lp_hooked"):
        if not oracle.available(name):
            pytest.skip(f"{name} not built (make -C oracle ref ref-tests)")
    inst = instances.lp_uniform(5, 400, 1000, 5)
    _, simplex = oracle.ref_solve_lp(inst, oracle.LP_SIMPLEX, hooked=True)
    assert simplex["status_name"] == "OPTIMAL"
    return inst, simplex["objective"]


def _close(a, b, tol):
    return abs(a - b) <= tol * (1 + abs(b))


def test_first_order_through_the_engine(oracle, case):
    inst, obj = case
    x, r = oracle.ref_solve_lp(inst, oracle.LP_FIRST_ORDER, hooked=True)
    assert r["status_name"] == "OPTIMAL" and r["used_first_order"] and r["pdlp_converged"], r
    assert r["primal_residual"] <= 1e-6
    assert _close(r["objective"], obj, 1e-6), (r["objective"], obj)
    assert _close(float(inst["c"] @ x), r["objective"], 1e-12)
    # the unmodified core, whose run_first_order is the reference's GpuPdlp
    _, ref = oracle.ref_solve_lp(inst, oracle.LP_FIRST_ORDER, hooked=False)
    assert ref["status_name"] == "OPTIMAL" and _close(ref["objective"], obj, 1e-6), ref


def test_hybrid_first_order_leads(oracle, case):
    inst, obj = case
    _, r = oracle.ref_solve_lp(inst, oracle.LP_HYBRID, hooked=True, hybrid_row_threshold=0)
    assert r["status_name"] == "OPTIMAL" and r["used_first_order"] and not r["first_order_fallback_used"], r
    assert _close(r["objective"], obj, 1e-6)


def test_hybrid_falls_back_to_simplex_when_the_engine_stops_early(oracle, case):
    inst, obj = case
    _, r = oracle.ref_solve_lp(inst, oracle.LP_HYBRID, hooked=True, hybrid_row_threshold=0, pdlp_max_iterations=32)
    assert r["status_name"] == "OPTIMAL" and not r["used_first_order"] and not r["pdlp_converged"], r
    assert _close(r["objective"], obj, 1e-9)


def test_hybrid_falls_back_to_the_engine_when_simplex_runs_out_of_budget(oracle, case):
    inst, obj = case
    _, r = oracle.ref_solve_lp(inst, oracle.LP_HYBRID, hooked=True, hybrid_row_threshold=10 ** 9,
                               hybrid_simplex_budget=1e-6)
    assert r["status_name"] == "OPTIMAL" and r["used_first_order"] and r["first_order_fallback_used"], r
    assert _close(r["objective"], obj, 1e-6)
