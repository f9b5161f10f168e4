"""The engine's restarted PDLP answer taken to a certified vertex by the crossover
source (include/integration/sk_crossover.c, built against the reference's C core into
oracle/_ref): the chain a caller of both runs. The vertex must be the reference
simplex's certified optimum."""
import json
import os

import pytest

pytestmark = pytest.mark.gpu

CASES = {"lp60": (12, 60, 150, 4), "lp300": (11, 300, 700, 5)}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("polished", [False, True])
def test_engine_point_to_certified_vertex(engine, instances, oracle, golden_dir, name, polished):
    if not oracle.available("ref_crossover"):
        pytest.skip("crossover source not built against the reference core (make -C oracle ref)")
    inst = instances.lp_uniform(*CASES[name])
    g = json.load(open(os.path.join(golden_dir, f"simplex_{name}.json")))
    A = engine.Matrix.from_instance(inst)
    s = engine.pdlp_default_settings()
    s.eps_optimal, s.max_iterations, s.time_limit = 1e-6, 400000, 20.0
    if polished:
        rc, x, y, r, _ = engine.pdlp_solve_polished(A, inst, s)
    else:
        rc, x, y, r = engine.pdlp_solve(A, inst, s)
    assert rc == 0 and r["status"] == 0, r
    rc, out = oracle.ref_crossover(inst, x, y)
    assert rc == 0 and out["result"] == 0, out
    assert out["primal_infeasibility"] <= 1e-9 and out["dual_infeasibility"] <= 1e-9, out
    assert abs(out["objective"] - g["objective"]) <= 1e-9 * (1.0 + abs(g["objective"])), (out["objective"], g)


@pytest.mark.parametrize("name", sorted(CASES))
def test_engine_point_seats_a_basis_in_the_cpp_core(engine, instances, oracle, golden_dir, name):
    """The same answer seated as a basis in the reference C++ core's warm-start simplex
    (include/integration/sihps_crossover.cpp): the core's gate accepts it at the optimum."""
    if not oracle.available("ref_sihps_crossover"):
        pytest.skip("crossover source not built against the reference C++ core (make -C oracle ref)")
    inst = instances.lp_uniform(*CASES[name])
    g = json.load(open(os.path.join(golden_dir, f"simplex_{name}.json")))
    A = engine.Matrix.from_instance(inst)
    s = engine.pdlp_default_settings()
    s.eps_optimal, s.max_iterations, s.time_limit = 1e-6, 400000, 20.0
    rc, x, y, r = engine.pdlp_solve(A, inst, s)
    assert rc == 0 and r["status"] == 0, r
    rc, out = oracle.ref_sihps_crossover(inst, x, y)
    assert rc == 0 and out["status"] == 0, out
    assert out["primal_residual"] <= 1e-6 and out["dual_residual"] <= 1e-6, out
    assert abs(out["objective"] - g["objective"]) <= 1e-9 * (1.0 + abs(g["objective"])), (out["objective"], g)
