"""The reference's own branch and bound (sk_milp.c) run through the engine on a B200:
every node LP relaxation goes to sk_solve's first-order branch, which the sk_solve
integration block hands to sankhya_b200_pdhg_loop (oracle/_ref/
libsankhya_ref_milp_hooked.so, built from the reference's sources with
include/integration/sk_milp_node.inc and sk_solve_hook.inc spliced in); the revised
simplex takes the nodes the loop does not finish.

  - 20 binaries: the search reaches the optimum found by enumerating all 2^20 points
    (the reference's own simplex-based search stops at a worse point on this
    instance, which it reports as optimal);
  - 32 binaries, 373 nodes: the same optimum and node count as the reference's own
    search, with the simplex taking a small fraction of its pivots.
The engine's timing record after each search shows that its loop ran the nodes."""
import pytest

from test_milp_node_integration import binary_milp, brute_force_optimum

pytestmark = pytest.mark.gpu


@pytest.fixture
def hooked(oracle):
    for name in ("ref", "ref_milp_hooked"):
        if not oracle.available(name):
            pytest.skip(f"{name} not built (make -C oracle ref ref-tests)")
    return oracle


def test_search_through_the_engine_reaches_the_enumerated_optimum(engine, hooked, instances):
    inst = binary_milp(instances, 41, 10, 20)
    engine.set_timing(1)
    try:
        st, r = hooked.ref_sk_solve(inst, lib_name="ref_milp_hooked", primal_tol=1e-6, dual_tol=1e-6)
        t = engine.last_timing()
    finally:
        engine.set_timing(0)
    assert st == 0 and r["result"] == 0
    assert abs(r["objective"] - brute_force_optimum(inst)) <= 1e-9
    assert t["iterations"] > 0 and t["checkpoints"] > 0, t


def test_search_through_the_engine_matches_the_reference_search(engine, hooked, instances):
    inst = binary_milp(instances, 46, 16, 32)
    st0, r0 = hooked.ref_sk_solve(inst, lib_name="ref", primal_tol=1e-6, dual_tol=1e-6)
    engine.set_timing(1)
    try:
        st1, r1 = hooked.ref_sk_solve(inst, lib_name="ref_milp_hooked", primal_tol=1e-6, dual_tol=1e-6)
        t = engine.last_timing()
    finally:
        engine.set_timing(0)
    assert st0 == st1 == 0 and r0["result"] == r1["result"] == 0
    assert abs(r1["objective"] - r0["objective"]) <= 1e-9 * (1 + abs(r0["objective"]))
    assert r1["iterations"] < r0["iterations"] / 10, (r1["iterations"], r0["iterations"])
    assert t["iterations"] > 0 and t["checkpoints"] > 0, t
    print(f"\n32 binaries: {r1['nodes']} nodes through the engine, {r1['iterations']} simplex pivots "
          f"(reference: {r0['nodes']} nodes, {r0['iterations']} pivots)")
