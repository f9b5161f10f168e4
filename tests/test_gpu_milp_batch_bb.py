"""A small branch-and-bound search whose node relaxations are solved in batches by
sankhya_b200_shared_batch_pdhg, the replacement for one milp_solve_lp call per node
(c/src/sk_milp.c:432-459; the caller is include/integration/sk_milp_batch.inc).

The binary MILP is the node-relaxation recipe at 40 x 80 (A >= 0, rows <= 0.3 row
sum, c <= 0, x in {0, 1}). Each level takes the open nodes, solves them as one batch
(the shared matrix with per-node column bounds), and branches every converged,
fractional node on its most fractional variable (fix to 0 / fix to 1), eight nodes a
level at most, four levels. Every node is checked against the reference:
  - a converged node's objective equals the reference simplex's objective of the same
    LP (sk_solve with SK_LP_SIMPLEX from the reference's C core) to 1e-6 relative,
    and its point equals the oracle's restatement of the first-order loop bit for bit;
  - a node bound never falls below its parent's (fixing only restricts) and never
    rises above the MILP optimum that the reference's own branch and bound finds
    (sk_solve on the MILP), so every bound the batch returns is a valid bound."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
PTOL = DTOL = 1e-7
ITERS = 200_000


def _root(instances):
    base = dict(instances.milp_nodes(41, 1, m=40, n=80)[0])
    base.pop("csc", None)
    base["cl"], base["cu"] = np.zeros(base["n"]), np.ones(base["n"])
    return base


def test_branch_and_bound_node_batches_match_the_reference(engine, oracle, instances):
    base = _root(instances)
    milp = dict(base)
    milp["vartype"] = np.ones(base["n"], dtype=np.uint8)   # SK_INTEGER: every column binary
    st, ref_milp = oracle.ref_sk_solve(milp, primal_tol=1e-9, dual_tol=1e-9)
    assert st == 0 and ref_milp["result"] == 0
    optimum = ref_milp["objective"]

    A = engine.Matrix.from_instance(base)
    s = engine.batch_default_settings()
    s.max_iterations, s.primal_tol, s.dual_tol = ITERS, PTOL, DTOL
    open_nodes = [(base["cl"].copy(), base["cu"].copy(), -np.inf)]
    solved = converged = 0
    for level in range(4):
        if not open_nodes:
            break
        cl = np.stack([nd[0] for nd in open_nodes])
        cu = np.stack([nd[1] for nd in open_nodes])
        rc, X, _, res = engine.shared_batch_pdhg(A, len(open_nodes), base["c"], base["rl"], base["ru"], cl, cu, s)
        assert rc == 0, engine.last_error()
        children = []
        for k, (lo, hi, parent_bound) in enumerate(open_nodes):
            node = dict(base)
            node["cl"], node["cu"] = lo, hi
            solved += 1
            xo, _, _, out = oracle.sk_loop(node, ITERS, PTOL, DTOL)
            assert np.array_equal(X[k], xo) and res[k]["iterations"] == out["iterations"], (level, k)
            if res[k]["status"] != 0:
                continue
            converged += 1
            bound = float(base["c"] @ X[k])
            st, lp = oracle.ref_sk_solve(node, lp_engine=1, primal_tol=1e-9, dual_tol=1e-9)
            assert st == 0 and lp["result"] == 0
            assert abs(bound - lp["objective"]) <= 1e-6 * (1 + abs(lp["objective"])), (level, k, bound, lp)
            assert bound >= parent_bound - 1e-6 and bound <= optimum + 1e-6, (bound, parent_bound, optimum)
            frac = np.abs(X[k] - np.round(X[k]))
            j = int(np.argmax(frac))
            if frac[j] > 1e-6:
                for v in (0.0, 1.0):
                    a, b = lo.copy(), hi.copy()
                    a[j] = b[j] = v
                    children.append((a, b, bound))
        open_nodes = children[:8]
    assert solved >= 10 and converged >= 10, (solved, converged)
