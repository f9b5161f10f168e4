"""Batched PDHG (sankhya_b200_batch_pdhg): every LP of the batch must equal a
separate run of sk_solve's first-order loop (the oracle's restatement, itself
bit-exact against the reference core) -- same iterates bit for bit, same
stopping iteration."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check_against_oracle(engine, oracle, lps, max_iterations, ptol=1e-6, dtol=1e-6):
    blk, rseg, cseg = engine.block_diagonal(lps)
    A = engine.Matrix.from_instance(blk)
    s = engine.batch_default_settings()
    s.max_iterations, s.primal_tol, s.dual_tol = max_iterations, ptol, dtol
    rc, x, y, res = engine.batch_pdhg(A, blk, rseg, cseg, s, want_dual=True)
    assert rc == 0, engine.last_error()
    for k, inst in enumerate(lps):
        xo, yo, act, out = oracle.sk_loop(inst, max_iterations, ptol, dtol)
        xs, ys = x[cseg[k]:cseg[k + 1]], y[rseg[k]:rseg[k + 1]]
        assert res[k]["iterations"] == out["iterations"], (k, res[k], out)
        assert (res[k]["status"] == 0) == bool(out["converged"])
        assert np.array_equal(xs, xo) and np.array_equal(ys, yo), k
        assert res[k]["anorm"] == out["anorm"]
    return res


def test_uneven_batch_matches_separate_solves(engine, oracle, instances):
    lps = instances.lp_batch_uneven(31, 48, 20, 300)
    res = _check_against_oracle(engine, oracle, lps, 20000, ptol=1e-4, dtol=1e-4)
    assert sum(r["status"] == 0 for r in res) >= 30   # most converge ...
    assert len({r["iterations"] for r in res}) > 10    # ... each at its own iteration


def test_config3a_size_range_matches_separate_solves(engine, oracle, instances):
    """64 LPs drawn with config 3a's recipe over its whole size range (m log-uniform in
    [50, 5,000], n = 2m, 4-8 per column; 0.86M nonzeros in all): bit-identical iterates
    and stopping iterations against separate oracle runs, most LPs stopping at their own
    gate and some at the iteration limit."""
    lps = instances.lp_batch_uneven(35, 64, 50, 5000)
    assert max(lp["m"] for lp in lps) > 4000
    res = _check_against_oracle(engine, oracle, lps, 4000, ptol=3e-3, dtol=3e-3)
    assert 40 <= sum(r["status"] == 0 for r in res) < 64
    assert len({r["iterations"] for r in res}) > 30


def test_iteration_limit_not_multiple_of_check(engine, oracle, instances):
    lps = instances.lp_batch_uneven(32, 12, 30, 120)
    res = _check_against_oracle(engine, oracle, lps, 137, ptol=1e-12, dtol=1e-12)
    assert all(r["status"] == 1 and r["iterations"] == 137 for r in res)


def test_node_relaxations_sharing_a(engine, oracle, instances):
    nodes = instances.milp_nodes(33, 8, m=300, n=600)
    _check_against_oracle(engine, oracle, nodes, 20000, ptol=1e-3, dtol=1e-3)


def test_rejects_non_block_diagonal(engine, instances):
    lps = instances.lp_batch_uneven(34, 3, 20, 40)
    blk, rseg, cseg = engine.block_diagonal(lps)
    blk = dict(blk)
    blk["idx"] = blk["idx"].copy()
    blk["idx"][0] = blk["n"] - 1       # row 0 (LP 0) touching the last LP's column
    A = engine.Matrix.from_instance(blk)
    rc, *_ = engine.batch_pdhg(A, blk, rseg, cseg)
    assert rc == -1 and "block-diagonal" in engine.last_error()
