"""Batched PDHG over LPs sharing one matrix (sankhya_b200_shared_batch_pdhg): the
node relaxations of a branch-and-bound search (milp_solve_lp, c/src/sk_milp.c:432-459,
re-solves the same model with new column bounds). Every LP must equal a separate
run of sk_solve's first-order loop (the oracle's restatement, itself bit-exact
against the reference core) bit for bit, with the same stopping iteration, and the
block-diagonal batch of the same LPs must give the same bits."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _settings(engine, max_iterations, ptol, dtol):
    s = engine.batch_default_settings()
    s.max_iterations, s.primal_tol, s.dual_tol = max_iterations, ptol, dtol
    return s


def _shared(engine, nodes, s, per_lp_cost=False, per_lp_rows=False):
    base = nodes[0]
    A = engine.Matrix.from_instance(base)
    b = len(nodes)
    stack = lambda key: np.stack([nd[key] for nd in nodes])
    c = stack("c") if per_lp_cost else base["c"]
    rl, ru = (stack("rl"), stack("ru")) if per_lp_rows else (base["rl"], base["ru"])
    return engine.shared_batch_pdhg(A, b, c, rl, ru, stack("cl"), stack("cu"), s, want_dual=True)


def _check_node(oracle, nd, x, y, r, max_iterations, ptol, dtol):
    xo, yo, act, out = oracle.sk_loop(nd, max_iterations, ptol, dtol)
    assert r["iterations"] == out["iterations"], (r, out)
    assert (r["status"] == 0) == bool(out["converged"])
    assert np.array_equal(x, xo) and np.array_equal(y, yo)
    assert r["anorm"] == out["anorm"]


def test_nodes_match_separate_solves(engine, oracle, instances):
    nodes = instances.milp_nodes(35, 40, m=300, n=600)
    s = _settings(engine, 20000, 1e-3, 1e-3)
    rc, x, y, res = _shared(engine, nodes, s)
    assert rc == 0, engine.last_error()
    for k, nd in enumerate(nodes):
        _check_node(oracle, nd, x[k], y[k], res[k], 20000, 1e-3, 1e-3)
    assert sum(r["status"] == 0 for r in res) >= len(nodes) // 2


def test_nodes_equal_block_diagonal_batch(engine, instances):
    nodes = instances.milp_nodes(36, 24, m=400, n=800)
    s = _settings(engine, 3000, 1e-4, 1e-4)
    rc, x, y, res = _shared(engine, nodes, s)
    assert rc == 0, engine.last_error()
    blk, rseg, cseg = engine.block_diagonal(nodes)
    rc2, xb, yb, resb = engine.batch_pdhg(engine.Matrix.from_instance(blk), blk, rseg, cseg, s, want_dual=True)
    assert rc2 == 0, engine.last_error()
    for k in range(len(nodes)):
        assert np.array_equal(x[k], xb[cseg[k]:cseg[k + 1]]) and np.array_equal(y[k], yb[rseg[k]:rseg[k + 1]]), k
        assert res[k] == resb[k], (k, res[k], resb[k])


def test_per_lp_costs_and_row_bounds(engine, oracle, instances):
    base = instances.lp_uniform(37, 120, 300, 4)
    rng = np.random.default_rng(37)
    lps = []
    for _ in range(9):
        lp = dict(base)
        lp["c"] = base["c"] + 0.1 * rng.standard_normal(base["n"])
        shift = 0.05 * rng.standard_normal(base["m"]) * np.abs(base["rl"])
        lp["rl"], lp["ru"] = base["rl"] + shift, base["ru"] + shift
        lps.append(lp)
    s = _settings(engine, 5000, 1e-5, 1e-5)
    rc, x, y, res = _shared(engine, lps, s, per_lp_cost=True, per_lp_rows=True)
    assert rc == 0, engine.last_error()
    for k, lp in enumerate(lps):
        _check_node(oracle, lp, x[k], y[k], res[k], 5000, 1e-5, 1e-5)
        assert res[k]["objective"] == float(np.sum(lp["c"] * x[k])) or np.isclose(
            res[k]["objective"], float(np.dot(lp["c"], x[k])), rtol=1e-14)


def test_more_than_one_warp_group_and_ragged_batch(engine, oracle, instances):
    # 300 LPs: 10 slabs of 32 (the last one padded), two warp groups per row
    nodes = instances.milp_nodes(38, 300, m=60, n=120, fix_hi=10)
    s = _settings(engine, 137, 1e-12, 1e-12)
    rc, x, y, res = _shared(engine, nodes, s)
    assert rc == 0, engine.last_error()
    assert all(r["status"] == 1 and r["iterations"] == 137 for r in res)
    for k in (0, 31, 32, 255, 256, 299):
        _check_node(oracle, nodes[k], x[k], y[k], res[k], 137, 1e-12, 1e-12)


def test_rejects_crossed_bounds(engine, instances):
    nodes = instances.milp_nodes(39, 3, m=50, n=100)
    nodes[1] = dict(nodes[1])
    nodes[1]["cl"] = nodes[1]["cl"].copy()
    nodes[1]["cl"][5] = 2.0                  # above the upper bound of 1
    rc, *_ = _shared(engine, nodes, _settings(engine, 100, 1e-6, 1e-6))
    assert rc == -1 and "bound" in engine.last_error()


def test_every_warp_schedule_gives_the_same_bits(engine, instances):
    # 70 LPs: 3 slabs, so each shape (1 x 8, 2 x 4, 4 x 4) has a partly filled group
    nodes = instances.milp_nodes(40, 70, m=300, n=600)
    outs = []
    for schedule in (0, 1, 2, 3):
        s = _settings(engine, 400, 1e-5, 1e-5)
        s.schedule = schedule
        rc, x, y, res = _shared(engine, nodes, s)
        assert rc == 0, engine.last_error()
        outs.append((x, y, res))
    for x, y, res in outs[1:]:
        assert np.array_equal(x, outs[0][0]) and np.array_equal(y, outs[0][1]) and res == outs[0][2]
    s = _settings(engine, 10, 1e-5, 1e-5)
    s.schedule = 4
    rc, *_ = _shared(engine, nodes, s)
    assert rc == -1 and "settings" in engine.last_error()
