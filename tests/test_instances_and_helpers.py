"""Host-side pieces that need no GPU: the seeded instance recipes (shapes, sizes,
value ranges and feasibility by construction, as the workload descriptions state
them) and the learned warm start's host helpers."""
import numpy as np


def _csr_ok(inst):
    ptr, idx = inst["ptr"], inst["idx"]
    assert ptr[0] == 0 and ptr[-1] == idx.size and np.all(np.diff(ptr) >= 0)
    assert np.all((idx >= 0) & (idx < inst["n"]))
    for r in range(min(inst["m"], 200)):
        row = idx[ptr[r]:ptr[r + 1]]
        assert np.all(np.diff(row) > 0)   # columns ascend and are distinct inside a row


def test_uniform_recipe(instances):
    inst = instances.lp_uniform(3, 400, 1000, 5)
    _csr_ok(inst)
    assert inst["idx"].size == 5 * 1000
    assert np.array_equal(np.bincount(inst["idx"], minlength=1000), np.full(1000, 5))
    act = instances.csr_matvec(inst["ptr"], inst["idx"], inst["val"], inst["x0"])
    assert np.all(inst["rl"] <= act) and np.all(act <= inst["ru"])      # x0 is feasible
    assert np.all((inst["x0"] >= 0) & (inst["x0"] <= 10))
    again = instances.lp_uniform(3, 400, 1000, 5)
    assert np.array_equal(again["val"], inst["val"]) and np.array_equal(again["c"], inst["c"])


def test_power_law_recipe(instances):
    inst = instances.lp_powerlaw(5, 4000, 8000, 80000)
    _csr_ok(inst)
    deg = np.bincount(inst["idx"], minlength=8000)
    assert abs(inst["idx"].size - 80000) <= 0.01 * 80000 and deg.max() <= 1000 and deg.min() >= 1
    mag = np.abs(inst["val"])
    assert mag.min() >= 1e-3 and mag.max() <= 1e3


def test_family_and_node_recipes(instances):
    base = instances.lp_family_base(11, 150, 375, 4)
    member = instances.lp_family_member(base, 1001)
    assert member["ptr"] is base["ptr"] and member["idx"] is base["idx"]     # same matrix
    assert not np.array_equal(member["c"], base["c"]) and np.all(member["rl"] <= member["ru"])
    np.testing.assert_allclose(member["ru"] - member["rl"], base["ru"] - base["rl"], rtol=1e-12, atol=1e-12)
    nodes = instances.milp_nodes(3, 6, m=200, n=400)
    for nd in nodes:
        assert np.all((nd["cl"] == nd["cu"]) | ((nd["cl"] == 0) & (nd["cu"] == 1)))
        fixed = int(np.sum(nd["cl"] == nd["cu"]))
        assert 1 <= fixed <= 50
        assert np.all(nd["rl"] <= -1e30)


def test_batch_recipe_and_block_diagonal(engine, instances):
    lps = instances.lp_batch_uneven(7, 5, 20, 60)
    blk, rseg, cseg = engine.block_diagonal(lps)
    assert rseg[-1] == blk["m"] == sum(lp["m"] for lp in lps) and cseg[-1] == blk["n"]
    rows = np.repeat(np.arange(blk["m"]), np.diff(blk["ptr"]))
    for k in range(len(lps)):
        inside = (rows >= rseg[k]) & (rows < rseg[k + 1])
        assert np.all((blk["idx"][inside] >= cseg[k]) & (blk["idx"][inside] < cseg[k + 1]))


def test_transpose_helper_is_stable(instances):
    inst = instances.lp_uniform(4, 50, 80, 3)
    tp, ti, tv = instances.transpose_csr(inst["m"], inst["n"], inst["ptr"], inst["idx"], inst["val"])
    assert tp[-1] == inst["idx"].size
    for j in range(inst["n"]):
        assert np.all(np.diff(ti[tp[j]:tp[j + 1]]) > 0)   # row indices ascend inside each column


def test_learned_host_helpers(learned):
    data = [(None, np.zeros(3), np.array([3.0, -4.0]), 2.0), (None, np.zeros(3), np.array([0.0, 0.0]), 8.0),
            (None, np.zeros(3), np.array([1.0, 1.0]), 4.0)]
    assert np.isclose(learned.dual_scale(data), np.sqrt((9 + 16 + 0 + 0 + 1 + 1) / 6))
    assert learned.learned_weight(data) == 4.0
    assert learned.dual_scale([(None, None, np.zeros(4), 1.0)]) == 1e-12


def test_qp_recipe(instances):
    """The convex QP recipe (config 2 at a small size): A with a_per_col entries per
    column, Q = D + L L^T full symmetric CSR and positive semidefinite, D log-uniform in
    [1e-2, 1e2], boxes [-5, 5], rows feasible at x0."""
    inst = instances.qp_diag_plus_lowrank(9, 300, 600, a_per_col=10, l_per_col=3)
    _csr_ok(inst)
    assert np.array_equal(np.bincount(inst["idx"], minlength=600), np.full(600, 10))
    n = inst["n"]
    Q = np.zeros((n, n))
    for i in range(n):
        Q[i, inst["q_idx"][inst["q_ptr"][i]:inst["q_ptr"][i + 1]]] = inst["q_val"][inst["q_ptr"][i]:inst["q_ptr"][i + 1]]
    assert np.allclose(Q, Q.T, rtol=0, atol=1e-14)
    assert np.linalg.eigvalsh(Q).min() > 0                           # D > 0 makes it definite
    d = inst["qdiag"]
    assert d.min() >= 1e-2 and d.max() <= 1e2
    assert np.all(np.diag(Q) >= d - 1e-12)                          # L L^T adds a non-negative diagonal
    assert np.all(inst["cl"] == -5.0) and np.all(inst["cu"] == 5.0)
    act = instances.csr_matvec(inst["ptr"], inst["idx"], inst["val"], inst["x0"])
    assert np.all(inst["rl"] <= act) and np.all(act <= inst["ru"])
