"""The reference's own branch and bound (sk_milp.c) with its node LP relaxations sent
through sk_solve's first-order branch (include/integration/sk_milp_node.inc spliced
into milp_solve_lp, on top of the sk_solve loop hook; oracle/_ref/
libsankhya_ref_milp_hooked.so), the revised simplex taking nodes that do not converge.

On the CPU (no device) the loop hook falls back to the reference's own first-order
loop, so these tests check the splice and the driver logic: the spliced search reaches
the true optimum. The same searches run through the engine on a B200 in
tests/test_gpu_milp_node_integration.py."""
import os

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def binary_milp(instances, seed, m, n):
    base = dict(instances.milp_nodes(seed, 1, m=m, n=n, fix_lo=1, fix_hi=2)[0])
    base.pop("csc", None)
    base["cl"], base["cu"] = np.zeros(base["n"]), np.ones(base["n"])
    base["vartype"] = np.ones(base["n"], dtype=np.uint8)   # SK_INTEGER: every column binary
    return base


def brute_force_optimum(inst):
    """min c'x over x in {0, 1}^n with rl <= A x <= ru, by enumeration (n <= 22)."""
    n, m = inst["n"], inst["m"]
    A = np.zeros((m, n))
    A[np.repeat(np.arange(m), np.diff(inst["ptr"])), inst["idx"]] = inst["val"]
    X = ((np.arange(1 << n)[:, None] >> np.arange(n)) & 1).astype(float)
    act = X @ A.T
    feasible = np.all(act <= inst["ru"] + 1e-9, axis=1) & np.all(act >= inst["rl"] - 1e-9, axis=1)
    return float((X @ inst["c"])[feasible].min())


def test_splice_replaces_the_lp_branch(oracle):
    import hooked_core
    ref = oracle.reference_tree()
    if ref is None:
        pytest.skip("reference sources absent")
    text = open(os.path.join(ref, "c", "src", "sk_milp.c")).read()
    out = hooked_core.patched_milp(text, hooked_core.milp_node_snippet())
    body = out[out.index("static sk_result milp_solve_lp("):]
    body = body[:body.index("\n}\n")]
    assert "fo.lp_engine = SK_LP_FIRST_ORDER" in body and body.count("sk_simplex_solve(") == 1
    assert hooked_core.MILP_LP_BRANCH in text and hooked_core.MILP_LP_BRANCH not in out


@pytest.fixture
def hooked(oracle):
    for name in ("ref", "ref_milp_hooked"):
        if not oracle.available(name):
            pytest.skip(f"{name} not built (make -C oracle ref ref-tests)")
    return oracle


def test_spliced_search_reaches_the_enumerated_optimum(hooked, instances):
    inst = binary_milp(instances, 41, 10, 20)
    st, r = hooked.ref_sk_solve(inst, lib_name="ref_milp_hooked", primal_tol=1e-6, dual_tol=1e-6)
    assert st == 0 and r["result"] == 0
    assert abs(r["objective"] - brute_force_optimum(inst)) <= 1e-9


def test_spliced_search_matches_the_reference_search(hooked, instances):
    inst = binary_milp(instances, 46, 16, 32)
    st0, r0 = hooked.ref_sk_solve(inst, lib_name="ref", primal_tol=1e-6, dual_tol=1e-6)
    st1, r1 = hooked.ref_sk_solve(inst, lib_name="ref_milp_hooked", primal_tol=1e-6, dual_tol=1e-6)
    assert st0 == st1 == 0 and r0["result"] == r1["result"] == 0
    assert abs(r1["objective"] - r0["objective"]) <= 1e-9 * (1 + abs(r0["objective"]))
    # the simplex only takes the nodes the first-order loop does not finish
    assert r1["iterations"] < r0["iterations"] / 10, (r1["iterations"], r0["iterations"])
