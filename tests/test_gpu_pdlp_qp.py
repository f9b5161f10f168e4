"""Restarted PDLP with a quadratic objective (sankhya_b200_pdlp_solve_qp): hand-solved
QPs, and seeded convex QPs against the reference's own sk_solve QP answer (its first-
order loop finished by its active-set polish, certified by its sk_verify to ~1e-14;
c/src/sk_solve.c:908-954), for the diagonal Hessian (exact prox) and the general
Hessian (gradient step, curvature in the adaptive step), in FP64, with FP32
iterations refined in FP64, and with those iterations over bf16 values of A."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
INF = float("inf")


def _settings(engine, **kw):
    s = engine.pdlp_default_settings()
    s.eps_optimal = 1e-9
    s.max_iterations = 1_000_000
    s.time_limit = 60.0
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def _diag_hessian_inst(inst):
    """The same QP with only Q's diagonal, as a CSR the reference's sk_solve reads."""
    n = inst["n"]
    d = {k: v for k, v in inst.items() if k not in ("csc", "q_ptr", "q_idx", "q_val")}
    d["q_ptr"] = np.arange(n + 1, dtype=np.int32)
    d["q_idx"] = np.arange(n, dtype=np.int32)
    d["q_val"] = np.asarray(inst["qdiag"], dtype=np.float64).copy()
    return d


@pytest.mark.parametrize("form", ["diagonal", "hessian"])
@pytest.mark.parametrize("precision", ["FP64", "FP32_REFINE", "BF16_REFINE"])
def test_hand_solved_qps(engine, instances, form, precision):
    # min x^2 - 4x, 0 <= x <= 10 (row and column): x = 2, objective -4 (the reference's
    # diagonal_qp_smoke answer); and min x'Qx/2 - 1'x with Q = [[2, 1], [1, 2]], x >= 0,
    # x1 + x2 <= 10: x = (1/3, 1/3), objective -1/3
    cases = [(instances.small_dense_lp(1, 1, [1.0], [-4.0], [0.0], [10.0], [0.0], [INF]), np.array([[2.0]]),
              np.array([2.0]), -4.0),
             (instances.small_dense_lp(1, 2, [1.0, 1.0], [-1.0, -1.0], [-INF], [10.0], [0.0, 0.0], [INF, INF]),
              np.array([[2.0, 1.0], [1.0, 2.0]]), np.array([1.0, 1.0]) / 3.0, -1.0 / 3.0)]
    for inst, Q, x_star, obj_star in cases:
        if form == "diagonal" and np.count_nonzero(Q - np.diag(np.diag(Q))):
            continue
        A = engine.Matrix.from_instance(inst)
        n = inst["n"]
        kw = {}
        H = None
        if form == "diagonal":
            kw["qdiag"] = np.diag(Q).copy()
        else:
            r, c = np.nonzero(Q)
            ptr = np.zeros(n + 1, dtype=np.int32)
            np.cumsum(np.bincount(r, minlength=n), out=ptr[1:])
            H = engine.Matrix(n, n, ptr, c.astype(np.int32), Q[r, c])
            kw["hessian"] = H
        rc, x, y, res = engine.pdlp_solve_qp(A, inst, _settings(engine, precision=getattr(engine, precision)), **kw)
        assert rc == 0 and res["status"] == 0, (res, engine.last_error())
        assert np.allclose(x, x_star, atol=1e-6), x
        obj = float(inst["c"] @ x + 0.5 * x @ Q @ x)
        assert abs(obj - obj_star) <= 1e-6
        assert abs(res["primal_objective"] - obj_star) <= 1e-6


@pytest.mark.parametrize("form", ["diagonal", "hessian"])
@pytest.mark.parametrize("precision", ["FP64", "FP32_REFINE", "BF16_REFINE"])
def test_qp_matches_reference_sk_solve(engine, oracle, instances, form, precision):
    inst = instances.qp_diag_plus_lowrank(31, 100, 200, a_per_col=3, l_per_col=2)
    ref_inst = inst if form == "hessian" else _diag_hessian_inst(inst)
    st, ref = oracle.ref_sk_solve(ref_inst, quadratic=True, primal_tol=1e-9, dual_tol=1e-9)
    assert st == 0 and ref["result"] == 0
    A = engine.Matrix.from_instance(inst)
    kw = {"hessian": engine.Matrix.from_instance(inst, hessian=True)} if form == "hessian" else \
        {"qdiag": inst["qdiag"]}
    rc, x, y, r = engine.pdlp_solve_qp(A, inst, _settings(engine, precision=getattr(engine, precision),
                                                          eps_optimal=1e-8), **kw)
    assert rc == 0 and r["status"] == 0, (r, engine.last_error())
    assert max(r["relative_primal_residual"], r["relative_dual_residual"], r["relative_gap"]) <= 1e-8
    if form == "hessian":
        Q = np.zeros((inst["n"], inst["n"]))
        rows = np.repeat(np.arange(inst["n"]), np.diff(inst["q_ptr"]))
        Q[rows, inst["q_idx"]] = inst["q_val"]
        obj = float(inst["c"] @ x + 0.5 * x @ Q @ x)
    else:
        obj = float(inst["c"] @ x + 0.5 * np.sum(inst["qdiag"] * x * x))
    assert abs(obj - ref["objective"]) <= 1e-6 * (1 + abs(ref["objective"])), (obj, ref["objective"])
    # the reference's own certificate of the engine's point
    vs, cert = oracle.ref_sk_verify(ref_inst, x, y, quadratic=True)
    assert cert["primal_infeasibility"] <= 1e-6


def test_qp_entry_rejects_bad_input(engine, instances):
    inst = instances.small_dense_lp(1, 2, [1.0, 1.0], [-1.0, -1.0], [-INF], [10.0], [0.0, 0.0], [INF, INF])
    A = engine.Matrix.from_instance(inst)
    H = engine.Matrix(2, 2, [0, 1, 2], np.array([0, 1], dtype=np.int32), [1.0, 1.0])
    rc, *_ = engine.pdlp_solve_qp(A, inst, _settings(engine), hessian=H, qdiag=np.ones(2))
    assert rc == -1 and "not both" in engine.last_error()
    rc, *_ = engine.pdlp_solve_qp(A, inst, _settings(engine), qdiag=np.array([1.0, -1.0]))
    assert rc == -1 and "diagonal" in engine.last_error()
    rc, *_ = engine.pdlp_solve_qp(A, inst, _settings(engine, algorithm=engine.PDLP_HALPERN), qdiag=np.ones(2))
    assert rc == -1 and "adaptive" in engine.last_error()
