"""CPU checks of the MPS / QPS files the reference-program GPU tests feed to
apps/sankhya_pdhg.cu and apps/sankhya_qp_cuda.cu: each file reads back through the
reference's own reader (sk_read_mps, c/src/sk_core.c) as the generated instance bit
for bit; the LP optimum agrees with an independent simplex (HiGHS through scipy);
and the oracle, run with the steps those programs choose, converges within their
iteration limit to a point the reference's verifier accepts (the programs' exit
conditions)."""
import os

import numpy as np
import pytest

import mps_files as mf

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
HAVE_REF = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libsankhya_ref.so"))
needs_ref = pytest.mark.skipif(not HAVE_REF, reason="reference C core not built (make -C oracle ref)")
KEYS = ("ptr", "idx", "val", "c", "rl", "ru", "cl", "cu")
QKEYS = KEYS + ("q_ptr", "q_idx", "q_val")
APP_SETTINGS = dict(max_iterations=100000, check_every=100, theta=1.0, tolerance=1e-6)


def _dense(inst):
    A = np.zeros((inst["m"], inst["n"]))
    for i in range(inst["m"]):
        for p in range(inst["ptr"][i], inst["ptr"][i + 1]):
            A[i, inst["idx"][p]] = inst["val"][p]
    return A


def _highs(inst):
    from scipy.optimize import linprog
    A = _dense(inst)
    a_ub, b_ub, a_eq, b_eq = [], [], [], []
    for i in range(inst["m"]):
        lo, hi = inst["rl"][i], inst["ru"][i]
        if lo == hi:
            a_eq.append(A[i]); b_eq.append(lo)
            continue
        if np.isfinite(hi):
            a_ub.append(A[i]); b_ub.append(hi)
        if np.isfinite(lo):
            a_ub.append(-A[i]); b_ub.append(-lo)
    bounds = [(None if np.isneginf(l) else l, None if np.isposinf(u) else u) for l, u in zip(inst["cl"], inst["cu"])]
    return linprog(inst["c"], A_ub=np.array(a_ub), b_ub=b_ub, A_eq=np.array(a_eq), b_eq=b_eq, bounds=bounds,
                   method="highs")


def test_writer_rejects_what_the_reader_would_change(tmp_path):
    inst = mf.lp_instance(5)
    bad = dict(inst, rl=inst["rl"].copy(), ru=inst["ru"].copy())
    bad["rl"][1], bad["ru"][1] = -np.inf, np.inf
    with pytest.raises(ValueError, match="free"):
        mf.write_mps(str(tmp_path / "free.mps"), bad)
    bad = dict(inst, val=inst["val"].copy())
    bad["val"][0] = 0.0
    with pytest.raises(ValueError, match="zero"):
        mf.write_mps(str(tmp_path / "zero.mps"), bad)


def test_instance_has_every_row_and_bound_kind():
    inst = mf.lp_instance(5)
    rl, ru, cl, cu = inst["rl"], inst["ru"], inst["cl"], inst["cu"]
    assert np.any(rl == ru)
    assert np.any(np.isfinite(rl) & np.isposinf(ru))
    assert np.any(np.isneginf(rl) & np.isfinite(ru))
    assert np.any(np.isfinite(rl) & np.isfinite(ru) & (rl < ru))
    assert np.any(np.isneginf(cl) & np.isposinf(cu))
    assert np.any(np.isneginf(cl) & np.isfinite(cu))
    assert np.any(np.isfinite(cl) & (cl == cu))
    assert np.any((cl == 0.0) & np.isposinf(cu))


@needs_ref
@pytest.mark.parametrize("seed", [1, 5])
def test_lp_file_round_trips_and_solves(tmp_path, oracle, seed):
    inst = mf.lp_instance(seed)
    path = str(tmp_path / "lp.mps")
    mf.write_mps(path, inst)
    back = oracle.ref_read_mps(path)
    for k in KEYS:
        assert np.array_equal(back[k], inst[k]), k
    assert back["objshift"] == 0.0 and not back["integer"].any()
    ref = _highs(inst)
    assert ref.status == 0
    step = 0.5 / oracle.power_norm(back, 30)
    rc, x, _, r = oracle.fixed_pdhg(back, dict(APP_SETTINGS, tau=step, sigma=step), want_dual=False)
    assert rc == 0 and r["status"] == 0 and r["iterations"] < APP_SETTINGS["max_iterations"]
    assert abs(r["objective"] - ref.fun) <= 1e-6 * (1 + abs(ref.fun))
    assert r["maximum_row_violation"] <= APP_SETTINGS["tolerance"]


@needs_ref
@pytest.mark.parametrize("diagonal", [True, False])
def test_qp_file_round_trips_and_verifies(tmp_path, oracle, diagonal):
    inst = mf.qp_instance(5, diagonal=diagonal)
    path = str(tmp_path / "qp.qps")
    mf.write_mps(path, inst)
    back = oracle.ref_read_mps(path)
    for k in QKEYS:
        assert np.array_equal(back[k], inst[k]), k
    assert (mf.q_diagonal(back) is not None) == diagonal
    assert np.all(np.linalg.eigvalsh(inst["Q"]) > 0)
    primal, dual = mf.app_qp_steps(back)
    qd = mf.q_diagonal(back)
    kw = dict(qdiag=qd) if diagonal else dict(hessian=True)
    rc, x, y, r = oracle.fixed_pdhg(back, dict(APP_SETTINGS, tau=0.0, sigma=0.0), primal_steps=primal,
                                    dual_steps=dual, want_dual=True, **kw)
    assert rc == 0 and r["status"] == 0 and r["iterations"] < APP_SETTINGS["max_iterations"]
    st, v = oracle.ref_sk_verify(back, x, y, quadratic=True)
    assert st == 0
    for k in ("primal_infeasibility", "dual_infeasibility", "complementarity"):
        assert v[k] <= 100 * APP_SETTINGS["tolerance"], k


def test_app_steps_follow_column_order():
    """Masses summed column by column (A's CSC, then Q's column), as the program does."""
    inst = mf.qp_instance(3)
    primal, dual = mf.app_qp_steps(inst)
    A = np.abs(_dense(inst))
    col = A.sum(axis=0) + np.abs(inst["Q"]).sum(axis=0)
    np.testing.assert_allclose(primal, 0.9 / (1 + col), rtol=1e-15)
    np.testing.assert_allclose(dual, 0.9 / (1 + A.sum(axis=1)), rtol=1e-15)


SMOKE = os.path.join(ROOT, "oracle", "_ref", "smoke")
needs_smoke = pytest.mark.skipif(not os.path.isdir(SMOKE), reason="reference CLI model files not copied")


@needs_ref
@needs_smoke
def test_cli_model_files_known_answers(oracle):
    """The reference's CLI model files (bench/smoke/, run by cuda/CMakeLists.txt:31-48)
    read through its own reader, solved by the oracle with the programs' steps and
    settings: the known answers the gpu runs of those programs are held to."""
    unit = oracle.ref_read_mps(os.path.join(SMOKE, "unit_lp.mps"))
    step = 0.5 / oracle.power_norm(unit, 30)
    rc, x, _, r = oracle.fixed_pdhg(unit, dict(APP_SETTINGS, max_iterations=5000, tolerance=1e-5, tau=step,
                                               sigma=step), want_dual=False)
    assert rc == 0 and r["status"] == 0 and abs(x[0] - 1.0) <= 1e-5 and abs(r["objective"] - 1.0) <= 1e-5

    tiny = oracle.ref_read_mps(os.path.join(SMOKE, "tiny_lp.mps"))
    step = 0.5 / oracle.power_norm(tiny, 30)
    rc, x, _, r = oracle.fixed_pdhg(tiny, dict(APP_SETTINGS, tau=step, sigma=step), want_dual=False)
    assert rc == 0 and r["status"] == 0
    assert np.allclose(x, [3.0, 1.0], atol=1e-6) and abs(r["objective"] + 11.0) <= 1e-6

    qp = oracle.ref_read_mps(os.path.join(SMOKE, "tiny_qp.qps"))
    assert mf.q_diagonal(qp) is None and np.diff(qp["ptr"]).sum() == 1
    primal, dual = mf.app_qp_steps(qp)
    rc, x, y, r = oracle.fixed_pdhg(qp, dict(APP_SETTINGS, max_iterations=100000, tolerance=1e-5, tau=0.0,
                                             sigma=0.0), primal_steps=primal, dual_steps=dual, hessian=True)
    assert rc == 0 and r["status"] == 0 and np.allclose(x, [2.0, 0.0], atol=1e-5)
    assert abs(r["objective"] + 4.0) <= 1e-5
    st, v = oracle.ref_sk_verify(qp, x, y, quadratic=True)
    assert st == 0 and max(v["primal_infeasibility"], v["dual_infeasibility"], v["complementarity"]) <= 1e-3

    with pytest.raises(ValueError):   # no constraint rows: the reader rejects the guard's file
        oracle.ref_read_mps(os.path.join(SMOKE, "nonconvex_qp.qps"))
