"""Pins the oracle (oracle/pdhg_oracle.c) to the reference.

1. Against the committed golden fixtures made by tests/golden/make_golden.py from
   the reference's own compiled C core: bit-exact x, y, rowact of sk_solve's
   first-order loop, sk_verify's residuals, sk_scale_model's factors.
2. Against the reference's known-answer tests for this path, restated:
   cuda/tests/pdhg_smoke.cu, cuda/tests/diagonal_qp_smoke.cu,
   tests/lp/test_pdlp.cpp:53-150 (hand-solved LPs).
3. Live against oracle/_ref/libsankhya_ref.so when it is present.
"""
import json
import os

import numpy as np
import pytest

INF = float("inf")


def _manifest(golden_dir):
    with open(os.path.join(golden_dir, "manifest.json")) as f:
        return json.load(f)


def test_sk_loop_matches_reference_fixtures_bit_exact(oracle, instances, golden_dir):
    man = _manifest(golden_dir)
    for name, seed, m, n, per_col, limits in man["lp"]:
        inst = instances.lp_uniform(seed, m, n, per_col)
        for lim in limits:
            g = np.load(os.path.join(golden_dir, f"sk_loop_{name}_it{lim}.npz"))
            x, y, act, out = oracle.sk_loop(inst, lim, 1e-300, 1e-300)
            assert out["iterations"] == int(g["iterations"])
            assert np.array_equal(x, g["x"]), f"{name} it{lim} x"
            assert np.array_equal(y, g["y"]), f"{name} it{lim} y"
            assert np.array_equal(act, g["rowact"]), f"{name} it{lim} rowact"
            v = oracle.sk_verify(inst, x, y)
            gv = np.load(os.path.join(golden_dir, f"sk_verify_{name}_it{lim}.npz"))
            for k in ("objective", "primal_infeasibility", "dual_infeasibility", "complementarity"):
                assert v[k] == float(gv[k]), (name, lim, k)


def test_sk_qp_loop_matches_reference_fixtures_bit_exact(oracle, instances, golden_dir):
    man = _manifest(golden_dir)
    for name, seed, m, n, limits in man["qp"]:
        inst = instances.qp_diag_plus_lowrank(seed, m, n, a_per_col=4, l_per_col=2)
        for lim in limits:
            g = np.load(os.path.join(golden_dir, f"sk_qp_{name}_it{lim}.npz"))
            x, y, act, out = oracle.sk_loop(inst, lim, 1e-300, 1e-300, quadratic=True)
            assert out["iterations"] == int(g["iterations"])
            assert np.array_equal(x, g["x"])
            assert np.array_equal(y, g["y"])


def test_pow2_scaling_matches_reference_fixtures(oracle, instances, golden_dir):
    man = _manifest(golden_dir)
    for name, seed, m, n, per_col, _ in man["lp"]:
        inst = instances.lp_uniform(seed, m, n, per_col)
        g = np.load(os.path.join(golden_dir, f"sk_scale_{name}.npz"))
        r, c = oracle.pow2_scale(inst, 4)
        assert np.array_equal(r, g["R"]) and np.array_equal(c, g["C"])
        # powers of two: exact in binary
        assert np.all(np.frexp(r)[0] == 0.5) and np.all(np.frexp(c)[0] == 0.5)


def _one_var(cost, lower, upper=INF, value=1.0):
    import sankhya_b200_instances as I
    return I.small_dense_lp(1, 1, [value], [cost], [lower], [upper], [0.0], [INF])


def test_fixed_pdhg_known_answers(oracle):
    # cuda/tests/pdhg_smoke.cu:8-17, 108-123: min x s.t. x >= 1, x >= 0 -> x = 1
    inst = _one_var(1.0, 1.0)
    s = dict(max_iterations=5000, check_every=10, tau=0.25, sigma=2.0, theta=1.0, tolerance=1e-5, time_limit=0.0)
    rc, x, y, r = oracle.fixed_pdhg(inst, s)
    assert rc == 0 and r["status"] == 0
    assert abs(x[0] - 1.0) <= 1e-3
    for k in ("maximum_row_violation", "maximum_kkt_residual", "maximum_dual_residual", "maximum_complementarity"):
        assert np.isfinite(r[k]) and r[k] <= 1e-5
    # :86-91 NaN cost rejected
    rc, *_ = oracle.fixed_pdhg(inst, s, c=np.array([np.nan]))
    assert rc != 0
    # :94-106 overflow in the product is a numeric failure (-2)
    import sankhya_b200_instances as I
    big = I.small_dense_lp(1, 1, [1e308], [1.0], [1e308], [INF], [0.0], [INF])
    rc, x, y, r = oracle.fixed_pdhg(big, s)
    assert rc == -2 and r["status"] == -2


def test_diagonal_qp_known_answers(oracle):
    # cuda/tests/diagonal_qp_smoke.cu:8-33: min x^2 - 4x s.t. x >= 1 -> x = 2, obj -4
    inst = _one_var(-4.0, 1.0)
    s = dict(max_iterations=10000, check_every=10, tau=0.15, sigma=0.5, theta=1.0, tolerance=1e-7, time_limit=0.0)
    rc, x, y, r = oracle.fixed_pdhg(inst, s, qdiag=np.array([2.0]))
    assert rc == 0 and r["status"] == 0
    assert abs(x[0] - 2.0) <= 1e-5 and abs(r["objective"] + 4.0) <= 1e-5
    for k in ("maximum_row_violation", "maximum_kkt_residual", "maximum_dual_residual", "maximum_complementarity"):
        assert r[k] <= 1e-7
    # :35-53 preconditioned + dual: y ~ 0
    s0 = dict(s, tau=0.0, sigma=0.0)
    rc, x, y, r = oracle.fixed_pdhg(inst, s0, qdiag=np.array([2.0]), primal_steps=np.array([0.15]),
                                    dual_steps=np.array([0.5]))
    assert rc == 0 and r["status"] == 0 and abs(x[0] - 2.0) <= 1e-5 and abs(y[0]) <= 1e-6
    # :54-61 zero primal step rejected
    rc, *_ = oracle.fixed_pdhg(inst, s0, qdiag=np.array([2.0]), primal_steps=np.array([0.0]),
                               dual_steps=np.array([0.5]))
    assert rc != 0


HAND_LPS = [
    # tests/lp/test_pdlp.cpp:53-80: max 3x+5y, x<=4, 2y<=12, 3x+2y<=18 -> (2, 6)
    (dict(rows=3, cols=2, dense=[1, 0, 0, 2, 3, 2], c=[-3, -5], rl=[-INF] * 3, ru=[4, 12, 18],
          cl=[0, 0], cu=[INF, INF]), lambda x: np.allclose(x, [2, 6], atol=1e-5)),
    # :82-103 x + y == 5 on [0,10]^2, min x + y
    (dict(rows=1, cols=2, dense=[1, 1], c=[1, 1], rl=[5], ru=[5], cl=[0, 0], cu=[10, 10]),
     lambda x: abs(x.sum() - 5) <= 1e-6),
    # :105-128 2 <= x <= 7 as a row, x in [0,100], min -x -> 7
    (dict(rows=1, cols=1, dense=[1], c=[-1], rl=[2], ru=[7], cl=[0], cu=[100]), lambda x: abs(x[0] - 7) <= 1e-6),
    # :130-150 x + y <= 100, x in [0,3], y in [0,4], min -x-y -> (3, 4)
    (dict(rows=1, cols=2, dense=[1, 1], c=[-1, -1], rl=[-INF], ru=[100], cl=[0, 0], cu=[3, 4]),
     lambda x: np.allclose(x, [3, 4], atol=1e-6)),
]


@pytest.mark.parametrize("case", range(len(HAND_LPS)))
def test_pdlp_oracle_hand_solved_lps(oracle, case):
    import sankhya_b200_instances as I
    spec, ok = HAND_LPS[case]
    inst = I.small_dense_lp(**spec)
    x, y, st = oracle.pdlp(inst, eps=1e-9, max_iterations=400000, restart_period=64)
    assert st["converged"] == 1, st
    assert ok(x), (x, st)


def test_pdlp_oracle_reaches_simplex_objective(oracle, instances, golden_dir):
    with open(os.path.join(golden_dir, "simplex_lp60.json")) as f:
        ref = json.load(f)
    inst = instances.lp_uniform(12, 60, 150, 4)
    x, y, st = oracle.pdlp(inst, eps=1e-8, max_iterations=200000)
    assert st["converged"] == 1
    obj = float(np.dot(inst["c"], x))
    assert abs(obj - ref["objective"]) <= 1e-6 * (1 + abs(ref["objective"]))


def test_config0_simplex_golden_is_certified():
    """The config-0 objective golden (tests/golden/make_simplex_config0.py): the
    reference's simplex reached optimality, its own sk_verify certified the point, and
    an independent simplex (HiGHS) agrees to 1e-12 relative."""
    here = os.path.join(os.path.dirname(__file__), "golden", "simplex_lp_config0.json")
    g = json.load(open(here))
    assert g["status"] == 0 and g["result"] == 0
    cert = g["sk_verify"]
    assert max(cert["primal_infeasibility"], cert["dual_infeasibility"], cert["complementarity"]) <= 1e-9
    assert abs(g["objective"] - g["highs_objective"]) <= 1e-12 * (1 + abs(g["objective"]))


def test_pdlp_oracle_reaches_config0_simplex_objective(oracle, instances, golden_dir):
    """The oracle's restatement of GpuPdlp on the 2,000 x 5,000 LP to 1e-8 relative
    KKT lands on the reference simplex's objective."""
    g = json.load(open(os.path.join(golden_dir, "simplex_lp_config0.json")))
    inst = instances.lp_config0(0)
    x, y, st = oracle.pdlp(inst, eps=1e-8, max_iterations=400000)
    assert st["converged"] == 1
    assert max(st["relative_primal_residual"], st["relative_dual_residual"], st["relative_gap"]) <= 1e-8
    obj = float(np.dot(inst["c"], x))
    assert abs(obj - g["objective"]) <= 1e-8 * (1 + abs(g["objective"])), (obj, g["objective"])


def test_ruiz_and_pock_chambolle_properties(oracle, instances):
    inst = instances.lp_uniform(5, 80, 200, 4)
    r, c, conv = oracle.ruiz(inst, 100, 1e-2)
    assert conv
    # scaled infinity norms of every row and column within 1 +- tol
    rows = np.repeat(np.arange(inst["m"]), np.diff(inst["ptr"]))
    scaled = np.abs(inst["val"]) * r[rows] * c[inst["idx"]]
    rmax = np.zeros(inst["m"]); np.maximum.at(rmax, rows, scaled)
    cmax = np.zeros(inst["n"]); np.maximum.at(cmax, inst["idx"], scaled)
    # the factors are the ones BEFORE the converged norms were measured, so the
    # norms of the returned scaling are within tol
    assert np.all(np.abs(rmax - 1) < 1e-2 + 1e-12) and np.all(np.abs(cmax - 1) < 1e-2 + 1e-12)
    pr, pc = oracle.pock_chambolle(inst, 1.0)
    racc = np.zeros(inst["m"]); np.add.at(racc, rows, np.abs(inst["val"]))
    cacc = np.zeros(inst["n"]); np.add.at(cacc, inst["idx"], np.abs(inst["val"]))
    assert np.allclose(pr, 1 / np.sqrt(racc), rtol=1e-14)
    assert np.allclose(pc, 1 / np.sqrt(cacc), rtol=1e-14)
    # non-convergence within the budget returns the identity (Scaling.cpp:87-91)
    r1, c1, conv1 = oracle.ruiz(inst, 1, 1e-12)
    assert not conv1 and np.all(r1 == 1) and np.all(c1 == 1)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                    "libsankhya_ref.so")), reason="reference core not built")
def test_oracle_live_against_reference_core(oracle, instances):
    inst = instances.lp_config0(0)
    for lim in (3, 40):
        st, ref = oracle.ref_sk_solve(inst, primal_tol=1e-300, dual_tol=1e-300, iteration_limit=lim)
        x, y, act, out = oracle.sk_loop(inst, lim, 1e-300, 1e-300)
        assert np.array_equal(x, ref["x"]) and np.array_equal(y, ref["y"]) and np.array_equal(act, ref["rowact"])
    st, v = oracle.ref_sk_verify(inst, x, y)
    assert v == oracle.sk_verify(inst, x, y)


def test_openmp_build_of_the_reference_core_gives_the_same_bits(oracle, instances):
    """The OpenMP build (the timed CPU legs' core) splits only csc_tmv over columns, each
    column's sum still in stored order: its sk_solve iterates equal the serial build's."""
    import os
    if not os.path.exists(os.path.join(os.path.dirname(oracle.__file__), "_ref", "libsankhya_ref_omp.so")):
        pytest.skip("OpenMP build of the reference core absent")
    inst = instances.lp_powerlaw(3, 20000, 40000, 400000)    # above csc_tmv's threading threshold
    st0, ser = oracle.ref_sk_solve(inst, primal_tol=1e-300, dual_tol=1e-300, iteration_limit=60)
    for threads in (1, 4, 8):
        st, par = oracle.ref_sk_solve(inst, lib_name="ref_omp", threads=threads, primal_tol=1e-300, dual_tol=1e-300,
                                      iteration_limit=60)
        assert st == st0 == 0 and par["iterations"] == ser["iterations"] == 60
        for k in ("x", "y", "rowact"):
            assert np.array_equal(par[k], ser[k]), (threads, k)


@pytest.mark.parametrize("name", ["lp60", "powerlaw20k", "config0"])
def test_scaling_restatements_match_the_reference_cpp_core(oracle, instances, name):
    """The oracle's Ruiz and Pock-Chambolle factors equal, bit for bit, those of the
    reference C++ core's own compute_ruiz_scaling / compute_pock_chambolle_scaling
    (src/lp/Scaling.cpp, compiled into oracle/_ref), including a Ruiz run that does not
    reach its tolerance (the reference then falls back to the identity)."""
    import os
    if not os.path.exists(os.path.join(os.path.dirname(oracle.__file__), "_ref", "libsihps_scaling_ref.so")):
        pytest.skip("reference scaling checker not built (make -C oracle ref)")
    inst = {"lp60": lambda: instances.lp_uniform(12, 60, 150, 4),
            "powerlaw20k": lambda: instances.lp_powerlaw(3, 20000, 40000, 400000),
            "config0": lambda: instances.lp_config0(0)}[name]()
    for max_iters, tol in ((100, 1e-2), (2, 1e-12)):
        r0, c0, conv = oracle.ruiz(inst, max_iters, tol)
        r1, c1 = oracle.ref_ruiz(inst, max_iters, tol)
        assert np.array_equal(r0, r1) and np.array_equal(c0, c1), (max_iters, tol)
        if not conv:
            assert np.all(r1 == 1.0) and np.all(c1 == 1.0)
    for alpha in (1.0, 0.5):
        p0, q0 = oracle.pock_chambolle(inst, alpha)
        p1, q1 = oracle.ref_pock_chambolle(inst, alpha)
        assert np.array_equal(p0, p1) and np.array_equal(q0, q1), alpha


def test_reference_gpu_pdlp_checker_loads_and_fails_cleanly_without_a_device(oracle, instances):
    """The reference C++ core's GPU PDLP (GpuPdlp, oracle/_ref/libsihps_pdlp_ref.so) is
    built from the reference tree for comparisons on a B200. Here it must load and, with
    no device, report failure through its C entry point instead of crashing."""
    import os
    import torch
    if not os.path.exists(os.path.join(os.path.dirname(oracle.__file__), "_ref", "libsihps_pdlp_ref.so")):
        pytest.skip("reference GPU PDLP checker not built (make -C oracle ref)")
    oracle.load("ref_pdlp")
    if torch.cuda.is_available():
        return
    with pytest.raises(RuntimeError):
        oracle.ref_gpupdlp(instances.lp_uniform(12, 60, 150, 4), eps=1e-6)
