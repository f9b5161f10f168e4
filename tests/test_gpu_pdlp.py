"""Restarted PDLP (sankhya_b200_pdlp_solve) against the reference's PDLP tests
(tests/lp/test_pdlp.cpp:53-206) and the oracle's restatement of GpuPdlp."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
INF = float("inf")

HAND = [
    (dict(rows=3, cols=2, dense=[1, 0, 0, 2, 3, 2], c=[-3, -5], rl=[-INF] * 3, ru=[4, 12, 18], cl=[0, 0],
          cu=[INF, INF]), lambda x: np.allclose(x, [2, 6], atol=1e-5)),
    (dict(rows=1, cols=2, dense=[1, 1], c=[1, 1], rl=[5], ru=[5], cl=[0, 0], cu=[10, 10]),
     lambda x: abs(x.sum() - 5) <= 1e-6),
    (dict(rows=1, cols=1, dense=[1], c=[-1], rl=[2], ru=[7], cl=[0], cu=[100]), lambda x: abs(x[0] - 7) <= 1e-6),
    (dict(rows=1, cols=2, dense=[1, 1], c=[-1, -1], rl=[-INF], ru=[100], cl=[0, 0], cu=[3, 4]),
     lambda x: np.allclose(x, [3, 4], atol=1e-6)),
]


def settings(engine, **kw):
    s = engine.pdlp_default_settings()
    s.eps_optimal = 1e-9
    s.max_iterations = 400000
    s.time_limit = 20.0
    for k, v in kw.items():
        setattr(s, k, v)
    return s


@pytest.mark.parametrize("case", range(len(HAND)))
@pytest.mark.parametrize("scaling", [0, 3])
def test_hand_solved_lps(engine, instances, case, scaling):
    spec, ok = HAND[case]
    inst = instances.small_dense_lp(**spec)
    A = engine.Matrix.from_instance(inst)
    rc, x, y, r = engine.pdlp_solve(A, inst, settings(engine, scaling=scaling))
    assert rc == 0 and r["status"] == 0, r
    assert ok(x), (x, r)


def test_fixed_step_variant(engine, instances):
    spec, ok = HAND[0]
    inst = instances.small_dense_lp(**spec)
    A = engine.Matrix.from_instance(inst)
    rc, x, y, r = engine.pdlp_solve(A, inst, settings(engine, adaptive_step=0, scaling=0))
    assert rc == 0 and r["status"] == 0 and ok(x)


def test_sync_count_and_reproducibility(engine, instances):
    # test_pdlp.cpp:152-206: host syncs far below iterations; bit-identical repeats
    spec, ok = HAND[0]
    inst = instances.small_dense_lp(**spec)
    A = engine.Matrix.from_instance(inst)
    s = settings(engine, scaling=0, restart_period=128)
    runs = [engine.pdlp_solve(A, inst, s) for _ in range(3)]
    rc, x, y, r = runs[0]
    assert rc == 0 and r["status"] == 0
    assert r["host_syncs"] < r["iterations"] / 8 + 16
    for rc2, x2, y2, r2 in runs[1:]:
        assert r2["iterations"] == r["iterations"] and np.array_equal(x2, x) and np.array_equal(y2, y)


@pytest.mark.parametrize("name,seed,m,n,per_col", [("lp60", 12, 60, 150, 4), ("lp300", 11, 300, 700, 5)])
def test_objective_matches_reference_simplex(engine, instances, golden_dir, name, seed, m, n, per_col):
    ref = json.load(open(os.path.join(golden_dir, f"simplex_{name}.json")))
    inst = instances.lp_uniform(seed, m, n, per_col)
    A = engine.Matrix.from_instance(inst)
    rc, x, y, r = engine.pdlp_solve(A, inst, settings(engine, eps_optimal=1e-8))
    assert rc == 0 and r["status"] == 0, r
    obj = float(np.dot(inst["c"], x))
    assert abs(obj - ref["objective"]) <= 1e-6 * (1 + abs(ref["objective"])), (obj, ref)


def test_against_oracle_restatement(engine, oracle, instances):
    """Unscaled PDLP: same matrix norm, same converged objective as the oracle's GpuPdlp restatement."""
    inst = instances.lp_uniform(12, 60, 150, 4)
    A = engine.Matrix.from_instance(inst)
    rc, x, y, r = engine.pdlp_solve(A, inst, settings(engine, scaling=0, eps_optimal=1e-8))
    xo, yo, so = oracle.pdlp(inst, eps=1e-8, max_iterations=400000)
    assert rc == 0 and r["status"] == 0 and so["converged"] == 1
    assert abs(r["matrix_norm"] - so["matrix_norm"]) <= 1e-12 * so["matrix_norm"]
    obj, objo = float(np.dot(inst["c"], x)), float(np.dot(inst["c"], xo))
    assert abs(obj - objo) <= 1e-6 * (1 + abs(objo))
    # same trajectory up to rounding: iteration counts agree within a few windows
    assert abs(r["iterations"] - so["iterations"]) <= max(256, 0.2 * so["iterations"]), (r, so)


def test_warm_start_from_solution(engine, instances):
    inst = instances.lp_uniform(12, 60, 150, 4)
    A = engine.Matrix.from_instance(inst)
    rc, x, y, r = engine.pdlp_solve(A, inst, settings(engine, eps_optimal=1e-8))
    rc2, x2, y2, r2 = engine.pdlp_solve(A, inst, settings(engine, eps_optimal=1e-6), x0=x, y0=y)
    assert rc2 == 0 and r2["status"] == 0 and r2["iterations"] <= 256, r2


# ------------------------------------------------------------------ FP32 refinement

@pytest.mark.parametrize("case", range(len(HAND)))
def test_fp32_refined_hand_lps(engine, instances, case):
    spec, ok = HAND[case]
    inst = instances.small_dense_lp(**spec)
    A = engine.Matrix.from_instance(inst)
    rc, x, y, r = engine.pdlp_solve(A, inst, settings(engine, precision=engine.FP32_REFINE))
    assert rc == 0 and r["status"] == 0, r
    assert r["refinements"] >= 1
    assert ok(x), (x, r)


@pytest.mark.parametrize("name,seed,m,n,per_col", [("lp60", 12, 60, 150, 4), ("lp300", 11, 300, 700, 5)])
def test_fp32_refined_reaches_simplex_objective(engine, instances, golden_dir, name, seed, m, n, per_col):
    """FP32 inner iterations, FP64 refinement: the FP64 certificate reaches 1e-8 and the
    objective matches the reference simplex to 1e-6 relative."""
    ref = json.load(open(os.path.join(golden_dir, f"simplex_{name}.json")))
    inst = instances.lp_uniform(seed, m, n, per_col)
    A = engine.Matrix.from_instance(inst)
    rc, x, y, r = engine.pdlp_solve(A, inst, settings(engine, precision=engine.FP32_REFINE, eps_optimal=1e-8))
    assert rc == 0 and r["status"] == 0, r
    assert max(r["relative_primal_residual"], r["relative_dual_residual"], r["relative_gap"]) <= 1e-8
    obj = float(np.dot(inst["c"], x))
    assert abs(obj - ref["objective"]) <= 1e-6 * (1 + abs(ref["objective"])), (obj, ref)


@pytest.mark.parametrize("precision", ["FP64", "FP32_REFINE", "BF16_REFINE"])
def test_config0_to_1e8_reaches_the_simplex_objective(engine, instances, golden_dir, precision):
    """The 2,000 x 5,000 LP (instances.lp_config0, seed 0) to 1e-8 relative KKT, FP64,
    FP32 iterations refined in FP64, and FP32 iterations over bf16 matrix values refined
    in FP64: the objective matches the reference simplex's (certified by its sk_verify,
    cross-checked with HiGHS) to 1e-6 relative."""
    g = json.load(open(os.path.join(golden_dir, "simplex_lp_config0.json")))
    inst = instances.lp_config0(0)
    A = engine.Matrix.from_instance(inst)
    rc, x, y, r = engine.pdlp_solve(A, inst, settings(engine, precision=getattr(engine, precision),
                                                      eps_optimal=1e-8, time_limit=120.0))
    assert rc == 0 and r["status"] == 0, r
    assert max(r["relative_primal_residual"], r["relative_dual_residual"], r["relative_gap"]) <= 1e-8
    obj = float(np.dot(inst["c"], x))
    assert abs(obj - g["objective"]) <= 1e-6 * (1 + abs(g["objective"])), (obj, g["objective"])


@pytest.mark.parametrize("precision", ["FP32_REFINE", "BF16_REFINE"])
def test_refined_agrees_with_fp64_on_power_law(engine, instances, precision):
    """|a| over six decades. The restarted loop's progress past ~1e-5 on such matrices
    depends on the exact rounding of its trajectory (FP64 runs of two implementations
    stall at different gaps), so the check is at 1e-5, where both converge. A relative
    gap of 1e-5 (over 1 + |primal| + |dual|) leaves each objective up to ~2e-5 from
    the optimum, so two converged points agree to 1e-4."""
    inst = instances.lp_powerlaw(21, 4000, 8000, 80000)
    A = engine.Matrix.from_instance(inst)
    rc64, x64, y64, r64 = engine.pdlp_solve(A, inst, settings(engine, eps_optimal=1e-5, time_limit=60.0))
    rc32, x32, y32, r32 = engine.pdlp_solve(A, inst, settings(engine, precision=getattr(engine, precision),
                                                              eps_optimal=1e-5, time_limit=60.0))
    assert rc64 == 0 and rc32 == 0 and r64["status"] == 0 and r32["status"] == 0, (r64, r32)
    o64, o32 = float(np.dot(inst["c"], x64)), float(np.dot(inst["c"], x32))
    assert abs(o64 - o32) <= 1e-4 * (1 + abs(o64))


@pytest.mark.parametrize("eps", [1e-6, 1e-8])
def test_fp32_centered_loop_follows_fp64(engine, instances, eps):
    """FP32 iterations on deviations from an FP64 center that moves to each restart
    point: the restart decisions see FP64 residuals of the combined point, so the
    solve takes about the FP64 solve's iterations (plain FP32 arithmetic takes several
    times more on such instances) and reaches FP64 accuracy; every restart is one
    refinement."""
    inst = instances.lp_uniform(3, 5000, 10000, 5)
    A = engine.Matrix.from_instance(inst)
    rc64, x64, _, r64 = engine.pdlp_solve(A, inst, settings(engine, eps_optimal=eps, time_limit=60.0))
    rc32, x32, _, r32 = engine.pdlp_solve(A, inst, settings(engine, precision=engine.FP32_REFINE, eps_optimal=eps,
                                                            time_limit=60.0))
    assert rc64 == rc32 == 0 and r64["status"] == r32["status"] == 0, (r64, r32)
    assert r32["refinements"] == r32["restarts"] + 1 and r32["refinements"] > 1
    assert r32["iterations"] <= 1.15 * r64["iterations"] + 256, (r32["iterations"], r64["iterations"])
    assert max(r32["relative_primal_residual"], r32["relative_dual_residual"], r32["relative_gap"]) <= eps
    o64, o32 = float(np.dot(inst["c"], x64)), float(np.dot(inst["c"], x32))
    assert abs(o64 - o32) <= 10 * eps * (1 + abs(o64)), (o64, o32)


def test_bf16_values_centered_loop(engine, instances):
    """bf16 matrix values under the FP32 deviations: the residuals and restart decisions
    stay in FP64 on the exact matrix, so the solve still reaches the FP64 tolerance
    and objective, in a number of iterations near the FP64 solve's (printed with -s);
    the mode needs the adaptive loop."""
    inst = instances.lp_uniform(3, 5000, 10000, 5)
    A = engine.Matrix.from_instance(inst)
    rc64, x64, _, r64 = engine.pdlp_solve(A, inst, settings(engine, eps_optimal=1e-6, time_limit=60.0))
    rc16, x16, _, r16 = engine.pdlp_solve(A, inst, settings(engine, precision=engine.BF16_REFINE, eps_optimal=1e-6,
                                                            time_limit=60.0))
    assert rc64 == rc16 == 0 and r64["status"] == r16["status"] == 0, (r64, r16)
    assert r16["refinements"] > 1
    assert r16["iterations"] <= 2 * r64["iterations"] + 256, (r16["iterations"], r64["iterations"])
    assert max(r16["relative_primal_residual"], r16["relative_dual_residual"], r16["relative_gap"]) <= 1e-6
    o64, o16 = float(np.dot(inst["c"], x64)), float(np.dot(inst["c"], x16))
    assert abs(o64 - o16) <= 1e-5 * (1 + abs(o64)), (o64, o16)
    print(f"\nBF16_REFINE {r16['iterations']} it {r16['seconds']:.3f} s vs FP64 {r64['iterations']} it "
          f"{r64['seconds']:.3f} s")
    rc, *_ = engine.pdlp_solve(A, inst, settings(engine, precision=engine.BF16_REFINE, algorithm=engine.PDLP_HALPERN))
    assert rc == -1 and "BF16_REFINE" in engine.last_error()


# ------------------------------------------------------- reflected Halpern PDHG option

@pytest.mark.parametrize("case", range(len(HAND)))
def test_halpern_hand_solved_lps(engine, instances, case):
    spec, ok = HAND[case]
    inst = instances.small_dense_lp(**spec)
    A = engine.Matrix.from_instance(inst)
    rc, x, y, r = engine.pdlp_solve(A, inst, settings(engine, algorithm=engine.PDLP_HALPERN))
    assert rc == 0 and r["status"] == 0, r
    assert r["rejected_steps"] == 0
    assert ok(x), (x, r)


@pytest.mark.parametrize("name,seed,m,n,per_col", [("lp60", 12, 60, 150, 4), ("lp300", 11, 300, 700, 5)])
def test_halpern_reaches_simplex_objective(engine, instances, golden_dir, name, seed, m, n, per_col):
    ref = json.load(open(os.path.join(golden_dir, f"simplex_{name}.json")))
    inst = instances.lp_uniform(seed, m, n, per_col)
    A = engine.Matrix.from_instance(inst)
    rc, x, y, r = engine.pdlp_solve(A, inst, settings(engine, algorithm=engine.PDLP_HALPERN, eps_optimal=1e-8))
    assert rc == 0 and r["status"] == 0, r
    assert max(r["relative_primal_residual"], r["relative_dual_residual"], r["relative_gap"]) <= 1e-8
    obj = float(np.dot(inst["c"], x))
    assert abs(obj - ref["objective"]) <= 1e-6 * (1 + abs(ref["objective"])), (obj, ref)


def test_halpern_agrees_with_adaptive_on_power_law(engine, instances):
    inst = instances.lp_powerlaw(21, 4000, 8000, 80000)
    A = engine.Matrix.from_instance(inst)
    rc_a, xa, ya, ra = engine.pdlp_solve(A, inst, settings(engine, eps_optimal=1e-6, time_limit=60.0))
    rc_h, xh, yh, rh = engine.pdlp_solve(A, inst, settings(engine, algorithm=engine.PDLP_HALPERN, eps_optimal=1e-6,
                                                             time_limit=60.0))
    assert rc_a == 0 and rc_h == 0 and ra["status"] == 0 and rh["status"] == 0, (ra, rh)
    oa, oh = float(np.dot(inst["c"], xa)), float(np.dot(inst["c"], xh))
    assert abs(oa - oh) <= 1e-4 * (1 + abs(oa))


def test_settings_version_one_means_adaptive(engine, instances):
    import ctypes as C
    spec, ok = HAND[0]
    inst = instances.small_dense_lp(**spec)
    A = engine.Matrix.from_instance(inst)
    s = settings(engine, scaling=0)
    s.struct_version = 1
    s.algorithm = 99                      # not part of a version-1 struct: ignored
    rc, x, y, r = engine.pdlp_solve(A, inst, s)
    assert rc == 0 and r["status"] == 0 and ok(x)
    s.struct_version = 2
    rc, *_ = engine.pdlp_solve(A, inst, s)
    assert rc == -1 and "invalid" in engine.last_error()
