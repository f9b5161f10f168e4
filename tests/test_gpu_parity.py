"""CUDA path vs the oracle on the same seeded inputs.

Rows of at most 32 entries are summed sequentially in stored order on the
device and every elementwise update uses round-to-nearest intrinsics without
contraction, so on such instances the device iterates are BIT-IDENTICAL to the
oracle's. Instances with longer rows (power-law columns) use warp/block trees
and are compared with a relative tolerance of 1e-9 on the iterates."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
INF = float("inf")


def fixed_settings(engine, **kw):
    base = dict(max_iterations=200, check_every=50, tau=0.0, sigma=0.0, theta=1.0, tolerance=1e-12, time_limit=0.0)
    base.update(kw)
    return base


def run_both(engine, oracle, inst, s, **kw):
    """Device and oracle on the same input. Entry points without a dual output
    are compared on x and the result fields; y is compared through the
    *_with_dual entry point (scalar steps passed as constant step vectors, which
    is the same arithmetic)."""
    A = engine.Matrix.from_instance(inst)
    H = engine.Matrix.from_instance(inst, hessian=True) if kw.pop("hessian", False) else None
    rc, x, y, r = engine.pdhg(A, inst, engine.settings(**s), hessian=H, want_dual=True,
                              entry="with_dual" if "primal_steps" in kw else None, **kw)
    rc2, x2, y2, r2 = oracle.fixed_pdhg(inst, s, hessian=H is not None, **kw)
    if y is None and "primal_steps" not in kw:
        ps = np.full(inst["n"], s["tau"])
        ds = np.full(inst["m"], s["sigma"])
        rcd, xd, y, rd = engine.pdhg(A, inst, engine.settings(**s), hessian=H, want_dual=True, entry="with_dual",
                                     primal_steps=ps, dual_steps=ds, **kw)
        assert rcd == rc and np.array_equal(xd, x) and rd == r
    return (rc, x, y, r), (rc2, x2, y2, r2)


def _steps(inst):
    rows = np.repeat(np.arange(inst["m"]), np.diff(inst["ptr"]))
    rmass = np.zeros(inst["m"]); np.add.at(rmass, rows, np.abs(inst["val"]))
    cmass = np.zeros(inst["n"]); np.add.at(cmass, inst["idx"], np.abs(inst["val"]))
    return 0.9 / (1 + cmass), 0.9 / (1 + rmass)


@pytest.mark.parametrize("seed", [0, 1])
def test_lp_pdhg_bit_exact_config0(engine, oracle, instances, seed):
    inst = instances.lp_config0(seed)
    s = fixed_settings(engine, max_iterations=300, check_every=100, tau=0.05, sigma=0.05)
    (rc, x, y, r), (rc2, x2, y2, r2) = run_both(engine, oracle, inst, s)
    assert rc == rc2 == 0
    assert np.array_equal(x, x2) and np.array_equal(y, y2)
    assert r["iterations"] == r2["iterations"] and r["status"] == r2["status"]
    for k in ("maximum_row_violation", "maximum_step", "maximum_kkt_residual", "maximum_dual_residual"):
        assert r[k] == r2[k], k
    assert abs(r["objective"] - r2["objective"]) <= 1e-12 * (1 + abs(r2["objective"]))
    assert abs(r["maximum_complementarity"] - r2["maximum_complementarity"]) <= 1e-12 * (1 + r2["maximum_complementarity"])


@pytest.mark.parametrize("theta", [0.0, 0.5, 1.0])
def test_preconditioned_theta_bit_exact(engine, oracle, instances, theta):
    inst = instances.lp_uniform(3, 400, 900, 5)
    ps, ds = _steps(inst)
    s = fixed_settings(engine, max_iterations=137, check_every=25, theta=theta)
    (rc, x, y, r), (rc2, x2, y2, r2) = run_both(engine, oracle, inst, s, primal_steps=ps, dual_steps=ds)
    assert rc == rc2 == 0
    assert np.array_equal(x, x2) and np.array_equal(y, y2)
    assert r["iterations"] == r2["iterations"] == 137


def test_diagonal_and_sparse_qp_bit_exact(engine, oracle, instances):
    inst = instances.qp_diag_plus_lowrank(7, 300, 600, a_per_col=4, l_per_col=2)
    s = fixed_settings(engine, max_iterations=120, check_every=40, tau=0.02, sigma=0.02)
    (rc, x, y, r), (rc2, x2, y2, r2) = run_both(engine, oracle, inst, s, qdiag=inst["qdiag"])
    assert rc == rc2 == 0 and np.array_equal(x, x2) and np.array_equal(y, y2)
    (rc, x, y, r), (rc2, x2, y2, r2) = run_both(engine, oracle, inst, s, hessian=True)
    assert rc == rc2 == 0 and np.array_equal(x, x2) and np.array_equal(y, y2)
    assert abs(r["objective"] - r2["objective"]) <= 1e-12 * (1 + abs(r2["objective"]))


def test_qp_config2_within_tolerance(engine, oracle, instances):
    """The config-2 QP itself (n = 200,000, m = 100,000, 2M nonzeros in A, explicit
    Q = D + L L^T with 1.4M): 40 fixed-step iterations of the diagonal-proximal and
    the sparse-Hessian entry points against the oracle. Some rows of A are longer than
    32 entries (warp-tree sums), so the comparison is at 1e-9 relative."""
    inst = instances.qp_config2(2)
    s = fixed_settings(engine, max_iterations=40, check_every=20, tau=0.005, sigma=0.5)
    for kw in (dict(qdiag=inst["qdiag"]), dict(hessian=True)):
        (rc, x, y, r), (rc2, x2, y2, r2) = run_both(engine, oracle, inst, s, **kw)
        assert rc == rc2 == 0, kw.keys()
        assert np.abs(x - x2).max() <= 1e-9 * (1 + np.abs(x2).max()), kw.keys()
        assert np.abs(y - y2).max() <= 1e-9 * (1 + np.abs(y2).max()), kw.keys()
        assert abs(r["objective"] - r2["objective"]) <= 1e-9 * (1 + abs(r2["objective"]))


def test_converges_like_the_oracle(engine, oracle, instances):
    """Same stopping iteration and status when the gates fire."""
    inst = instances.lp_uniform(4, 50, 120, 3)
    ps, ds = _steps(inst)
    s = fixed_settings(engine, max_iterations=200000, check_every=100, tolerance=1e-6)
    (rc, x, y, r), (rc2, x2, y2, r2) = run_both(engine, oracle, inst, s, primal_steps=ps, dual_steps=ds)
    assert rc == rc2 == 0
    assert r["status"] == r2["status"] and r["iterations"] == r2["iterations"]
    assert np.array_equal(x, x2)


def test_power_law_rows_within_tolerance(engine, oracle, instances):
    """Long rows (> 32 and > 2048 entries) take the warp / block reductions."""
    inst = instances.lp_powerlaw(5, 20000, 40000, 400000)
    assert np.diff(instances.transpose_csr(inst["m"], inst["n"], inst["ptr"], inst["idx"], inst["val"])[0]).max() > 32
    ps, ds = _steps(inst)
    s = fixed_settings(engine, max_iterations=60, check_every=30)
    (rc, x, y, r), (rc2, x2, y2, r2) = run_both(engine, oracle, inst, s, primal_steps=ps, dual_steps=ds)
    assert rc == rc2 == 0
    scale_x = 1 + np.abs(x2).max()
    scale_y = 1 + np.abs(y2).max()
    assert np.abs(x - x2).max() <= 1e-9 * scale_x
    assert np.abs(y - y2).max() <= 1e-9 * scale_y


def test_device_spmv_matches_numpy(engine, instances):
    import torch
    inst = instances.lp_powerlaw(6, 30000, 60000, 600000)
    # a few rows longer than a whole tile
    A = engine.Matrix.from_instance(inst)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(inst["n"])
    y = rng.standard_normal(inst["m"])
    dx = torch.tensor(x, device="cuda")
    dy = torch.zeros(inst["m"], dtype=torch.float64, device="cuda")
    L = engine.lib()
    assert L.sankhya_cuda_spmv_device_f64(A.handle, dx.data_ptr(), dy.data_ptr()) == 0
    ref = instances.csr_matvec(inst["ptr"], inst["idx"], inst["val"], x)
    got = dy.cpu().numpy()
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(inst["val"]).max() * np.abs(x).max())
    dyv = torch.tensor(y, device="cuda")
    dxo = torch.zeros(inst["n"], dtype=torch.float64, device="cuda")
    assert L.sankhya_cuda_spmv_transpose_device_f64(A.handle, dyv.data_ptr(), dxo.data_ptr()) == 0
    tp, ti, tv = instances.transpose_csr(inst["m"], inst["n"], inst["ptr"], inst["idx"], inst["val"])
    ref_t = instances.csr_matvec(tp, ti, tv, y)
    assert np.allclose(dxo.cpu().numpy(), ref_t, rtol=1e-11, atol=1e-9)


def test_bit_reproducible_across_calls(engine, instances):
    inst = instances.lp_powerlaw(8, 5000, 10000, 100000)
    A = engine.Matrix.from_instance(inst)
    s = engine.settings(80, 40, 1e-4, 1e-4, 1.0, 1e-12)
    outs = [engine.pdhg(A, inst, s, want_dual=True) for _ in range(3)]
    for rc, x, y, r in outs[1:]:
        assert np.array_equal(x, outs[0][1]) and np.array_equal(y, outs[0][2]) and r == outs[0][3]


def _sk_model_args(oracle, inst, quadratic=False):
    keep = oracle._Keep()
    model = oracle.build_sk_model(keep, inst, quadratic)
    return keep, model


def test_sk_loop_bridge_bit_exact_vs_reference_fixtures(engine, oracle, instances, golden_dir):
    import ctypes as C
    import json
    import os
    man = json.load(open(os.path.join(golden_dir, "manifest.json")))
    for name, seed, m, n, per_col, limits in man["lp"]:
        inst = instances.lp_uniform(seed, m, n, per_col)
        for lim in limits:
            g = np.load(os.path.join(golden_dir, f"sk_loop_{name}_it{lim}.npz"))
            keep, model = _sk_model_args(oracle, inst)
            opts = oracle.SkOptions(primal_tol=1e-300, dual_tol=1e-300, iteration_limit=lim, threads=1)
            x, y, act = np.zeros(n), np.zeros(m), np.zeros(m)
            res = engine.LoopResult()
            rc = engine.lib().sankhya_b200_pdhg_loop(C.byref(model), C.byref(opts), engine._p(x), engine._p(y),
                                                     engine._p(act), C.byref(res))
            assert rc == 0
            assert res.iterations == int(g["iterations"])
            assert np.array_equal(x, g["x"]) and np.array_equal(y, g["y"]) and np.array_equal(act, g["rowact"])


def test_sk_loop_bridge_qp_bit_exact(engine, oracle, instances, golden_dir):
    import ctypes as C
    import json
    import os
    man = json.load(open(os.path.join(golden_dir, "manifest.json")))
    for name, seed, m, n, limits in man["qp"]:
        inst = instances.qp_diag_plus_lowrank(seed, m, n, a_per_col=4, l_per_col=2)
        for lim in limits:
            g = np.load(os.path.join(golden_dir, f"sk_qp_{name}_it{lim}.npz"))
            keep, model = _sk_model_args(oracle, inst, quadratic=True)
            opts = oracle.SkOptions(primal_tol=1e-300, dual_tol=1e-300, iteration_limit=lim, threads=1)
            x, y, act = np.zeros(n), np.zeros(m), np.zeros(m)
            res = engine.LoopResult()
            rc = engine.lib().sankhya_b200_pdhg_loop(C.byref(model), C.byref(opts), engine._p(x), engine._p(y),
                                                     engine._p(act), C.byref(res))
            assert rc == 0 and res.iterations == lim
            assert np.array_equal(x, g["x"]) and np.array_equal(y, g["y"])


def test_sk_loop_bridge_converges_like_reference(engine, oracle, instances):
    import ctypes as C
    inst = instances.lp_uniform(12, 60, 150, 4)
    x2, y2, act2, out2 = oracle.sk_loop(inst, 100000, 1e-6, 1e-6)
    keep, model = _sk_model_args(oracle, inst)
    opts = oracle.SkOptions(primal_tol=1e-6, dual_tol=1e-6, iteration_limit=100000, threads=1)
    x, y, act = np.zeros(inst["n"]), np.zeros(inst["m"]), np.zeros(inst["m"])
    res = engine.LoopResult()
    assert engine.lib().sankhya_b200_pdhg_loop(C.byref(model), C.byref(opts), engine._p(x), engine._p(y),
                                               engine._p(act), C.byref(res)) == 0
    assert res.converged == out2["converged"] and res.iterations == out2["iterations"]
    assert np.array_equal(x, x2) and np.array_equal(act, act2)
