"""sk_solve through the reference's C core with the integration block
include/integration/sk_solve_hook.inc applied (oracle/_ref/libsankhya_ref_hooked.so, built by oracle/hooked_core.py
where the reference sources are present). On a GPU the block hands the first-order
loop of solve_continuous to the engine's sankhya_b200_pdhg_loop, whose iterates equal
the reference's own loop; so sk_solve's answer through the patched core must equal,
bit for bit, the unpatched core's (oracle/_ref/libsankhya_ref.so), and the engine's
timing record for this thread must hold the hook's iteration count, which shows the
hook, not the block's CPU fallback, produced it. (Named to run after every other gpu
file, the allocation-free entry point's included.)"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


@pytest.mark.parametrize("case", ["lp_first_order", "qp"])
def test_sk_solve_through_the_hook_equals_the_reference(engine, oracle, instances, case):
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libsankhya_ref_hooked.so")):
        pytest.skip("patched reference core not built (reference sources absent at build time)")
    if case == "lp_first_order":
        inst, quad = instances.lp_uniform(12, 60, 150, 4), False
        opts = dict(primal_tol=1e-6, dual_tol=1e-6, iteration_limit=2000)
    else:
        inst, quad = instances.qp_diag_plus_lowrank(3, 40, 80, a_per_col=4, l_per_col=2), True
        opts = dict(primal_tol=1e-6, dual_tol=1e-6, iteration_limit=3000)
    st_ref, ref = oracle.ref_sk_solve(inst, quadratic=quad, **opts)

    # leave a distinctive count in this thread's timing record first
    small = instances.lp_uniform(5, 20, 40, 3)
    A = engine.Matrix.from_instance(small)
    rc, *_ = engine.pdhg(A, small, engine.settings(max_iterations=7, check_every=7, tau=0.05, sigma=0.05,
                                                   theta=1.0, tolerance=1e-12))
    A.close()
    assert rc == 0 and engine.last_timing()["iterations"] == 7

    st, out = oracle.ref_sk_solve(inst, quadratic=quad, lib_name="ref_hooked", **opts)
    assert st == st_ref == 0
    assert out["iterations"] == ref["iterations"] and out["result"] == ref["result"]
    assert engine.last_timing()["iterations"] == out["iterations"] != 7     # the hook ran
    for k in ("x", "y", "rowact"):
        assert np.array_equal(out[k], ref[k]), k
    assert out["objective"] == ref["objective"]
