"""CUDA path vs the oracle on the instance the headline measurement runs: the
power-law LP with m = 1,000,000, n = 2,000,000 and about 20,000,000 nonzeros
(instances.lp_config1, seed 1), through the entry point the bench calls
(sankhya_cuda_qp_pdhg_preconditioned; its *_with_dual twin for y), with the
per-row / per-column steps 0.9 / (1 + mass) of the reference's CPU loop.

Rows of A have about 20 entries and columns up to ~200 (Zipf degrees), so the
A^T-side product takes the owning-lane sums for short columns and the warp tree
for columns longer than 32: those sums round differently from the oracle's
serial loops, so the iterates are compared with a relative tolerance of 1e-9
(sums of products spanning six decades of |a|). Rows of at most 32 entries are
bit-identical, and on this instance every row of A is that short, so the dual
iterate's discrepancies come only through the primal side."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_config1_iterates_match_oracle(engine, oracle, instances):
    inst = instances.lp_config1(1)
    m, n = inst["m"], inst["n"]
    tptr = instances.transpose_csr(m, n, inst["ptr"], inst["idx"], inst["val"])[0]
    col_len, row_len = np.diff(tptr), np.diff(inst["ptr"])
    assert col_len.max() > 32 and row_len.max() <= 256   # warp-tree columns are present
    rows = np.repeat(np.arange(m), row_len)
    rmass = np.bincount(rows, weights=np.abs(inst["val"]), minlength=m)
    cmass = np.bincount(inst["idx"], weights=np.abs(inst["val"]), minlength=n)
    ps, ds = 0.9 / (1 + cmass), 0.9 / (1 + rmass)
    s = dict(max_iterations=20, check_every=10, tau=0.0, sigma=0.0, theta=1.0, tolerance=1e-12, time_limit=0.0)
    A = engine.Matrix.from_instance(inst)
    rc, x, y, r = engine.pdhg(A, inst, engine.settings(**s), primal_steps=ps, dual_steps=ds, want_dual=True,
                              entry="with_dual")
    rc_p, x_p, _, r_p = engine.pdhg(A, inst, engine.settings(**s), primal_steps=ps, dual_steps=ds,
                                    entry="preconditioned")
    A.close()
    assert rc == rc_p == 0, engine.last_error()
    assert np.array_equal(x, x_p) and r == r_p     # both entry points run the same kernels
    rc2, x2, y2, r2 = oracle.fixed_pdhg(inst, s, primal_steps=ps, dual_steps=ds)
    assert rc2 == 0
    assert r["iterations"] == r2["iterations"] == 20
    assert np.abs(x - x2).max() <= 1e-9 * (1 + np.abs(x2).max())
    assert np.abs(y - y2).max() <= 1e-9 * (1 + np.abs(y2).max())
    # the checkpoint's fields (objective, row violation, residuals) agree too
    for k in ("objective", "maximum_row_violation", "maximum_kkt_residual", "maximum_dual_residual"):
        assert abs(r[k] - r2[k]) <= 1e-8 * (1 + abs(r2[k])), (k, r[k], r2[k])
    # and the iterate moved: 20 iterations from x0 = clamp(0) are not a fixed point
    assert np.abs(x).max() > 0 and np.abs(y).max() > 0
