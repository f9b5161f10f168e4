"""Shapes at the edges of the fixed-step solver against the oracle: empty rows and
columns, one-sided and free bounds given as IEEE infinities, a single row, and rows
whose lengths sit at the warp-chunk limits (32 / 33 entries: sequential sum vs warp
tree; 256 / 257: a chunk of its own vs the streamed path). Bit-identical where every
row has at most 32 entries, 1e-9 relative otherwise."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
INF = float("inf")


def _settings(**kw):
    s = dict(max_iterations=240, check_every=80, tau=0.02, sigma=0.02, theta=1.0, tolerance=1e-12, time_limit=0.0)
    s.update(kw)
    return s


def _both(engine, oracle, inst, s):
    A = engine.Matrix.from_instance(inst)
    ps, ds = np.full(inst["n"], s["tau"]), np.full(inst["m"], s["sigma"])
    rc, x, y, r = engine.pdhg(A, inst, engine.settings(**s), want_dual=True, entry="with_dual", primal_steps=ps,
                              dual_steps=ds)
    rc2, x2, y2, r2 = oracle.fixed_pdhg(inst, s, primal_steps=ps, dual_steps=ds)
    assert rc == rc2, (rc, rc2, engine.last_error())
    assert r["iterations"] == r2["iterations"] and r["status"] == r2["status"]
    return (x, y, r), (x2, y2, r2)


def _from_rows(rng, m, n, lengths):
    rows = [np.sort(rng.choice(n, size=k, replace=False)) if k else np.zeros(0, dtype=np.int64) for k in lengths]
    ptr = np.concatenate([[0], np.cumsum(lengths)]).astype(np.int32)
    idx = (np.concatenate(rows) if ptr[-1] else np.zeros(0)).astype(np.int32)
    val = rng.standard_normal(idx.size)
    x0 = rng.uniform(0, 10, n)
    act = np.bincount(np.repeat(np.arange(m), lengths), weights=val * x0[idx], minlength=m)
    return dict(m=m, n=n, ptr=ptr, idx=idx, val=val, c=rng.standard_normal(n), rl=act - 1.0, ru=act + 1.0,
                cl=np.zeros(n), cu=np.full(n, 10.0), x0=x0)


def test_empty_rows_and_columns(engine, oracle):
    rng = np.random.default_rng(10)
    m, n = 120, 300
    lengths = [0 if i % 7 == 0 else int(rng.integers(1, 9)) for i in range(m)]
    inst = _from_rows(rng, m, n, lengths)
    keep = inst["idx"] % 11 != 0                     # columns 0, 11, 22, ... become empty
    rows = np.repeat(np.arange(m), np.diff(inst["ptr"]))[keep]
    inst["idx"], inst["val"] = inst["idx"][keep], inst["val"][keep]
    inst["ptr"] = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=m))]).astype(np.int32)
    (x, y, r), (x2, y2, r2) = _both(engine, oracle, inst, _settings())
    assert np.array_equal(x, x2) and np.array_equal(y, y2)


def test_infinite_bounds(engine, oracle):
    rng = np.random.default_rng(11)
    m, n = 80, 200
    inst = _from_rows(rng, m, n, [int(rng.integers(2, 10)) for _ in range(m)])
    inst["cu"][::3] = INF                            # lower bound only
    inst["cl"][1::5], inst["cu"][1::5] = -INF, INF   # free
    inst["rl"][::4] = -INF                           # <= rows
    inst["ru"][2::6] = INF                           # >= rows
    inst["c"] = np.abs(inst["c"])                    # bounded below on the free columns' directions
    (x, y, r), (x2, y2, r2) = _both(engine, oracle, inst, _settings())
    assert np.array_equal(x, x2) and np.array_equal(y, y2)


def test_single_row(engine, oracle):
    rng = np.random.default_rng(12)
    inst = _from_rows(rng, 1, 25, [20])
    (x, y, r), (x2, y2, r2) = _both(engine, oracle, inst, _settings())
    assert np.array_equal(x, x2) and np.array_equal(y, y2)


@pytest.mark.parametrize("lengths,exact", [((32, 5, 32, 1), True), ((33, 5, 33, 1), False),
                                           ((256, 3, 4), False), ((257, 3, 4), False)])
def test_rows_at_chunk_limits(engine, oracle, lengths, exact):
    rng = np.random.default_rng(13)
    m, n = 60, 400
    pattern = (list(lengths) * (m // len(lengths) + 1))[:m]
    inst = _from_rows(rng, m, n, pattern)
    (x, y, r), (x2, y2, r2) = _both(engine, oracle, inst, _settings(tau=0.005, sigma=0.005))
    if exact:
        assert np.array_equal(x, x2) and np.array_equal(y, y2)
    else:
        assert np.allclose(x, x2, rtol=1e-9, atol=1e-12) and np.allclose(y, y2, rtol=1e-9, atol=1e-12)
