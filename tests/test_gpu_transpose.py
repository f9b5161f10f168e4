"""The matrix store's device transpose (built by sankhya_cuda_csr_create, read
back with sankhya_b200_csr_transpose) against the stable host transpose: each
column's row indices ascending, values carried along, bit for bit. Shapes cover
empty rows and columns, no entries at all, one column, columns longer than a
radix tile, and enough columns for three radix passes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(engine, instances, m, n, ptr, idx, val):
    inst = dict(m=m, n=n, ptr=np.asarray(ptr, dtype=np.int32), idx=np.asarray(idx, dtype=np.int32),
                val=np.asarray(val, dtype=np.float64))
    A = engine.Matrix.from_instance(inst)
    tp, ti, tv = engine.csr_transpose(A)
    ep, ei, ev = instances.transpose_csr(m, n, inst["ptr"], inst["idx"], inst["val"])
    assert np.array_equal(tp, ep) and np.array_equal(ti, ei) and np.array_equal(tv, ev)


def _random(rng, m, n, density_rows):
    rows = []
    for r in range(m):
        k = density_rows(r)
        rows.append(np.sort(rng.choice(n, size=min(k, n), replace=False)))
    ptr = np.concatenate([[0], np.cumsum([len(c) for c in rows])])
    idx = np.concatenate(rows) if rows and ptr[-1] else np.zeros(0, dtype=np.int64)
    return ptr, idx, rng.standard_normal(idx.size)


def test_uniform_and_power_law(engine, instances):
    for inst in (instances.lp_uniform(1, 300, 700, 5), instances.lp_powerlaw(2, 2000, 5000, 60000)):
        _check(engine, instances, inst["m"], inst["n"], inst["ptr"], inst["idx"], inst["val"])


def test_empty_rows_and_columns(engine, instances):
    rng = np.random.default_rng(3)
    ptr, idx, val = _random(rng, 400, 900, lambda r: 0 if r % 3 == 0 else int(rng.integers(0, 6)))
    _check(engine, instances, 400, 900, ptr, idx, val)


def test_no_entries_and_one_column(engine, instances):
    _check(engine, instances, 5, 7, np.zeros(6), np.zeros(0), np.zeros(0))
    rng = np.random.default_rng(4)
    ptr, idx, val = _random(rng, 50, 1, lambda r: r % 2)
    _check(engine, instances, 50, 1, ptr, idx, val)


def test_dense_column_longer_than_a_tile(engine, instances):
    # column 7 appears in every row: 6,000 entries in one row of the transpose
    rng = np.random.default_rng(5)
    m, n = 6000, 40
    rows = [np.union1d([7], rng.choice(n, size=3, replace=False)) for _ in range(m)]
    ptr = np.concatenate([[0], np.cumsum([len(c) for c in rows])])
    idx = np.concatenate(rows)
    _check(engine, instances, m, n, ptr, idx, rng.standard_normal(idx.size))


def test_three_radix_passes(engine, instances):
    inst = instances.lp_uniform(6, 1000, 300_000, 1)     # 300,000 columns: 19 bits of keys
    _check(engine, instances, inst["m"], inst["n"], inst["ptr"], inst["idx"], inst["val"])
