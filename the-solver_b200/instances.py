"""Seeded synthetic LP / QP instances for the PDHG engine.

Every generator returns a dict with
  m, n            rows and columns of A
  ptr, idx, val   CSR of A (int32, int32, float64); column indices ascend inside a row
  c, rl, ru       cost, row lower / row upper (float64)
  cl, cu          column lower / column upper (float64)
  x0              the interior point the rows are centred on
and, for QPs, q_ptr/q_idx/q_val (CSR of the full symmetric Q) and/or qdiag.

Random numbers come from numpy's PCG64 stream seeded with the given seed, so
an instance is a pure function of (recipe, sizes, seed). The recipes follow
the workload descriptions the engine is measured on:

  lp_config0   m=2,000, n=5,000, 5 distinct uniform rows per column, N(0,1)
               values, x0~U[0,10], bounds [0,10], rows A x0 -/+ U(0,1), c~N(0,1).
  lp_config1   m=1e6, n=2e6, column degrees Zipf(1.5) capped at 1,000 and
               scaled so nnz ~ 2e7, rows uniform, |a| log-uniform [1e-3,1e3]
               with a random sign; x0, bounds and rows as in lp_config0.
  qp_config2   n=2e5, m=1e5, 10 N(0,1) entries per column of A,
               Q = diag(log-U[1e-2,1e2]) + L L^T with L having 3 N(0,0.1)
               entries per column, c~N(0,1), bounds [-5,5], rows A x0 -/+ U(0,1).
  lp_batch_uneven  count LPs, m log-uniform in [m_lo, m_hi], n = 2m, 4-8 distinct
               uniform rows per column, otherwise the lp_config0 recipe.
  milp_nodes   node relaxations of one binary MILP: m=5e3, n=1e4, A >= 0 with 6
               U[1,10] entries per column, rows <= 0.3 * row sum, c ~ -U[0,1],
               x in [0,1]; each node fixes 1-50 random variables to 0 or 1.
  lp_family    a parametric LP family on one matrix (the learned warm start's
               workload): the lp_config0 recipe at (m, n) as the base; member s has
               c = c0 + 0.1 N(0,1) and both bounds of row i shifted by
               0.05 N(0,1) max(|rl_i|, |ru_i|). config 4: m=5e4, n=1e5, 10 per column.
"""
from __future__ import annotations

import numpy as np

SK_INFINITY = 1.0e30


def _distinct_rows(rng, m: int, degrees: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Row indices for every column: degrees[j] distinct uniform rows for column j.

    Returns (col, row) entry arrays sorted by (col, row).
    """
    n = degrees.shape[0]
    col = np.repeat(np.arange(n, dtype=np.int64), degrees)
    row = rng.integers(0, m, size=col.shape[0], dtype=np.int64)
    for _ in range(64):
        key = col * m + row
        order = np.argsort(key, kind="stable")
        col, row, key = col[order], row[order], key[order]
        dup = np.zeros(key.shape[0], dtype=bool)
        dup[1:] = key[1:] == key[:-1]
        k = int(dup.sum())
        if k == 0:
            return col, row
        row[dup] = rng.integers(0, m, size=k, dtype=np.int64)
    raise RuntimeError("could not draw distinct rows")


def _csr_from_entries(m: int, row: np.ndarray, col: np.ndarray, val: np.ndarray):
    order = np.lexsort((col, row))
    ptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(np.bincount(row, minlength=m), out=ptr[1:])
    return (ptr.astype(np.int32), col[order].astype(np.int32),
            np.ascontiguousarray(val[order], dtype=np.float64))


def csr_matvec(ptr, idx, val, x):
    rows = np.repeat(np.arange(ptr.shape[0] - 1), np.diff(ptr))
    return np.bincount(rows, weights=val * x[idx], minlength=ptr.shape[0] - 1)


def _finish_lp(rng, m, n, ptr, idx, val, lo=0.0, hi=10.0):
    x0 = rng.uniform(lo, hi, size=n)
    act = csr_matvec(ptr, idx, val, x0)
    rl = act - rng.uniform(0.0, 1.0, size=m)
    ru = act + rng.uniform(0.0, 1.0, size=m)
    c = rng.standard_normal(n)
    return dict(m=m, n=n, ptr=ptr, idx=idx, val=val, c=c, rl=rl, ru=ru,
                cl=np.full(n, lo), cu=np.full(n, hi), x0=x0)


def lp_uniform(seed: int, m: int, n: int, per_col: int = 5):
    """The lp_config0 recipe at any size: per_col distinct uniform rows per column."""
    rng = np.random.Generator(np.random.PCG64(seed))
    degrees = np.full(n, per_col, dtype=np.int64)
    col, row = _distinct_rows(rng, m, degrees)
    val = rng.standard_normal(col.shape[0])
    ptr, idx, val = _csr_from_entries(m, row, col, val)
    return _finish_lp(rng, m, n, ptr, idx, val)


def lp_config0(seed: int = 0):
    return lp_uniform(seed, 2000, 5000, 5)


def zipf_degrees(rng, n: int, nnz_target: int, exponent: float = 1.5, cap: int = 1000):
    raw = np.minimum(rng.zipf(exponent, size=n), cap).astype(np.float64)
    scale = nnz_target / raw.sum()
    deg = np.maximum(1, np.rint(raw * scale)).astype(np.int64)
    for _ in range(20):
        total = deg.sum()
        if abs(total - nnz_target) <= 0.002 * nnz_target:
            break
        scale *= nnz_target / total
        deg = np.maximum(1, np.rint(raw * scale)).astype(np.int64)
    return np.minimum(deg, cap)


def lp_powerlaw(seed: int, m: int, n: int, nnz_target: int):
    """The lp_config1 recipe at any size."""
    rng = np.random.Generator(np.random.PCG64(seed))
    degrees = zipf_degrees(rng, n, nnz_target)
    col, row = _distinct_rows(rng, m, degrees)
    mag = 10.0 ** rng.uniform(-3.0, 3.0, size=col.shape[0])
    sign = np.where(rng.integers(0, 2, size=col.shape[0]) == 0, -1.0, 1.0)
    ptr, idx, val = _csr_from_entries(m, row, col, mag * sign)
    return _finish_lp(rng, m, n, ptr, idx, val)


def lp_config1(seed: int = 1):
    return lp_powerlaw(seed, 1_000_000, 2_000_000, 20_000_000)


def qp_diag_plus_lowrank(seed: int, m: int, n: int, a_per_col: int = 10, l_per_col: int = 3,
                         explicit: bool = True):
    """The qp_config2 recipe at any size. With explicit=True the Hessian
    Q = D + L L^T is returned as a full symmetric CSR (q_ptr/q_idx/q_val);
    qdiag always holds D."""
    import scipy.sparse as sp

    rng = np.random.Generator(np.random.PCG64(seed))
    col, row = _distinct_rows(rng, m, np.full(n, a_per_col, dtype=np.int64))
    val = rng.standard_normal(col.shape[0])
    ptr, idx, val = _csr_from_entries(m, row, col, val)
    d = 10.0 ** rng.uniform(-2.0, 2.0, size=n)
    lcol, lrow = _distinct_rows(rng, n, np.full(n, l_per_col, dtype=np.int64))
    lval = rng.normal(0.0, 0.1, size=lcol.shape[0])
    inst = _finish_lp(rng, m, n, ptr, idx, val, lo=-5.0, hi=5.0)
    inst["qdiag"] = d
    if explicit:
        L = sp.csr_matrix((lval, (lrow, lcol)), shape=(n, n))
        Q = (sp.diags(d) + L @ L.T).tocsr()
        Q.sort_indices()
        inst["q_ptr"] = Q.indptr.astype(np.int32)
        inst["q_idx"] = Q.indices.astype(np.int32)
        inst["q_val"] = Q.data.astype(np.float64)
    return inst


def qp_config2(seed: int = 2, explicit: bool = True):
    return qp_diag_plus_lowrank(seed, 100_000, 200_000, explicit=explicit)


def transpose_csr(m: int, n: int, ptr, idx, val):
    """CSR of A^T (= CSC of A), rows of A in ascending order inside each column."""
    rows = np.repeat(np.arange(m, dtype=np.int32), np.diff(ptr))
    order = np.argsort(idx, kind="stable")
    tptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(idx, minlength=n), out=tptr[1:])
    return tptr.astype(np.int32), rows[order].astype(np.int32), val[order].copy()


def small_dense_lp(rows, cols, dense, c, rl, ru, cl, cu):
    """Instance dict from a small dense matrix (tests)."""
    a = np.asarray(dense, dtype=np.float64).reshape(rows, cols)
    r, cidx = np.nonzero(a)
    ptr, idx, val = _csr_from_entries(rows, r.astype(np.int64), cidx.astype(np.int64), a[r, cidx])
    f = lambda v: np.asarray(v, dtype=np.float64)
    return dict(m=rows, n=cols, ptr=ptr, idx=idx, val=val, c=f(c), rl=f(rl), ru=f(ru),
                cl=f(cl), cu=f(cu), x0=np.zeros(cols))


def lp_variable_degree(rng, m: int, n: int, deg_lo: int, deg_hi: int):
    degrees = rng.integers(deg_lo, deg_hi + 1, size=n).astype(np.int64)
    degrees = np.minimum(degrees, m)
    col, row = _distinct_rows(rng, m, degrees)
    val = rng.standard_normal(col.shape[0])
    ptr, idx, val = _csr_from_entries(m, row, col, val)
    return _finish_lp(rng, m, n, ptr, idx, val)


def lp_batch_uneven(seed: int, count: int, m_lo: int = 50, m_hi: int = 5000):
    """count independent LPs (the batched-LP workload); returns a list of instance dicts."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ms = np.exp(rng.uniform(np.log(m_lo), np.log(m_hi), size=count)).astype(np.int64)
    return [lp_variable_degree(rng, int(m), 2 * int(m), 4, 8) for m in ms]


def milp_nodes(seed: int, nodes: int, m: int = 5000, n: int = 10000, per_col: int = 6,
               fix_lo: int = 1, fix_hi: int = 50):
    """Node relaxations of one binary MILP sharing A; returns (list of instances, shared CSR)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    col, row = _distinct_rows(rng, m, np.full(n, per_col, dtype=np.int64))
    val = rng.uniform(1.0, 10.0, size=col.shape[0])
    ptr, idx, val = _csr_from_entries(m, row, col, val)
    rowsum = csr_matvec(ptr, idx, val, np.ones(n))
    base = dict(m=m, n=n, ptr=ptr, idx=idx, val=val, c=-rng.uniform(0.0, 1.0, size=n),
                rl=np.full(m, -SK_INFINITY), ru=0.3 * rowsum, cl=np.zeros(n), cu=np.ones(n), x0=np.zeros(n))
    out = []
    for _ in range(nodes):
        k = int(rng.integers(fix_lo, fix_hi + 1))
        which = rng.choice(n, size=k, replace=False)
        to = rng.integers(0, 2, size=k).astype(np.float64)
        cl, cu = base["cl"].copy(), base["cu"].copy()
        cl[which] = to
        cu[which] = to
        node = dict(base)
        node["cl"], node["cu"] = cl, cu
        out.append(node)
    return out


def lp_family_base(seed: int, m: int, n: int, per_col: int = 10):
    """Fixed part of a parametric family (the lp_config0 recipe at any size)."""
    return lp_uniform(seed, m, n, per_col)


def lp_family_member(base, seed: int):
    """Member `seed` of the family: perturbed cost and shifted row bounds, same A."""
    rng = np.random.Generator(np.random.PCG64(seed))
    inst = dict(base)
    inst["c"] = base["c"] + 0.1 * rng.standard_normal(base["n"])
    shift = 0.05 * rng.standard_normal(base["m"]) * np.maximum(np.abs(base["rl"]), np.abs(base["ru"]))
    inst["rl"] = base["rl"] + shift
    inst["ru"] = base["ru"] + shift
    return inst


def lp_config4_base(seed: int = 4):
    return lp_family_base(seed, 50_000, 100_000, 10)
