"""Seeded small LPs / convex QPs written as free-format MPS / QPS files, for running
the reference's command-line programs (apps/sankhya_pdhg.cu, apps/sankhya_qp_cuda.cu)
on this library.

The writer emits what the reference's reader accepts (c/src/sankhya_mps.c
read_mps_impl, c/src/sk_core.c read_qps_quadratic): indented data records, one
(row, value) pair per COLUMNS record, an L row with a RANGES record for a two-sided
row (the reader sets lower = rhs - |range|), FR / MI / LO / UP / FX bounds, and a
QUADOBJ section listing the lower triangle of Q once (the reader mirrors the
off-diagonal entries). Every number is written as the shortest repr that parses back
to the same double, and the generators build two-sided rows as rl = ru - w, the
reader's own arithmetic, so the model read back equals the instance bit for bit.
"""
from __future__ import annotations

import numpy as np


def _num(v: float) -> str:
    return repr(float(v))


def lp_instance(seed: int = 7, m: int = 10, n: int = 14, density: float = 0.35) -> dict:
    """A bounded feasible LP with E, G, L and ranged rows, and default, boxed, free
    (FR), upper-only (MI + UP) and fixed (FX) columns. Column 0 is free and sits in
    row 0, an equality row, so it is pinned by the boxed columns there."""
    rng = np.random.default_rng(seed)
    mask = rng.random((m, n)) < density
    mask[0, :4] = True
    for j in range(n):
        if not mask[:, j].any():
            mask[rng.integers(m), j] = True
    A = np.where(mask, np.round(rng.uniform(-2.0, 2.0, (m, n)) * 8.0) / 8.0, 0.0)
    A[mask & (A == 0.0)] = 0.5
    cl = np.zeros(n)
    cu = np.full(n, np.inf)
    for j in range(1, n):
        kind = j % 4
        if kind == 1:
            cl[j], cu[j] = -1.0, 3.0
        elif kind == 2:
            cl[j], cu[j] = 0.5, 2.5
    cl[0], cu[0] = -np.inf, np.inf
    cl[3], cu[3] = -np.inf, 2.0
    cl[n - 2], cu[n - 2] = 1.25, 1.25
    x0 = np.empty(n)
    for j in range(n):
        if np.isfinite(cl[j]) and np.isfinite(cu[j]):
            x0[j] = 0.5 * (cl[j] + cu[j])
        elif np.isfinite(cl[j]):
            x0[j] = cl[j] + 0.75
        elif np.isfinite(cu[j]):
            x0[j] = cu[j] - 0.75
        else:
            x0[j] = 0.3
    act = A @ x0
    rl = np.empty(m)
    ru = np.empty(m)
    for i in range(m):
        kind = 0 if i == 0 else i % 4
        slack = 0.25 + 0.25 * (i % 3)
        if kind == 0:
            rl[i] = ru[i] = act[i]
        elif kind == 1:
            rl[i], ru[i] = act[i] - slack, np.inf
        elif kind == 2:
            rl[i], ru[i] = -np.inf, act[i] + slack
        else:
            ru[i] = act[i] + slack
            rl[i] = ru[i] - 2.0 * slack
    c = np.round(rng.uniform(-1.0, 1.0, n) * 16.0) / 16.0
    c[0] = 0.0
    c[3] = -abs(c[3]) - 0.25
    for j in range(1, n):
        if np.isfinite(cl[j]) and np.isposinf(cu[j]):
            c[j] = abs(c[j]) + 0.125
    ptr = np.zeros(m + 1, np.int32)
    ptr[1:] = np.cumsum(mask.sum(axis=1))
    idx = np.concatenate([np.nonzero(mask[i])[0] for i in range(m)]).astype(np.int32)
    val = np.concatenate([A[i, mask[i]] for i in range(m)])
    return dict(m=m, n=n, ptr=ptr, idx=idx, val=val, c=c, rl=rl, ru=ru, cl=cl, cu=cu)


def qp_instance(seed: int = 11, m: int = 8, n: int = 12, diagonal: bool = False) -> dict:
    """The LP family above with a convex objective 0.5 x'Qx + c'x: Q = B'B + I/4
    (sparse B, full symmetric Q in CSR) or, with diagonal=True, a positive diagonal."""
    inst = lp_instance(seed, m, n)
    rng = np.random.default_rng(seed + 1)
    if diagonal:
        Q = np.diag(np.round(rng.uniform(0.5, 2.0, n) * 8.0) / 8.0)
    else:
        B = np.where(rng.random((n // 2, n)) < 0.3, np.round(rng.uniform(-1.0, 1.0, (n // 2, n)) * 4.0) / 4.0, 0.0)
        Q = B.T @ B + 0.25 * np.eye(n)
    Q[np.abs(Q) < 1e-15] = 0.0
    q_ptr = np.zeros(n + 1, np.int32)
    q_ptr[1:] = np.cumsum((Q != 0.0).sum(axis=1))
    inst["q_ptr"] = q_ptr
    inst["q_idx"] = np.concatenate([np.nonzero(Q[i])[0] for i in range(n)]).astype(np.int32)
    inst["q_val"] = np.concatenate([Q[i, Q[i] != 0.0] for i in range(n)])
    inst["Q"] = Q
    return inst


def write_mps(path: str, inst: dict, name: str = "B200TEST") -> None:
    """Free-format MPS (QPS when the instance carries q_ptr/q_idx/q_val)."""
    m, n = inst["m"], inst["n"]
    rl, ru, cl, cu = inst["rl"], inst["ru"], inst["cl"], inst["cu"]
    kinds, rhs, rng_w = [], {}, {}
    for i in range(m):
        lo, hi = rl[i], ru[i]
        if np.isfinite(lo) and np.isfinite(hi) and lo == hi:
            kinds.append("E"); rhs[i] = lo
        elif np.isfinite(lo) and not np.isfinite(hi):
            kinds.append("G"); rhs[i] = lo
        elif not np.isfinite(lo) and np.isfinite(hi):
            kinds.append("L"); rhs[i] = hi
        elif np.isfinite(lo) and np.isfinite(hi):
            kinds.append("L"); rhs[i] = hi; rng_w[i] = hi - lo
            if hi - abs(hi - lo) != lo:
                raise ValueError(f"row {i}: rl is not ru - (ru - rl) in float64; the file would not round-trip")
        else:
            raise ValueError(f"row {i} is free: the reader drops free rows")
    cols = [[] for _ in range(n)]
    for i in range(m):
        for p in range(inst["ptr"][i], inst["ptr"][i + 1]):
            if inst["val"][p] == 0.0:
                raise ValueError("explicit zero in A: the reader drops it")
            cols[inst["idx"][p]].append((i, inst["val"][p]))
    out = [f"NAME {name}", "ROWS", " N OBJ"]
    out += [f" {k} R{i}" for i, k in enumerate(kinds)]
    out.append("COLUMNS")
    for j in range(n):
        out.append(f"    X{j} OBJ {_num(inst['c'][j])}")
        out += [f"    X{j} R{i} {_num(v)}" for i, v in sorted(cols[j])]
    out.append("RHS")
    out += [f"    RHS R{i} {_num(v)}" for i, v in sorted(rhs.items()) if v != 0.0]
    if rng_w:
        out.append("RANGES")
        out += [f"    RNG R{i} {_num(w)}" for i, w in sorted(rng_w.items())]
    out.append("BOUNDS")
    for j in range(n):
        lo, hi = cl[j], cu[j]
        if np.isneginf(lo) and np.isposinf(hi):
            out.append(f" FR BND X{j}")
        elif np.isfinite(lo) and lo == hi:
            out.append(f" FX BND X{j} {_num(lo)}")
        else:
            if np.isneginf(lo):
                out.append(f" MI BND X{j}")
            elif lo != 0.0:
                out.append(f" LO BND X{j} {_num(lo)}")
            if np.isfinite(hi):
                out.append(f" UP BND X{j} {_num(hi)}")
    if "q_ptr" in inst:
        out.append("QUADOBJ")
        for i in range(n):
            for p in range(inst["q_ptr"][i], inst["q_ptr"][i + 1]):
                j = inst["q_idx"][p]
                if j <= i:
                    out.append(f"    X{i} X{j} {_num(inst['q_val'][p])}")
    out.append("ENDATA")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def app_qp_steps(inst: dict):
    """The primal / dual steps apps/sankhya_qp_cuda.cu builds (0.9 / (1 + mass)),
    accumulated in the same order: column by column over A's CSC (rows ascending),
    then Q's entries of that column; row masses in column order."""
    m, n = inst["m"], inst["n"]
    rows = np.repeat(np.arange(m), np.diff(inst["ptr"]))
    order = np.lexsort((rows, inst["idx"]))
    col_mass = [0.0] * n
    row_mass = [0.0] * m
    for p in order:
        v = abs(float(inst["val"][p]))
        col_mass[int(inst["idx"][p])] += v
        row_mass[int(rows[p])] += v
    if "q_ptr" in inst:
        qrows = np.repeat(np.arange(n), np.diff(inst["q_ptr"]))
        qorder = np.lexsort((qrows, inst["q_idx"]))
        for p in qorder:
            col_mass[int(inst["q_idx"][p])] += abs(float(inst["q_val"][p]))
    primal = np.array([0.9 / (1.0 + v) for v in col_mass])
    dual = np.array([0.9 / (1.0 + v) for v in row_mass])
    return primal, dual


def q_diagonal(inst: dict) -> np.ndarray | None:
    """Q's diagonal when Q is diagonal (the app's diagonal-Hessian path), else None."""
    n = inst["n"]
    d = np.zeros(n)
    for i in range(n):
        for p in range(inst["q_ptr"][i], inst["q_ptr"][i + 1]):
            if inst["q_idx"][p] != i:
                return None
            d[i] += inst["q_val"][p]
    return d
