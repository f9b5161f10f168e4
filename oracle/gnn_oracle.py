"""CPU restatement (numpy, FP64) of the warm-start network: test infrastructure
only -- the checker for the device forward / backward kernels, never a path that
ships.

The reference has no learned component; this network is defined by the engine
(bipartite message passing over the constraint matrix, 4 rounds, hidden 64). The
device rounds the inputs of every dense layer (activations, features, weights) to
bf16 and accumulates in fp32 (in the backward pass also the incoming gradient
dZ); with bf16=True this restatement applies the same input rounding and
accumulates in fp64, so the two agree to accumulation error. With bf16=False it
is the exact fp64 function, whose gradient is checked against finite differences.

Parameter vector (flat, in this order; W stored row-major [in][out]):
  Ev[16][H], bev[H], Ec[16][H], bec[H],
  for t in 1..R: Wc_t[2H][H], bc_t[H], Wv_t[2H][H], bv_t[H],
  wx[H], bx, wy[H], by
Forward:
  Hv0 = relu(Fv Ev + bev), Hc0 = relu(Fc Ec + bec)
  round t: Hc_t = relu([Hc_{t-1}, D_r A Hv_{t-1}] Wc_t + bc_t)
           Hv_t = relu([Hv_{t-1}, D_c A' Hc_t] Wv_t + bv_t)
  (D_r, D_c: 1 / max(1, row / column nonzero count))
  x_hat = lo + (hi - lo) sigmoid(Hv_R wx + bx) on boxed columns, else clamp(bs (Hv_R wx + bx))
  y_hat = ys (Hc_R wy + by)
  loss  = mean_j ((x_hat - x*) / w_j)^2 + mean_i ((y_hat - y*) / ys)^2,
          w_j = hi - lo on boxed columns (at least 1e-12), else bs
"""
from __future__ import annotations

import numpy as np

INF = 1.0e30
FEATURES = 16


def bf16(a):
    """Round to bfloat16 (nearest, ties to even) through float32, back to float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = rounded.astype(np.uint32).view(np.float32)
    out = np.where(np.isfinite(f), out, f)
    return out.astype(np.float64)


def param_shapes(hidden=64, rounds=4):
    H = hidden
    shapes = [("Ev", (FEATURES, H)), ("bev", (H,)), ("Ec", (FEATURES, H)), ("bec", (H,))]
    for t in range(rounds):
        shapes += [(f"Wc{t}", (2 * H, H)), (f"bc{t}", (H,)), (f"Wv{t}", (2 * H, H)), (f"bv{t}", (H,))]
    shapes += [("wx", (H,)), ("bx", (1,)), ("wy", (H,)), ("by", (1,))]
    return shapes


def n_params(hidden=64, rounds=4):
    return sum(int(np.prod(s)) for _, s in param_shapes(hidden, rounds))


def unpack(theta, hidden=64, rounds=4):
    out, o = {}, 0
    for name, shape in param_shapes(hidden, rounds):
        k = int(np.prod(shape))
        out[name] = np.asarray(theta[o:o + k], dtype=np.float64).reshape(shape)
        o += k
    return out


def pack(grads, hidden=64, rounds=4):
    return np.concatenate([np.asarray(grads[name], dtype=np.float64).ravel()
                           for name, _ in param_shapes(hidden, rounds)])


def _present(v):
    return np.abs(v) < INF


def features(inst):
    """Node features and scales of one instance (dict with m, n, ptr, idx, val, c, rl, ru, cl, cu)."""
    m, n = inst["m"], inst["n"]
    ptr, idx, val = inst["ptr"], inst["idx"], inst["val"]
    rows = np.repeat(np.arange(m), np.diff(ptr))
    absval = np.abs(val)
    row_norm = np.bincount(rows, weights=absval, minlength=m)
    col_norm = np.bincount(idx, weights=absval, minlength=n)
    row_deg = np.diff(ptr).astype(np.float64)
    col_deg = np.bincount(idx, minlength=n).astype(np.float64)
    an = max(row_norm.max(initial=0.0), col_norm.max(initial=0.0), 1e-300)
    c, cl, cu, rl, ru = (np.asarray(inst[k], dtype=np.float64) for k in ("c", "cl", "cu", "rl", "ru"))
    cs = max(np.abs(c).max(initial=0.0), 1e-300)
    hl, hu = _present(cl), _present(cu)
    bs = max(np.abs(np.concatenate([cl[hl], cu[hu]])).max(initial=0.0), 1e-300) if (hl.any() or hu.any()) else 1.0
    gl, gu = _present(rl), _present(ru)
    rs = max(np.abs(np.concatenate([rl[gl], ru[gu]])).max(initial=0.0), 1e-300) if (gl.any() or gu.any()) else 1.0
    fv = np.zeros((n, FEATURES))
    fv[:, 0] = c / cs
    fv[:, 1] = np.where(hl, cl / bs, 0.0)
    fv[:, 2] = np.where(hu, cu / bs, 0.0)
    fv[:, 3] = hl
    fv[:, 4] = hu
    fv[:, 5] = col_norm / an
    fv[:, 6] = col_deg / max(col_deg.max(initial=0.0), 1.0)
    fv[:, 7] = 1.0
    fc = np.zeros((m, FEATURES))
    fc[:, 0] = np.where(gl, rl / rs, 0.0)
    fc[:, 1] = np.where(gu, ru / rs, 0.0)
    fc[:, 2] = gl
    fc[:, 3] = gu
    fc[:, 4] = row_norm / an
    fc[:, 5] = row_deg / max(row_deg.max(initial=0.0), 1.0)
    fc[:, 6] = 1.0
    return dict(fv=fv, fc=fc, bs=bs, rows=rows, inv_row=1.0 / np.maximum(row_deg, 1.0),
                inv_col=1.0 / np.maximum(col_deg, 1.0), hl=hl, hu=hu, cl=cl, cu=cu)


def _spmm(inst, rows, X):
    """A @ X with A in CSR (rows ascending), fp64."""
    out = np.zeros((inst["m"], X.shape[1]))
    np.add.at(out, rows, inst["val"][:, None] * X[inst["idx"]])
    return out


def _spmm_t(inst, rows, Y):
    """A' @ Y."""
    out = np.zeros((inst["n"], Y.shape[1]))
    np.add.at(out, inst["idx"], inst["val"][:, None] * Y[rows])
    return out


def forward_backward(theta, inst, x_target=None, y_target=None, ys=1.0, hidden=64, rounds=4,
                     use_bf16=True, want_grad=True):
    """Returns dict(x_hat, y_hat, loss, grad) (loss / grad None without targets)."""
    p = unpack(theta, hidden, rounds)
    f = features(inst)
    q = bf16 if use_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    rows = f["rows"]

    def dense(X, W, b):
        return q(X) @ q(W) + b

    zv = dense(f["fv"], p["Ev"], p["bev"])
    zc = dense(f["fc"], p["Ec"], p["bec"])
    hv, hc = np.maximum(zv, 0.0), np.maximum(zc, 0.0)
    tape = []
    for t in range(rounds):
        agg_c = f["inv_row"][:, None] * _spmm(inst, rows, hv)
        xc = np.concatenate([hc, agg_c], axis=1)
        hc_new = np.maximum(dense(xc, p[f"Wc{t}"], p[f"bc{t}"]), 0.0)
        agg_v = f["inv_col"][:, None] * _spmm_t(inst, rows, hc_new)
        xv = np.concatenate([hv, agg_v], axis=1)
        hv_new = np.maximum(dense(xv, p[f"Wv{t}"], p[f"bv{t}"]), 0.0)
        tape.append((xc, hc_new, xv, hv_new))
        hc, hv = hc_new, hv_new
    box = f["hl"] & f["hu"]
    lo, hi = f["cl"], f["cu"]
    width = np.where(box, np.maximum(hi - lo, 1e-12), f["bs"])
    sx = hv @ p["wx"] + p["bx"][0]
    sig = 1.0 / (1.0 + np.exp(-sx))
    lin = f["bs"] * sx
    clamped = np.minimum(np.maximum(lin, np.where(f["hl"], lo, -np.inf)), np.where(f["hu"], hi, np.inf))
    x_hat = np.where(box, lo + (hi - lo) * sig, clamped)
    sy = hc @ p["wy"] + p["by"][0]
    y_hat = ys * sy
    out = dict(x_hat=x_hat, y_hat=y_hat, loss=None, grad=None)
    if x_target is None:
        return out
    n, m = inst["n"], inst["m"]
    ex = (x_hat - x_target) / width
    ey = (y_hat - y_target) / ys
    out["loss"] = float(np.mean(ex ** 2) + np.mean(ey ** 2))
    if not want_grad:
        return out
    g = {}
    dxh = 2.0 * ex / width / n
    inside = (lin > np.where(f["hl"], lo, -np.inf)) & (lin < np.where(f["hu"], hi, np.inf))
    dsx = np.where(box, dxh * (hi - lo) * sig * (1.0 - sig), np.where(inside, dxh * f["bs"], 0.0))
    dyh = 2.0 * ey / ys / m
    dsy = dyh * ys
    g["wx"], g["bx"] = hv.T @ dsx, np.array([dsx.sum()])
    g["wy"], g["by"] = hc.T @ dsy, np.array([dsy.sum()])
    dhv = np.outer(dsx, p["wx"])
    dhc = np.outer(dsy, p["wy"])
    for t in reversed(range(rounds)):
        xc, hc_t, xv, hv_t = tape[t]
        dz = dhv * (hv_t > 0)
        g[f"Wv{t}"] = q(xv).T @ q(dz)
        g[f"bv{t}"] = dz.sum(axis=0)
        dxv = q(dz) @ q(p[f"Wv{t}"]).T
        dhv = dxv[:, :hidden]
        dhc = dhc + _spmm(inst, rows, f["inv_col"][:, None] * dxv[:, hidden:])
        dz = dhc * (hc_t > 0)
        g[f"Wc{t}"] = q(xc).T @ q(dz)
        g[f"bc{t}"] = dz.sum(axis=0)
        dxc = q(dz) @ q(p[f"Wc{t}"]).T
        dhc = dxc[:, :hidden]
        dhv = dhv + _spmm_t(inst, rows, f["inv_row"][:, None] * dxc[:, hidden:])
    dz = dhv * (zv > 0)
    g["Ev"], g["bev"] = q(f["fv"]).T @ q(dz), dz.sum(axis=0)
    dz = dhc * (zc > 0)
    g["Ec"], g["bec"] = q(f["fc"]).T @ q(dz), dz.sum(axis=0)
    out["grad"] = pack(g, hidden, rounds)
    return out
