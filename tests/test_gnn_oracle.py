"""The warm-start network's CPU restatement (oracle/gnn_oracle.py) is itself
checked here: its backward pass against central finite differences of its exact
fp64 forward pass (every head path: boxed, one-sided and free columns, an absent
row bound), and its bf16 rounding against hand-computed values."""
import numpy as np

import gnn_oracle as G


def _instance(instances):
    inst = dict(instances.lp_uniform(5, 12, 20, 3))
    for k in ("cl", "cu", "ru"):
        inst[k] = inst[k].copy()
    inst["cu"][3] = 1e30                     # lower bound only
    inst["cl"][4], inst["cu"][4] = -1e30, 1e30   # free
    inst["ru"][2] = 1e30                     # row without an upper bound
    return inst


def test_oracle_gradient_matches_finite_differences(instances):
    inst = _instance(instances)
    rng = np.random.default_rng(0)
    H, R = 8, 2
    theta = 0.3 * rng.standard_normal(G.n_params(H, R))
    xt, yt = rng.uniform(0, 10, inst["n"]), rng.standard_normal(inst["m"])
    kw = dict(ys=2.0, hidden=H, rounds=R, use_bf16=False)
    g = G.forward_backward(theta, inst, xt, yt, **kw)["grad"]
    worst = 0.0
    for k in rng.choice(theta.size, 80, replace=False):
        e = 1e-6
        tp, tm = theta.copy(), theta.copy()
        tp[k] += e
        tm[k] -= e
        fd = (G.forward_backward(tp, inst, xt, yt, want_grad=False, **kw)["loss"]
              - G.forward_backward(tm, inst, xt, yt, want_grad=False, **kw)["loss"]) / (2 * e)
        worst = max(worst, abs(fd - g[k]) / max(1e-8, abs(fd) + abs(g[k])))
    assert worst < 1e-5


def test_bf16_rounding():
    # exactly representable values are unchanged; halfway cases go to the even neighbour
    assert np.array_equal(G.bf16(np.array([1.0, -2.5, 0.0, 3.0])), [1.0, -2.5, 0.0, 3.0])
    one_ulp = 2.0 ** -7                      # bf16 spacing at 1.0
    assert G.bf16(np.array([1.0 + one_ulp / 2]))[0] == 1.0
    assert G.bf16(np.array([1.0 + 3 * one_ulp / 2]))[0] == 1.0 + 2 * one_ulp
    assert G.bf16(np.array([1.0 + 0.6 * one_ulp]))[0] == 1.0 + one_ulp


def test_parameter_layout():
    assert G.n_params(64, 4) == 2 * (16 * 64 + 64) + 4 * 2 * (128 * 64 + 64) + 2 * (64 + 1)
    theta = np.arange(G.n_params(8, 2), dtype=np.float64)
    assert np.array_equal(G.pack(G.unpack(theta, 8, 2), 8, 2), theta)
