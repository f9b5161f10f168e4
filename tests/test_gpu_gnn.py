"""The warm-start network on the device (sankhya_b200_gnn_*): its forward pass,
loss and gradient against the oracle's restatement with the same bf16 input
rounding (the device accumulates in fp32, the oracle in fp64), determinism, the
parameter interface, and what a trained network gains over cold-started PDLP on
held-out members of a parametric family."""
import numpy as np
import pytest

import gnn_oracle as G

pytestmark = pytest.mark.gpu


def _instance(instances):
    inst = dict(instances.lp_uniform(5, 60, 150, 4))
    for k in ("cl", "cu", "ru"):
        inst[k] = inst[k].copy()
    inst["cu"][3] = 1e30
    inst["cl"][4], inst["cu"][4] = -1e30, 1e30
    inst["ru"][7] = 1e30
    return inst


def test_gradient_matches_oracle(engine, instances):
    inst = _instance(instances)
    A = engine.Matrix.from_instance(inst)
    rng = np.random.default_rng(0)
    xt, yt = rng.uniform(0, 10, inst["n"]), rng.standard_normal(inst["m"])
    net = engine.Gnn(seed=7, y_scale=2.0)
    theta = net.parameters().astype(np.float64)
    loss, grad = net.gradient(A, inst, xt, yt)
    ref = G.forward_backward(theta, inst, xt, yt, ys=2.0)
    assert abs(loss - ref["loss"]) <= 1e-5 * ref["loss"]
    assert np.linalg.norm(grad - ref["grad"]) <= 1e-4 * np.linalg.norm(ref["grad"])
    off = 0
    for name, shape in G.param_shapes():
        k = int(np.prod(shape))
        a, b = grad[off:off + k], ref["grad"][off:off + k]
        off += k
        assert np.linalg.norm(a - b) <= 1e-3 * max(np.linalg.norm(b), 1e-12), name
    x, y = net.predict(A, inst)
    assert np.max(np.abs(x - ref["x_hat"])) <= 1e-4 and np.max(np.abs(y - ref["y_hat"])) <= 1e-5


def test_deterministic_and_parameters_roundtrip(engine, instances):
    inst = _instance(instances)
    A = engine.Matrix.from_instance(inst)
    rng = np.random.default_rng(1)
    xt, yt = rng.uniform(0, 10, inst["n"]), rng.standard_normal(inst["m"])
    net = engine.Gnn(seed=3)
    l1, g1 = net.gradient(A, inst, xt, yt)
    l2, g2 = net.gradient(A, inst, xt, yt)
    assert l1 == l2 and np.array_equal(g1, g2)
    theta = net.parameters()
    other = engine.Gnn(seed=99)
    other.set_parameters(theta)
    assert np.array_equal(other.parameters(), theta)
    assert np.array_equal(other.gradient(A, inst, xt, yt)[1], g1)
    bad = theta.copy()
    bad[5] = np.nan
    with pytest.raises(RuntimeError, match="non-finite"):
        other.set_parameters(bad)


def test_rejects_invalid_inputs(engine, instances):
    inst = _instance(instances)
    A = engine.Matrix.from_instance(inst)
    net = engine.Gnn(seed=2)
    before = net.parameters()
    bad = dict(inst)
    bad["c"] = inst["c"].copy()
    bad["c"][3] = np.nan
    with pytest.raises(RuntimeError, match="cost or column bound"):
        net.predict(A, bad)
    bad = dict(inst)
    bad["rl"] = inst["rl"].copy()
    bad["rl"][2] = inst["ru"][2] + 1.0
    with pytest.raises(RuntimeError, match="row bound"):
        net.train_step(A, bad, np.zeros(inst["n"]), np.zeros(inst["m"]))
    xt = np.zeros(inst["n"])
    xt[0] = np.inf
    with pytest.raises(RuntimeError, match="training target"):
        net.train_step(A, inst, xt, np.zeros(inst["m"]))
    assert np.array_equal(net.parameters(), before)   # nothing was applied


def test_prediction_inside_bounds(engine, instances):
    inst = _instance(instances)
    A = engine.Matrix.from_instance(inst)
    x, _ = engine.Gnn(seed=5).predict(A, inst)
    lo = np.where(np.abs(inst["cl"]) < 1e30, inst["cl"], -np.inf)
    hi = np.where(np.abs(inst["cu"]) < 1e30, inst["cu"], np.inf)
    assert np.all(x >= lo) and np.all(x <= hi)


def test_what_training_gains_on_held_out_members(engine, instances, learned):
    """Trained on 64 solved members of a family, measured on 64 others: the held-out
    loss falls far below the untrained network's, the predictions are closer to the
    solutions than the training mean is (the trivial predictor), every warm-started
    PDLP solve converges (PDLP's own KKT test decides it), and the warm starts need
    fewer iterations on average than cold starts."""
    base = instances.lp_family_base(11, 150, 375, 4)
    A = engine.Matrix.from_instance(base)
    train = learned.dataset(engine, A, [instances.lp_family_member(base, 1000 + s) for s in range(64)], 1e-6)
    held = learned.dataset(engine, A, [instances.lp_family_member(base, 5000 + s) for s in range(64)], 1e-6)
    assert len(train) == 64 and len(held) == 64
    scale = learned.dual_scale(train)
    net, untrained = engine.Gnn(seed=3, y_scale=scale), engine.Gnn(seed=3, y_scale=scale)
    history = learned.train(net, A, train, 40)
    assert history[-1] < 0.25 * history[0]
    loss = lambda g: np.mean([g.gradient(A, d[0], d[1], d[2])[0] for d in held])
    assert loss(net) < 0.2 * loss(untrained)
    mx, my = np.mean([d[1] for d in train], axis=0), np.mean([d[2] for d in train], axis=0)

    def err(xp, yp, d):
        return np.sqrt(np.mean((xp - d[1]) ** 2)), np.sqrt(np.mean((yp - d[2]) ** 2))

    e_net = np.mean([err(*net.predict(A, d[0]), d) for d in held], axis=0)
    e_mean = np.mean([err(mx, my, d) for d in held], axis=0)
    assert e_net[0] < e_mean[0] and e_net[1] < e_mean[1], (e_net, e_mean)
    rows = learned.evaluate(engine, net, A, [d[0] for d in held], 1e-6)
    assert all(r["cold_status"] == 0 and r["warm_status"] == 0 for r in rows)
    cold = np.mean([r["cold_iterations"] for r in rows])
    warm = np.mean([r["warm_iterations"] for r in rows])
    assert warm <= 0.97 * cold, (warm, cold)
