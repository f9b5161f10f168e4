"""Training and evaluation of the warm-start network (sankhya_b200_gnn_*) on a
parametric LP family that shares one matrix.

The work happens behind the C ABI: PDLP solves (sankhya_b200_pdlp_solve) make
the (instance, solution) pairs, every training step is one call of
sankhya_b200_gnn_train_step (features, forward, backward and the Adam update on
the device), and a prediction is one sankhya_b200_gnn_predict. This module only
orders those calls. Cold start is the fallback: `evaluate` solves every member
both ways and PDLP's own relative-KKT test decides convergence in both.
"""
from __future__ import annotations

import time

import numpy as np


def solve(engine, matrix, inst, eps, x0=None, y0=None, max_iterations=200_000, omega0=None):
    s = engine.pdlp_default_settings()
    s.eps_optimal = eps
    s.max_iterations = max_iterations
    if omega0:
        s.initial_primal_weight = omega0
    t = time.perf_counter()
    rc, x, y, res = engine.pdlp_solve(matrix, inst, s, x0=x0, y0=y0)
    return rc, x, y, res, time.perf_counter() - t


def dataset(engine, matrix, members, eps, progress=None, workers=1):
    """(member, x*, y*, final primal weight) for every member whose PDLP solve converged,
    in member order. With workers > 1 the solves run concurrently from that many host
    threads: each thread's calls go to its own stream with their own buffers (the
    matrix is only read), and every solve is deterministic, so the pairs are the same
    as with one worker."""
    import sys

    def one(inst):
        rc, x, y, res, _ = solve(engine, matrix, inst, eps)
        return (inst, x, y, res["primal_weight"]) if rc == 0 and res["status"] == 0 else None

    results = []
    if workers <= 1:
        for k, inst in enumerate(members):
            results.append(one(inst))
            if progress and (k + 1) % progress == 0:
                print(f"solved {k + 1} / {len(members)}", file=sys.stderr, flush=True)
    else:
        from concurrent.futures import ThreadPoolExecutor

        with ThreadPoolExecutor(max_workers=workers) as pool:
            for k, r in enumerate(pool.map(one, members)):
                results.append(r)
                if progress and (k + 1) % progress == 0:
                    print(f"solved {k + 1} / {len(members)}", file=sys.stderr, flush=True)
    return [r for r in results if r is not None]


def dual_scale(data):
    """Scale of the dual targets: their root mean square (at least 1e-12)."""
    ys = np.concatenate([d[2] for d in data])
    return float(max(np.sqrt(np.mean(ys ** 2)), 1e-12))


def train(gnn, matrix, data, epochs, seed=0):
    """Adam steps over the data in a seeded order; mean loss per epoch."""
    rng = np.random.default_rng(seed)
    history = []
    for _ in range(epochs):
        losses = [gnn.train_step(matrix, data[k][0], data[k][1], data[k][2]) for k in rng.permutation(len(data))]
        history.append(float(np.mean(losses)))
    return history


def learned_weight(data):
    """The family's primal weight: the median of the training solves' final weights."""
    return float(np.median([d[3] for d in data]))


def evaluate(engine, gnn, matrix, members, eps, mean_x=None, mean_y=None, omega=None):
    """Per member: cold-start and network-warm-started PDLP (and, given the
    training mean, a mean-solution warm start; given a learned primal weight, both
    starts again from that weight): iterations, seconds, status."""
    rows = []
    if members:  # one untimed solve first: graph capture and allocations are not a start's cost
        solve(engine, matrix, members[0], eps)
    for inst in members:
        rc_c, _, _, cold, t_cold = solve(engine, matrix, inst, eps)
        tp = time.perf_counter()
        xp, yp = gnn.predict(matrix, inst)
        t_pred = time.perf_counter() - tp
        rc_w, _, _, warm, t_warm = solve(engine, matrix, inst, eps, x0=xp, y0=yp)
        row = dict(cold_iterations=cold["iterations"], cold_seconds=t_cold, cold_status=cold["status"],
                   warm_iterations=warm["iterations"], warm_seconds=t_warm + t_pred, predict_seconds=t_pred,
                   warm_status=warm["status"], cold_objective=cold["primal_objective"],
                   warm_objective=warm["primal_objective"])
        if mean_x is not None:
            _, _, _, mean, t_mean = solve(engine, matrix, inst, eps, x0=mean_x, y0=mean_y)
            row.update(mean_iterations=mean["iterations"], mean_seconds=t_mean, mean_status=mean["status"])
        if omega:
            _, _, _, cw, t_cw = solve(engine, matrix, inst, eps, omega0=omega)
            _, _, _, ww, t_ww = solve(engine, matrix, inst, eps, x0=xp, y0=yp, omega0=omega)
            row.update(cold_weight_iterations=cw["iterations"], cold_weight_seconds=t_cw,
                       cold_weight_status=cw["status"], warm_weight_iterations=ww["iterations"],
                       warm_weight_seconds=t_ww + t_pred, warm_weight_status=ww["status"])
        rows.append(row)
    return rows


def _load(name, path):
    import importlib.util
    import sys
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def main(argv=None):
    """Time to a relative-KKT tolerance, network warm start vs cold start, on a
    seeded parametric family (config 4: m=50,000, n=100,000, 10 per column).
    Prints one JSON line."""
    import argparse
    import json
    import os

    here = os.path.dirname(os.path.abspath(__file__))
    engine = _load("sankhya_b200", os.path.join(here, "__init__.py"))
    instances = _load("sankhya_b200_instances", os.path.join(here, "instances.py"))
    ap = argparse.ArgumentParser()
    ap.add_argument("--m", type=int, default=50_000)
    ap.add_argument("--n", type=int, default=100_000)
    ap.add_argument("--per-col", type=int, default=10)
    ap.add_argument("--train", type=int, default=128)
    ap.add_argument("--eval", type=int, default=16)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--eps", type=float, default=1e-6)
    ap.add_argument("--train-eps", type=float, default=1e-6)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--workers", type=int, default=1, help="concurrent solves while making the training set")
    ap.add_argument("--eval-seed", type=int, default=900_000, help="first seed of the evaluation members")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="only time this many training steps (zero targets, no PDLP solves) and one prediction")
    a = ap.parse_args(argv)
    base = instances.lp_family_base(a.seed, a.m, a.n, a.per_col)
    matrix = engine.Matrix.from_instance(base)
    if a.profile_steps:
        net = engine.Gnn(seed=a.seed)
        x0, y0 = np.zeros(a.n), np.zeros(a.m)
        net.train_step(matrix, base, x0, y0)
        t = time.perf_counter()
        for _ in range(a.profile_steps):
            net.train_step(matrix, base, x0, y0)
        t_steps = time.perf_counter() - t
        t = time.perf_counter()
        net.predict(matrix, base)
        print(json.dumps(dict(workload=f"lp_family: m={a.m}, n={a.n}, {a.per_col} per column, seed {a.seed}",
                              nnz=int(base["ptr"][-1]), steps=a.profile_steps,
                              ms_per_step=1e3 * t_steps / a.profile_steps,
                              predict_ms=1e3 * (time.perf_counter() - t))))
        return
    t = time.perf_counter()
    data = dataset(engine, matrix, [instances.lp_family_member(base, 1000 + s) for s in range(a.train)], a.train_eps,
                   progress=50, workers=a.workers)
    t_data = time.perf_counter() - t
    net = engine.Gnn(seed=a.seed, y_scale=dual_scale(data))
    t = time.perf_counter()
    history = train(net, matrix, data, a.epochs)
    t_train = time.perf_counter() - t
    mean_x = np.mean([d[1] for d in data], axis=0)
    mean_y = np.mean([d[2] for d in data], axis=0)
    omega = learned_weight(data)
    rows = evaluate(engine, net, matrix, [instances.lp_family_member(base, a.eval_seed + s) for s in range(a.eval)],
                    a.eps, mean_x, mean_y, omega)
    avg = lambda k: float(np.mean([r[k] for r in rows])) if rows else None
    out = dict(workload=f"lp_family: m={a.m}, n={a.n}, {a.per_col} per column, seed {a.seed}",
               nnz=int(base["ptr"][-1]), eps=a.eps, train_members=len(data), train_eps=a.train_eps,
               epochs=a.epochs, train_steps=a.epochs * len(data), data_seconds=t_data, train_seconds=t_train,
               steps_per_second=a.epochs * len(data) / t_train, loss_first_epoch=history[0],
               loss_last_epoch=history[-1], eval_members=len(rows),
               converged_cold=sum(r["cold_status"] == 0 for r in rows),
               converged_warm=sum(r["warm_status"] == 0 for r in rows),
               cold_iterations=avg("cold_iterations"), warm_iterations=avg("warm_iterations"),
               mean_start_iterations=avg("mean_iterations"), cold_seconds=avg("cold_seconds"),
               warm_seconds=avg("warm_seconds"), predict_seconds=avg("predict_seconds"),
               mean_start_seconds=avg("mean_seconds"), learned_primal_weight=omega,
               cold_weight_iterations=avg("cold_weight_iterations"), cold_weight_seconds=avg("cold_weight_seconds"),
               warm_weight_iterations=avg("warm_weight_iterations"), warm_weight_seconds=avg("warm_weight_seconds"),
               converged_warm_weight=sum(r["warm_weight_status"] == 0 for r in rows))
    out["speedup_warm_vs_cold"] = out["cold_seconds"] / out["warm_seconds"] if rows else None
    out["speedup_weight_vs_cold"] = out["cold_seconds"] / out["cold_weight_seconds"] if rows else None
    out["speedup_warm_weight_vs_cold"] = out["cold_seconds"] / out["warm_weight_seconds"] if rows else None
    print(json.dumps(out))


if __name__ == "__main__":
    main()
