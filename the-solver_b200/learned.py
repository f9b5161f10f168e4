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


def solve(engine, matrix, inst, eps, x0=None, y0=None, max_iterations=200_000):
    s = engine.pdlp_default_settings()
    s.eps_optimal = eps
    s.max_iterations = max_iterations
    t = time.perf_counter()
    rc, x, y, res = engine.pdlp_solve(matrix, inst, s, x0=x0, y0=y0)
    return rc, x, y, res, time.perf_counter() - t


def dataset(engine, matrix, members, eps):
    """(member, x*, y*) for every member whose PDLP solve converged."""
    out = []
    for inst in members:
        rc, x, y, res, _ = solve(engine, matrix, inst, eps)
        if rc == 0 and res["status"] == 0:
            out.append((inst, x, y))
    return out


def dual_scale(data):
    """Scale of the dual targets: their root mean square (at least 1e-12)."""
    ys = np.concatenate([y for _, _, y in data])
    return float(max(np.sqrt(np.mean(ys ** 2)), 1e-12))


def train(gnn, matrix, data, epochs, seed=0):
    """Adam steps over the data in a seeded order; mean loss per epoch."""
    rng = np.random.default_rng(seed)
    history = []
    for _ in range(epochs):
        losses = [gnn.train_step(matrix, data[k][0], data[k][1], data[k][2]) for k in rng.permutation(len(data))]
        history.append(float(np.mean(losses)))
    return history


def evaluate(engine, gnn, matrix, members, eps, mean_x=None, mean_y=None):
    """Per member: cold-start and network-warm-started PDLP (and, given the
    training mean, a mean-solution warm start): iterations, seconds, status."""
    rows = []
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
        rows.append(row)
    return rows
