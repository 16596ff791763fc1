"""Training data, training and judging of the learned troubled-cell indicator.

The network (wasl_mlp_* / wasl_gpu_set_indicator in include/wasl_b200.h) is
trained on the flags the reference modal-decay sensor produces on the
method's own runs: every ``every`` steps of a seeded run with the reference
sensor, the features and flags of the current state are recorded
(``Solver.indicator_data``).  The training runs on the GPU with the
project's own forward/backward and Adam kernels.  The judge is the reference
sensor: missed and false flags of the learned decisions, the share handed to
the fallback, and the change in the solution.
"""
from __future__ import annotations

import numpy as np

from . import Mlp, Solver, cases, meshgen


def collect_run(arrays, problem, p, steps, every, cfl=0.1, precision="mixed", **solver_kw):
    """Features and reference flags from one run with the reference sensor."""
    xs, ys = [], []
    with Solver(*arrays, polynomial_order=p, precision=precision, limiting=True,
                volume_rule_order=p if precision == "mixed" else 0, **solver_kw) as g:
        cases.project_initial(g, problem.conserved)
        g.limit()
        for k in range(steps):
            if k % every == 0:
                x, y = g.indicator_data()
                xs.append(x)
                ys.append(y)
            g.step(g.stable_dt(cfl))
    return np.concatenate(xs), np.concatenate(ys)


def balance(features, labels, negatives_per_positive=3, seed=0):
    """All troubled samples and a seeded random subset of the others, shuffled."""
    rng = np.random.Generator(np.random.PCG64(seed))
    pos = np.nonzero(labels)[0]
    neg = np.nonzero(labels == 0)[0]
    keep = rng.choice(neg, size=min(len(neg), negatives_per_positive * max(len(pos), 1)),
                      replace=False)
    idx = np.concatenate([pos, keep])
    rng.shuffle(idx)
    # whole mini-batches of 64
    idx = idx[: max(64, len(idx) // 64 * 64)]
    return features[idx], labels[idx]


def train(features, labels, steps=3000, batch=4096, learning_rate=2e-3, positive_weight=8.0,
          seed=0, device=0):
    """Train on the GPU; returns (weights, final mean loss)."""
    with Mlp(features.shape[1], seed=seed, device=device) as net:
        net.set_data(features, labels)
        loss = net.train(steps, batch=batch, learning_rate=learning_rate,
                         positive_weight=positive_weight)
        return net.weights(), loss


def shock_vortex_mesh(nx, seed):
    """[0,2] x [0,1] with 2 nx x nx quads, jittered, split along random diagonals."""
    return meshgen.jittered_box(2 * nx, 0.0, 2.0, 0.0, 1.0, jitter=0.15, seed=seed, ny=nx)
