"""The learned troubled-cell indicator end to end: training data from the
method's own runs with the reference sensor (seeded two-state Riemann
problems), training on the GPU, then held-out runs judged against the
reference sensor.  What the network gains over running without a troubled
-cell indicator: its solutions stay close to the reference-limited ones
(far closer than with no indicator), while it decides almost every cell
itself and hands few to the fallback."""
import numpy as np
import pytest

import wasl_b200
from wasl_b200 import cases, indicator, meshgen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    xs, ys = [], []
    for seed in range(12):
        arrays = meshgen.jittered_box(24, jitter=0.15, seed=seed)
        x, y = indicator.collect_run(arrays, cases.PlanarRiemann(seed=seed), 2, 100, 4,
                                     boundary="transmissive", positivity_all=True)
        xs.append(x)
        ys.append(y)
    x, y = np.concatenate(xs), np.concatenate(ys)
    assert y.mean() > 0.002  # the reference sensor fires on these runs
    xb, yb = indicator.balance(x, y, 3, seed=0)
    w, loss = indicator.train(xb, yb, steps=3000, batch=4096, learning_rate=2e-3,
                              positive_weight=8.0)
    return w, loss


def run(arrays, problem, mode, w, steps=80):
    with wasl_b200.Solver(*arrays, polynomial_order=2, precision="mixed", volume_rule_order=2,
                          limiting=True, boundary="transmissive", positivity_all=True,
                          sensor_threshold=2.0 if mode == "none" else 1e-3) as g:
        cases.project_initial(g, problem.conserved)
        g.limit()
        if mode == "learned":
            g.set_indicator(w, 0.05, 0.95)
        for _ in range(steps):
            g.step(g.stable_dt(0.1))
        rho = g.get_state().reshape(4, g.modes, g.elements)[0, 0] / np.sqrt(2.0)
        return rho, g.indicator_stats() if mode == "learned" else None


def test_training_fits_the_reference_flags(trained):
    w, loss = trained
    assert loss < 0.1


@pytest.mark.parametrize("seed", [100, 101])
def test_held_out_runs_against_the_reference_sensor(trained, seed):
    w, _ = trained
    arrays = meshgen.jittered_box(20, jitter=0.15, seed=seed)
    problem = cases.PlanarRiemann(seed=seed)
    ref, _ = run(arrays, problem, "reference", w)
    learned, stats = run(arrays, problem, "learned", w)
    none, _ = run(arrays, problem, "none", w)
    cell_stages = sum(stats[k] for k in ("network_troubled", "network_smooth", "fallback"))
    # measured on these seeds: fallback ~3%, missed ~17-21% of the reference's
    # flags, false ~1-2% of all cell-stages, distance 4-8% of no-indicator's
    assert stats["fallback"] <= 0.1 * cell_stages
    assert stats["missed"] <= 0.4 * stats["reference_troubled"]
    assert stats["false"] <= 0.03 * cell_stages
    d_learned = np.mean(np.abs(learned - ref))
    d_none = np.mean(np.abs(none - ref))
    assert d_learned <= 0.15 * d_none
