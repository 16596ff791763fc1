"""The learned troubled-cell indicator end to end: training data from the
method's own runs with the reference sensor (seeded two-state Riemann
problems), training on the GPU, then held-out runs judged against the
reference sensor and against the exact solution.  What the network gains
over running without a troubled-cell indicator: its solutions stay close to
the reference-limited ones (far closer than with no indicator), with the
same L1 error against the exact solution, while it decides almost every cell
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


# The network decides a cell itself when sigmoid(logit) is outside this band
# and hands it to the reference sensor otherwise.
BAND = (0.005, 0.999)


def run(arrays, problem, mode, w, steps=80, band=BAND):
    """(cell-average densities, indicator counts, L1 density error against
    the exact solution) after `steps` steps."""
    with wasl_b200.Solver(*arrays, polynomial_order=2, precision="mixed", volume_rule_order=2,
                          limiting=True, boundary="transmissive", positivity_all=True,
                          sensor_threshold=2.0 if mode == "none" else 1e-3) as g:
        cases.project_initial(g, problem.conserved)
        g.limit()
        if mode == "learned":
            g.set_indicator(w, *band)
        t = 0.0
        for _ in range(steps):
            dt = g.stable_dt(0.1)
            g.step(dt)
            t += dt
        rho = g.get_state().reshape(4, g.modes, g.elements)[0, 0] / np.sqrt(2.0)
        l1 = cases.l1_density_error(
            g, lambda x, y: np.repeat(problem.density(x, y, t)[..., None], 4, axis=-1))
        return rho, g.indicator_stats() if mode == "learned" else None, l1


def test_training_fits_the_reference_flags(trained):
    w, loss = trained
    assert loss < 0.1


@pytest.mark.parametrize("seed", [100, 101, 102, 103])
def test_held_out_runs_against_the_reference_sensor(trained, seed):
    """Held-out seeded runs, judged by the reference sensor and by the exact
    solution.  Measured on these seeds with the band (0.005, 0.999): the
    network decides ~95% of cell-stages itself (fallback 4-5%), misses 6-25%
    of the reference's flags, flags 0.2-1% falsely, and its L1 density error
    against the exact planar Riemann solution is within -1%..+2% of the
    reference-limited run's; its densities stay far closer to the
    reference-limited ones than a run without any troubled-cell indicator
    (4-8% of that distance on seeds 100 and 101)."""
    w, _ = trained
    arrays = meshgen.jittered_box(20, jitter=0.15, seed=seed)
    problem = cases.PlanarRiemann(seed=seed)
    ref, _, l1_ref = run(arrays, problem, "reference", w)
    learned, stats, l1_learned = run(arrays, problem, "learned", w)
    none, _, _ = run(arrays, problem, "none", w)
    cell_stages = sum(stats[k] for k in ("network_troubled", "network_smooth", "fallback"))
    assert stats["fallback"] <= 0.06 * cell_stages
    assert stats["missed"] <= 0.3 * stats["reference_troubled"]
    assert stats["false"] <= 0.02 * cell_stages
    assert abs(l1_learned / l1_ref - 1.0) <= 0.05
    d_learned = np.mean(np.abs(learned - ref))
    d_none = np.mean(np.abs(none - ref))
    assert d_learned <= 0.3 * d_none
