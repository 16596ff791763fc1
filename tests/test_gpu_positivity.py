"""Always-on positivity (an extension of the reference, which limits
positivity in troubled cells only): every unflagged element also passes
through the positivity limiter after each stage."""
import numpy as np
import pytest

import wasl_b200
from golden.make_golden import seeded_state
from wasl_b200 import cases, meshgen

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_no_change_on_a_positive_state(precision):
    """Where every check point is already physical the limiter scales by 1:
    the trajectory is bit-identical to the reference behaviour's."""
    arrays = meshgen.jittered_box(12, jitter=0.15, seed=8)
    out = []
    for positivity_all in (False, True):
        with wasl_b200.Solver(*arrays, polynomial_order=2, precision=precision, limiting=True,
                              positivity_all=positivity_all) as g:
            g.set_state(seeded_state(g.elements, 2, 5, amplitude=0.01))
            for _ in range(5):
                g.step(g.stable_dt(0.15))
            out.append(g.get_state())
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("p", [1, 2, 3])
def test_point_values_stay_physical(p):
    """A sharp seeded four-quadrant Riemann problem: after every step the
    density and pressure at the volume check points are above the floors (to
    round-off)."""
    arrays = meshgen.jittered_box(24, jitter=0.15, seed=p)
    problem = cases.QuadrantRiemann(seed=11)
    with wasl_b200.Solver(*arrays, polynomial_order=p, precision="mixed", limiting=True,
                          positivity_all=True, boundary="transmissive") as g:
        cases.project_initial(g, problem.conserved)
        g.limit()
        for _ in range(15):
            g.step(g.stable_dt(0.1))
            values = g.evaluate(p)
            rho = values[..., 0]
            kinetic = 0.5 * (values[..., 1] ** 2 + values[..., 2] ** 2) / rho
            pressure = 0.4 * (values[..., 3] - kinetic)
            assert rho.min() >= 1e-10 - 1e-12
            assert pressure.min() >= 1e-10 - 1e-9 * np.abs(values[..., 3]).max()
