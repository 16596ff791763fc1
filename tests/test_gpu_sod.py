"""Sod's shock tube on the 1D Euler GPU path against the reference's own
published verification (cases/tutorials/euler/sod-shock-tube/README.md:36-45,
scripts/sod_shock_tube.py:175-176): P2, HLLC, characteristic WENO and
positivity on troubled cells, CFL 0.2, outflow ends, t = 0.2, uniform meshes
of 50/100/200 elements; the L1 error of the density cell averages against
the exact Riemann solution's cell averages (400 samples per cell)."""
import numpy as np
import pytest

import wasl_b200
from wasl_b200 import cases, meshgen

pytestmark = pytest.mark.gpu

PUBLISHED = {50: 1.083e-2, 100: 5.673e-3, 200: 2.992e-3}


def sod_error(n, precision="plain"):
    arrays = meshgen.jittered_line(n, jitter=0.0)
    exact = cases.ExactRiemann((1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    left, right = cases.conserved(1.0, 0.0, 0.0, 1.0), cases.conserved(0.125, 0.0, 0.0, 0.1)
    with wasl_b200.Solver(*arrays, dimensions=1, equation="euler", polynomial_order=2,
                          boundary="outflow", limiting=True, precision=precision) as g:
        cases.project_line(g, lambda x: np.where((x < 0.5)[..., None], left, right))
        g.limit()
        steps, t = g.run(0.2, 0.0, 0.2)
        assert t == 0.2
        state = g.get_state().reshape(4, g.modes, g.elements)
        error = cases.sod_density_l1(g, exact)
    return error, state


@pytest.mark.parametrize("n", [50, 100, 200])
def test_published_density_l1_errors(n):
    """The published errors are given to four digits: agreement to within
    half a unit in the last digit."""
    error, state = sod_error(n)
    last_digit = 1e-3 * 10 ** np.floor(np.log10(PUBLISHED[n]))
    assert abs(error - PUBLISHED[n]) <= 0.5 * last_digit
    rho = state[0, 0] / np.sqrt(2.0)
    assert rho.min() > 0


def test_verifier_thresholds():
    """The reference verifier's bars: ratio >= 1.6 per doubling, and an L1
    error <= 4e-3 on 200 elements."""
    errors = [sod_error(n)[0] for n in (50, 100, 200)]
    assert errors[0] / errors[1] >= 1.6 and errors[1] / errors[2] >= 1.6
    assert errors[2] <= 4e-3
