"""The plain FP64 path against the reference on the benchmark meshes themselves.

tests/golden/digests_<config>.json holds, for each step of the reference's
own SSP-RK3 steps (oracle/_ref, run by tests/golden/make_config_digests.py),
the CFL time step and the sha256 of the state and of the troubled-cell flag
sets.  Here the GPU plain path starts from the same input (the seeded mesh and
initial data projected on the CPU by the oracle's L2 projection, then, for
limited runs, one limiter application) and must reproduce every dt, state and
flag set bit for bit:

* the isentropic vortex on 256x256 quads (131,072 triangles), P2, periodic,
  100 steps: the metric's own workload;
* the four-quadrant Riemann problem on 1024x1024 quads (2,097,152 triangles),
  P3, transmissive, limiter, 2 steps;
* the shock-vortex on 2048x1024 quads (4,194,304 triangles), P3, transmissive,
  limiter, 1 step.

Bit-identical states give the north star's bars at once: cell averages
within 1e-11 relative, mass and energy conserved as the reference conserves
them, identical flag sets.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import wasl_b200
from golden.make_config_digests import GAMMA, configs, initial_state

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def digests(name):
    path = os.path.join(HERE, "golden", f"digests_{name}.json")
    if not os.path.exists(path):
        pytest.skip(f"no reference digests for {name}")
    with open(path) as f:
        return json.load(f)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", ["vortex256", "quadrant1024", "shockvortex1024"])
def test_plain_path_reproduces_reference_steps(oracle, name):
    golden = digests(name)
    make_arrays, field, p, boundary, limiting, cfl, _ = configs()[name]
    arrays = make_arrays()
    c = initial_state(oracle, arrays, field, p)
    assert sha(c) == golden["initial_sha256"], "the projected input differs from the reference's"
    with wasl_b200.Solver(*arrays, polynomial_order=p, precision="plain", limiting=limiting,
                          boundary=boundary, gamma=GAMMA) as g:
        assert g.elements == golden["elements"]
        g.set_state(c)
        if limiting:
            g.limit()
            assert sha(g.get_state()) == golden["limited_initial_sha256"]
        for k, row in enumerate(golden["steps"]):
            dt = g.stable_dt(cfl)
            assert dt.hex() == row["dt"], f"step {k + 1}: dt"
            g.step(dt)
            assert sha(g.get_state()) == row["state_sha256"], f"step {k + 1}: state"
            if limiting:
                flags = g.flags()
                assert [int(s) for s in flags.sum(axis=1)] == row["troubled"], f"step {k + 1}"
                assert sha(flags) == row["flags_sha256"], f"step {k + 1}: flag sets"
