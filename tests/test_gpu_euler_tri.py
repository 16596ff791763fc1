"""2D Euler on triangles: the CUDA plain FP64 path against the oracle, bit for bit.

Parity bar: bit-exact states (np.array_equal) after single steps and short
runs, identical troubled-cell flag sets per stage, identical CFL time steps;
the reference's own vectors (tests/golden/ref_vectors.npz) and its stored
case regression (tests/golden/case_regression.json, relative 1e-10)."""
import json
import os

import numpy as np
import pytest

import golden_cases as gc
import wasl_b200
from golden.make_golden import seeded_state
from wasl_b200 import meshgen

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "case_regression.json")))
VECTORS = np.load(os.path.join(HERE, "golden", "ref_vectors.npz"))


def same(a, b):
    return np.array_equal(a, b, equal_nan=True)


def solver(arrays, p, **kw):
    return wasl_b200.Solver(*arrays, dimensions=2, equation="euler", polynomial_order=p, **kw)


def quadrant_state(oracle, arrays, p, seed):
    """Projected four-quadrant Riemann data on [0,1]^2 (seeded states)."""
    mesh = oracle.tri_mesh(*arrays)
    rng = np.random.Generator(np.random.PCG64(seed))
    states = [gc.conserved(rng.uniform(0.1, 1.5), rng.uniform(-1.2, 1.2), rng.uniform(-1.2, 1.2),
                           rng.uniform(0.02, 1.5)) for _ in range(4)]
    rule = max(p, 5)
    xs, ys = mesh.rule_points(rule)
    q = (xs >= 0.5).astype(int) + 2 * (ys >= 0.5).astype(int)
    vals = np.array(states)[q]
    return mesh, mesh.project(p, rule, vals)


@pytest.mark.parametrize("p", [0, 1, 2, 3])
def test_mesh_normalization_matches(oracle, p):
    arrays = meshgen.jittered_box(6, jitter=0.15, seed=p)
    om = oracle.tri_mesh(*arrays)
    with solver(arrays, p) as g:
        assert g.elements == om.ne and g.faces == om.nf
        assert same(g.vertices(), om.vertices)


@pytest.mark.parametrize("p", [0, 1, 2, 3])
@pytest.mark.parametrize("limiting", [False, True])
def test_single_step_periodic(oracle, p, limiting):
    arrays = meshgen.irregular_box(5)
    om = oracle.tri_mesh(*arrays)
    c = seeded_state(om.ne, p, 100 + p)
    donors, basis = om.periodic_trace(p)
    st = om.stencil(p, donors) if limiting else None
    with solver(arrays, p, limiting=limiting) as g:
        g.set_state(c)
        dt = g.stable_dt(0.2)
        assert dt == om.cfl(gc.GAMMA, c, p, 0.2)
        g.step(dt)
        ref = c.copy()
        flags = om.euler_step(gc.GAMMA, p, dt, ref, donors=donors, basis=basis, stencil=st,
                              return_flags=True)
        assert same(g.get_state(), ref)
        if limiting and p > 0:
            assert same(g.flags(), flags)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_reference_vectors(p):
    arrays = meshgen.irregular_box(5)
    with solver(arrays, p, limiting=True) as g:
        g.set_state(VECTORS[f"state_p{p}"])
        g.step(2e-3)
        assert same(g.get_state(), VECTORS[f"limited_step_p{p}"])


@pytest.mark.parametrize("name,d,p,limiting", [c for c in gc.euler_cases() if c[1] == 2])
def test_case_regression(oracle, name, d, p, limiting):
    """The reference's golden 2D Euler runs, through the run loop on the GPU."""
    mesh, c = gc.euler_initial(oracle, 2, p, limiting)
    with solver(meshgen.irregular_box(5), p, limiting=limiting, sensor_threshold=1e-4) as g:
        g.set_state(c)
        g.limit()
        steps, time = g.run(0.2, 0.0, 0.03, 1000)
        state = g.get_state()
        mass, _ = g.mass_energy()
    metrics = gc.metrics(steps, time, state, mass)
    expected = GOLDEN[name]
    assert metrics["step"] == expected["step"]
    for key in ("time", "coefficient_sum", "coefficient_l2", "final_mass"):
        assert gc.close(metrics[key], expected[key]), (key, metrics[key], expected[key])
    # and bit-exact against the oracle run
    donors, basis = mesh.periodic_trace(p)
    st = mesh.stencil(p, donors)
    if limiting:
        st.limit(gc.GAMMA, 1e-4, 1e-10, 1e-10, c)
    gc.run_loop(c, lambda s: mesh.cfl(gc.GAMMA, s, p, 0.2),
                lambda dt, s: mesh.euler_step(gc.GAMMA, p, dt, s, donors=donors, basis=basis,
                                              stencil=st if limiting else None, threshold=1e-4),
                0.0, 0.03)
    assert same(state, c)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_transmissive_quadrant_riemann_limited(oracle, p):
    """Four-quadrant Riemann data, transmissive boundaries, limiter and positivity."""
    arrays = meshgen.jittered_box(12, jitter=0.15, seed=40 + p)
    mesh, c = quadrant_state(oracle, arrays, p, seed=7)
    st = mesh.stencil(p)
    with solver(arrays, p, limiting=True, boundary="transmissive") as g:
        g.set_state(c)
        g.limit()
        st.limit(gc.GAMMA, 1e-3, 1e-10, 1e-10, c)
        assert same(g.get_state(), c)
        troubled = 0
        for _ in range(5):
            dt = g.stable_dt(0.1)
            assert dt == mesh.cfl(gc.GAMMA, c, p, 0.1)
            g.step(dt)
            flags = mesh.euler_step(gc.GAMMA, p, dt, c, boundary="transmissive", stencil=st,
                                    return_flags=True)
            assert same(g.flags(), flags)
            troubled += int(flags.sum())
            assert same(g.get_state(), c)
        assert troubled > 0


def test_larger_periodic_mesh_many_steps(oracle):
    p = 2
    arrays = meshgen.jittered_box(32, 0.0, 10.0, 0.0, 10.0, jitter=0.15, seed=1)
    om = oracle.tri_mesh(*arrays)
    c = seeded_state(om.ne, p, 5, amplitude=0.02)
    donors, basis = om.periodic_trace(p)
    with solver(arrays, p) as g:
        g.set_state(c)
        for _ in range(10):
            dt = g.stable_dt(0.15)
            assert dt == om.cfl(gc.GAMMA, c, p, 0.15)
            g.step(dt)
            om.euler_step(gc.GAMMA, p, dt, c, donors=donors, basis=basis)
        assert same(g.get_state(), c)


def test_mass_energy_conserved_periodic():
    p = 2
    arrays = meshgen.jittered_box(16, jitter=0.15, seed=2)
    with solver(arrays, p) as g:
        g.set_state(seeded_state(g.elements, p, 9, amplitude=0.02))
        m0, e0 = g.mass_energy()
        for _ in range(50):
            g.step(g.stable_dt(0.15))
        m1, e1 = g.mass_energy()
    assert abs(m1 - m0) <= 1e-13 * abs(m0)
    assert abs(e1 - e0) <= 1e-13 * abs(e0)


def test_checkpoint_round_trip(tmp_path):
    p = 2
    arrays = meshgen.irregular_box(4)
    with solver(arrays, p) as g:
        c = seeded_state(g.elements, p, 3)
        g.set_state(c)
        g.write_checkpoint(tmp_path / "c.bin", 0.25, 7, "box.mesh")
        g.set_state(np.zeros_like(c))
        assert g.read_checkpoint(tmp_path / "c.bin") == (0.25, 7)
        assert same(g.get_state(), c)
    with solver(meshgen.irregular_box(3), p) as other:
        with pytest.raises(wasl_b200.WaslError, match="layout or mesh provenance"):
            other.read_checkpoint(tmp_path / "c.bin")


def test_nonphysical_average_is_an_error_status():
    p = 1
    arrays = meshgen.irregular_box(3)
    with solver(arrays, p) as g:
        c = seeded_state(g.elements, p, 4)
        c[5] = -1.0  # negative density average in element 5
        g.set_state(c)
        with pytest.raises(wasl_b200.WaslError, match="not physical") as err:
            g.stable_dt(0.1)
        assert err.value.status == -4
        c[5] = 1.0
        g.set_state(c)
        assert g.stable_dt(0.1) > 0.0  # the handle stays usable


def test_positivity_floor_error_status(oracle):
    p = 1
    arrays = meshgen.irregular_box(5)
    mesh, c = gc.euler_initial(oracle, 2, p, True)
    with solver(arrays, p, limiting=True, density_floor=0.5, sensor_threshold=1e-4) as g:
        g.set_state(c)
        with pytest.raises(wasl_b200.WaslError, match="below a floor") as err:
            g.limit()
        assert err.value.status == -5


def test_hundred_limited_steps_match_the_oracle(oracle):
    """The plain path against the oracle for 100 steps with the limiter:
    every step's troubled-cell flag set identical, the same dt, and the final
    state identical (the bar is cell averages within 1e-11 relative); mass
    conserved to 1e-13."""
    p = 2
    arrays = meshgen.jittered_box(24, jitter=0.15, seed=12)
    om = oracle.tri_mesh(*arrays)
    c = seeded_state(om.ne, p, 21, amplitude=0.02)
    donors, basis = om.periodic_trace(p)
    st = om.stencil(p, donors)
    troubled = 0
    with solver(arrays, p, limiting=True) as g:
        g.set_state(c)
        m0, _ = g.mass_energy()
        for _ in range(100):
            dt = g.stable_dt(0.15)
            assert dt == om.cfl(gc.GAMMA, c, p, 0.15)
            g.step(dt)
            flags = om.euler_step(gc.GAMMA, p, dt, c, donors=donors, basis=basis, stencil=st,
                                  return_flags=True)
            assert same(g.flags(), flags)
            troubled += int(flags.sum())
        state = g.get_state()
        m1, _ = g.mass_energy()
    assert same(state, c)
    assert troubled > 0
    assert abs(m1 - m0) <= 1e-13 * abs(m0)
