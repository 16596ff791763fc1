"""1D Euler, 1D scalar advection and 2D scalar advection: the CUDA plain FP64
paths against the oracle, bit for bit.

Parity bar: bit-exact states (np.array_equal) after single steps and whole
runs, identical troubled-cell flag sets per stage and identical CFL steps;
the reference's stored case regression (tests/golden/case_regression.json,
relative 1e-10) for every 1D Euler and scalar run it holds.  Scalar states
cross the C-ABI in the checkpoint layout [mode][element]; the oracle keeps the
reference's solver layout [element][mode], so tests transpose.
"""
import json
import os

import numpy as np
import pytest

import golden_cases as gc
import wasl_b200
from wasl_b200 import cases, meshgen

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "case_regression.json")))
KINDS = {"periodic": 0, "inflow": 1, "outflow": 2}


def same(a, b):
    return np.array_equal(a, b, equal_nan=True)


def line_state(ne, p, seed, amplitude=0.05):
    """Physical 1D Euler state U[variable][mode][element] with energy in every mode."""
    M = p + 1
    rng = np.random.Generator(np.random.PCG64(seed))
    c = amplitude * rng.standard_normal((4, M, ne))
    s2 = np.sqrt(2.0)
    c[0, 0] = s2 * (1.0 + 0.2 * rng.uniform(-1, 1, ne))
    c[1, 0] = s2 * 0.3 * rng.uniform(-1, 1, ne)
    c[2, 0] = s2 * 0.1 * rng.uniform(-1, 1, ne)
    c[3, 0] = s2 * (2.5 + 0.3 * rng.uniform(-1, 1, ne))
    return c.ravel()


def to_checkpoint(c, ne, M):
    """Solver layout [element][mode] -> checkpoint layout [mode][element]."""
    return np.ascontiguousarray(np.asarray(c).reshape(ne, M).T).ravel()


def line(arrays, p, equation="euler", **kw):
    return wasl_b200.Solver(*arrays, dimensions=1, equation=equation, polynomial_order=p, **kw)


def scalar_tri(arrays, p, **kw):
    return wasl_b200.Solver(*arrays, dimensions=2, equation="scalar", polynomial_order=p, **kw)


# ---- 1D Euler ------------------------------------------------------------------------

def test_line_mesh_normalization(oracle):
    arrays = meshgen.irregular_line(12)
    om = oracle.line_mesh(*arrays)
    with line(arrays, 1) as g:
        assert g.elements == om.ne and g.faces == om.nf
        v = g.vertices()
        assert same(v[:, 0], om.x_left) and same(v[:, 1], om.x_right)


@pytest.mark.parametrize("p", [0, 1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("ends", ["periodic", "outflow"])
@pytest.mark.parametrize("limiting", [False, True])
def test_euler_line_single_step(oracle, p, ends, limiting):
    arrays = meshgen.jittered_line(40, jitter=0.2, seed=p)
    om = oracle.line_mesh(*arrays)
    c = line_state(om.ne, p, 200 + p)
    k = KINDS[ends]
    st = om.stencil(p, periodic=k == 0) if limiting else None
    with line(arrays, p, boundary=ends, limiting=limiting) as g:
        g.set_state(c)
        dt = g.stable_dt(0.2)
        assert dt == om.cfl(gc.GAMMA, c, p, 0.2)
        g.step(dt)
        ref = c.copy()
        flags = om.euler_step(gc.GAMMA, p, dt, ref, k, k, st, return_flags=True)
        assert same(g.get_state(), ref)
        if limiting and p > 0:
            assert same(g.flags(), flags)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_euler_line_sod_limited(oracle, p):
    """Sod's shock tube, outflow ends, limiter and positivity: 60 steps bit for bit."""
    arrays = meshgen.jittered_line(200, jitter=0.2, seed=11 + p)
    om = oracle.line_mesh(*arrays)
    xs = om.rule_points(7)
    vals = np.where((xs < 0.5)[..., None], cases.conserved(1.0, 0.0, 0.0, 1.0),
                    cases.conserved(0.125, 0.0, 0.0, 0.1))
    c = om.project(p, 7, vals)
    st = om.stencil(p, periodic=False)
    with line(arrays, p, boundary="outflow", limiting=True) as g:
        g.set_state(c)
        g.limit()
        st.limit(gc.GAMMA, 1e-3, 1e-10, 1e-10, c)
        assert same(g.get_state(), c)
        troubled = 0
        for _ in range(60):
            dt = g.stable_dt(0.2)
            assert dt == om.cfl(gc.GAMMA, c, p, 0.2)
            g.step(dt)
            flags = om.euler_step(gc.GAMMA, p, dt, c, 2, 2, st, return_flags=True)
            assert same(g.flags(), flags)
            troubled += int(flags.sum())
        assert same(g.get_state(), c)
        assert troubled > 0


def test_euler_line_run_conserves_periodic(oracle):
    arrays = meshgen.jittered_line(64, jitter=0.2, seed=5)
    om = oracle.line_mesh(*arrays)
    c = line_state(om.ne, 2, 9)
    st = om.stencil(2, periodic=True)
    with line(arrays, 2, limiting=True) as g:
        g.set_state(c)
        m0, e0 = g.mass_energy()
        steps, time = g.run(0.2, 0.0, 0.05, 100000)
        m1, e1 = g.mass_energy()
        state = g.get_state()
    assert abs(m1 - m0) <= 1e-13 * abs(m0) and abs(e1 - e0) <= 1e-13 * abs(e0)
    n, t = gc.run_loop(c, lambda s: om.cfl(gc.GAMMA, s, 2, 0.2),
                       lambda dt, s: om.euler_step(gc.GAMMA, 2, dt, s, 0, 0, st),
                       0.0, 0.05, max_steps=100000)
    assert (n, t) == (steps, time)
    assert same(state, c)


def test_euler_line_rejects_inflow_and_one_periodic_end():
    arrays = meshgen.jittered_line(8)
    with pytest.raises(wasl_b200.WaslError) as e:
        line(arrays, 1, boundary="inflow", boundary_right="outflow")
    assert e.value.status == -1 and "inflow is not implemented" in str(e.value)
    with pytest.raises(wasl_b200.WaslError) as e:
        line(arrays, 1, boundary="periodic", boundary_right="outflow")
    assert e.value.status == -2 and "both line ends" in str(e.value)


def test_euler_line_nonphysical_average_reports():
    arrays = meshgen.jittered_line(16)
    c = line_state(16, 1, 3)
    c[0 * 2 * 16 + 5] = -1.0  # negative mean density in element 5
    with line(arrays, 1) as g:
        g.set_state(c)
        with pytest.raises(wasl_b200.WaslError) as e:
            g.stable_dt(0.2)
        assert e.value.status == -4


# ---- 1D scalar advection ---------------------------------------------------------------

@pytest.mark.parametrize("p", [0, 1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("ends,speed", [(("periodic", "periodic"), 0.7),
                                        (("inflow", "outflow"), 0.7),
                                        (("outflow", "inflow"), -0.9),
                                        (("outflow", "outflow"), 1.3)])
def test_scalar_line_steps(oracle, p, ends, speed):
    arrays = meshgen.jittered_line(50, jitter=0.2, seed=30 + p)
    om = oracle.line_mesh(*arrays)
    M = p + 1
    rng = np.random.Generator(np.random.PCG64(p))
    c = rng.standard_normal(om.ne * M)
    lk, rk = KINDS[ends[0]], KINDS[ends[1]]
    lv, rv = 0.8, -0.3
    with line(arrays, p, equation="scalar", velocity=(speed, 0.0), boundary=ends[0],
              boundary_right=ends[1], inflow=(lv, rv)) as g:
        g.set_state(to_checkpoint(c, om.ne, M))
        dt = g.stable_dt(0.3)
        assert dt == om.advection_cfl(speed, p, 0.3)
        for _ in range(10):
            g.step(dt)
            om.scalar_step(speed, p, dt, c, lk, lv, rk, rv)
            assert same(g.get_state(), to_checkpoint(c, om.ne, M))


def test_scalar_line_advected_pulse_full_run(oracle):
    """400 jittered cells, P2, a = 1, CFL 0.1, to t = 1: the whole run bit for bit."""
    arrays = cases.advection_line_mesh()
    om = oracle.line_mesh(*arrays)
    pulse = cases.AdvectedPulse(1.0)
    with line(arrays, 2, equation="scalar", velocity=(1.0, 0.0)) as g:
        cases.project_line(g, pulse.value)
        c0 = g.get_state()
        steps, time = g.run(0.1, 0.0, 1.0, 10 ** 9)
        state = g.get_state()
        mass0 = om.mass(c0, 1)
        mass, _ = g.mass_energy()
        error = cases.l1_line_error(g, lambda x: pulse.value(x, time))
    xs = om.rule_points(7)
    c = om.project(2, 7, pulse.value(xs)[..., None])
    assert same(c, c0)
    c = c.reshape(3, om.ne).T.ravel().copy()
    dt = om.advection_cfl(1.0, 2, 0.1)
    n, t = gc.run_loop(c, lambda s: dt, lambda d, s: om.scalar_step(1.0, 2, d, s), 0.0, 1.0,
                       max_steps=10 ** 9)
    assert (n, t) == (steps, time) and steps > 10000
    assert same(state, to_checkpoint(c, om.ne, 3))
    # Round-off of ~33,000 steps; the state itself is the reference's, bit for bit.
    assert abs(mass - mass0) <= 1e-11 * max(1.0, abs(mass0))
    assert error < 1e-3


def test_resident_run_is_the_host_loop_bit_for_bit():
    """The whole 400-cell advection run (P2, a = 1, CFL 0.1, to t = 1: ~33,000
    steps) in one kernel launch gives the host loop's step count, final time
    and state bit for bit (the host loop's run is the reference's, above)."""
    arrays = cases.advection_line_mesh()
    pulse = cases.AdvectedPulse(1.0)
    out = []
    for resident in (False, True):
        with line(arrays, 2, equation="scalar", velocity=(1.0, 0.0)) as g:
            cases.project_line(g, pulse.value)
            run = g.run_resident if resident else g.run
            steps, time = run(0.1, 0.0, 1.0, 10 ** 9)
            out.append((steps, time, g.get_state()))
    assert out[0][:2] == out[1][:2] and out[0][0] > 10000
    assert same(out[0][2], out[1][2])


@pytest.mark.parametrize("p,ends,n", [(1, "periodic", 96), (2, "periodic", 96),
                                      (2, "outflow", 96), (2, "periodic", 40),
                                      (2, "outflow", 192), (2, "periodic", 397),
                                      (3, "periodic", 397)])
def test_resident_euler_run_is_the_host_loop_bit_for_bit(p, ends, n):
    """1D Euler with the CFL step taken from the state every step, on the
    device in one launch, on line meshes of 40 to 397 elements: the host
    loop's steps, time and state."""
    arrays = meshgen.jittered_line(n, jitter=0.2, seed=3)
    rng = np.random.Generator(np.random.PCG64(8))
    M = p + 1
    c = 0.02 * rng.standard_normal((4, M, n))
    c[0, 0] = np.sqrt(2) * (1.0 + 0.2 * rng.uniform(-1, 1, n))
    c[1, 0] = np.sqrt(2) * 0.3
    c[3, 0] = np.sqrt(2) * 2.5
    out = []
    for resident in (False, True):
        with line(arrays, p, boundary=ends) as g:
            g.set_state(c.ravel())
            run = g.run_resident if resident else g.run
            out.append((*run(0.3, 0.0, 0.05), g.get_state()))
    assert out[0][:2] == out[1][:2] and out[0][0] > 5
    assert same(out[0][2], out[1][2])


def test_resident_run_limits():
    """Runs with the limiter, or meshes whose state does not fit in one
    CTA's shared memory, are refused with a status."""
    with line(meshgen.jittered_line(64, jitter=0.2, seed=1), 2, limiting=True) as g:
        with pytest.raises(wasl_b200.WaslError, match="limiter"):
            g.run_resident(0.3, 0.0, 0.01)
    with line(meshgen.jittered_line(20000, jitter=0.2, seed=1), 2, equation="scalar",
              velocity=(1.0, 0.0)) as g:
        with pytest.raises(wasl_b200.WaslError, match="shared memory"):
            g.run_resident(0.1, 0.0, 0.01)


def test_scalar_line_large_mesh_single_step(oracle):
    """A 2^20-cell line: parity does not depend on size."""
    arrays = meshgen.jittered_line(1 << 20, jitter=0.2, seed=1)
    om = oracle.line_mesh(*arrays)
    rng = np.random.Generator(np.random.PCG64(4))
    c = rng.standard_normal(om.ne * 4)
    with line(arrays, 3, equation="scalar", velocity=(-0.6, 0.0)) as g:
        g.set_state(to_checkpoint(c, om.ne, 4))
        dt = g.stable_dt(0.2)
        g.step(dt)
        om.scalar_step(-0.6, 3, dt, c)
        assert same(g.get_state(), to_checkpoint(c, om.ne, 4))


# ---- 2D scalar advection -----------------------------------------------------------------

@pytest.mark.parametrize("p", [0, 1, 2, 3])
@pytest.mark.parametrize("mesh_kind", ["irregular", "jittered"])
def test_scalar_tri_steps(oracle, p, mesh_kind):
    arrays = (meshgen.irregular_box(5) if mesh_kind == "irregular"
              else meshgen.jittered_box(9, jitter=0.15, seed=p, ny=7))
    om = oracle.tri_mesh(*arrays)
    M = (p + 1) * (p + 2) // 2
    donors, basis = om.periodic_trace(p)
    rng = np.random.Generator(np.random.PCG64(50 + p))
    c = rng.standard_normal(om.ne * M)
    with scalar_tri(arrays, p, velocity=(0.7, -0.4)) as g:
        g.set_state(to_checkpoint(c, om.ne, M))
        dt = g.stable_dt(0.3)
        assert dt == om.scalar_cfl(0.7, -0.4, p, 0.3)
        m0, _ = g.mass_energy()
        for _ in range(8):
            g.step(dt)
            om.scalar_step(0.7, -0.4, p, dt, c, donors, basis)
            assert same(g.get_state(), to_checkpoint(c, om.ne, M))
        m1, _ = g.mass_energy()
        assert abs(m1 - m0) <= 1e-13 * max(1.0, abs(m0))


def test_scalar_tri_rejects_open_boundaries():
    with pytest.raises(wasl_b200.WaslError) as e:
        scalar_tri(meshgen.irregular_box(3), 1, velocity=(1.0, 0.0), boundary="transmissive")
    assert e.value.status == -2 and "must be periodic" in str(e.value)


# ---- the reference's stored case regression ----------------------------------------------

def check(name, metrics):
    expected = GOLDEN[name]
    assert metrics["step"] == expected["step"], name
    for key in ("time", "coefficient_sum", "coefficient_l2", "final_mass"):
        assert gc.close(metrics[key], expected[key]), (name, key, metrics[key], expected[key])


@pytest.mark.parametrize("name,d,p,limiting", [c for c in gc.euler_cases() if c[1] == 1])
def test_case_regression_euler_line(oracle, name, d, p, limiting):
    mesh, c = gc.euler_initial(oracle, 1, p, limiting)
    with line(meshgen.irregular_line(12), p, limiting=limiting, sensor_threshold=1e-4) as g:
        g.set_state(c)
        g.limit()
        steps, time = g.run(0.2, 0.0, 0.03, 1000)
        state = g.get_state()
        mass, _ = g.mass_energy()
    check(name, gc.metrics(steps, time, state, mass))
    st = mesh.stencil(p, periodic=True)
    if limiting:
        st.limit(gc.GAMMA, 1e-4, 1e-10, 1e-10, c)
    gc.run_loop(c, lambda s: mesh.cfl(gc.GAMMA, s, p, 0.2),
                lambda dt, s: mesh.euler_step(gc.GAMMA, p, dt, s, 0, 0,
                                              st if limiting else None, 1e-4),
                0.0, 0.03)
    assert same(state, c)


@pytest.mark.parametrize("name,d,p", gc.scalar_cases())
def test_case_regression_scalar(oracle, tmp_path, name, d, p):
    """Fresh run to t = 0.2 with a checkpoint, then the restart to t = 0.3."""
    mesh, c = gc.scalar_initial(oracle, d, p)
    M = c.shape[1]
    arrays = meshgen.irregular_line(12) if d == 1 else meshgen.irregular_box(5)
    kw = dict(velocity=(0.7, 0.0)) if d == 1 else dict(velocity=(0.7, -0.4))
    make = (lambda: line(arrays, p, equation="scalar", **kw)) if d == 1 else \
        (lambda: scalar_tri(arrays, p, **kw))
    path = str(tmp_path / "restart.ckpt")
    with make() as g:
        g.set_state(to_checkpoint(c, mesh.ne, M))
        steps, time = g.run(0.3, 0.0, 0.2, 1000)
        mass, _ = g.mass_energy()
        check(name, gc.metrics(steps, time, g.get_state(), mass))
        g.write_checkpoint(path, time, steps)
    with make() as g:
        t0, s0 = g.read_checkpoint(path)
        n, time = g.run(0.3, t0, 0.3, 1000 - s0)
        mass, _ = g.mass_energy()
        state = g.get_state()
        check(name + "-restart", gc.metrics(s0 + n, time, state, mass))
    c = c.ravel().copy()
    if d == 1:
        dt0 = mesh.advection_cfl(0.7, p, 0.3)
        adv = lambda dt, s: mesh.scalar_step(0.7, p, dt, s)  # noqa: E731
    else:
        donors, basis = mesh.periodic_trace(p)
        dt0 = mesh.scalar_cfl(0.7, -0.4, p, 0.3)
        adv = lambda dt, s: mesh.scalar_step(0.7, -0.4, p, dt, s, donors, basis)  # noqa: E731
    step, t = gc.run_loop(c, lambda s: dt0, adv, 0.0, 0.2)
    gc.run_loop(c, lambda s: dt0, adv, t, 0.3, step0=step)
    assert same(state, to_checkpoint(c, mesh.ne, M))
