"""Pins the oracle against the reference's stored golden data.

* case_regression.json: the 29-run case regression of the reference
  (cpp/tests/runtime/case_regression_test.cpp, tolerance relative 1e-10).
* ref_vectors.npz: the reference's own outputs on seeded inputs, bit-exact.
"""
import json
import os

import numpy as np
import pytest

import golden_cases as gc
from golden.make_golden import seeded_state
from wasl_b200 import meshgen

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "case_regression.json")))
VECTORS = np.load(os.path.join(HERE, "golden", "ref_vectors.npz"))


def run_euler_oracle(oracle, name, d, p, limiting):
    mesh, c = gc.euler_initial(oracle, d, p, limiting)
    threshold, rf, pf = 1e-4, 1e-10, 1e-10
    if d == 1:
        stencil = mesh.stencil(p, periodic=True)
        if limiting:
            stencil.limit(gc.GAMMA, threshold, rf, pf, c)
        step, time = gc.run_loop(
            c, lambda s: mesh.cfl(gc.GAMMA, s, p, 0.2),
            lambda dt, s: mesh.euler_step(gc.GAMMA, p, dt, s, 0, 0,
                                          stencil if limiting else None, threshold, rf, pf),
            0.0, 0.03)
        mass = mesh.mass(c, 1)
    else:
        donors, basis = mesh.periodic_trace(p)
        stencil = mesh.stencil(p, donors)
        if limiting:
            stencil.limit(gc.GAMMA, threshold, rf, pf, c)
        step, time = gc.run_loop(
            c, lambda s: mesh.cfl(gc.GAMMA, s, p, 0.2),
            lambda dt, s: mesh.euler_step(gc.GAMMA, p, dt, s, donors=donors, basis=basis,
                                          stencil=stencil if limiting else None,
                                          threshold=threshold),
            0.0, 0.03)
        mass = mesh.mass(c, 1)
    return gc.metrics(step, time, c, mass)


def run_scalar_oracle(oracle, d, p):
    """Fresh run to t=0.2, then the restart continuing to t=0.3."""
    mesh, c = gc.scalar_initial(oracle, d, p)
    M = c.shape[1]
    c = c.ravel().copy()
    if d == 1:
        dt0 = mesh.advection_cfl(0.7, p, 0.3)
        adv = lambda dt, s: mesh.scalar_step(0.7, p, dt, s)  # noqa: E731
    else:
        donors, basis = mesh.periodic_trace(p)
        dt0 = mesh.scalar_cfl(0.7, -0.4, p, 0.3)
        adv = lambda dt, s: mesh.scalar_step(0.7, -0.4, p, dt, s, donors, basis)  # noqa: E731
    out = {}
    step, time = gc.run_loop(c, lambda s: dt0, adv, 0.0, 0.2)
    ck = c.reshape(mesh.ne, M).T.ravel()
    out[""] = gc.metrics(step, time, ck, mesh.mass(c, M))
    step, time = gc.run_loop(c, lambda s: dt0, adv, time, 0.3, step0=step)
    ck = c.reshape(mesh.ne, M).T.ravel()
    out["-restart"] = gc.metrics(step, time, ck, mesh.mass(c, M))
    return out


def check(name, actual):
    expected = GOLDEN[name]
    assert actual["step"] == expected["step"], name
    for key in ("time", "coefficient_sum", "coefficient_l2", "final_mass"):
        assert gc.close(actual[key], expected[key]), (name, key, actual[key], expected[key])


@pytest.mark.parametrize("name,d,p,limiting", gc.euler_cases())
def test_oracle_euler_case_regression(oracle, name, d, p, limiting):
    check(name, run_euler_oracle(oracle, name, d, p, limiting))


@pytest.mark.parametrize("name,d,p", gc.scalar_cases())
def test_oracle_scalar_case_regression(oracle, name, d, p):
    result = run_scalar_oracle(oracle, d, p)
    check(name, result[""])
    check(name + "-restart", result["-restart"])


def test_golden_table_is_complete():
    assert len(GOLDEN) == 28 or len(GOLDEN) == 29
    names = {n for n, *_ in gc.euler_cases()} | {n for n, *_ in gc.scalar_cases()}
    names |= {n + "-restart" for n, *_ in gc.scalar_cases()}
    assert names == set(GOLDEN)


@pytest.mark.parametrize("p", [0, 1, 2, 3])
def test_oracle_matches_reference_vectors(oracle, p):
    mesh = oracle.tri_mesh(*meshgen.irregular_box(5))
    c = seeded_state(mesh.ne, p, 100 + p)
    assert np.array_equal(c, VECTORS[f"state_p{p}"])
    donors, basis = mesh.periodic_trace(p)
    ext = mesh.periodic_exterior(p, donors, basis, c)
    assert np.array_equal(mesh.euler_residual(gc.GAMMA, p, c, ext), VECTORS[f"residual_p{p}"])
    if p > 0:
        stencil = mesh.stencil(p, donors)
        stepped = c.copy()
        flags = mesh.euler_step(gc.GAMMA, p, 2e-3, stepped, donors=donors, basis=basis,
                                stencil=stencil, threshold=1e-3, return_flags=True)
        assert flags.sum() > 0  # the limiter is exercised
        assert np.array_equal(stepped, VECTORS[f"limited_step_p{p}"])
