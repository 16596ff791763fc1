"""The case-level regression of the reference, restated as test input.

cpp/tests/runtime/case_regression_test.cpp:135-203 runs every serial driver on
an irregular 12-cell line and a 5x5 irregular box and reduces each run to
(step, time, sum of checkpoint coefficients, their L2 norm, final mass).  This
module rebuilds the same inputs (meshes, piecewise-constant initial data, run
control) and drives any stepper through the run loop of
cpp/src/case/serial_case_runner.cpp:117-149, so the oracle and the CUDA product
can both be checked against tests/golden/case_regression.json.
"""
from __future__ import annotations

import math

import numpy as np

from wasl_b200 import meshgen

GAMMA = 1.4


def euler_cases():
    out = []
    for d in (1, 2):
        for p in (0, 1, 2):
            for limiting in (False, True):
                out.append((f"euler-d{d}-p{p}" + ("-limited" if limiting else ""), d, p, limiting))
    return out


def scalar_cases():
    return [(f"scalar-d{d}-p{p}", d, p) for d in (1, 2) for p in (0, 1, 2, 3)]


def conserved(rho, u, v, p):
    """cpp/include/wasl/equations/euler/primitive.hpp:10-17"""
    kinetic_energy = 0.5 * rho * (u * u + v * v)
    return (rho, rho * u, rho * v, p / (GAMMA - 1.0) + kinetic_energy)


def euler_regions(d, limiting):
    default = (1.0, 0.3, 0.2 if d == 2 else 0.0, 1.0)
    inside = (0.2, 0.0, 0.0, 0.15) if limiting else (0.9, 0.25, 0.1 if d == 2 else 0.0, 0.95)
    return default, inside


def euler_initial_value(d, limiting, x, y=0.0):
    """cpp/src/case/initial_regions.cpp:36-57 for the regression's two regions."""
    default, inside = euler_regions(d, limiting)
    if d == 1:
        if 0.3 <= x <= 0.6:
            return inside
    else:
        dx, dy = x - 0.5, y - 0.5
        if dx * dx + dy * dy <= 0.25 * 0.25:
            return inside
    return default


def scalar_initial_value(d, p, x, y=0.0):
    """cpp/src/case/initial_regions.cpp:17-34 with the regression's settings."""
    if d == 1:
        if p == 2:
            return 1.5 * math.sin(2.0 * math.pi * x)
        if 0.2 <= x <= 0.55:
            return 1.0
        return 0.25
    dx, dy = x - 0.5, y - 0.4
    if dx * dx + dy * dy <= 0.25 * 0.25:
        return 2.0
    return 0.25


def meshes():
    return meshgen.irregular_line(12), meshgen.irregular_box(5)


def euler_initial(oracle, d, p, limiting):
    """Projected initial coefficients U[var][mode][elem] (initial_state.cpp:48-64)."""
    line, box = meshes()
    if d == 1:
        mesh = oracle.line_mesh(*line)
        xs = mesh.rule_points(7)
        vals = np.array([[conserved(*euler_initial_value(1, limiting, x)) for x in row]
                         for row in xs])
        return mesh, mesh.project(p, 7, vals)
    mesh = oracle.tri_mesh(*box)
    rule = max(p, 5)
    xs, ys = mesh.rule_points(rule)
    vals = np.array([[conserved(*euler_initial_value(2, limiting, x, y)) for x, y in zip(rx, ry)]
                     for rx, ry in zip(xs, ys)])
    return mesh, mesh.project(p, rule, vals)


def scalar_initial(oracle, d, p):
    """Projected, then transposed to the solver layout U[element][mode]
    (initial_state.cpp:31-46, scalar_coefficient_layout.cpp:22-31)."""
    line, box = meshes()
    if d == 1:
        mesh = oracle.line_mesh(*line)
        xs = mesh.rule_points(7)
        vals = np.array([[[scalar_initial_value(1, p, x)] for x in row] for row in xs])
        c = mesh.project(p, 7, vals)
        M = p + 1
    else:
        mesh = oracle.tri_mesh(*box)
        rule = max(p, 5)
        xs, ys = mesh.rule_points(rule)
        vals = np.array([[[scalar_initial_value(2, p, x, y)] for x, y in zip(rx, ry)]
                         for rx, ry in zip(xs, ys)])
        c = mesh.project(p, rule, vals)
        M = (p + 1) * (p + 2) // 2
    return mesh, c.reshape(M, mesh.ne).T.copy()


def next_time_step(end_time, time, stable):
    """cpp/src/case/serial_case_runner.cpp:107-113"""
    remaining = end_time - time
    step = min(stable if stable > 0.0 else remaining, remaining)
    if step <= 0.0 or time + step == time:
        raise RuntimeError("simulation: timestep cannot advance time")
    return step


def run_loop(state, stable_time_step, advance, start_time, end_time, max_steps=1000, step0=0):
    """The hot loop of run_serial_case (serial_case_runner.cpp:129-142)."""
    time, step = start_time, step0
    while time < end_time and step < max_steps:
        dt = next_time_step(end_time, time, stable_time_step(state))
        advance(dt, state)
        time += dt
        step += 1
    return step, time


def metrics(step, time, checkpoint_coefficients, mass):
    total, l2 = 0.0, 0.0
    for v in checkpoint_coefficients.tolist():
        total += v
        l2 += v * v
    return dict(step=step, time=time, coefficient_sum=total, coefficient_l2=math.sqrt(l2),
                final_mass=mass)


def close(actual, expected, tol=1e-10):
    """case_regression_test.cpp:233-235"""
    return abs(actual - expected) <= tol * max(1.0, abs(expected))
