"""Seeded synthetic workloads (initial data and exact solutions).

Each workload builds the mesh with ``meshgen``, projects its initial data with
the solver's own L2 projection (the rule the reference's initial state uses:
order max(p, 5) on triangles, 7 Gauss points on lines), and knows its exact
solution where one exists.  No public dataset is involved.
"""
from __future__ import annotations

import math

import numpy as np

from . import meshgen

GAMMA = 1.4


def conserved(rho, u, v, p, gamma=GAMMA):
    """cpp/include/wasl/equations/euler/primitive.hpp:10-17, elementwise."""
    rho, u, v, p = (np.asarray(a, dtype=np.float64) for a in (rho, u, v, p))
    kinetic = 0.5 * rho * (u * u + v * v)
    return np.stack(np.broadcast_arrays(rho, rho * u, rho * v, p / (gamma - 1.0) + kinetic),
                    axis=-1)


# ---- isentropic vortex on a periodic square -------------------------------------

class IsentropicVortex:
    """Shu's isentropic vortex of strength eps advected with (u0, v0) over the
    periodic square [0, L]^2; the exact solution is the translated initial
    field."""

    def __init__(self, strength=5.0, center=(5.0, 5.0), velocity=(1.0, 1.0), length=10.0,
                 gamma=GAMMA):
        self.eps, self.center, self.velocity = strength, center, velocity
        self.length, self.gamma = length, gamma

    def primitive(self, x, y, t=0.0):
        L = self.length
        xc = self.center[0] + self.velocity[0] * t
        yc = self.center[1] + self.velocity[1] * t
        dx = np.mod(x - xc + 0.5 * L, L) - 0.5 * L
        dy = np.mod(y - yc + 0.5 * L, L) - 0.5 * L
        r2 = dx * dx + dy * dy
        g = self.gamma
        bump = np.exp(0.5 * (1.0 - r2))
        du = -self.eps / (2.0 * math.pi) * bump * dy
        dv = self.eps / (2.0 * math.pi) * bump * dx
        temperature = 1.0 - (g - 1.0) * self.eps ** 2 / (8.0 * g * math.pi ** 2) * bump * bump
        rho = temperature ** (1.0 / (g - 1.0))
        return rho, self.velocity[0] + du, self.velocity[1] + dv, rho * temperature

    def conserved(self, x, y, t=0.0):
        return conserved(*self.primitive(x, y, t), gamma=self.gamma)


def vortex_mesh(n=256, seed=2025):
    """n x n quads on [0,10]^2, random diagonals, interior jitter +-0.15h."""
    return meshgen.jittered_box(n, 0.0, 10.0, 0.0, 10.0, jitter=0.15, seed=seed)


def project_initial(solver, field, rule_order=None):
    """Project field(x, y) -> [..., 4] conserved values onto the solver's modes."""
    p = solver.config.polynomial_order
    rule = max(p, 5) if rule_order is None else rule_order
    x, y, _ = solver.quadrature(rule)
    solver.project(rule, field(x, y))


def l1_density_error(solver, exact, rule_order=5):
    """Integral of |rho_h - rho_exact| with the order-5 triangle rule
    (the measure of cpp/tests/dg/euler_triangle_residual_test.cpp:161-183)."""
    x, y, w = solver.quadrature(rule_order)
    rho_h = solver.evaluate(rule_order)[..., 0]
    return float(np.sum(w * np.abs(rho_h - exact(x, y)[..., 0])))


# ---- 1D periodic advection -------------------------------------------------------------

class AdvectedPulse:
    """u0 = sin(2 pi x) + exp(-300 (x - 0.5)^2) on the periodic unit line,
    advected with speed a; the exact solution is the translated initial data."""

    def __init__(self, speed=1.0):
        self.speed = speed

    def value(self, x, t=0.0):
        y = np.mod(np.asarray(x, dtype=np.float64) - self.speed * t, 1.0)
        return np.sin(2.0 * math.pi * y) + np.exp(-300.0 * (y - 0.5) ** 2)


def advection_line_mesh(n=400, seed=2024):
    """n cells on [0,1], interior nodes moved uniformly within +-0.2h."""
    return meshgen.jittered_line(n, 0.0, 1.0, jitter=0.2, seed=seed)


def project_line(solver, field, points=7):
    """Project field(x) -> [..., variables] with the 7-point Gauss rule
    (cpp/src/case/initial_state.cpp:16-29)."""
    x, _, _ = solver.quadrature(points - 1)
    values = np.asarray(field(x), dtype=np.float64)
    if values.ndim == 2:
        values = values[..., None]
    solver.project(points - 1, values)


def l1_line_error(solver, exact, points=7):
    """Integral of |u_h - u_exact| (first variable) with a Gauss rule."""
    x, _, w = solver.quadrature(points - 1)
    u_h = solver.evaluate(points - 1)[..., 0]
    return float(np.sum(w * np.abs(u_h - exact(x))))


# ---- Riemann problems ----------------------------------------------------------------

def random_state(rng):
    """rho in [0.1,1.5], p in [0.02,1.5], |u|,|v| <= 1.2."""
    return (rng.uniform(0.1, 1.5), rng.uniform(-1.2, 1.2), rng.uniform(-1.2, 1.2),
            rng.uniform(0.02, 1.5))


def star_pressure(left, right, nx, ny, gamma=GAMMA):
    """Two-rarefaction estimate of the star pressure of the 1D Riemann problem
    between primitive states (rho, u, v, p) along the normal (nx, ny) (Toro,
    Riemann Solvers and Numerical Methods, eq. 9.32); <= 0 when the exact
    solution contains vacuum (u_R - u_L >= 2 (c_L + c_R) / (gamma - 1))."""
    rl, ul, vl, pl = left
    rr, ur, vr, pr = right
    cl, cr = math.sqrt(gamma * pl / rl), math.sqrt(gamma * pr / rr)
    z = (gamma - 1.0) / (2.0 * gamma)
    numerator = cl + cr - 0.5 * (gamma - 1.0) * ((ur - ul) * nx + (vr - vl) * ny)
    if numerator <= 0.0:
        return 0.0
    return (numerator / (cl / pl ** z + cr / pr ** z)) ** (1.0 / z)


def resolvable(left, right, nx, ny, gamma=GAMMA, fraction=0.1):
    """Whether the interface's star pressure is at least `fraction` of the
    smaller initial pressure: the discontinuous Galerkin method with density
    and pressure floors (the reference's limiter included) cannot follow a
    flow into vacuum, so seeded problems that would open one are redrawn."""
    return star_pressure(left, right, nx, ny, gamma) >= fraction * min(left[3], right[3])


class QuadrantRiemann:
    """Seeded four-quadrant Riemann problem on [0,1]^2 (states redrawn until
    every interface between neighbouring quadrants is resolvable)."""

    def __init__(self, seed=3, gamma=GAMMA):
        rng = np.random.Generator(np.random.PCG64(seed))
        while True:
            prim = [random_state(rng) for _ in range(4)]
            # quadrants 0 (SW), 1 (SE), 2 (NW), 3 (NE)
            if (resolvable(prim[0], prim[1], 1, 0, gamma) and resolvable(prim[2], prim[3], 1, 0, gamma)
                    and resolvable(prim[0], prim[2], 0, 1, gamma)
                    and resolvable(prim[1], prim[3], 0, 1, gamma)):
                break
        self.primitive_states = prim
        self.states = np.array([conserved(*s, gamma=gamma) for s in prim])

    def conserved(self, x, y, t=0.0):
        q = (x >= 0.5).astype(int) + 2 * (y >= 0.5).astype(int)
        return self.states[q]


class PlanarRiemann:
    """Two seeded states split by a line through (cx, cy) at a random angle
    (states redrawn until the interface is resolvable)."""

    def __init__(self, seed=0, gamma=GAMMA):
        rng = np.random.Generator(np.random.PCG64(seed))
        self.gamma = gamma
        self.angle = rng.uniform(0.0, 2.0 * math.pi)
        self.cx, self.cy = rng.uniform(0.3, 0.7, size=2)
        nx, ny = math.cos(self.angle), math.sin(self.angle)
        while True:
            left, right = random_state(rng), random_state(rng)
            if resolvable(left, right, nx, ny, gamma):
                break
        self.left = conserved(*left, gamma=gamma)
        self.right = conserved(*right, gamma=gamma)

    def conserved(self, x, y, t=0.0):
        side = (x - self.cx) * math.cos(self.angle) + (y - self.cy) * math.sin(self.angle) >= 0.0
        return np.where(side[..., None], self.right, self.left)

    def density(self, x, y, t):
        """Exact density at time t > 0 (before any wave reaches the boundary):
        the 1D Riemann solution along the interface normal, whose tangential
        velocity only rides along."""
        nx, ny = math.cos(self.angle), math.sin(self.angle)

        def normal(state):
            rho, mx, my, e = map(float, state)
            u, v = mx / rho, my / rho
            return rho, u * nx + v * ny, (self.gamma - 1.0) * (e - 0.5 * rho * (u * u + v * v))

        exact = ExactRiemann(normal(self.left), normal(self.right), gamma=self.gamma)
        s = ((x - self.cx) * nx + (y - self.cy) * ny) / t
        return exact.sample(s)[0]


class ShockVortex:
    """Stationary Mach 1.1 normal shock at x=0.5 on [0,2]x[0,1]: supersonic
    upstream flow (rho=1, p=1) on the left, the Rankine-Hugoniot state on the
    right, and an isentropic vortex of seeded strength in [0.2, 0.4] (radius
    0.05) centred at (0.25, 0.5) in the upstream flow."""

    def __init__(self, seed=0, mach=1.1, gamma=GAMMA):
        rng = np.random.Generator(np.random.PCG64(seed))
        self.strength = rng.uniform(0.2, 0.4)
        g = gamma
        self.gamma = g
        # upstream (left of the shock, moving right at Mach 1.1)
        rho_u, p_u = 1.0, 1.0
        c_u = math.sqrt(g * p_u / rho_u)
        u_u = mach * c_u
        # stationary normal shock relations
        m2 = mach * mach
        rho_d = rho_u * (g + 1.0) * m2 / ((g - 1.0) * m2 + 2.0)
        p_d = p_u * (2.0 * g * m2 - (g - 1.0)) / (g + 1.0)
        u_d = u_u * rho_u / rho_d
        self.upstream = (rho_u, u_u, 0.0, p_u)
        self.downstream = (rho_d, u_d, 0.0, p_d)

    def primitive(self, x, y):
        rho_u, u_u, _, p_u = self.upstream
        g = self.gamma
        dx, dy = x - 0.25, y - 0.5
        r2 = (dx * dx + dy * dy) / 0.05 ** 2
        bump = np.exp(0.5 * (1.0 - r2))
        eps = self.strength
        c = math.sqrt(g * p_u / rho_u)
        du = -eps * c * bump * dy / 0.05
        dv = eps * c * bump * dx / 0.05
        t_ratio = 1.0 - (g - 1.0) * eps ** 2 / (2.0 * g) * bump * bump
        rho = rho_u * t_ratio ** (1.0 / (g - 1.0))
        p = p_u * t_ratio ** (g / (g - 1.0))
        left = x < 0.5
        rho_d, u_d, _, p_d = self.downstream
        return (np.where(left, rho, rho_d), np.where(left, u_u + du, u_d),
                np.where(left, dv, 0.0), np.where(left, p, p_d))

    def conserved(self, x, y, t=0.0):
        return conserved(*self.primitive(x, y), gamma=self.gamma)


# ---- batched cases ---------------------------------------------------------------------

def batched_riemann_cases(count, seed=4, min_triangles=2_000, max_triangles=128_000,
                          orders=(1, 2, 3)):
    """Independent planar two-state Riemann problems on [0,1]^2: per case a
    triangle count drawn log-uniformly in [min, max] (n x n quads, n =
    round(sqrt(count / 2)), jittered +-0.15h), an order drawn from `orders`,
    and seeded states.  Returns [(node_tags, coordinates, triangles, p,
    problem)]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for c in range(count):
        triangles = math.exp(rng.uniform(math.log(min_triangles), math.log(max_triangles)))
        n = max(2, int(round(math.sqrt(triangles / 2.0))))
        p = int(rng.choice(orders))
        case_seed = int(rng.integers(1 << 31))
        arrays = meshgen.jittered_box(n, 0.0, 1.0, 0.0, 1.0, jitter=0.15, seed=case_seed)
        out.append((*arrays, p, PlanarRiemann(seed=case_seed)))
    return out


def project_batch_case(batch, c, field, p):
    """Project field(x, y) -> [..., 4] onto case c of a Batch (rule max(p, 5))."""
    rule = max(p, 5)
    x, y, _ = batch.quadrature(c, rule)
    batch.project(c, rule, field(x, y))


# ---- exact Riemann solution ------------------------------------------------------------

class ExactRiemann:
    """Exact solution of the 1D Riemann problem for an ideal gas between
    primitive states (rho, u, p) (Toro, Riemann Solvers and Numerical Methods
    for Fluid Dynamics, ch. 4): the star pressure by Newton's method on the
    sum of the two wave functions, started from the primitive-variable
    estimate, then each similarity coordinate sampled across the left wave,
    the contact and the right wave.  Vectorised over samples."""

    def __init__(self, left, right, gamma=GAMMA):
        self.gamma = g = gamma
        self.left, self.right = tuple(map(float, left)), tuple(map(float, right))
        (rl, ul, pl), (rr, ur, pr) = self.left, self.right
        self.cl, self.cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
        if 2.0 * (self.cl + self.cr) / (g - 1.0) <= ur - ul:
            raise ValueError("exact Riemann solution: the states open a vacuum")
        p = max(1e-12, 0.5 * (pl + pr) - 0.125 * (ur - ul) * (rl + rr) * (self.cl + self.cr))
        for _ in range(100):
            fl, dl = self._wave(p, rl, pl, self.cl)
            fr, dr = self._wave(p, rr, pr, self.cr)
            step = (fl + fr + ur - ul) / (dl + dr)
            p_new = max(1e-14, p - step)
            if abs(p_new - p) <= 1e-15 * (p_new + p):
                p = p_new
                break
            p = p_new
        self.p_star = p
        fl, _ = self._wave(p, rl, pl, self.cl)
        fr, _ = self._wave(p, rr, pr, self.cr)
        self.u_star = 0.5 * (ul + ur) + 0.5 * (fr - fl)

    def _wave(self, p, rho, pk, c):
        """The velocity jump across the wave from pressure pk to p, and its
        derivative in p (shock for p > pk, rarefaction otherwise)."""
        g = self.gamma
        if p > pk:
            a, b = 2.0 / ((g + 1.0) * rho), (g - 1.0) / (g + 1.0) * pk
            root = math.sqrt(a / (b + p))
            return (p - pk) * root, root * (1.0 - 0.5 * (p - pk) / (b + p))
        ratio = p / pk
        return (2.0 * c / (g - 1.0) * (ratio ** ((g - 1.0) / (2.0 * g)) - 1.0),
                ratio ** (-(g + 1.0) / (2.0 * g)) / (rho * c))

    def _side(self, s, state, c, sign):
        """Samples on one side of the contact; sign +1 left, -1 right (the
        right side is the left side's mirror image)."""
        g = self.gamma
        rho, u, p = state
        ps, us = self.p_star, self.u_star
        out_rho, out_u, out_p = (np.full_like(s, rho), np.full_like(s, u), np.full_like(s, p))
        ratio = ps / p
        if ps > p:  # shock
            speed = u - sign * c * math.sqrt((g + 1.0) / (2.0 * g) * ratio + (g - 1.0) / (2.0 * g))
            behind = sign * (s - speed) > 0.0
            k = (g - 1.0) / (g + 1.0)
            out_rho = np.where(behind, rho * (ratio + k) / (k * ratio + 1.0), out_rho)
            out_u = np.where(behind, us, out_u)
            out_p = np.where(behind, ps, out_p)
            return out_rho, out_u, out_p
        c_star = c * ratio ** ((g - 1.0) / (2.0 * g))
        head, tail = u - sign * c, us - sign * c_star
        star = sign * (s - tail) >= 0.0
        fan = (sign * (s - head) > 0.0) & ~star
        out_rho = np.where(star, rho * ratio ** (1.0 / g), out_rho)
        out_u = np.where(star, us, out_u)
        out_p = np.where(star, ps, out_p)
        cf = 2.0 / (g + 1.0) * (c + sign * (g - 1.0) / 2.0 * (u - s))
        uf = 2.0 / (g + 1.0) * (sign * c + (g - 1.0) / 2.0 * u + s)
        cf = np.maximum(cf, 0.0)
        out_rho = np.where(fan, rho * (cf / c) ** (2.0 / (g - 1.0)), out_rho)
        out_u = np.where(fan, uf, out_u)
        out_p = np.where(fan, p * (cf / c) ** (2.0 * g / (g - 1.0)), out_p)
        return out_rho, out_u, out_p

    def sample(self, s):
        """(rho, u, p) at similarity coordinates s = (x - x0) / t."""
        s = np.asarray(s, dtype=np.float64)
        left = self._side(s, self.left, self.cl, 1.0)
        right = self._side(s, self.right, self.cr, -1.0)
        on_left = s <= self.u_star
        return tuple(np.where(on_left, a, b) for a, b in zip(left, right))


def sod_density_l1(solver, exact, interface=0.5, time=0.2, samples=400):
    """L1 error of the density cell averages against the exact cell averages
    (each averaged over `samples` evenly spaced points), on a line mesh."""
    ends = solver.vertices().reshape(-1, 2)
    state = solver.get_state().reshape(4, solver.modes, solver.elements)
    average = state[0, 0] / math.sqrt(2.0)
    width = ends[:, 1] - ends[:, 0]
    points = ends[:, :1] + (np.arange(samples) + 0.5)[None, :] / samples * width[:, None]
    exact_average = exact.sample((points - interface) / time)[0].mean(axis=1)
    return float(np.sum(width * np.abs(average - exact_average)))
