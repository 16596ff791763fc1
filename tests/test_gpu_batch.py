"""The batched form: independent cases of uneven size and order advanced
together (per-order launches of the tile kernel over a work list of element
tiles, per-case CFL time steps, the step replayed from a CUDA graph).  Each
case must evolve bit for bit as the same case run alone through the
single-case mixed solver with the same kernel shape and volume rule."""
import numpy as np
import pytest

import wasl_b200
from wasl_b200 import cases, meshgen

pytestmark = pytest.mark.gpu

# Launch shapes of the tile kernels (see wasl_gpu_tuning): the batch tunes
# over the tile kernels' shapes 0-7 and the persistent tile kernel's 14-15.
TILE_SHAPES = 16
BATCH_SHAPES = list(range(8)) + [14, 15]


def small_cases(seed, count=5):
    out = []
    rng = np.random.Generator(np.random.PCG64(seed))
    for c in range(count):
        n = int(rng.integers(4, 15))
        p = int(rng.integers(1, 4))
        arrays = meshgen.jittered_box(n, 0.0, 1.0, 0.0, 1.0, jitter=0.15, seed=seed * 100 + c)
        out.append((*arrays, p, cases.PlanarRiemann(seed=seed * 100 + c)))
    return out


def smooth_field(x, y):
    rho = 1.0 + 0.2 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y)
    return cases.conserved(rho, 0.3 + 0.1 * np.cos(2 * np.pi * y), -0.2 + 0 * x, 1.0 + 0.1 * rho)


def milder(problem):
    """The Riemann data pulled halfway to the mean of its two states (still
    discontinuous, so the limiter acts; convex mixtures stay physical)."""
    mean = 0.5 * (problem.left + problem.right)
    return lambda x, y: 0.5 * (problem.conserved(x, y) + mean)


@pytest.mark.parametrize("limiting", [False, True])
@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("shape", [0, 3, 4, 6, 14, 15])
def test_batch_matches_single_case_solver(limiting, use_graph, shape):
    """Bit-identical states per case, or, if a case fails alone (a positivity
    floor), the same failure from the batch."""
    specs = small_cases(7 + shape)
    field = (lambda pr: milder(pr)) if limiting else (lambda pr: smooth_field)
    single, failure = [], None
    for s in specs:
        with wasl_b200.Solver(*s[:3], polynomial_order=s[3], precision="mixed",
                              volume_rule_order=s[3], mixed_kernel=2 + shape,
                              boundary="transmissive", limiting=limiting) as g:
            cases.project_initial(g, field(s[4]))
            try:
                g.advance(0.1, 4)
                single.append(g.get_state())
            except wasl_b200.WaslError as err:
                failure = failure or err.status
                single.append(None)
    with wasl_b200.Batch([s[:4] for s in specs], limiting=limiting, tile_shape=1 + shape,
                         use_graph=use_graph) as b:
        for c, s in enumerate(specs):
            cases.project_batch_case(b, c, field(s[4]), s[3])
        if failure is not None:
            with pytest.raises(wasl_b200.WaslError) as err:
                b.advance(0.1, 4)
            assert err.value.status == failure
            return
        b.advance(0.1, 4)
        time, dt = b.times()
        per_step, graph, total = b.launches()
        assert graph == use_graph and per_step > 0 and total == 4 * per_step
        for c, s in enumerate(specs):
            assert np.array_equal(b.get_state(c), single[c]), f"case {c} (P{s[3]}) differs"
            assert time[c] > 0 and dt[c] > 0


def test_periodic_batch_matches_single_case_solver():
    specs = small_cases(3, count=4)
    with wasl_b200.Batch([s[:4] for s in specs], boundary="periodic", tile_shape=1) as b:
        for c, s in enumerate(specs):
            cases.project_batch_case(b, c, smooth_field, s[3])
        b.advance(0.15, 5)
        got = [b.get_state(c) for c in range(len(specs))]
    for c, s in enumerate(specs):
        with wasl_b200.Solver(*s[:3], polynomial_order=s[3], precision="mixed",
                              volume_rule_order=s[3], mixed_kernel=2) as g:
            cases.project_initial(g, smooth_field)
            g.advance(0.15, 5)
            assert np.array_equal(got[c], g.get_state()), f"case {c} differs"


def test_batch_autotunes_each_order_and_conserves():
    specs = small_cases(11, count=6)
    with wasl_b200.Batch([s[:4] for s in specs], boundary="periodic") as b:
        for c, s in enumerate(specs):
            cases.project_batch_case(b, c, smooth_field, s[3])
        masses0 = [b.get_state(c).reshape(4, -1)[0] for c in range(len(specs))]
        b.advance(0.15, 10)
        for p in set(s[3] for s in specs):
            choice, ms = b.tuning(p)
            assert len(ms) == TILE_SHAPES and choice in BATCH_SHAPES
            assert all(ms[k] > 0 for k in BATCH_SHAPES)
            assert ms[choice] == min(ms[k] for k in BATCH_SHAPES)
        for c, s in enumerate(specs):
            ne, nm = b.case_size(c)
            state = b.get_state(c).reshape(4, nm, ne)
            x, y, w = b.quadrature(c, 1)
            area = w.sum(axis=1)  # |det J| x 2 per element (reference triangle area 2)
            before = masses0[c].reshape(nm, ne)[0]
            assert abs(np.sum(area * state[0, 0]) - np.sum(area * before)) <= 1e-12 * np.sum(
                area * before)


@pytest.mark.parametrize("limiting", [False, True])
def test_failed_case_is_frozen_and_the_rest_go_on(limiting):
    """A case with a non-physical cell average (made on the host) is frozen
    and reported; the other cases advance exactly as in a batch without it."""
    specs = small_cases(5, count=3)
    states = {}
    for bad in (True, False):
        with wasl_b200.Batch([s[:4] for s in specs], limiting=limiting, tile_shape=1) as b:
            for c, s in enumerate(specs):
                cases.project_batch_case(b, c, smooth_field, s[3])
            if bad:
                ne, nm = b.case_size(1)
                state = b.get_state(1).reshape(4, nm, ne)
                state[0, 0, ne // 2] = -0.5  # a negative cell-average density
                b.set_state(1, state)
            b.advance(0.1, 3)
            status = b.status()
            time, _ = b.times()
            states[bad] = [b.get_state(c) for c in (0, 2)]
            if bad:
                assert status.tolist() == [0, 1, 0]
                assert time[1] == 0.0 and time[0] > 0 and time[2] > 0
            else:
                assert not status.any()
    for a, b_ in zip(states[True], states[False]):
        assert np.array_equal(a, b_)


def test_bad_arguments_rejected():
    specs = small_cases(6, count=2)
    with pytest.raises(wasl_b200.WaslError, match="polynomial order"):
        wasl_b200.Batch([(*specs[0][:3], 4)])
    with wasl_b200.Batch([s[:4] for s in specs]) as b:
        with pytest.raises(wasl_b200.WaslError, match="out of range"):
            b.get_state(5)


def test_batch_limit_matches_single_case_limit():
    """wasl_batch_limit applies the same stage limiter as wasl_gpu_limit."""
    specs = small_cases(13, count=4)
    with wasl_b200.Batch([s[:4] for s in specs], limiting=True) as b:
        for c, s in enumerate(specs):
            cases.project_batch_case(b, c, s[4].conserved, s[3])
        b.limit()
        got = [b.get_state(c) for c in range(len(specs))]
    for c, s in enumerate(specs):
        with wasl_b200.Solver(*s[:3], polynomial_order=s[3], precision="mixed",
                              volume_rule_order=s[3], boundary="transmissive", limiting=True) as g:
            cases.project_initial(g, s[4].conserved)
            g.limit()
            assert np.array_equal(got[c], g.get_state()), f"case {c} differs"


def test_batched_riemann_runs_with_always_on_positivity():
    """The batched workload's configuration (limiter on, positivity on every
    element, initial limiting) on a few small seeded cases: 30 steps, every
    case advances and stays physical."""
    specs = cases.batched_riemann_cases(6, seed=21, min_triangles=200, max_triangles=3000)
    with wasl_b200.Batch([s[:4] for s in specs], limiting=True, positivity_all=True) as b:
        for c, s in enumerate(specs):
            cases.project_batch_case(b, c, s[4].conserved, s[3])
        b.limit()
        b.advance(0.1, 30)
        time, dt = b.times()
        assert np.all(time > 0) and np.all(dt > 0)
        for c in range(len(specs)):
            ne, nm = b.case_size(c)
            assert np.all(b.get_state(c).reshape(4, nm, ne)[0, 0] > 0)
