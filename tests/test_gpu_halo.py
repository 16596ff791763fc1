"""A mesh split over two solver handles reproduces one solver over the whole
mesh.  Both handles live on one GPU in one process and run one after the
other (their kernels never wait on each other); the ghost rows move through
the host between steps (wasl_b200.halo.exchange_in_process) and the time step
is reduced from each handle's wave speed and element length, as the ranks of
a multi-GPU run reduce them."""
import numpy as np
import pytest

import wasl_b200
from golden.make_golden import seeded_state
from wasl_b200 import halo, meshgen

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,limiting", [("plain", False), ("plain", True),
                                                ("mixed", False), ("mixed", True)])
def test_two_handles_reproduce_one(precision, limiting):
    p, ranks, cfl = 2, 2, 0.1
    tags, xy, tris = meshgen.jittered_box(16, jitter=0.15, seed=31)
    ne, M = len(tris), (p + 1) * (p + 2) // 2
    c = seeded_state(ne, p, 8, amplitude=0.02 if limiting else 0.005)
    kw = dict(polynomial_order=p, precision=precision, limiting=limiting,
              boundary="transmissive", positivity_all=limiting and precision == "mixed")
    if precision == "mixed":
        kw["mixed_kernel"] = 8  # one kernel for every handle (all tile shapes agree bit for bit)
    depth = halo.halo_depth(limiting)
    meshes = [halo.local_mesh(tags, xy, tris, r, ranks, depth) for r in range(ranks)]
    schedules = [halo.build_halo_schedule(meshes, ranks, ne, r) for r in range(ranks)]
    serial = wasl_b200.Solver(tags, xy, tris, **kw)
    parts = [wasl_b200.Solver(*m.arrays, **kw) for m in meshes]
    try:
        serial.set_state(c)
        for g, m in zip(parts, meshes):
            g.set_state(np.ascontiguousarray(c.reshape(4 * M, ne)[:, m.elements]).ravel())
        flagged = 0
        for _ in range(4):
            dt = serial.stable_dt(cfl)
            speeds, lengths = zip(*(g.cfl_parts() for g in parts))
            assert halo.dt_from_parts(cfl, max(speeds), min(lengths), p) == dt
            serial.step(dt)
            for g in parts:
                g.step(dt)
            states = [g.get_state().reshape(4 * M, -1) for g in parts]
            halo.exchange_in_process(states, meshes, schedules)
            for g, s in zip(parts, states):
                g.set_state(np.ascontiguousarray(s).ravel())
            full = serial.get_state().reshape(4 * M, ne)
            for s, m in zip(states, meshes):
                assert np.array_equal(s, full[:, m.elements])
            if limiting:
                flagged += int(serial.flags().sum())
        assert flagged > 0 or not limiting
    finally:
        serial.close()
        for g in parts:
            g.close()


def test_device_state_view_shares_the_handle_memory():
    """halo.device_state sees the handle's state in place: what it reads is
    get_state, and what the exchange writes through it the next step uses."""
    import torch
    tags, xy, tris = meshgen.jittered_box(6, jitter=0.15, seed=3)
    with wasl_b200.Solver(tags, xy, tris, polynomial_order=2, boundary="transmissive") as g:
        c = seeded_state(g.elements, 2, 4, amplitude=0.005)
        g.set_state(c)
        g.sync()
        view = halo.device_state(g)
        assert view.shape == (4 * g.modes, g.elements)
        assert np.array_equal(view.cpu().numpy().ravel(), c)
        cols = torch.tensor([0, 5, 9], device="cuda")
        view.index_copy_(1, cols, view.index_select(1, cols) * 1.0 + 0.25)
        torch.cuda.current_stream().synchronize()
        expect = c.reshape(4 * g.modes, -1).copy()
        expect[:, [0, 5, 9]] += 0.25
        assert np.array_equal(g.get_state().reshape(4 * g.modes, -1), expect)
