"""A mesh split over solver handles reproduces one solver over the whole
mesh, with transmissive and with periodic boundaries.  Both handles live on one GPU in one process and run one after the
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


def run_split(tags, xy, tris, ranks, depth, kw, c, steps, cfl, p, pairs=None, vars_=4):
    """Serial handle against one part handle per rank (run one after the
    other on this GPU, ghost rows exchanged through the host); returns the
    flags the serial run raised."""
    ne, M = len(tris), (p + 1) * (p + 2) // 2
    meshes = [halo.local_mesh(tags, xy, tris, r, ranks, depth, pairs=pairs)
              for r in range(ranks)]
    schedules = [halo.build_halo_schedule(meshes, ranks, ne, r) for r in range(ranks)]
    serial = wasl_b200.Solver(tags, xy, tris, **kw)
    parts = [wasl_b200.Solver(*m.arrays, part_boundary=m.part_boundary, **kw) for m in meshes]
    flagged = 0
    try:
        serial.set_state(c)
        for g, m in zip(parts, meshes):
            halo.check_partitioned_solver(g)
            g.set_state(np.ascontiguousarray(c.reshape(vars_ * M, ne)[:, m.elements]).ravel())
        for _ in range(steps):
            dt = serial.stable_dt(cfl)
            if vars_ == 4:
                speeds, lengths = zip(*(g.cfl_parts() for g in parts))
                assert halo.dt_from_parts(cfl, max(speeds), min(lengths), p) == dt
            serial.step(dt)
            for g in parts:
                g.step(dt)
            states = [g.get_state().reshape(vars_ * M, -1) for g in parts]
            halo.exchange_in_process(states, meshes, schedules)
            for g, st in zip(parts, states):
                g.set_state(np.ascontiguousarray(st).ravel())
            full = serial.get_state().reshape(vars_ * M, ne)
            for st, m in zip(states, meshes):
                assert np.array_equal(st, full[:, m.elements])
            if kw.get("limiting"):
                flagged += int(serial.flags().sum())
    finally:
        serial.close()
        for g in parts:
            g.close()
    return flagged


@pytest.mark.parametrize("precision,limiting,kernel", [
    ("plain", False, 0), ("plain", True, 0),
    ("mixed", False, 11),  # patch kernel, 128 elements x 5 CTAs per SM
    ("mixed", False, 8),   # shared-face tile kernel
    ("mixed", False, 1),   # face-centric kernels
    ("mixed", True, 8)])
@pytest.mark.parametrize("ranks", [2, 3])
def test_periodic_parts_reproduce_one(precision, limiting, kernel, ranks):
    """A periodic mesh split into parts across its seams (part handles built
    on the boundary that halo.local_mesh derives from the whole mesh's
    periodic trace) reproduces one periodic handle bit for bit, for the plain
    path and for the mixed form with each kernel family (both handles run
    the same kernel)."""
    p, cfl = 2, 0.1
    tags, xy, tris = meshgen.jittered_box(18, jitter=0.15, seed=33, ny=14)
    c = seeded_state(len(tris), p, 12, amplitude=0.02 if limiting else 0.005)
    kw = dict(polynomial_order=p, precision=precision, limiting=limiting, boundary="periodic",
              positivity_all=limiting and precision == "mixed")
    if precision == "mixed":
        kw["mixed_kernel"] = kernel
    pairs = halo.periodic_pairs(tags, xy, tris, p)
    flagged = run_split(tags, xy, tris, ranks, halo.halo_depth(limiting), kw, c, 4, cfl, p,
                        pairs)
    assert flagged > 0 or not limiting


def test_periodic_scalar_parts_reproduce_one():
    p = 3
    tags, xy, tris = meshgen.jittered_box(14, jitter=0.15, seed=34)
    rng = np.random.default_rng(1)
    M = (p + 1) * (p + 2) // 2
    c = rng.normal(size=M * len(tris))
    kw = dict(equation="scalar_advection", polynomial_order=p, velocity=(1.0, -0.6),
              boundary="periodic")
    run_split(tags, xy, tris, 2, 3, kw, c, 3, 0.1, p, halo.periodic_pairs(tags, xy, tris, p),
              vars_=1)


def test_part_boundary_is_checked():
    tags, xy, tris = meshgen.jittered_box(8, jitter=0.15, seed=35)
    pairs = halo.periodic_pairs(tags, xy, tris, 2)
    m = halo.local_mesh(tags, xy, tris, 0, 2, 3, pairs=pairs)
    donors, basis = m.part_boundary
    with pytest.raises(wasl_b200.WaslError, match="faces given"):
        wasl_b200.Solver(*m.arrays, polynomial_order=2, part_boundary=(donors[1:], basis[1:]))
    bad = donors.copy()
    bad[np.flatnonzero(bad[:, 0] >= 0)[0], 1] = 10 ** 6
    with pytest.raises(wasl_b200.WaslError, match="donor outside"):
        wasl_b200.Solver(*m.arrays, polynomial_order=2, part_boundary=(bad, basis))
    with pytest.raises(wasl_b200.WaslError, match="must be periodic"):
        wasl_b200.Solver(*m.arrays, polynomial_order=2, boundary="transmissive",
                         part_boundary=m.part_boundary)


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


def device_rows(pointer, rows, columns):
    import torch
    return torch.as_tensor(halo._DeviceRows(pointer, rows, columns), device="cuda")


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_native_halo_moves_the_ghost_rows(precision):
    """The library's halo (wasl_halo_*): pack on each part's stream, its
    device send buffers copied into the peer's receive buffers (the
    transport), unpack; two periodic parts stay bit-identical to the whole
    mesh for four limited steps."""
    import torch
    p, ranks, cfl = 2, 2, 0.1
    tags, xy, tris = meshgen.jittered_box(16, jitter=0.15, seed=36, ny=12)
    ne, M = len(tris), (p + 1) * (p + 2) // 2
    c = seeded_state(ne, p, 13, amplitude=0.02)
    kw = dict(polynomial_order=p, precision=precision, limiting=True, boundary="periodic",
              positivity_all=precision == "mixed")
    if precision == "mixed":
        kw["mixed_kernel"] = 8
    pairs = halo.periodic_pairs(tags, xy, tris, p)
    meshes = [halo.local_mesh(tags, xy, tris, r, ranks, halo.halo_depth(True), pairs=pairs)
              for r in range(ranks)]
    schedules = [halo.build_halo_schedule(meshes, ranks, ne, r) for r in range(ranks)]
    serial = wasl_b200.Solver(tags, xy, tris, **kw)
    parts = [wasl_b200.Solver(*m.arrays, part_boundary=m.part_boundary, **kw) for m in meshes]
    halos = [halo.NativeHalo(g, m, s) for g, m, s in zip(parts, meshes, schedules)]
    try:
        serial.set_state(c)
        for g, m in zip(parts, meshes):
            g.set_state(np.ascontiguousarray(c.reshape(4 * M, ne)[:, m.elements]).ravel())
        assert halos[0].peers == [1] and halos[1].peers == [0]
        for _ in range(4):
            dt = serial.stable_dt(cfl)
            serial.step(dt)
            for g, h in zip(parts, halos):
                g.step(dt)
                h.pack()
                g.sync()
            for r in range(ranks):
                send, _, ns, _, rows = halos[r].buffers(0)
                _, recv, _, nr, _ = halos[1 - r].buffers(0)
                assert ns == nr
                device_rows(recv, rows, nr).copy_(device_rows(send, rows, ns))
            torch.cuda.synchronize()
            for h in halos:
                h.unpack()
            full = serial.get_state().reshape(4 * M, ne)
            for g, m in zip(parts, meshes):
                assert np.array_equal(g.get_state().reshape(4 * M, -1), full[:, m.elements])
    finally:
        for h in halos:
            h.close()
        serial.close()
        for g in parts:
            g.close()


def test_nccl_transport_on_one_rank():
    """The NCCL transport bound at run time: a one-rank communicator, the
    CFL parts all-reduced (the handle's own dt), and an exchange with no
    peers (pack, an empty group, unpack) that leaves the state unchanged."""
    tags, xy, tris = meshgen.jittered_box(10, jitter=0.15, seed=37)
    c = seeded_state(len(tris), 2, 14, amplitude=0.005)
    comm = halo.nccl_communicator(1, halo.nccl_unique_id(), 0, 0)
    try:
        with wasl_b200.Solver(tags, xy, tris, polynomial_order=2, boundary="periodic") as g:
            g.set_state(c)
            assert halo.stable_dt_nccl(g, comm, 0.1) == g.stable_dt(0.1)
            pairs = halo.periodic_pairs(tags, xy, tris, 2)
            m = halo.local_mesh(tags, xy, tris, 0, 1, 3, pairs=pairs)
            h = halo.NativeHalo(g, m, halo.build_halo_schedule([m], 1, len(tris), 0))
            assert h.peers == []
            h.exchange_nccl(comm)
            g.sync()
            assert np.array_equal(g.get_state(), c)
            h.close()
    finally:
        halo.nccl_destroy(comm)
