"""Partition, ghost region and halo exchange (wasl_b200.halo), on the CPU.

The reference checks its distributed path by splitting a mesh over ranks in
one process and requiring the serial result for every owned element
(cpp/tests/communication/halo_exchange_test.cpp:1-12); the same check runs
here on the oracle's full SSP-RK3 step, with and without the limiter, and the
torch.distributed transport is exercised by two gloo ranks."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from golden.make_golden import seeded_state
from wasl_b200 import halo, meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GAMMA = 1.4


def test_partition_is_the_reference_block_rule():
    owners = halo.element_owners(10, 3)
    assert owners.tolist() == [0, 0, 0, 0, 1, 1, 1, 2, 2, 2]
    for ne, ranks in [(7, 7), (1000, 3), (131072, 8)]:
        o = halo.element_owners(ne, ranks)
        assert np.all(np.diff(o) >= 0) and set(o.tolist()) == set(range(ranks))
        assert np.array_equal(o, (np.arange(ne) * ranks // ne))
    with pytest.raises(ValueError):
        halo.element_owners(10, 0)


def test_face_neighbors_are_symmetric():
    tags, xy, tris = meshgen.jittered_box(9, jitter=0.15, seed=1, ny=7)
    nbr = halo.face_neighbors(tris)
    assert (nbr < 0).sum() == 2 * (9 + 7)  # boundary edges of a 9 x 7 box
    for e, row in enumerate(nbr):
        for n in row[row >= 0]:
            assert e in nbr[n]


def test_first_ghost_layer_is_the_reference_ghost_set():
    """Depth 1: every off-rank element that shares a face with an owned one
    (rank_ghost_elements); deeper layers grow one face step at a time."""
    tags, xy, tris = meshgen.jittered_box(10, jitter=0.15, seed=2)
    nbr = halo.face_neighbors(tris)
    owners = halo.element_owners(len(tris), 3)
    for rank in range(3):
        owned = owners == rank
        expect = sorted({int(n) for e in np.nonzero(owned)[0] for n in nbr[e]
                         if n >= 0 and owners[n] != rank})
        layers = halo.ghost_layers(nbr, owned, 3)
        assert layers[0].tolist() == expect
        reach = owned.copy()
        for layer in layers:
            assert not np.any(reach[layer])
            assert all(np.any(reach[nbr[g][nbr[g] >= 0]]) for g in layer)
            reach[layer] = True


def test_schedule_is_symmetric_and_sorted():
    tags, xy, tris = meshgen.jittered_box(12, jitter=0.15, seed=3)
    ranks, depth = 4, 3
    meshes = [halo.local_mesh(tags, xy, tris, r, ranks, depth) for r in range(ranks)]
    schedules = [halo.build_halo_schedule(meshes, ranks, len(tris), r) for r in range(ranks)]
    for r, s in enumerate(schedules):
        assert [p for p, _ in s.sends] == sorted(p for p, _ in s.sends)
        for peer, send in s.sends:
            assert np.all(np.diff(send) > 0)
            recv = dict(schedules[peer].recvs)[r]
            assert np.array_equal(send, recv)
        ghosts = meshes[r].elements[~meshes[r].owned]
        assert np.array_equal(np.sort(np.concatenate([g for _, g in s.recvs])), ghosts)


@pytest.mark.parametrize("p", [1, 2])
@pytest.mark.parametrize("limiting", [False, True])
@pytest.mark.parametrize("ranks", [2, 3])
def test_split_reproduces_the_serial_step(oracle, p, limiting, ranks):
    """Each rank steps its owned elements and ghost layers with the oracle's
    SSP-RK3 step (transmissive boundaries), one in-process exchange per step:
    every owned element equals the serial run bit for bit."""
    tags, xy, tris = meshgen.jittered_box(14, jitter=0.15, seed=20 + p)
    ne = len(tris)
    serial = oracle.tri_mesh(tags, xy, tris)
    c = seeded_state(ne, p, 5 + p, amplitude=0.02 if limiting else 0.005)
    M = (p + 1) * (p + 2) // 2
    depth = halo.halo_depth(limiting)
    meshes = [halo.local_mesh(tags, xy, tris, r, ranks, depth) for r in range(ranks)]
    schedules = [halo.build_halo_schedule(meshes, ranks, ne, r) for r in range(ranks)]
    locals_ = [oracle.tri_mesh(*m.arrays) for m in meshes]
    stencils = [lm.stencil(p) if limiting else None for lm in locals_]
    st_serial = serial.stencil(p) if limiting else None
    states = [np.ascontiguousarray(c.reshape(4 * M, ne)[:, m.elements]) for m in meshes]
    flagged = 0
    for _ in range(4):
        dt = serial.cfl(GAMMA, c, p, 0.1)
        flags = serial.euler_step(GAMMA, p, dt, c, boundary="transmissive", stencil=st_serial,
                                  return_flags=True)
        flagged += int(flags.sum())
        for r, m in enumerate(meshes):
            u = states[r].ravel()
            lf = locals_[r].euler_step(GAMMA, p, dt, u, boundary="transmissive",
                                       stencil=stencils[r], return_flags=True)
            states[r] = u.reshape(4 * M, -1)
            assert np.array_equal(lf[:, m.owned], flags[:, m.elements[m.owned]])
        halo.exchange_in_process(states, meshes, schedules)
        full = c.reshape(4 * M, ne)
        for r, m in enumerate(meshes):
            assert np.array_equal(states[r], full[:, m.elements]), f"rank {r}"
    assert flagged > 0 or not limiting


@pytest.mark.parametrize("p, pressure, width", [(1, 1.0, 0.0), (2, 10.0, 0.02)])
def test_split_strong_shock_across_the_cut(oracle, p, pressure, width):
    """A planar shock on the two-rank cut (density ratio 8; pressure ratio 10
    with a sharp jump at P1, 100 with the jump smoothed over a third of a cell
    at P2: the reference's algorithm goes non-finite on the projection of
    stronger or sharper jumps, serial or split), limiter on: the ghost layers
    that the cut spoils stay physical (no rank's step raises) and every owned
    element equals the serial run bit for bit while the shock crosses from one
    rank into the other."""
    tags, xy, tris = meshgen.jittered_box(16, jitter=0.15, seed=40 + p)
    ne, ranks = len(tris), 2
    serial = oracle.tri_mesh(tags, xy, tris)
    rule = max(p, 5)
    xs, ys = serial.rule_points(rule)
    cut_y = float(ys[: ne // 2].mean(axis=1).max())  # rank 0 holds the first half

    def state(rho, p_):
        return np.array([rho, 0.0, 0.0, p_ / (GAMMA - 1.0)])

    below, above = state(1.0, pressure), state(0.125, 0.1)
    if width > 0.0:
        vals = below + (above - below) * (0.5 * (1.0 + np.tanh((ys - cut_y) / width)))[..., None]
    else:
        vals = np.where((ys < cut_y)[..., None], below, above)
    c = serial.project(p, rule, vals)
    M = (p + 1) * (p + 2) // 2
    depth = halo.halo_depth(True)
    meshes = [halo.local_mesh(tags, xy, tris, r, ranks, depth) for r in range(ranks)]
    schedules = [halo.build_halo_schedule(meshes, ranks, ne, r) for r in range(ranks)]
    locals_ = [oracle.tri_mesh(*m.arrays) for m in meshes]
    stencils = [lm.stencil(p) for lm in locals_]
    st_serial = serial.stencil(p)
    states = [np.ascontiguousarray(c.reshape(4 * M, ne)[:, m.elements]) for m in meshes]
    start = c.reshape(4 * M, ne)[0].copy()
    flagged = 0
    for _ in range(8):
        dt = serial.cfl(GAMMA, c, p, 0.1)
        flags = serial.euler_step(GAMMA, p, dt, c, boundary="transmissive", stencil=st_serial,
                                  return_flags=True)
        flagged += int(flags.sum())
        for r, m in enumerate(meshes):
            u = states[r].ravel()
            locals_[r].euler_step(GAMMA, p, dt, u, boundary="transmissive", stencil=stencils[r])
            states[r] = u.reshape(4 * M, -1)
        halo.exchange_in_process(states, meshes, schedules)
        full = c.reshape(4 * M, ne)
        assert np.all(np.isfinite(full))
        for r, m in enumerate(meshes):
            assert np.array_equal(states[r], full[:, m.elements]), f"rank {r}"
    assert flagged > 0
    # the shock moved into rank 1's elements
    rank1 = meshes[1].elements[meshes[1].owned]
    assert np.count_nonzero(np.abs(c.reshape(4 * M, ne)[0, rank1] - start[rank1])
                            > 0.02 * start[rank1]) >= 8


def dense_part_trace(oracle, om, part, p):
    """A part's boundary (LocalMesh.part_boundary) as the oracle's per-face
    periodic trace: owner faces (donor -1) take the face's own element and its
    basis at its edge points; the stencil's donors keep -1 there."""
    Q, M = p + 1, (p + 1) * (p + 2) // 2
    donors = np.full(om.nf * Q, -1, dtype=np.int32)
    stencil_donors = donors.copy()
    basis = np.zeros(om.nf * Q * M)
    faces = np.flatnonzero(om.face_right < 0)
    part_donors, part_basis = part
    assert len(faces) == len(part_donors)
    xi, eta = oracle.tri_edge_rules(p)[:2]
    for b, f in enumerate(faces):
        rows = slice(f * Q, (f + 1) * Q)
        if part_donors[b, 0] < 0:
            le = om.face_left_edge[f]
            donors[rows] = om.face_left[f]
            for q in range(Q):
                basis[(f * Q + q) * M:(f * Q + q + 1) * M] = oracle.dubiner(
                    xi[le * Q + q], eta[le * Q + q], p)
        else:
            donors[rows] = stencil_donors[rows] = part_donors[b]
            basis[f * Q * M:(f + 1) * Q * M] = part_basis[b].ravel()
    return donors, basis, stencil_donors


@pytest.mark.parametrize("p", [1, 2])
@pytest.mark.parametrize("limiting", [False, True])
@pytest.mark.parametrize("ranks", [2, 3])
def test_periodic_split_reproduces_the_serial_step(oracle, p, limiting, ranks):
    """A periodic mesh split over ranks: ghost layers across the periodic
    seams and each part's boundary from the whole mesh's periodic trace
    (halo.periodic_pairs, from the library's host setup); every rank steps its
    part with the oracle's SSP-RK3 step on that boundary, one in-process
    exchange per step, and every owned element equals the serial periodic run
    bit for bit."""
    tags, xy, tris = meshgen.jittered_box(12, jitter=0.15, seed=40 + p, ny=10)
    ne = len(tris)
    serial = oracle.tri_mesh(tags, xy, tris)
    gd, gb = serial.periodic_trace(p)
    st_serial = serial.stencil(p, gd) if limiting else None
    c = seeded_state(ne, p, 9 + p, amplitude=0.02 if limiting else 0.005)
    M = (p + 1) * (p + 2) // 2
    pairs = halo.periodic_pairs(tags, xy, tris, p)
    depth = halo.halo_depth(limiting)
    meshes = [halo.local_mesh(tags, xy, tris, r, ranks, depth, pairs=pairs)
              for r in range(ranks)]
    schedules = [halo.build_halo_schedule(meshes, ranks, ne, r) for r in range(ranks)]
    locals_ = [oracle.tri_mesh(*m.arrays) for m in meshes]
    traces = [dense_part_trace(oracle, lm, m.part_boundary, p)
              for lm, m in zip(locals_, meshes)]
    stencils = [lm.stencil(p, t[2]) if limiting else None for lm, t in zip(locals_, traces)]
    states = [np.ascontiguousarray(c.reshape(4 * M, ne)[:, m.elements]) for m in meshes]
    assert any(np.any(m.part_boundary[0][:, 0] >= 0) for m in meshes)  # seams inside parts
    for _ in range(4):
        dt = serial.cfl(GAMMA, c, p, 0.1)
        flags = serial.euler_step(GAMMA, p, dt, c, donors=gd, basis=gb, stencil=st_serial,
                                  return_flags=True)
        for r, m in enumerate(meshes):
            u = states[r].ravel()
            lf = locals_[r].euler_step(GAMMA, p, dt, u, donors=traces[r][0],
                                       basis=traces[r][1], stencil=stencils[r],
                                       return_flags=True)
            states[r] = u.reshape(4 * M, -1)
            assert np.array_equal(lf[:, m.owned], flags[:, m.elements[m.owned]])
        halo.exchange_in_process(states, meshes, schedules)
        full = c.reshape(4 * M, ne)
        for r, m in enumerate(meshes):
            assert np.array_equal(states[r], full[:, m.elements]), f"rank {r}"


def test_periodic_pairs_are_the_oracle_trace(oracle):
    tags, xy, tris = meshgen.jittered_box(9, jitter=0.15, seed=5, ny=6)
    om = oracle.tri_mesh(tags, xy, tris)
    for p in (0, 1, 2, 3):
        pairs = halo.periodic_pairs(tags, xy, tris, p)
        Q, M = p + 1, (p + 1) * (p + 2) // 2
        donors, basis = om.periodic_trace(p)
        faces = np.flatnonzero(om.face_right < 0)
        assert np.array_equal(pairs.element, om.face_left[faces])
        assert np.array_equal(pairs.edge, om.face_left_edge[faces])
        assert np.array_equal(pairs.donors, donors.reshape(om.nf, Q)[faces])
        assert np.array_equal(pairs.basis, basis.reshape(om.nf, Q, M)[faces])


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _Parts:
    """Stands in for a solver's cfl_parts on one rank."""

    def __init__(self, speed, length):
        self.parts = (speed, length)

    def cfl_parts(self):
        return self.parts


def rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    from wasl_b200 import halo, meshgen
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    tags, xy, tris = meshgen.jittered_box(10, jitter=0.15, seed=4)
    ne, rows = len(tris), 6
    meshes = [halo.local_mesh(tags, xy, tris, r, world, 3) for r in range(world)]
    sched = halo.build_halo_schedule(meshes, world, ne, rank)
    m = meshes[rank]
    coded = np.arange(rows)[:, None] * 1e6 + m.elements[None, :].astype(np.float64)
    state = torch.tensor(np.where(m.owned[None, :], coded, np.nan))
    halo.HaloExchange(m, sched, rows).exchange(state)
    ok = bool(np.array_equal(state.numpy(), coded))
    dt = halo.global_dt(_Parts([2.0, 3.0][rank], [0.5, 0.25][rank]), 0.1, 2)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, ok, dt))


def test_two_gloo_ranks_exchange_ghost_rows():
    """Every ghost column holds its owner's values after one exchange, and
    the reduced time step uses the largest speed and the smallest length."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, out)) for r in range(2)]
    for proc in procs:
        proc.start()
    results = {r: (ok, dt) for r, ok, dt in (out.get(timeout=120) for _ in procs)}
    for proc in procs:
        proc.join(timeout=60)
        assert proc.exitcode == 0
    assert results[0][0] and results[1][0]
    assert results[0][1] == results[1][1] == halo.dt_from_parts(0.1, 3.0, 0.25, 2)


def test_partitioned_runs_refuse_periodic_handles_without_a_part_boundary():
    """A rank's periodic handle built by its own donor search would pair its
    cut faces across the period; the partitioned step refuses it up front,
    and accepts a handle built on its part's boundary."""
    class Config:
        boundary_left = 0  # periodic

    class Handle:
        config = Config()
        part = False

    with pytest.raises(ValueError, match="periodic"):
        halo.check_partitioned_solver(Handle())
    Handle.part = True
    halo.check_partitioned_solver(Handle())
    Handle.part = False
    Handle.config.boundary_left = 3  # transmissive
    halo.check_partitioned_solver(Handle())
