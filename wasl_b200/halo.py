"""Element partition, ghost region and halo exchange for a run over several
ranks (one process and one GPU each).

The pieces follow the reference's partition and communication layer:

* ownership is the contiguous block partition rank(e) = floor(e R / N)
  (cpp/include/wasl/mesh/partition/partition.hpp:7-13 and :37);
* a rank imports the off-rank elements next to its owned ones
  (rank_ghost_elements, cpp/src/mesh/partition/partition.cpp:48-77), here
  `depth` face-adjacent layers deep;
* the halo schedule lists, per peer rank and in ascending order, the owned
  elements a peer imports (sends) and the ghosts imported from it (recvs)
  (cpp/include/wasl/communication/halo_schedule.hpp:17-42,
  cpp/src/communication/halo_schedule.cpp:37-61);
* `exchange_in_process` is the transport-free exchange the reference checks
  its MPI transport against (cpp/src/communication/in_process_halo_exchange.cpp:8-37);
  `HaloExchange` moves the same rows over torch.distributed (NCCL between
  GPUs, gloo on CPU) in one batch of point-to-point transfers.

One difference in the schedule: the reference exchanges one ghost layer
before every residual evaluation.  Here a rank holds its owned elements and
`depth` ghost layers as one mesh (in ascending global order, so every face
keeps its orientation and every element its slot order) and advances all of
them through a whole SSP-RK3 step, exchanging once per step.  The ghosts'
outermost faces lead nowhere (they take the transmissive exterior), so each
stage spoils one more layer from the outside in, and the limiter, which reads
the neighbours' unlimited stage values, one more: `halo_depth(limiting)` is 3
without the limiter and 6 with it, and the owned elements come out of every
step bit-identical to a run over the whole mesh.  The time step is reduced
over ranks from each rank's largest wave speed and smallest element length
(`global_dt`), which gives the whole-mesh dt bit for bit.

Periodic domains are partitioned through the whole mesh's periodic trace
(`periodic_pairs`): the ghost layers grow across the periodic seams as well,
and each rank's handle is built with its boundary given explicitly
(`LocalMesh.part_boundary`, wasl_gpu_create_part): a periodic face whose
donors are on the rank keeps its donors and basis from the whole mesh's
trace, and every other face of the part's boundary (where the ghost region
ends) takes its own element's trace.  A rank's own periodic donor search
would instead pair those cut faces across the period.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def halo_depth(limiting: bool) -> int:
    """Ghost layers that keep the owned elements exact through one step."""
    return 6 if limiting else 3


def element_owners(element_count: int, ranks: int) -> np.ndarray:
    """rank(e) = floor(e * ranks / element_count), a contiguous block per rank."""
    if ranks < 1:
        raise ValueError("partition: rank count must be at least 1")
    e = np.arange(element_count, dtype=np.int64)
    return (e * ranks // max(element_count, 1)).astype(np.int32)


def face_neighbors(element_nodes) -> np.ndarray:
    """[elements][3] index of the element across each edge (-1 on the
    boundary), edges matched by their node tags."""
    tris = np.asarray(element_nodes, dtype=np.int64)
    ne = tris.shape[0]
    a = tris[:, [0, 1, 2]].ravel()
    b = tris[:, [1, 2, 0]].ravel()
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    owner = np.repeat(np.arange(ne, dtype=np.int64), 3)
    slot = np.tile(np.arange(3), ne)
    order = np.lexsort((hi, lo))
    lo, hi, owner, slot = lo[order], hi[order], owner[order], slot[order]
    same = (lo[1:] == lo[:-1]) & (hi[1:] == hi[:-1])
    if np.any(same[1:] & same[:-1]):
        raise ValueError("triangle mesh: an edge is shared by more than two elements")
    nbr = np.full((ne, 3), -1, dtype=np.int64)
    i = np.nonzero(same)[0]
    nbr[owner[i], slot[i]] = owner[i + 1]
    nbr[owner[i + 1], slot[i + 1]] = owner[i]
    return nbr


@dataclass
class PeriodicPairs:
    """The whole mesh's periodic trace: boundary face b (ascending face
    order) lies on edge `edge[b]` of element `element[b]` (local edges of the
    counter-clockwise normalized element), and its edge points' periodic
    images lie in donors[b][q], whose basis there is basis[b][q][mode]."""
    element: np.ndarray
    edge: np.ndarray
    donors: np.ndarray
    basis: np.ndarray


def periodic_pairs(node_tags, node_coordinates, element_nodes,
                   polynomial_order: int) -> PeriodicPairs:
    """The periodic trace of the whole mesh, from the library's host setup."""
    from . import mesh_periodic_trace
    pairs = PeriodicPairs(*mesh_periodic_trace(node_tags, node_coordinates, element_nodes,
                                               polynomial_order))
    if np.any(pairs.donors != pairs.donors[:, :1]):
        raise ValueError("partition: a periodic face's points have different donors"
                         " (non-conforming periodic faces)")
    return pairs


def normalized_edge(node_tags, node_coordinates, element_nodes) -> np.ndarray:
    """[elements][3]: the caller's local edge (nodes k, k+1) that is the
    normalized element's edge j.  The library turns clockwise triangles
    counter-clockwise by swapping their second and third nodes, which maps
    edge j to the caller's edge 2 - j."""
    tags = np.asarray(node_tags, dtype=np.int64)
    xy = np.asarray(node_coordinates, dtype=np.float64).reshape(-1, 2)
    tris = np.asarray(element_nodes, dtype=np.int64)
    order = np.argsort(tags, kind="stable")
    pos = order[np.searchsorted(tags[order], tris)]
    x, y = xy[pos, 0], xy[pos, 1]
    area2 = (x[:, 0] * (y[:, 1] - y[:, 2]) + x[:, 1] * (y[:, 2] - y[:, 0])
             + x[:, 2] * (y[:, 0] - y[:, 1]))
    edges = np.tile(np.arange(3), (len(tris), 1))
    edges[area2 < 0] = 2 - edges[area2 < 0]
    return edges


def periodic_neighbors(neighbors: np.ndarray, caller_edge: np.ndarray,
                       pairs: PeriodicPairs) -> np.ndarray:
    """face_neighbors with every boundary edge's periodic partner filled in."""
    nbr = neighbors.copy()
    nbr[pairs.element, caller_edge[pairs.element, pairs.edge]] = pairs.donors[:, 0]
    return nbr


def ghost_layers(neighbors: np.ndarray, owned: np.ndarray, depth: int) -> list[np.ndarray]:
    """The ghost layers around a set of owned elements (boolean mask): layer k
    holds the elements k face steps away, ascending."""
    inside = owned.copy()
    front = np.nonzero(owned)[0]
    layers = []
    for _ in range(depth):
        cand = neighbors[front].ravel()
        cand = np.unique(cand[cand >= 0])
        cand = cand[~inside[cand]]
        inside[cand] = True
        layers.append(cand)
        front = cand
    return layers


@dataclass
class LocalMesh:
    """One rank's mesh: its owned elements and ghost layers, ascending."""
    rank: int
    elements: np.ndarray          # global indices of the local elements, ascending
    owned: np.ndarray             # bool per local element
    node_tags: np.ndarray         # the nodes the local elements use, ascending
    node_coordinates: np.ndarray
    element_nodes: np.ndarray     # local elements' node tags
    # For a periodic mesh: (donors [b][Q] int32, basis [b][Q][modes]) of the
    # part's boundary faces, the handle's wasl_gpu_create_part input.
    part_boundary: tuple | None = None

    @property
    def arrays(self):
        """(node tags, coordinates, element nodes): the solver's mesh input."""
        return self.node_tags, self.node_coordinates, self.element_nodes

    def local_index(self, global_elements) -> np.ndarray:
        idx = np.searchsorted(self.elements, global_elements)
        if np.any(idx >= self.elements.size) or np.any(self.elements[idx] != global_elements):
            raise ValueError("halo: element is not on this rank")
        return idx


def local_mesh(node_tags, node_coordinates, element_nodes, rank: int, ranks: int,
               depth: int, neighbors: np.ndarray | None = None,
               pairs: PeriodicPairs | None = None) -> LocalMesh:
    """The rank's owned elements plus `depth` ghost layers as a mesh; with
    the whole mesh's periodic pairs, the layers also grow across the periodic
    seams and the part's boundary is given (LocalMesh.part_boundary)."""
    tris = np.asarray(element_nodes, dtype=np.int64)
    owners = element_owners(tris.shape[0], ranks)
    nbr = face_neighbors(tris) if neighbors is None else neighbors
    caller_edge = None
    if pairs is not None:
        caller_edge = normalized_edge(node_tags, node_coordinates, tris)
        geometric, nbr = nbr, periodic_neighbors(nbr, caller_edge, pairs)
    owned_mask = owners == rank
    layers = ghost_layers(nbr, owned_mask, depth)
    elements = np.sort(np.concatenate([np.nonzero(owned_mask)[0]] + layers))
    local_tris = tris[elements]
    tags = np.asarray(node_tags, dtype=np.int64)
    used = np.unique(local_tris)
    order = np.argsort(tags, kind="stable")
    pos = order[np.searchsorted(tags[order], used)]
    if np.any(tags[pos] != used):
        raise ValueError("halo: an element uses an unknown node tag")
    coords = np.asarray(node_coordinates, dtype=np.float64)[pos]
    boundary = None
    if pairs is not None:
        boundary = part_boundary(elements, geometric, caller_edge, pairs)
    return LocalMesh(rank, elements, owners[elements] == rank, used, coords, local_tris,
                     boundary)


def part_boundary(elements: np.ndarray, geometric: np.ndarray, caller_edge: np.ndarray,
                  pairs: PeriodicPairs):
    """The boundary faces of the part made of `elements` (ascending global
    indices), in the part's face order (by element, then normalized edge):
    a face of the whole mesh's boundary whose donors are all in the part keeps
    them (as part indices) and their basis; any other face (a cut face, or a
    periodic face whose donor lies beyond the ghost region) gets donor -1,
    its own element's trace."""
    Q, M = pairs.basis.shape[1], pairs.basis.shape[2]
    inside = np.full(geometric.shape[0], -1, dtype=np.int64)
    inside[elements] = np.arange(elements.size)
    face_of = {(int(e), int(j)): b for b, (e, j) in enumerate(zip(pairs.element, pairs.edge))}
    donors, basis = [], []
    for g in elements:
        for j in range(3):
            h = geometric[g, caller_edge[g, j]]
            if h >= 0 and inside[h] >= 0:
                continue  # an interior face of the part
            d = np.full(Q, -1, dtype=np.int32)
            v = np.zeros((Q, M))
            if h < 0:
                b = face_of[(int(g), j)]
                local = inside[pairs.donors[b]]
                if np.all(local >= 0):
                    d, v = local.astype(np.int32), pairs.basis[b]
            donors.append(d)
            basis.append(v)
    return (np.array(donors, dtype=np.int32).reshape(-1, Q),
            np.array(basis, dtype=np.float64).reshape(-1, Q, M))


@dataclass
class HaloSchedule:
    """Per peer rank (ascending), the global elements this rank sends (owned
    ones the peer holds as ghosts) and receives (its ghosts the peer owns)."""
    rank: int
    sends: list[tuple[int, np.ndarray]] = field(default_factory=list)
    recvs: list[tuple[int, np.ndarray]] = field(default_factory=list)


def build_halo_schedule(meshes: list[LocalMesh], ranks: int, element_count: int,
                        rank: int) -> HaloSchedule:
    """The schedule of `rank` from every rank's local mesh (a function of the
    mesh alone, so every rank builds the same set)."""
    owners = element_owners(element_count, ranks)
    s = HaloSchedule(rank)
    mine = meshes[rank]
    ghosts = mine.elements[~mine.owned]
    for peer in range(ranks):
        if peer == rank:
            continue
        recv = ghosts[owners[ghosts] == peer]
        if recv.size:
            s.recvs.append((peer, recv))
        other = meshes[peer]
        their_ghosts = other.elements[~other.owned]
        send = their_ghosts[owners[their_ghosts] == rank]
        if send.size:
            s.sends.append((peer, send))
    return s


def exchange_in_process(states: list[np.ndarray], meshes: list[LocalMesh],
                        schedules: list[HaloSchedule]) -> None:
    """Copy every rank's owned rows into the matching ghost columns of the
    ranks that import them; states[r] is [rows][local elements]."""
    for sender, sched in enumerate(schedules):
        for peer, elements in sched.sends:
            src = meshes[sender].local_index(elements)
            dst = meshes[peer].local_index(elements)
            states[peer][:, dst] = states[sender][:, src]


class HaloExchange:
    """The exchange of one rank over torch.distributed: for every peer, the
    owned columns it imports are gathered into one contiguous buffer and sent,
    and the ghost columns it owns are received and scattered, all as one
    batch of point-to-point operations (NCCL requires the batch; gloo takes
    it as well)."""

    def __init__(self, mesh: LocalMesh, schedule: HaloSchedule, rows: int, device="cpu",
                 group=None, element_order=None):
        """element_order: the handle's storage order (Solver.element_order()),
        when the exchanged state is its device storage; None: the local mesh's
        own element order."""
        import torch
        self.torch = torch
        self.group = group
        self.rows = rows
        column = None
        if element_order is not None:
            column = np.empty(len(element_order), dtype=np.int64)
            column[np.asarray(element_order)] = np.arange(len(element_order))

        def index(elements):
            local = mesh.local_index(elements)
            return torch.as_tensor(local if column is None else column[local], device=device)

        self.sends = [(peer, index(el)) for peer, el in schedule.sends]
        self.recvs = [(peer, index(el)) for peer, el in schedule.recvs]

    def exchange(self, state) -> None:
        """state: [rows][local elements] float64 tensor on the rank's device."""
        torch = self.torch
        dist = torch.distributed
        ops, inbox = [], []
        for peer, idx in self.sends:
            buf = state.index_select(1, idx).contiguous()
            ops.append(dist.P2POp(dist.isend, buf, peer, group=self.group))
        for peer, idx in self.recvs:
            buf = torch.empty((self.rows, idx.numel()), dtype=state.dtype, device=state.device)
            inbox.append((idx, buf))
            ops.append(dist.P2POp(dist.irecv, buf, peer, group=self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for idx, buf in inbox:
            state.index_copy_(1, idx, buf)


class NativeHalo:
    """One rank's halo exchange in the library (wasl_halo_*), on its
    handle's device state: pack and unpack kernels on the handle's stream,
    per-peer device buffers [rows][columns], and the NCCL transport.  The
    same schedule as HaloExchange, without torch on the data path."""

    def __init__(self, solver, mesh: LocalMesh, schedule: HaloSchedule):
        import ctypes as C

        from . import WaslError, _i64, _ptr, library
        self._lib, self._C, self.solver = library(), C, solver
        sends, recvs = dict(schedule.sends), dict(schedule.recvs)
        self.peers = sorted(set(sends) | set(recvs))
        empty = np.zeros(0, dtype=np.int64)
        send_lists = [mesh.local_index(sends[p]) if p in sends else empty for p in self.peers]
        recv_lists = [mesh.local_index(recvs[p]) if p in recvs else empty for p in self.peers]
        ranks = np.array(self.peers, dtype=np.int32)
        send_counts = np.array([len(x) for x in send_lists], dtype=np.int64)
        recv_counts = np.array([len(x) for x in recv_lists], dtype=np.int64)
        send_elems = np.ascontiguousarray(np.concatenate([empty] + send_lists), dtype=np.int64)
        recv_elems = np.ascontiguousarray(np.concatenate([empty] + recv_lists), dtype=np.int64)
        err = C.create_string_buffer(1024)
        h = C.c_void_p()
        rc = self._lib.wasl_halo_create(
            solver._h, len(self.peers), ranks.ctypes.data_as(C.POINTER(C.c_int32)),
            _ptr(send_counts, _i64), _ptr(send_elems, _i64), _ptr(recv_counts, _i64),
            _ptr(recv_elems, _i64), C.byref(h), err, len(err))
        if rc != 0:
            raise WaslError(rc, err.value.decode())
        self._h = h

    def _check(self, rc):
        from . import WaslError
        if rc != 0:
            raise WaslError(rc, self._lib.wasl_halo_last_error(self._h).decode())

    def pack(self):
        self._check(self._lib.wasl_halo_pack(self._h))

    def unpack(self):
        self._check(self._lib.wasl_halo_unpack(self._h))

    def buffers(self, k: int):
        """(send pointer, receive pointer, send columns, receive columns, rows)
        of the k-th peer (self.peers[k])."""
        C = self._C
        send, recv = C.c_void_p(), C.c_void_p()
        ns, nr, rows = C.c_int64(), C.c_int64(), C.c_int64()
        self._check(self._lib.wasl_halo_buffers(self._h, k, C.byref(send), C.byref(recv),
                                                C.byref(ns), C.byref(nr), C.byref(rows)))
        return send.value, recv.value, ns.value, nr.value, rows.value

    def exchange_nccl(self, comm: int):
        self._check(self._lib.wasl_halo_exchange_nccl(self._h, self._C.c_void_p(comm)))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.wasl_halo_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def nccl_unique_id() -> bytes:
    """A new NCCL communicator id (128 bytes), made on one rank and shared."""
    import ctypes as C

    from . import WaslError, library
    buf = (C.c_uint8 * 128)()
    rc = library().wasl_nccl_unique_id(buf)
    if rc != 0:
        raise WaslError(rc, "NCCL: no unique id")
    return bytes(buf)


def nccl_communicator(ranks: int, uid: bytes, rank: int, device: int) -> int:
    """An NCCL communicator (ncclComm_t as an int) of this rank."""
    import ctypes as C

    from . import WaslError, library
    buf = (C.c_uint8 * 128).from_buffer_copy(uid)
    comm, err = C.c_void_p(), C.create_string_buffer(1024)
    rc = library().wasl_nccl_comm_create(ranks, buf, rank, device, C.byref(comm), err, len(err))
    if rc != 0:
        raise WaslError(rc, err.value.decode())
    return comm.value


def nccl_destroy(comm: int) -> None:
    import ctypes as C

    from . import library
    library().wasl_nccl_comm_destroy(C.c_void_p(comm))


def stable_dt_nccl(solver, comm: int, cfl: float) -> float:
    """The whole mesh's CFL step, the CFL parts all-reduced over comm."""
    import ctypes as C
    dt = C.c_double()
    solver._check(solver._lib.wasl_gpu_stable_dt_nccl(solver._h, C.c_void_p(comm), cfl,
                                                      C.byref(dt)))
    return dt.value


class _DeviceRows:
    """A [rows][columns] float64 array in device memory, by its pointer."""

    def __init__(self, pointer: int, rows: int, columns: int):
        self.__cuda_array_interface__ = {"shape": (rows, columns), "typestr": "<f8",
                                         "data": (pointer, False), "version": 3,
                                         "strides": None}


def device_state(solver):
    """The handle's device state U[variable][mode][element] as a
    [4 M][elements] torch tensor sharing its memory (no copy), its columns in
    the handle's storage order (Solver.element_order()).  The handle's
    stream must have finished (solver.sync()) before it is read, and writes
    through it must have finished before the handle's next step."""
    import torch
    rows = solver.variables * solver.modes
    return torch.as_tensor(_DeviceRows(solver.state_device_pointer(), rows, solver.elements),
                           device="cuda")


def check_partitioned_solver(solver) -> None:
    """A rank's periodic handle must have been built on its part's given
    boundary (Solver(..., part_boundary=mesh.part_boundary)): its own donor
    search would pair the faces where its ghost region is cut across the
    period and silently compute wrong values there.  Raises ValueError for
    such a handle."""
    from . import BOUNDARY_KINDS
    if (solver.config.boundary_left == BOUNDARY_KINDS["periodic"]
            and not getattr(solver, "part", False)):
        raise ValueError("partitioned runs: a periodic handle needs its part's boundary (build"
                         " it with part_boundary=LocalMesh.part_boundary from a local_mesh"
                         " given the periodic pairs); otherwise its cut faces would be paired"
                         " across the period")


def step_partitioned(solver, exchange: HaloExchange, cfl: float, polynomial_order: int,
                     group=None) -> float:
    """One step of a rank of a partitioned run on its GPU: the whole-mesh dt
    from the reduced CFL parts, the step, then the ghost exchange.

    The handle checks every local element, ghosts included: a non-physical
    cell average or a mean below a positivity floor in a ghost layer (the
    outer layers are spoiled by the cut, by design, and overwritten by the
    exchange) raises the error on this rank even though another rank owns the
    element."""
    import torch
    check_partitioned_solver(solver)
    dt = global_dt(solver, cfl, polynomial_order, group=group, device="cuda")
    solver.step(dt)
    solver.sync()
    exchange.exchange(device_state(solver))
    torch.cuda.current_stream().synchronize()
    return dt


def dt_from_parts(cfl: float, speed: float, length: float, polynomial_order: int) -> float:
    """cfl length / (speed (2p + 1)), in the order the solver evaluates it
    (cpp/src/time/cfl_timestep.cpp:70-84); 0 for a state at rest."""
    return cfl * length / (speed * (2 * polynomial_order + 1)) if speed > 0.0 else 0.0


def global_dt(solver, cfl: float, polynomial_order: int, group=None, device="cpu") -> float:
    """The whole-mesh CFL step of a partitioned run: the largest wave speed
    and the smallest element length reduced over ranks."""
    import torch
    speed, length = solver.cfl_parts()
    v = torch.tensor([speed, -length], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(v, op=torch.distributed.ReduceOp.MAX, group=group)
    return dt_from_parts(cfl, float(v[0]), -float(v[1]), polynomial_order)
