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

Domains whose boundary is periodic are not partitioned here: the periodic
pairing of a rank's boundary faces would also pair the faces where its ghost
region ends.
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
               depth: int, neighbors: np.ndarray | None = None) -> LocalMesh:
    """The rank's owned elements plus `depth` ghost layers as a mesh."""
    tris = np.asarray(element_nodes, dtype=np.int64)
    owners = element_owners(tris.shape[0], ranks)
    nbr = face_neighbors(tris) if neighbors is None else neighbors
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
    return LocalMesh(rank, elements, owners[elements] == rank, used, coords, local_tris)


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
    """A rank's handle must treat its boundary faces as transmissive: with
    periodic boundaries it would pair the faces where its ghost region is cut
    across the period and silently compute wrong values there.  Raises
    ValueError for such a handle."""
    from . import BOUNDARY_KINDS
    if solver.config.boundary_left == BOUNDARY_KINDS["periodic"]:
        raise ValueError("partitioned runs: periodic boundaries are not supported (a rank's"
                         " cut faces would be paired across the period); build each rank's"
                         " handle with boundary='transmissive'")


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
