"""Advection borders between ranks: the reference's guard exchange
(lib/isaac.hpp:1856-1913), with ``torch.distributed`` (NCCL, or gloo on the CPU)
in place of MPI.

Each rank's field sources carry advection textures with a guard band
(``isaacb_advection_guard``).  After every rank has advected (``isaacb_advect``),
for each field source and each neighbour direction i (1-26, the reference's
indices, lib/isaac/isaac_types.hpp:133-161) with a neighbour rank:

* the rank packs its own slab i (``isaacb_pack_guard``, SyncToOwnGuard) and sends
  it to ``neighbours[i]`` with tag ``mirrored(i)``;
* it receives slab i from ``neighbours[i]`` with tag i and unpacks it into the
  guard band (``isaacb_unpack_guard``, SyncFromNeighbourGuard).

These are the reference's MPI_Isend / MPI_Irecv pairs.  Sends and receives are
posted in order of their tags on every rank, so that a transport which matches
messages between two ranks in issue order (NCCL) pairs them as the tags do.  A
rank that is its own neighbour (periodic with one rank along an axis) copies
locally.  Pack and unpack are parameters so that the exchange can be exercised
with gloo ranks on the CPU against the oracle; on the GPU the defaults call the
CUDA kernels through the C ABI.
"""

from __future__ import annotations


def direction_of(index: int) -> tuple:
    """Neighbour index -> (dx, dy, dz): base-3 digits x, y, z, digit 2 meaning -1."""
    d = []
    for _ in range(3):
        m = index % 3
        d.append(-1 if m == 2 else m)
        index //= 3
    return tuple(d)


def index_of(direction) -> int:
    return sum((2 if v == -1 else v) * 3**a for a, v in enumerate(direction))


def mirrored(index: int) -> int:
    """The index of the opposite direction (toMirroredIndex)."""
    return index_of(tuple(-v for v in direction_of(index)))


def slab_shape(direction: int, local_size, guard) -> tuple:
    """(x, y, z) extent of the guard slab of a direction: the guard across it, the local size along it."""
    return tuple(int(g) if d != 0 else int(l) for d, l, g in zip(direction_of(direction), local_size, guard))


class AdvectionBorders:
    """Per-frame guard exchange of one rank's field sources over a process group."""

    def __init__(self, neighbours, local_size, guard, pack, unpack, group=None, device="cuda"):
        import torch.distributed as dist

        if len(neighbours) != 27:
            raise ValueError("neighbours: 27 ranks (index 0 is this rank's own cell, ignored), -1 for none")
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.neighbours = [int(n) for n in neighbours]
        self.local_size = tuple(int(v) for v in local_size)
        self.guard = tuple(int(v) for v in guard)
        self.pack, self.unpack = pack, unpack
        self.device = device

    @classmethod
    def for_visualization(cls, viz, neighbours, group=None):
        """The exchange of an IsaacVisualization's field sources through the CUDA kernels."""
        import torch

        guard = viz.advectionGuard()

        def pack(src, direction):
            out = torch.empty(int(torch.tensor(slab_shape(direction, viz.localSize, guard)).prod()), dtype=torch.uint8,
                              device="cuda")
            viz.packGuard(src, direction, out)
            return out

        def unpack(src, direction, data):
            viz.unpackGuard(src, direction, data)

        return cls(neighbours, viz.localSize, guard, pack, unpack, group=group, device="cuda")

    def directions(self) -> list[int]:
        return [i for i in range(1, 27) if self.neighbours[i] >= 0]

    def exchange(self, src: int) -> None:
        """Exchange the guard slabs of field source ``src`` with every neighbour."""
        import torch

        dist = self.dist
        own = {i: self.pack(src, i) for i in self.directions()}
        recv = {}
        ops = []
        for i in sorted(self.directions()):  # receives, by tag i
            shape = slab_shape(i, self.local_size, self.guard)
            n = shape[0] * shape[1] * shape[2]
            if self.neighbours[i] == self.rank:
                # my own slab sent the other way (tag i is the send of direction mirrored(i))
                m = mirrored(i)
                recv[i] = (own[m] if m in own else self.pack(src, m)).clone()
                continue
            recv[i] = torch.empty(n, dtype=torch.uint8, device=self.device)
            ops.append(dist.P2POp(dist.irecv, recv[i], self.neighbours[i], self.group, tag=i))
        for i in sorted(self.directions(), key=mirrored):  # sends, by tag mirrored(i)
            if self.neighbours[i] != self.rank:
                ops.append(dist.P2POp(dist.isend, own[i], self.neighbours[i], self.group, tag=mirrored(i)))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        for i in sorted(recv):
            self.unpack(src, i, recv[i])
