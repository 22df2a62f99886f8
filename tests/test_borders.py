"""Advection borders between ranks on the host (no GPU).

The oracle restates the reference's guard band and its SyncToOwnGuard /
SyncFromNeighbourGuard index arithmetic (lib/isaac/isaac_common_kernel.hpp:454-498).
Here an in-process emulation of all ranks (each rank an oracle context over its
sub-volume, slabs handed over directly) is the reference for the exchange that
``isaac_b200.borders.AdvectionBorders`` runs over gloo ranks, tags and ordering
included (lib/isaac.hpp:1856-1913)."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from harness import Scene, build_oracle
from isaac_b200 import borders as B
from isaac_b200 import scenes
from oracle import oracle as OR


def test_directions_match_the_oracle():
    for i in range(27):
        assert B.direction_of(i) == OR.direction_of(i)
        assert B.mirrored(i) == OR.mirrored(i)
        assert B.index_of(B.direction_of(i)) == i
    assert B.direction_of(1) == (1, 0, 0) and B.direction_of(2) == (-1, 0, 0) and B.direction_of(26) == (-1, -1, -1)
    assert B.slab_shape(1, (16, 12, 8), (4, 4, 4)) == (4, 12, 8)
    assert B.slab_shape(13, (16, 12, 8), (4, 4, 4)) == (4, 4, 4)


def grid_neighbours(dims, coord):
    """The 27 neighbour ranks of grid cell ``coord`` (ranks x fastest), -1 outside the grid."""
    out = []
    for i in range(27):
        d = B.direction_of(i)
        c = [coord[a] + d[a] for a in range(3)]
        if i == 0 or any(c[a] < 0 or c[a] >= dims[a] for a in range(3)):
            out.append(-1)
        else:
            out.append(c[0] + dims[0] * (c[1] + dims[1] * c[2]))
    return out


def rank_scenes(n, dims):
    """The Gaussian pair of n^3 cut into dims boxes; source 1 (the curl) is the field source."""
    sc, curl = scenes.gaussian_scene(n, 3)
    sc, curl = sc.numpy(), curl.numpy()
    lx, ly, lz = n // dims[0], n // dims[1], n // dims[2]
    out = []
    for k in range(dims[2]):
        for j in range(dims[1]):
            for i in range(dims[0]):
                px, py, pz = i * lx, j * ly, k * lz
                s = Scene(n=(lx, ly, lz), global_n=(n, n, n), position=(px, py, pz), fb=(32, 24),
                          volumes=[(np.ascontiguousarray(sc[pz:pz + lz, py:py + ly, px:px + lx]), True),
                                   (np.ascontiguousarray(curl[pz:pz + lz, py:py + ly, px:px + lx]), True)])
                s.functions = ["idem", "length"]
                s.transfer = [scenes.transfer_4point(0.3), scenes.transfer_4point(1.7)]
                out.append(((i, j, k), s))
    return out


ADVECTION = (1.0, 0.95, 1, 1, 60)  # step factor, history weight, seeding period, duration, seeds


def oracle_rank(s):
    o = build_oracle(s)
    o.set_field(1)
    o.set_advection(*ADVECTION)
    return o


def emulate(n, dims, frames, exchange=True):
    """Every rank in this process: advect, hand the guard slabs over, merge."""
    ranks = rank_scenes(n, dims)
    ctx = [oracle_rank(s) for _, s in ranks]
    nbrs = [grid_neighbours(dims, c) for c, _ in ranks]
    for _ in range(frames):
        for o in ctx:
            o.advect()
        if exchange:
            own = [{i: o.pack_guard(1, i) for i in range(1, 27) if nb[i] >= 0} for o, nb in zip(ctx, nbrs)]
            for r, o in enumerate(ctx):
                for i in range(1, 27):
                    if nbrs[r][i] >= 0:
                        # rank r receives, as slab i, the neighbour's slab of the opposite direction
                        o.unpack_guard(1, i, own[nbrs[r][i]][B.mirrored(i)])
        for o in ctx:
            o.update()
    return [o.advection(1) for o in ctx]


def test_exchange_reaches_across_the_boundary():
    with_ex = emulate(32, (2, 1, 1), 3)
    without = emulate(32, (2, 1, 1), 3, exchange=False)
    # the field carries values over the x boundary only when the slabs are exchanged
    assert any(not np.array_equal(a, b) for a, b in zip(with_ex, without))
    # far from the boundary nothing changes (3 frames of at most 3 voxels each)
    assert np.array_equal(with_ex[0][:, :, :4], without[0][:, :, :4])


def _rank_main(rank, world, port, n, dims, frames, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        coord, s = rank_scenes(n, dims)[rank]
        o = oracle_rank(s)
        guard = tuple(int(np.ceil(np.float32(4.0) / np.float32(v))) for v in s.scale)
        ex = B.AdvectionBorders(grid_neighbours(dims, coord), s.n, guard,
                                pack=lambda src, i: torch.from_numpy(o.pack_guard(src, i)),
                                unpack=lambda src, i, t: o.unpack_guard(src, i, t.numpy()), device="cpu")
        for _ in range(frames):
            o.advect()
            ex.exchange(1)
            o.update()
        np.save(os.path.join(out_dir, f"adv{rank}.npy"), o.advection(1))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.mark.parametrize("dims", [(2, 1, 1), (2, 2, 1)])
def test_gloo_ranks_exchange_like_the_emulation(tmp_path, dims):
    n, frames = 24, 3
    world = dims[0] * dims[1] * dims[2]
    mp.start_processes(_rank_main, args=(world, _free_port(), n, dims, frames, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    ref = emulate(n, dims, frames)
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"adv{r}.npy"), ref[r]), r
