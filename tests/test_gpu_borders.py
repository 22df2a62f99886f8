"""Advection borders between ranks on one GPU: every rank is its own context over
its sub-volume (no rank waits on another), the guard slabs go from one context's
buffers to another's, and each frame's advection texture and combined textures
equal, bit for bit, the oracle's emulation of the same ranks (the reference's
guard band and SyncToOwnGuard / SyncFromNeighbourGuard arithmetic,
lib/isaac/isaac_common_kernel.hpp:454-498, lib/isaac.hpp:1856-1913)."""

import numpy as np
import pytest
import torch

from harness import build_gpu
from isaac_b200 import _lib
from isaac_b200 import borders as B
from test_borders import ADVECTION, grid_neighbours, oracle_rank, rank_scenes

pytestmark = pytest.mark.gpu


def _gpu_rank(s):
    viz = build_gpu(s)
    viz.setFieldSource(1)
    viz.setAdvection(*ADVECTION)
    return viz


@pytest.mark.parametrize("dims", [(2, 1, 1), (2, 2, 1), (1, 2, 2)])
def test_emulated_ranks_exchange_guards(dims):
    n = 32
    ranks = rank_scenes(n, dims)
    vizs = [_gpu_rank(s) for _, s in ranks]
    ors = [oracle_rank(s) for _, s in ranks]
    nbrs = [grid_neighbours(dims, c) for c, _ in ranks]
    assert vizs[0].advectionGuard() == (4, 4, 4)
    for frame in range(4):
        for v, o in zip(vizs, ors):
            v.advect()
            o.advect()
        own_g = []
        own_o = []
        for v, o, nb in zip(vizs, ors, nbrs):
            dg, do = {}, {}
            for i in range(1, 27):
                if nb[i] < 0:
                    continue
                e = B.slab_shape(i, v.localSize, v.advectionGuard())
                t = torch.empty(e[0] * e[1] * e[2], dtype=torch.uint8, device="cuda")
                v.packGuard(1, i, t)
                dg[i] = t
                do[i] = o.pack_guard(1, i)
            own_g.append(dg)
            own_o.append(do)
        torch.cuda.synchronize()
        for r in range(len(vizs)):
            for i in range(1, 27):
                if nbrs[r][i] >= 0:
                    src = nbrs[r][i]
                    assert np.array_equal(own_g[src][B.mirrored(i)].cpu().numpy(), own_o[src][B.mirrored(i)])
                    vizs[r].unpackGuard(1, i, own_g[src][B.mirrored(i)])
                    ors[r].unpack_guard(1, i, own_o[src][B.mirrored(i)])
        for v, o in zip(vizs, ors):
            v.update()
            o.update()
        torch.cuda.synchronize()
        for r, (v, o) in enumerate(zip(vizs, ors)):
            assert np.array_equal(v.advectionTexture(1), o.advection(1)), (frame, r)
            gv, gi = v.combinedTextures()
            rv, ri = o.combined()
            assert np.array_equal(gv, rv), (frame, r)
            assert np.array_equal(gi, ri), (frame, r)
    for v in vizs:
        v.close()


def test_guard_calls_check_their_arguments():
    _, s = rank_scenes(32, (2, 1, 1))[0]
    viz = _gpu_rank(s)
    t = torch.empty(4 * 32 * 32, dtype=torch.uint8, device="cuda")
    with pytest.raises(_lib.IsaacError):
        viz.packGuard(1, 1, t)  # no advection texture before the first advection step
    viz.advect()
    with pytest.raises(_lib.IsaacError):
        viz.packGuard(1, 27, t)  # directions are 1-26
    with pytest.raises(_lib.IsaacError):
        viz.packGuard(0, 1, t)  # source 0 is not a field source
    viz.packGuard(1, 1, t)
    # "advection border" off clears both textures
    viz.update()
    viz.setAdvectionBorder(False)
    assert not viz.advectionTexture(1).any()
    viz.close()
