"""Sort-last compositing on the host (no GPU): the per-rank camera distance and
the front-to-back order against the oracle's restatement of lib/isaac.hpp:2019-2047,
and the compositor's exchange (all-gather of distances, all-to-all of row stripes,
all-gather of the blended stripes) with gloo ranks on the CPU, the blend supplied
by the oracle.  The frame heights do not divide by the world size."""

import os
import socket
import time

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from isaac_b200 import sortlast as S
from isaac_b200.scenes import camera
from oracle import sortlast_oracle as O


def test_distance_and_order_match_oracle():
    rng = np.random.default_rng(3)
    for seed in range(20):
        _, mv = camera(64, 48, seed=seed, distance=float(rng.uniform(1.5, 4.0)))
        glo = tuple(int(v) for v in rng.integers(16, 80, 3))
        scale = tuple(float(v) for v in rng.uniform(0.5, 2.0, 3))
        ds, dso = [], []
        for r in range(6):
            loc = tuple(int(rng.integers(1, g + 1)) for g in glo)
            pos = tuple(int(rng.integers(0, g - l + 1)) for g, l in zip(glo, loc))
            ds.append(S.rank_distance(mv, pos, loc, glo, scale))
            dso.append(O.distance(mv, pos, loc, glo, scale))
        assert ds == dso
        assert S.composite_order(ds) == O.order(dso)


def test_order_is_front_to_back_with_stable_ties():
    # camera on the +z axis looking down -z: the upper z half is nearer
    mv = np.eye(4)
    mv[3][2] = -2.5
    near = S.rank_distance(mv, (0, 0, 32), (64, 64, 32), (64, 64, 64))
    far = S.rank_distance(mv, (0, 0, 0), (64, 64, 32), (64, 64, 64))
    assert near < far
    assert S.composite_order([far, near]) == [1, 0]
    assert S.composite_order([1.0, 0.5, 1.0, 0.5]) == [1, 3, 0, 2]


def _premultiplied(h, w, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 256, (h, w, 1))
    c = (rng.random((h, w, 3)) * (a + 1)).astype(np.int64).clip(0, a)
    return np.concatenate([c, a], axis=-1).astype(np.uint8)


def _oracle_blend(stripes, order, background):
    return torch.from_numpy(O.blend(list(stripes.numpy()), order, background))


def _rank_main(rank, world, port, h, w, distances, background, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        comp = S.SortLastCompositor(background=background, blend=_oracle_blend)
        frame = torch.from_numpy(_premultiplied(h, w, seed=100 + rank))
        out = comp.composite(frame, distances[rank])
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), out.numpy())
        np.save(os.path.join(out_dir, f"order{rank}.npy"), np.array(comp.lastOrder))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,h,w,distances,background", [
    (2, 7, 5, [2.0, 1.0], None),
    (3, 10, 6, [1.5, 3.0, 0.5], (10, 20, 30, 255)),
])
def test_gloo_ranks_composite_like_the_oracle(tmp_path, world, h, w, distances, background):
    mp.start_processes(_rank_main, args=(world, _free_port(), h, w, distances, background, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    order = O.order(distances)
    ref = O.blend([_premultiplied(h, w, seed=100 + r) for r in range(world)], order, background)
    for r in range(world):
        assert list(np.load(tmp_path / f"order{r}.npy")) == order
        got = np.load(tmp_path / f"rank{r}.npy")
        assert got.shape == (h, w, 4)
        assert np.array_equal(got, ref)


def _failing_rank_main(rank, world, port, out_dir):
    """Rank 1 leaves between frames (it raises after one composite); the survivors'
    next composite must end with an error from the short process-group timeout instead
    of waiting for good."""
    import datetime

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    comp = S.SortLastCompositor(blend=_oracle_blend)
    frame = torch.from_numpy(_premultiplied(6, 4, seed=100 + rank))
    comp.composite(frame, float(rank))  # a good frame first
    if rank == 1:
        os._exit(0)  # leaves between steps: nothing of it is in flight
    t0 = time.time()
    try:
        comp.composite(frame, float(rank))
        outcome = "completed"
    except Exception as ex:  # the collective reports the missing rank
        outcome = f"error:{type(ex).__name__}"
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(f"{outcome}\n{time.time() - t0:.1f}\n")
    os._exit(0)


def test_surviving_ranks_see_a_departed_rank_as_an_error(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_failing_rank_main, args=(r, 3, port, str(tmp_path))) for r in range(3)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a surviving rank waited for good"
    for r in (0, 2):
        outcome, secs = (tmp_path / f"rank{r}.txt").read_text().split("\n")[:2]
        assert outcome.startswith("error"), outcome
        assert float(secs) < 60.0
