"""Batched multi-view rendering (isaacb_batch_*) against single-view renders.

Every view of a batch must be bit-identical to the frame one context of the
view's size draws with the view's camera, for any tile shape, CTA count,
skipping choice and whether the frame comes from a captured CUDA graph."""

import dataclasses

import numpy as np
import pytest
import torch

from harness import build_gpu, build_oracle, gaussian_pair, image_diff
from isaac_b200 import _lib, scenes
from isaac_b200.batch import IsaacBatch

pytestmark = pytest.mark.gpu

# (context, width, height, camera seed): ragged sizes, views thinner than a tile, several per context
VIEWS = [
    (0, 64, 48, 1),
    (0, 37, 29, 5),
    (1, 8, 4, 2),
    (1, 100, 3, 7),
    (2, 45, 61, 3),
    (0, 129, 17, 9),
    (2, 16, 16, 11),
]


def _scenes():
    a = gaussian_pair(32, seed=1, background=(0.1, 0.2, 0.3, 0.4), clips=[(0.5, 0.5, 0.5, 0.3, -1.0, 0.2)])
    b = gaussian_pair(32, seed=2, interpolation=False, step=0.7, render_mode=2)
    c = gaussian_pair(24, seed=3, weights=[0.0, 0.0], background=(0.3, 0.0, 0.9, 1.0))
    return [a, b, c]


def _reference(s, w, h, seed):
    """The frame of one context of the view's size and camera."""
    r = dataclasses.replace(s, fb=(w, h), camera_seed=seed)
    return build_gpu(r).doVisualization()


def _camera(w, h, seed, s):
    return scenes.camera(w, h, seed=seed, distance=s.camera_distance)


@pytest.fixture(scope="module")
def setup():
    sc = _scenes()
    vis = [build_gpu(s) for s in sc]
    views = [(ci, w, h, *_camera(w, h, seed, sc[ci])) for ci, w, h, seed in VIEWS]
    batch = IsaacBatch(vis, views)
    refs = [_reference(sc[ci], w, h, seed) for ci, w, h, seed in VIEWS]
    return sc, vis, batch, refs


def _check(batch, refs):
    torch.cuda.synchronize()
    for i, ref in enumerate(refs):
        got = batch.frames[i].cpu().numpy()
        assert np.array_equal(got, ref), (i, image_diff(got, ref))


def test_batch_matches_single_views(setup):
    _, _, batch, refs = setup
    batch.render(update=True)
    _check(batch, refs)
    # three merges of two kernels (pass 1, pass 2) and the one batch render
    assert batch.launchCount() == 3 * 2 + 1


@pytest.mark.parametrize("tile", [(32, 8), (16, 16), (8, 32), (64, 4)])
@pytest.mark.parametrize("skip", [0, 1])
def test_batch_launch_shapes(setup, tile, skip):
    _, _, batch, refs = setup
    for f in batch.frames:
        f.zero_()
    batch.setConfig(tile[0], tile[1], blocks_per_sm=1 if skip else 0, skip_empty=skip)
    batch.render(update=False)
    _check(batch, refs)
    batch.setConfig()


def test_batch_view_matches_oracle(setup):
    sc, _, batch, _ = setup
    batch.render(update=True)
    torch.cuda.synchronize()
    ci, w, h, seed = VIEWS[0]
    ref = build_oracle(dataclasses.replace(sc[ci], fb=(w, h), camera_seed=seed)).frame()
    st = image_diff(batch.frames[0].cpu().numpy(), ref)
    assert st["frac_le1"] >= 0.999 and st["max"] <= 3, st


def test_batch_graph_and_camera_update(setup):
    sc, vis, batch, refs = setup
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        batch.capture(update=True)
        for f in batch.frames:
            f.zero_()
        batch.launchGraph()
        batch.launchGraph()
    s.synchronize()
    _check(batch, refs)
    # a new camera reaches the captured graph through the view table
    ci, w, h, _ = VIEWS[1]
    P, MV = _camera(w, h, 42, sc[ci])
    with torch.cuda.stream(s):
        batch.setCamera(1, P, MV)
        batch.launchGraph()
    s.synchronize()
    got = batch.frames[1].cpu().numpy()
    assert np.array_equal(got, _reference(sc[ci], w, h, 42))
    with torch.cuda.stream(s):
        batch.setCamera(1, *_camera(w, h, VIEWS[1][3], sc[ci]))
        batch.launchGraph()
    s.synchronize()
    _check(batch, refs)


def test_batch_graph_recaptures_after_weight_change():
    sc = _scenes()[:1]
    vis = [build_gpu(sc[0])]
    ci, w, h, seed = VIEWS[0]
    batch = IsaacBatch(vis, [(0, w, h, *_camera(w, h, seed, sc[0]))])
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        batch.capture(update=True)
        batch.launchGraph()
        vis[0].setWeight(1, 0.0)
        batch.launchGraph()
    s.synchronize()
    ref = _reference(dataclasses.replace(sc[0], weights=[2.0, 0.0]), w, h, seed)
    assert np.array_equal(batch.frames[0].cpu().numpy(), ref)
    batch.close()


def test_batch_sample_count_matches_single_views(setup):
    sc, _, batch, _ = setup
    batch.setCounting(True)
    batch.render(update=False)
    total = batch.samples()
    batch.setCounting(False)
    want = 0
    for ci, w, h, seed in VIEWS:
        v = build_gpu(dataclasses.replace(sc[ci], fb=(w, h), camera_seed=seed))
        v.setCounting(True)
        v.doVisualization()
        want += v.counters()[0]
    assert total == want


def test_batch_autotune_keeps_pixels(setup):
    _, _, batch, refs = setup
    cfg, ms = batch.autotune()
    assert cfg.tile_w * cfg.tile_h == 256 and ms > 0
    for f in batch.frames:
        f.zero_()
    batch.render(update=False)
    _check(batch, refs)
    batch.setConfig()


def test_batch_rejects_unbatchable_contexts():
    s = gaussian_pair(16, iso=[0.0, 0.5])
    v = build_gpu(s)
    with pytest.raises(_lib.IsaacError) as e:
        IsaacBatch([v], [(0, 16, 16, *_camera(16, 16, 1, s))])
    assert e.value.status == _lib.INVALID_ARG
    s2 = gaussian_pair(16)
    v2 = build_gpu(s2)
    with pytest.raises(_lib.IsaacError):
        IsaacBatch([v2], [(1, 16, 16, *_camera(16, 16, 1, s2))])  # context index out of range
    b = IsaacBatch([v2], [(0, 16, 16, *_camera(16, 16, 1, s2))])
    with pytest.raises(_lib.IsaacError):
        b.setConfig(24, 8)  # not 256 pixels
    b.close()
