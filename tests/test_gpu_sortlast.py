"""Sort-last compositing on one GPU.

* The blend kernel (``isaacb_blend_ordered``) against the oracle's restatement of
  IceT's ordered BLEND composite, bit-exact: 1 to 64 images, permuted orders, with
  and without a background, on the four-pixel path and the one-pixel path
  (pixel counts not a multiple of 4, or a buffer off a 16-byte boundary).
* Ranks emulated on one GPU (each rank is its own context rendering its own
  sub-volume; no rank waits on another): every rank's frame meets the parity bar
  against the oracle rendering the same sub-volume, the GPU composite equals the
  oracle's blend of the GPU frames, and the composite of the oracle's frames is
  within the bar of the GPU composite.  The composite is compared with the
  single-context render of the whole volume, which it approximates: the ranks'
  textures end at their box (trilinear taps clamp there instead of reading the
  neighbour) and each partial frame is rounded to bytes before blending.  The scene
  uses dense transfer functions, so the reversed order is clearly worse.
"""

import numpy as np
import pytest
import torch

from harness import Scene, assert_image_parity, build_gpu, build_oracle, image_diff
from isaac_b200 import scenes
from isaac_b200 import sortlast as S
from oracle import sortlast_oracle as O

pytestmark = pytest.mark.gpu


def _premultiplied(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 256, (n, 1))
    c = (rng.random((n, 3)) * (a + 1)).astype(np.int64).clip(0, a)
    return np.concatenate([c, a], axis=-1).astype(np.uint8)


@pytest.mark.parametrize("k", [1, 2, 3, 5, 8, 17, 64])
@pytest.mark.parametrize("pixels", [4096, 1023])
@pytest.mark.parametrize("background", [None, (12, 40, 90, 255)])
def test_blend_kernel_bit_exact(k, pixels, background):
    rng = np.random.default_rng(k * 1000 + pixels)
    imgs = np.stack([_premultiplied(pixels, seed=int(rng.integers(1 << 30))) for _ in range(k)])
    order = [int(v) for v in rng.permutation(k)]
    got = S.blend_cuda(torch.from_numpy(imgs).cuda(), order, background).cpu().numpy()
    assert np.array_equal(got, O.blend(list(imgs), order, background))


def test_blend_kernel_unaligned_buffers():
    imgs = np.stack([_premultiplied(1001, seed=s) for s in range(3)])
    dev = torch.zeros(3 * 1001 * 4 + 4, dtype=torch.uint8, device="cuda")
    dev[4:] = torch.from_numpy(imgs.reshape(-1)).cuda()  # every image 4 bytes off a 16-byte boundary
    view = dev[4:].view(3, 1001, 4)
    got = S.blend_cuda(view, [2, 0, 1]).cpu().numpy()
    assert np.array_equal(got, O.blend(list(imgs), [2, 0, 1]))


# dense transfer functions: the volume is mostly opaque, so the blend order shows
DENSE = [{0: (0.0, 0.0, 1.0, 0.0), 300: (0.0, 0.0, 1.0, 0.9), 600: (1.0, 0.0, 0.0, 1.0), 1024: (0.0, 1.0, 0.0, 1.0)},
         {0: (1.0, 1.0, 0.0, 0.0), 1024: (0.0, 1.0, 1.0, 1.0)}]


def _split_scenes(n, splits, fb=(96, 72), seed=3):
    """The two-source Gaussian scene of n^3 cut into splits = (sx, sy, sz) boxes."""
    sc, curl = scenes.gaussian_scene(n, seed)
    sc, curl = sc.numpy(), curl.numpy()
    out = []
    sx, sy, sz = splits
    lx, ly, lz = n // sx, n // sy, n // sz
    for k in range(sz):
        for j in range(sy):
            for i in range(sx):
                px, py, pz = i * lx, j * ly, k * lz
                s = Scene(n=(lx, ly, lz), global_n=(n, n, n), position=(px, py, pz), fb=fb,
                          volumes=[(np.ascontiguousarray(sc[pz:pz + lz, py:py + ly, px:px + lx]), True),
                                   (np.ascontiguousarray(curl[pz:pz + lz, py:py + ly, px:px + lx]), True)])
                out.append(s)
    full = Scene(n=(n, n, n), fb=fb, volumes=[(sc, True), (curl, True)])
    for s in out + [full]:
        s.functions = ["idem", "length"]
        s.transfer = DENSE
        s.weights = [8.0, 8.0]
    return out, full


def _psnr(a, b):
    d = a.astype(np.float64) - b.astype(np.float64)
    mse = float(np.mean(d * d))
    return float("inf") if mse == 0 else 10 * np.log10(255.0**2 / mse)


@pytest.mark.parametrize("splits", [(2, 1, 1), (2, 2, 1), (1, 2, 2)])
def test_emulated_ranks_composite(splits):
    n = 32
    parts, full = _split_scenes(n, splits)
    frames, ref_frames, dists = [], [], []
    for s in parts:
        viz = build_gpu(s)
        g = viz.doVisualization()
        o = build_oracle(s).frame()
        assert_image_parity(g, o)
        frames.append(g)
        ref_frames.append(o)
        dists.append(S.rank_distance(viz.modelview, s.position, s.n, s.global_n, s.scale))
        viz.close()
    order = S.composite_order(dists)
    stack = torch.from_numpy(np.stack([f.reshape(-1, 4) for f in frames])).cuda()
    comp = S.blend_cuda(stack, order).cpu().numpy().reshape(frames[0].shape)
    assert np.array_equal(comp, O.blend(frames, order))
    assert_image_parity(comp, O.blend(ref_frames, order))
    # against the whole volume in one context
    whole = build_gpu(full)
    ref_full = whole.doVisualization()
    whole.close()
    p = _psnr(comp, ref_full)
    assert p > 45.0, (p, image_diff(comp, ref_full))
    # the order matters: back to front is clearly further from the whole-volume render
    wrong = S.blend_cuda(stack, order[::-1]).cpu().numpy().reshape(frames[0].shape)
    assert _psnr(wrong, ref_full) < p - 3.0
