"""The configurable SSAO tap pattern (no reference counterpart; the full-feature
configuration asks for 16 samples within 8 px).  The reference's 7x7 grid stays the
default and the parity path.  With a pattern set, the AO buffer must equal the
occlusion count over the pattern's taps of the frame's own depth buffer, computed
here in numpy (float32, the same division), and resetting the pattern must restore
the grid's frame exactly."""

import numpy as np
import pytest

from harness import build_gpu, gaussian_pair
from isaac_b200 import scenes

pytestmark = pytest.mark.gpu


def _scene():
    off, pos, attr = scenes.particles_uniform(900, (8, 8, 8), seed=9)
    s = gaussian_pair(n=32, fb=(120, 90), iso=[0.5, 0.0], ao=(True, 0.7, False))
    s.particle_cells = (8, 8, 8)
    s.particles = [(off.numpy(), pos.numpy(), attr.numpy(), None, 0.6)]
    s.functions = ["idem", "length", "length"]
    return s


def _expected_ao(depth: np.ndarray, offsets: np.ndarray) -> np.ndarray:
    H, W = depth.shape
    ys, xs = np.mgrid[0:H, 0:W]
    occ = np.zeros((H, W), dtype=np.float32)
    for dx, dy in offsets:
        x = np.clip(xs + dx, 0, W - 1)
        y = np.clip(ys + dy, 0, H - 1)
        occ += (depth[y, x] < depth).astype(np.float32)
    return np.clip(occ / np.float32(len(offsets) * 42.0 / 48.0), np.float32(0), np.float32(1))


@pytest.mark.parametrize("samples,radius", [(16, 8.0), (32, 20.0), (5, 3.0)])
def test_ao_pattern_matches_its_definition(samples, radius):
    viz = build_gpu(_scene())
    grid = viz.doVisualization()
    viz.setAmbientOcclusionPattern(samples, radius)
    offs = viz.ambientOcclusionPattern()
    assert offs.shape == (samples, 2)
    assert (np.hypot(offs[:, 0], offs[:, 1]) <= radius + 0.75).all()
    got = viz.doVisualization()
    depth, _, ao = viz.gbuffer()
    hit = depth < 1e30
    assert hit.mean() > 0.05
    assert np.array_equal(ao, _expected_ao(depth, offs))
    assert not np.array_equal(got, grid)  # the pattern changes the shading
    viz.setAmbientOcclusionPattern(0)
    assert viz.ambientOcclusionPattern().shape == (0, 2)
    assert np.array_equal(viz.doVisualization(), grid)


def test_ao_pattern_rejects_bad_arguments():
    from isaac_b200 import _lib

    viz = build_gpu(gaussian_pair(n=16))
    for samples, radius in [(33, 8.0), (16, 0.5), (16, 200.0)]:
        with pytest.raises(_lib.IsaacError):
            viz.setAmbientOcclusionPattern(samples, radius)
