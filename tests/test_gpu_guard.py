"""Volume sources with guard cells (the reference's guardSize: the simulation's
field carries ghost cells around the local volume, and the source's operator[]
reaches them at coordinates -g..L+g-1).  The combined renderer's merge and the
min/max read the interior (lib/isaac/isaac_common_kernel.hpp:690-759,
lib/isaac/isaac_min_max_kernel.hpp:22-60), so the guard cells -- filled here with
noise that would show up if read -- must not change any byte: merged textures and
min/max bit-exact against the oracle reading the same guarded arrays, frames
within the parity bar."""

import numpy as np
import pytest
import torch

from harness import assert_image_parity, build_gpu, build_oracle, gaussian_pair

pytestmark = pytest.mark.gpu


def _pad(a: np.ndarray, g: int, rng) -> np.ndarray:
    """Surround a (Z, Y, X[, C]) array with g cells of large noise on every side."""
    if g == 0:
        return a
    shape = tuple(n + 2 * g for n in a.shape[:3]) + a.shape[3:]
    out = rng.uniform(-50.0, 50.0, shape).astype(np.float32)
    out[g:-g, g:-g, g:-g] = a
    return out


@pytest.mark.parametrize("persistent", [True, False])
@pytest.mark.parametrize("guards", [(2, 1), (1, 3), (0, 2)])
def test_guarded_sources_read_their_interior(guards, persistent):
    rng = np.random.default_rng(sum(guards))
    s = gaussian_pair(n=29, fb=(72, 56), iso=[0.45, 0.0])
    s.volumes = [(_pad(v, g, rng), persistent) for (v, _), g in zip(s.volumes, guards)]
    s.guard = list(guards)
    s.functions = ["mul(1.5)|add(-0.2)", "length"]
    o = build_oracle(s)
    o.update()
    rv, ri = o.combined()
    viz = build_gpu(s)
    viz.update()
    gv, gi = viz.combinedTextures()
    assert np.array_equal(gv, rv) and np.array_equal(gi, ri)
    rmn, rmx = o.minmax()
    gmn, gmx = viz.minMax()
    assert rmn.tobytes() == gmn.tobytes() and rmx.tobytes() == gmx.tobytes()
    got = viz.doVisualization()
    ref = o.frame()
    assert_image_parity(got, ref)
    # the same interior without guard cells renders the same frame
    plain = gaussian_pair(n=29, fb=(72, 56), iso=[0.45, 0.0])
    plain.volumes = [(v, persistent) for v, _ in plain.volumes]
    plain.functions = s.functions
    assert np.array_equal(build_gpu(plain).doVisualization(), got)


def test_guarded_sources_need_the_combined_renderer():
    from isaac_b200 import _lib

    rng = np.random.default_rng(1)
    s = gaussian_pair(n=16)
    s.volumes = [(_pad(v, 1, rng), True) for v, _ in s.volumes]
    s.guard = [1, 1]
    viz = build_gpu(s)
    viz.setRenderOptimization(False)
    with pytest.raises(_lib.IsaacError):
        viz.update()
