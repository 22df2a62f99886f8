"""Field-source advection against the oracle: the noise texture, the advection
texture over several frames, the merged combined texture (bit-exact) and the
rendered frames (parity bar)."""

import numpy as np
import pytest
import torch

from harness import assert_image_parity, build_gpu, build_oracle, gaussian_pair

pytestmark = pytest.mark.gpu


def _pair(seeds=40, **adv):
    s = gaussian_pair(n=28, fb=(64, 48))  # source 1: the float3 curl field, the last volume source
    viz, o = build_gpu(s), build_oracle(s)
    viz.setFieldSource(1)
    o.set_field(1)
    p = dict(step_factor=1.0, history_weight=0.95, seeding_period=1, seeding_duration=1, seed_points=seeds)
    p.update(adv)
    viz.setAdvection(**p)
    o.set_advection(*p.values())
    return s, viz, o


def test_noise_texture_bit_exact():
    _, viz, o = _pair(seeds=60)
    assert np.array_equal(viz.noiseTexture(), o.noise())


@pytest.mark.parametrize("adv", [dict(), dict(seeding_period=3, seeding_duration=1, history_weight=0.7, step_factor=0.5)])
def test_advection_frames_bit_exact(adv):
    s, viz, o = _pair(**adv)
    for frame in range(4):
        viz.update()
        o.update()
        torch.cuda.synchronize()
        assert np.array_equal(viz.advectionTexture(1), o.advection(1)), frame
        gv, gi = viz.combinedTextures()
        rv, ri = o.combined()
        assert np.array_equal(gv, rv), frame
        assert np.array_equal(gi, ri), frame


def test_advected_frames_match_oracle():
    s, viz, o = _pair(seeds=80)
    for _ in range(3):
        got = viz.doVisualization()
        ref = o.frame()
        assert_image_parity(got, ref)


def test_field_source_rules():
    s = gaussian_pair(n=16)
    viz = build_gpu(s)
    from isaac_b200 import _lib

    with pytest.raises(_lib.IsaacError):
        viz.setFieldSource(0)  # scalar source: not a vector field
    viz.setFieldSource(1)
    viz.setRenderOptimization(False)
    with pytest.raises(_lib.IsaacError):
        viz.update()  # the per-source renderer does not merge field sources
