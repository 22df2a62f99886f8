"""Ortho and stereo controllers and the GPU compositors against the oracle.

Each pass renders with the controller's projection; the oracle renders the same
camera; the parity bar is the usual one (<= 1 LSB on 99.9 % of pixels, <= 3 LSB
anywhere).  The compositors are byte operations, so they must equal the same
composition done in numpy on the same images."""

import numpy as np
import pytest
import torch

from harness import assert_image_parity, build_oracle, gaussian_pair
from isaac_b200 import controllers as K

pytestmark = pytest.mark.gpu


def _oracle_frame(s, P, MV):
    o = build_oracle(s)
    o.set_camera(P, MV)
    return o.frame()


@pytest.mark.parametrize("mode", ["ortho", "stereo_sbs", "stereo_anaglyph"])
def test_controller_passes_and_compositors(mode):
    s = gaussian_pair(n=32, fb=(64, 48))
    from harness import build_gpu

    viz = build_gpu(s)
    MV = viz.modelview.copy()
    if mode == "ortho":
        viz.controller = K.OrthoController
        viz.projections = K.OrthoController.projections(s.fb)
        viz.compositor = K.DefaultCompositor()
        viz.projection = viz.projections[0]
        viz._push_camera()
        got = viz.doVisualization()
        ref = _oracle_frame(s, viz.projections[0], MV)
        assert_image_parity(got, ref)
        return
    ctrl = K.StereoController(0.08)
    viz.controller = ctrl
    viz.projections = ctrl.projections(s.fb)
    viz.compositor = K.StereoCompositorSideBySide() if mode == "stereo_sbs" else K.StereoCompositorAnaglyph()
    got = viz.doVisualization()
    left = _oracle_frame(s, viz.projections[0], MV)
    right = _oracle_frame(s, viz.projections[1], MV)
    if mode == "stereo_sbs":
        assert got.shape == (48, 128, 4)
        assert_image_parity(got[:, :64], left)
        assert_image_parity(got[:, 64:], right)
    else:
        lw = left.view(np.uint32)[..., 0] & np.uint32(0x000000FF)
        rw = right.view(np.uint32)[..., 0] & np.uint32(0x00FFFF00)
        ref = (lw | rw).view(np.uint8).reshape(48, 64, 4)
        assert_image_parity(got, ref)


def test_composite_kernel_is_bytewise():
    g = torch.Generator().manual_seed(3)
    a = torch.randint(0, 256, (37, 53, 4), dtype=torch.uint8, generator=g)
    b = torch.randint(0, 256, (37, 53, 4), dtype=torch.uint8, generator=g)
    ad, bd = a.cuda(), b.cuda()
    sbs = K.composite(K.COMPOSITE_SIDE_BY_SIDE, ad, bd).cpu()
    assert torch.equal(sbs, torch.cat([a, b], dim=1))
    ana = K.composite(K.COMPOSITE_ANAGLYPH, ad, bd, left_filter=0xFF00FF00, right_filter=0x00FF00FF).cpu().numpy()
    an, bn = a.numpy().view(np.uint32), b.numpy().view(np.uint32)
    assert np.array_equal(ana.view(np.uint32), (an & np.uint32(0xFF00FF00)) | (bn & np.uint32(0x00FF00FF)))
    first = K.composite(K.COMPOSITE_FIRST, ad, None).cpu()
    assert torch.equal(first, a)
