"""Projection controllers (lib/isaac/isaac_controllers.hpp) against values
derived by hand from the reference's helper formulas, and the multi-pass
plumbing of the Python front end (no GPU)."""

import math

import numpy as np

from isaac_b200 import controllers as K


def test_orthographic_matches_set_orthographic():
    # setOrthographic(P, right = 2 w/h, top = 2, near, far) for 800 x 600
    P = K.OrthoController.updateProjection((800, 600))
    assert P[0][0] == 1.0 / (800 / 600 * 2.0) and P[1][1] == 0.5
    assert P[2][2] == -2.0 / (100.0 - 0.002) and P[3][2] == -(100.0 + 0.002) / (100.0 - 0.002)
    assert P[3][3] == 1.0 and P[2][3] == 0.0
    # an orthographic projection maps depth linearly and keeps w = 1
    v = P.T @ np.array([0.3, -0.2, -50.0, 1.0])
    assert v[3] == 1.0


def test_stereo_frustum_values():
    left, right = K.StereoController(0.06).projections((1000, 500))
    f = np.float32
    t = f(float(f(0.002)) * math.tan(45.0 * math.pi / 360.0))
    shift = f(0.06) / f(2.0) * f(0.002) / f(5.0)
    l, r = -t + shift, t + shift
    assert left[0][0] == float((f(0.002) * f(2)) / (r - l))
    assert left[2][0] == float((r + l) / (r - l))  # projection[8]: the off-axis term
    assert left[3][0] == float(f(0.06))  # projection[12] += distance
    assert right[3][0] == float(f(-0.06))
    assert left[2][3] == -1.0 and left[3][3] == 0.0
    # the eyes are mirror images: equal scale, opposite off-axis shift
    assert left[0][0] == right[0][0] and left[2][0] == -right[2][0]


def test_default_controller_is_glm_perspective_in_radians():
    P = K.DefaultController.updateProjection((640, 480))
    t = math.tan(45.0 / 2.0)  # glm reads 45.0 as radians
    assert abs(P[1][1] - 1.0 / t) < 1e-15
    assert K.DefaultController.passCount == 1 and K.StereoController.passCount == 2


def test_compositor_sizes():
    assert K.StereoCompositorSideBySide.size((64, 48)) == (128, 48)
    assert K.StereoCompositorAnaglyph.size((64, 48)) == (64, 48)
    assert K.DefaultCompositor().compose(["a", "b"]) == "a"
