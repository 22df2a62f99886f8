"""Projection controllers and stereo compositors.

The reference templates ``IsaacVisualization`` on a controller, which gives one
projection per render pass (lib/isaac/isaac_controllers.hpp:23-117), and on a
compositor, which combines the passes' images into the frame that is sent
(lib/isaac/isaac_compositors.hpp:37-116).  The same roles here: a controller
returns ``passCount`` column-major projection matrices; a compositor combines
the passes' RGBA8 frames on the GPU through ``isaacb_composite``.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import check

Z_NEAR, Z_FAR = 0.002, 100.0  # ISAAC_Z_NEAR / ISAAC_Z_FAR (lib/isaac/isaac_defines.hpp:53-54)


def perspective(fovy: float, aspect: float, znear: float, zfar: float) -> np.ndarray:
    """glm::perspective (right-handed, depth -1..1), column-major [col][row]."""
    t = math.tan(fovy / 2.0)
    m = np.zeros((4, 4))
    m[0][0] = 1.0 / (aspect * t)
    m[1][1] = 1.0 / t
    m[2][2] = -(zfar + znear) / (zfar - znear)
    m[2][3] = -1.0
    m[3][2] = -(2.0 * zfar * znear) / (zfar - znear)
    return m


def orthographic(right: float, top: float, znear: float, zfar: float) -> np.ndarray:
    """setOrthographic (lib/isaac/isaac_helper.hpp:328-340), in double."""
    m = np.eye(4)
    m[0][0] = 1.0 / right
    m[1][1] = 1.0 / top
    m[2][2] = -2.0 / (zfar - znear)
    m[3][2] = -(zfar + znear) / (zfar - znear)
    return m


def _frustum(left, right, bottom, top, znear, zfar) -> np.ndarray:
    """setFrustum (lib/isaac/isaac_helper.hpp:266-307): float arithmetic stored as double."""
    f = np.float32
    znear2 = f(znear) * f(2)
    width = f(right) - f(left)
    height = f(top) - f(bottom)
    zrange = f(znear) - f(zfar)
    p = np.zeros(16)
    p[0] = znear2 / width
    p[5] = znear2 / height
    p[8] = (f(right) + f(left)) / width
    p[9] = (f(top) + f(bottom)) / height
    p[10] = (f(zfar) + f(znear)) / zrange
    p[11] = -1.0
    p[14] = (znear2 * f(zfar)) / zrange
    return p.reshape(4, 4)


def perspective_stereoscopic(fovy_degrees, aspect, znear, zfar, z0, distance) -> np.ndarray:
    """spSetPerspectiveStereoscopic (lib/isaac/isaac_helper.hpp:309-325): an off-axis
    frustum for one eye shifted by ``distance``; float arithmetic as the reference."""
    f = np.float32
    # znear * tan(fovy * M_PI / 360): the float operands meet M_PI in double, rounded once to float
    t_z0 = f(float(f(znear)) * math.tan(float(f(fovy_degrees)) * math.pi / 360.0))
    shift = f(distance) / f(2.0) * f(znear) / f(z0)
    m = _frustum(-t_z0 + shift, t_z0 + shift, -t_z0 / f(aspect), t_z0 / f(aspect), znear, zfar)
    m[3][0] += float(f(distance))
    return m


class DefaultController:
    """isaac_controllers.hpp:23-43: perspective(45.0, w/h, Z_NEAR, Z_FAR), with 45.0 in
    radians as glm reads it."""

    passCount = 1

    @staticmethod
    def updateProjection(framebuffer_size) -> np.ndarray:
        w, h = framebuffer_size
        return perspective(45.0, float(w) / float(h), Z_NEAR, Z_FAR)

    @classmethod
    def projections(cls, framebuffer_size) -> list:
        return [cls.updateProjection(framebuffer_size)]

    @staticmethod
    def handleMessage(message: dict) -> bool:
        """Controller-specific keys of a server message; True when the projections changed."""
        return False

    @staticmethod
    def sendFeedback(root: dict, force: bool = False) -> None:
        """Controller state for the period message."""


class OrthoController:
    """isaac_controllers.hpp:45-63: orthographic, right = 2 w/h, top = 2."""

    passCount = 1

    @staticmethod
    def updateProjection(framebuffer_size) -> np.ndarray:
        w, h = framebuffer_size
        return orthographic(float(w) / float(h) * 2.0, 2.0, Z_NEAR, Z_FAR)

    @classmethod
    def projections(cls, framebuffer_size) -> list:
        return [cls.updateProjection(framebuffer_size)]

    handleMessage = DefaultController.handleMessage
    sendFeedback = DefaultController.sendFeedback


class StereoController:
    """isaac_controllers.hpp:65-117: two off-axis frusta (45 degrees, convergence at
    z0 = 5) for eyes at +eyeDistance and -eyeDistance."""

    passCount = 2

    def __init__(self, eye_distance: float = 0.06):
        self.eyeDistance = float(eye_distance)
        self.sendStereo = True

    def handleMessage(self, message: dict) -> bool:
        """"eye distance" sets the eye separation; True while the new projections
        have not been reported (updateProjection, isaac_controllers.hpp:75-101)."""
        if "eye distance" in message:
            self.sendStereo = True
            self.eyeDistance = float(message.pop("eye distance"))
        return self.sendStereo

    def sendFeedback(self, root: dict, force: bool = False) -> None:
        """"eye distance" in the period message after a change or on request."""
        if self.sendStereo or force:
            root["eye distance"] = float(np.float32(self.eyeDistance))  # an isaac_float in the reference
            self.sendStereo = False

    def updateProjection(self, framebuffer_size) -> np.ndarray:
        return self.projections(framebuffer_size)[0]

    def projections(self, framebuffer_size) -> list:
        w, h = framebuffer_size
        aspect = float(np.float32(w) / np.float32(h))
        return [
            perspective_stereoscopic(45.0, aspect, Z_NEAR, Z_FAR, 5.0, self.eyeDistance),
            perspective_stereoscopic(45.0, aspect, Z_NEAR, Z_FAR, 5.0, -self.eyeDistance),
        ]


# ---------------------------------------------------------------------------- compositors
COMPOSITE_FIRST, COMPOSITE_SIDE_BY_SIDE, COMPOSITE_ANAGLYPH = 0, 1, 2


def composite(mode: int, left, right, out=None, left_filter: int = 0, right_filter: int = 0):
    """Combine two (H, W, 4) uint8 CUDA frames: the first, side by side (H, 2W, 4), or an
    anaglyph (each pixel's 32-bit RGBA word masked and OR-ed)."""
    import torch

    h, w, _ = left.shape
    if out is None:
        shape = (h, 2 * w, 4) if mode == COMPOSITE_SIDE_BY_SIDE else (h, w, 4)
        out = torch.empty(shape, dtype=torch.uint8, device=left.device)
    check(
        _lib.load().isaacb_composite(
            int(mode), C.c_void_p(left.data_ptr()), C.c_void_p(right.data_ptr() if right is not None else 0), w, h,
            int(left_filter) & 0xFFFFFFFF, int(right_filter) & 0xFFFFFFFF, C.c_void_p(out.data_ptr()),
            C.c_void_p(torch.cuda.current_stream().cuda_stream),
        )
    )
    return out


class DefaultCompositor:
    """isaac_compositors.hpp:37-52: the first pass's image."""

    @staticmethod
    def size(framebuffer_size):
        return tuple(framebuffer_size)

    def compose(self, images):
        return images[0]


class StereoCompositorSideBySide:
    """isaac_compositors.hpp:54-90: left and right images side by side (2W x H)."""

    @staticmethod
    def size(framebuffer_size):
        return (2 * framebuffer_size[0], framebuffer_size[1])

    def compose(self, images):
        return composite(COMPOSITE_SIDE_BY_SIDE, images[0], images[1])


class StereoCompositorAnaglyph:
    """isaac_compositors.hpp:92-116: per pixel (left & LeftFilter) | (right & RightFilter)
    on the RGBA8 word, red/cyan by default (bytes R, G, B, A from the low end)."""

    def __init__(self, left_filter: int = 0x000000FF, right_filter: int = 0x00FFFF00):
        self.left_filter, self.right_filter = int(left_filter), int(right_filter)

    @staticmethod
    def size(framebuffer_size):
        return tuple(framebuffer_size)

    def compose(self, images):
        return composite(COMPOSITE_ANAGLYPH, images[0], images[1], left_filter=self.left_filter, right_filter=self.right_filter)
