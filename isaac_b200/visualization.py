"""Host-side mirror of ISAAC's ``IsaacVisualization`` for the rendering hot path.

The reference class (``lib/isaac.hpp:58-3036``) is a C++ template over source
lists.  This Python class keeps its roles and names -- source objects with
``featureDim``/``persistent``/``getName()``/``update()``, functor-chain strings,
per-source transfer functions, weights, iso thresholds, clipping planes, the
camera (projection, look-at, rotation, distance), ambient occlusion, render and
dither modes -- and drives the sm_100a kernels through the C ABI
(``include/isaac_b200.h``).  Steering messages use the reference's JSON keys
(``lib/isaac.hpp:1345-1803``).  Given a server URL, the object talks the
reference's streaming protocol through ``isaac_b200.protocol`` (register, period
messages with the frame as GPU-encoded JPEG, steering from the server).  The IceT
compositing and MPI are not part of this path.
"""

from __future__ import annotations

import ctypes as C
import math
from typing import Iterable, Sequence

import numpy as np

from . import _lib
from ._lib import check

from .controllers import Z_FAR, Z_NEAR, DefaultCompositor, DefaultController, perspective  # noqa: F401


def _torch():
    import torch

    return torch


def modelview(look_at=(0.0, 0.0, 0.0), rotation=None, distance=-4.5) -> np.ndarray:
    """updateModelview (lib/isaac.hpp:2878-2889): distanceM * rotationM * translationM."""
    rot = np.eye(3) if rotation is None else np.asarray(rotation, dtype=np.float64)
    T = np.eye(4)
    T[3, 0:3] = look_at  # column-major: translation in column 3
    R = np.eye(4)
    R[0:3, 0:3] = rot  # rot given column major [col][row]
    D = np.eye(4)
    D[3][2] = distance
    # column-major product A*B == (B^T A^T)^T with row-major numpy; keep [col][row] storage
    return _cm_mul(_cm_mul(D, R), T)


def _cm_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Product of two column-major [col][row] matrices, returned column-major."""
    return (a.T @ b.T).T


class VolumeSource:
    """A volume source over device memory: ``data`` is a CUDA tensor of shape
    (Z, Y, X, featureDim) or (Z, Y, X), float32, x fastest -- what the reference
    reads through ``operator[]`` (example/example.cpp:36-143).  With ``guard_size``
    g > 0 the tensor holds g guard cells on every side, (Z+2g, Y+2g, X+2g[, f]), as
    a simulation's field with ghost cells does; the combined renderer and min/max
    read its interior."""

    def __init__(self, name: str, data, feature_dim: int | None = None, persistent: bool = True, guard_size: int = 0):
        self._name = name
        self.data = data
        self.featureDim = int(feature_dim if feature_dim is not None else (data.shape[-1] if data.dim() == 4 else 1))
        self.persistent = bool(persistent)
        self.guardSize = int(guard_size)

    def getName(self) -> str:
        return self._name

    def update(self, enabled: bool, pointer=None) -> None:
        """Called before every buffer update, as the reference calls ``source.update``."""


class ParticleSource:
    """A particle source as a cell list (``getIterator`` of example/example.cpp:148-228):
    ``offsets`` (ncells+1, uint32 as int32/int64 tensor), ``positions`` (N,3)
    cell-relative in [0,1), ``attributes`` (N,featureDim), ``radii`` (N) or a constant."""

    def __init__(self, name: str, offsets, positions, attributes, radii=None, radius: float = 0.5):
        self._name = name
        self.offsets = offsets
        self.positions = positions
        self.attributes = attributes
        self.radii = radii
        self.radius = float(radius)
        self.featureDim = int(attributes.shape[1]) if attributes.dim() == 2 else 1

    def getName(self) -> str:
        return self._name

    def update(self, enabled: bool, pointer=None) -> None:
        pass


def _fa(vals) -> C.Array:
    vals = list(vals)
    return (C.c_float * len(vals))(*vals)


class IsaacVisualization:
    """drop-in host object for the rendering path; see the module docstring."""

    def __init__(
        self,
        name: str,
        framebuffer_size: Sequence[int],
        global_size: Sequence[int],
        local_size: Sequence[int],
        local_particle_size: Sequence[int],
        position: Sequence[int],
        volume_sources: Sequence[VolumeSource],
        particle_sources: Sequence[ParticleSource] = (),
        scale: Sequence[float] = (1.0, 1.0, 1.0),
        transfer_size: int = 1024,
        controller=DefaultController,
        compositor=None,
        server_url: str | None = None,
        server_port: int = 2458,
        jpeg: bool = True,
    ):
        self.lib = _lib.load()
        self.name = name
        self.globalSize = tuple(int(v) for v in global_size)
        self.localSize = tuple(int(v) for v in local_size)
        self.framebufferSize = tuple(int(v) for v in framebuffer_size)
        self.volumeSources = list(volume_sources)
        self.particleSources = list(particle_sources)
        self.scale = tuple(float(v) for v in scale)
        self.transferSize = int(transfer_size)
        n_vol, n_part = len(self.volumeSources), len(self.particleSources)
        d = _lib.Desc()
        d.framebuffer[:] = self.framebufferSize
        d.global_size[:] = [int(v) for v in global_size]
        d.local_size[:] = [int(v) for v in local_size]
        d.local_particle_size[:] = [int(v) for v in local_particle_size]
        d.position[:] = [int(v) for v in position]
        d.scale[:] = self.scale
        d.transfer_size = self.transferSize
        d.n_volume_sources = n_vol
        d.n_particle_sources = n_part
        for i, s in enumerate(self.volumeSources + self.particleSources):
            d.feature_dim[i] = s.featureDim
            d.persistent[i] = int(getattr(s, "persistent", True))
            d.guard_size[i] = int(getattr(s, "guardSize", 0))
        self.desc = d
        ctx = C.c_void_p()
        check(self.lib.isaacb_create(C.byref(d), C.byref(ctx)), None)
        self.ctx = ctx
        self.combinedSourceListSize = n_vol + n_part
        n = self.combinedSourceListSize
        # steering state with the reference defaults (lib/isaac.hpp:565-945)
        self.functions = ["idem"] * n
        self.functionErrors = [0] * n
        self.sourceWeight = [2.0] * n
        self.sourceIsoThreshold = [0.0] * n
        self.transferDescription: list[dict[int, tuple]] = [dict() for _ in range(n)]
        self.step = 0.5
        self.interpolation = False
        self.renderOptimization = True
        self.ambientOcclusion = {"isEnabled": False, "weight": 0.5}
        self.renderMode = 0
        self.ditherMode = 1
        self.backgroundColor = [0.0, 0.0, 0.0, 0.0]
        self.clipping: list[tuple] = []
        self.controller = controller
        self.compositor = compositor if compositor is not None else DefaultCompositor()
        # one projection per render pass (two for a stereo controller)
        self.projections = [np.asarray(m, dtype=np.float64) for m in controller.projections(self.framebufferSize)]
        self.projection = self.projections[0]
        self.lookAt = (0.0, 0.0, 0.0)
        self.rotation = np.eye(3)
        self.distance = -4.5
        self.modelview = modelview(self.lookAt, self.rotation, self.distance)
        self.kernelTime = 0.0
        self.mergeTime = 0.0
        self.copyTime = 0.0
        self._frame = None
        self._srcPtrs = [0] * len(self.volumeSources)
        for i, s in enumerate(self.volumeSources):
            check(self.lib.isaacb_set_source(ctx, i, C.c_void_p(s.data.data_ptr())), ctx)
            self._srcPtrs[i] = s.data.data_ptr()
        for j, p in enumerate(self.particleSources):
            self._set_particles(n_vol + j, p)
        self._push_camera()
        # the streaming server (the reference's communicator of the master rank)
        self.communicator = None
        self.session = None
        self.metadata = None
        self._frame_dev = None
        # advection borders between ranks (updateNeighbours; "advection border" defaults on)
        self.fieldSources: set[int] = set()
        self.neighbourNodeIds = [-1] * 27
        self.advectionBorder = True
        self.borderGroup = None
        self._borders = None
        if server_url is not None:
            self.setServer(server_url, server_port, jpeg)

    def setServer(self, url: str, port: int = 2458, jpeg: bool = True):
        """Attach the streaming server (the constructor's server URL and port); ``init``
        then connects and registers."""
        from .protocol import IsaacCommunicator, Session

        self.communicator = IsaacCommunicator(url, port, jpeg)
        self.session = Session(self, self.communicator)

    def init(self, communicator_setting: int = 0) -> int:
        """Connect to the server and register (lib/isaac.hpp:1276-1295): 0, or -1 when
        the connection fails (ReturnAtError = 0; RetryEverySend = 1 keeps retrying on
        each send).  Without a server URL there is nothing to do."""
        if self.session is None:
            return 0
        return self.session.init(communicator_setting)

    def getJsonMetaRoot(self) -> dict:
        """The metadata object sent with the next period message."""
        return self.session.metaRoot if self.session is not None else {}

    def setJpegQuality(self, quality: int):
        if self.communicator is not None:
            self.communicator.setJpegQuality(quality)

    # ------------------------------------------------------------------ lifecycle
    def close(self):
        if getattr(self, "session", None) is not None:
            self.session.exit()
            self.communicator.close()
            self.session = None
        if getattr(self, "ctx", None):
            self.lib.isaacb_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _set_particles(self, idx: int, p: ParticleSource):
        radii = C.c_void_p(p.radii.data_ptr()) if p.radii is not None else None
        check(
            self.lib.isaacb_set_particles(
                self.ctx,
                idx,
                C.c_void_p(p.offsets.data_ptr()),
                C.c_void_p(p.positions.data_ptr()),
                C.c_void_p(p.attributes.data_ptr()),
                radii,
                p.radius,
            ),
            self.ctx,
        )

    # ------------------------------------------------------------------ steering (reference setters)
    def updateFunctions(self) -> list[int]:
        """Parse ``self.functions`` (lib/isaac.hpp:1079-1241); returns the error codes."""
        codes = []
        for i, f in enumerate(self.functions):
            err = C.c_int32(0)
            st = self.lib.isaacb_set_functions(self.ctx, i, f.encode(), C.byref(err))
            if st not in (_lib.OK, _lib.PARSE_ERROR):
                check(st, self.ctx)
            codes.append(int(err.value))
        self.functionErrors = codes
        return codes

    def setTransferPoints(self, src: int, points: dict[int, Sequence[float]]):
        """Replace the control points of one source ("transfer points", lib/isaac.hpp:1591-1612)."""
        self.transferDescription[src] = {int(k): tuple(float(x) for x in v) for k, v in points.items()}
        self.updateTransfer(src)

    def updateTransfer(self, src: int | None = None):
        """Rebuild transfer tables from the control points (lib/isaac.hpp:1244-1266)."""
        srcs = range(self.combinedSourceListSize) if src is None else [src]
        for i in srcs:
            desc = self.transferDescription[i]
            if not desc:
                continue
            keys = (C.c_uint32 * len(desc))(*desc.keys())
            rgba = _fa([c for v in desc.values() for c in v])
            check(self.lib.isaacb_set_transfer(self.ctx, i, len(desc), keys, rgba), self.ctx)

    def getTransfer(self, src: int) -> np.ndarray:
        out = np.zeros((self.transferSize, 4), dtype=np.float32)
        check(self.lib.isaacb_get_transfer(self.ctx, src, out.ctypes.data_as(_lib._fp)), self.ctx)
        return out

    def setWeight(self, src: int, w: float):
        self.sourceWeight[src] = float(w)
        check(self.lib.isaacb_set_weight(self.ctx, src, float(w)), self.ctx)

    def setIsoThreshold(self, src: int, v: float):
        self.sourceIsoThreshold[src] = float(v)
        check(self.lib.isaacb_set_iso_threshold(self.ctx, src, float(v)), self.ctx)

    def setStep(self, step: float):
        self.step = max(float(step), 0.01)
        check(self.lib.isaacb_set_step(self.ctx, self.step), self.ctx)

    def setInterpolation(self, on: bool):
        self.interpolation = bool(on)
        check(self.lib.isaacb_set_interpolation(self.ctx, int(on)), self.ctx)

    def setSlotOrder(self, order: int = -1):
        """Slot order inside the combined texture's bricks: -1 chosen by each merge from its
        camera (textures beyond 4x L2), 0 x fastest, 1 y fastest.  Speed only."""
        check(self.lib.isaacb_set_slot_order(self.ctx, int(order)), self.ctx)

    def setRenderOptimization(self, on: bool):
        self.renderOptimization = bool(on)
        r = _lib.RENDERER_COMBINED if on else _lib.RENDERER_PER_SOURCE
        check(self.lib.isaacb_set_renderer(self.ctx, r), self.ctx)

    def setStorage(self, src: int, dtype: int):
        check(self.lib.isaacb_set_storage(self.ctx, src, int(dtype)), self.ctx)

    def setAmbientOcclusion(self, enabled: bool, weight: float = 0.5, filter: bool = False):
        self.ambientOcclusion = {"isEnabled": bool(enabled), "weight": float(weight)}
        check(self.lib.isaacb_set_ao(self.ctx, int(enabled), float(weight), int(filter)), self.ctx)

    def setAmbientOcclusionPattern(self, samples: int = 0, radius: float = 8.0):
        """SSAO taps (no reference counterpart): 0 = the reference's 7x7 grid 10 px apart;
        1..32 samples on a golden-angle spiral within ``radius`` pixels."""
        check(self.lib.isaacb_set_ao_pattern(self.ctx, int(samples), float(radius)), self.ctx)

    def ambientOcclusionPattern(self) -> np.ndarray:
        """The (x, y) pixel offsets of the SSAO taps, shape (samples, 2); empty for the grid."""
        n = C.c_uint32(0)
        check(self.lib.isaacb_get_ao_pattern(self.ctx, C.byref(n), None), self.ctx)
        out = np.zeros(2 * max(n.value, 1), dtype=np.int32)
        check(self.lib.isaacb_get_ao_pattern(self.ctx, C.byref(n), C.c_void_p(out.ctypes.data)), self.ctx)
        return out[: 2 * n.value].reshape(-1, 2)

    def setRenderMode(self, mode: int):
        self.renderMode = int(mode)
        check(self.lib.isaacb_set_render_mode(self.ctx, int(mode)), self.ctx)

    def setDitherMode(self, mode: int):
        self.ditherMode = int(mode)
        check(self.lib.isaacb_set_dither_mode(self.ctx, int(mode)), self.ctx)

    # ------------------------------------------------------------------ field sources and advection
    def setFieldSource(self, src: int, enabled: bool = True):
        """Make volume source ``src`` (a float3 vector field, after every plain volume
        source) an advected field source (the reference's FieldSourceList)."""
        check(self.lib.isaacb_set_field_source(self.ctx, int(src), int(enabled)), self.ctx)
        if enabled:
            self.fieldSources.add(int(src))
        else:
            self.fieldSources.discard(int(src))

    def setAdvection(self, step_factor=1.0, history_weight=0.95, seeding_period=1, seeding_duration=1, seed_points=1000):
        """The "advection step", "advection weight", "advection seeding period",
        "advection seeding duration" and "seed points" settings (lib/isaac.hpp:1636-1662)."""
        self.advection = dict(step=step_factor, weight=history_weight, period=seeding_period,
                              duration=seeding_duration, seeds=seed_points)
        check(self.lib.isaacb_set_advection(self.ctx, float(step_factor), float(history_weight), int(seeding_period),
                                             int(seeding_duration), int(seed_points)), self.ctx)

    # ------------------------------------------------------------------ advection borders between ranks
    def updateNeighbours(self, neighbours):
        """The ranks of the 26 neighbouring sub-volumes (index = the reference's direction
        index, -1 for none; lib/isaac.hpp:1049-1053).  With a process group (``group``,
        or the default one) the advection borders are exchanged with them every frame."""
        self.neighbourNodeIds = [int(v) for v in neighbours]

    def setAdvectionBorder(self, enabled: bool):
        """The "advection border" key: off clears the advection textures and stops the exchange."""
        self.advectionBorder = bool(enabled)
        if not enabled:
            check(self.lib.isaacb_clear_advection(self.ctx, self._stream()), self.ctx)

    def advectionGuard(self) -> tuple:
        g = (C.c_uint32 * 3)()
        check(self.lib.isaacb_advection_guard(self.ctx, g), self.ctx)
        return tuple(int(v) for v in g)

    def advect(self):
        """The advection step alone; the next update merges without advecting again."""
        check(self.lib.isaacb_advect(self.ctx, self._stream()), self.ctx)

    def packGuard(self, src: int, direction: int, out):
        check(self.lib.isaacb_pack_guard(self.ctx, int(src), int(direction), C.c_void_p(out.data_ptr()), self._stream()),
              self.ctx)

    def unpackGuard(self, src: int, direction: int, data):
        check(self.lib.isaacb_unpack_guard(self.ctx, int(src), int(direction), C.c_void_p(data.data_ptr()),
                                           self._stream()), self.ctx)

    def _exchange_borders(self):
        """Advect and swap guard slabs with the neighbour ranks (lib/isaac.hpp:1856-1913)."""
        if not any(n >= 0 for n in self.neighbourNodeIds[1:]) or not self.advectionBorder or not self.fieldSources:
            return
        if self._borders is None:
            from .borders import AdvectionBorders

            self._borders = AdvectionBorders.for_visualization(self, self.neighbourNodeIds, self.borderGroup)
        self._borders.neighbours = list(self.neighbourNodeIds)
        self.advect()
        for s in sorted(self.fieldSources):
            if self.sourceWeight[s] != 0 or self.sourceIsoThreshold[s] != 0:
                self._borders.exchange(s)

    def advectionTexture(self, src: int) -> np.ndarray:
        lx, ly, lz = (int(v) for v in self.desc.local_size)
        out = np.empty((lz, ly, lx), dtype=np.uint8)
        check(self.lib.isaacb_get_advection(self.ctx, self._stream(), int(src), C.c_void_p(out.ctypes.data)), self.ctx)
        return out

    def noiseTexture(self) -> np.ndarray:
        lx, ly, lz = (int(v) for v in self.desc.local_size)
        out = np.empty((lz, ly, lx), dtype=np.float32)
        check(self.lib.isaacb_get_noise(self.ctx, self._stream(), out.ctypes.data_as(_lib._fp)), self.ctx)
        return out

    def setBackgroundColor(self, rgba: Sequence[float]):
        self.backgroundColor = [float(v) for v in rgba]
        check(self.lib.isaacb_set_background(self.ctx, _fa(self.backgroundColor)), self.ctx)

    def editClipping(self, nr: int, px, py, pz, nx, ny, nz) -> bool:
        st = self.lib.isaacb_edit_clipping(self.ctx, int(nr), _fa([px, py, pz]), _fa([nx, ny, nz]))
        if st == _lib.OK and nr < len(self.clipping):
            self.clipping[nr] = (px, py, pz, nx, ny, nz)
        return st == _lib.OK

    def addClipping(self, px, py, pz, nx, ny, nz) -> bool:
        st = self.lib.isaacb_add_clipping(self.ctx, _fa([px, py, pz]), _fa([nx, ny, nz]))
        if st == _lib.OK:
            self.clipping.append((px, py, pz, nx, ny, nz))
        return st == _lib.OK

    def removeClipping(self, nr: int):
        if 0 <= nr < len(self.clipping):
            check(self.lib.isaacb_remove_clipping(self.ctx, int(nr)), self.ctx)
            del self.clipping[nr]

    # ------------------------------------------------------------------ camera
    def setCamera(self, projection: np.ndarray, modelview_m: np.ndarray):
        """Explicit projection and modelview, column-major [col][row] doubles."""
        self.projection = np.asarray(projection, dtype=np.float64)
        self.projections = [self.projection] + self.projections[1:]
        self.modelview = np.asarray(modelview_m, dtype=np.float64)
        self._push_camera()

    def updateModelview(self):
        self.modelview = modelview(self.lookAt, self.rotation, self.distance)
        self._push_camera()

    def _push_camera(self):
        p = np.ascontiguousarray(self.projection, dtype=np.float64).reshape(16)
        m = np.ascontiguousarray(self.modelview, dtype=np.float64).reshape(16)
        check(
            self.lib.isaacb_set_camera(self.ctx, p.ctypes.data_as(_lib._dp), m.ctypes.data_as(_lib._dp)),
            self.ctx,
        )

    # ------------------------------------------------------------------ JSON steering (reference keys)
    def steer(self, message: dict):
        """Apply a steering message with the reference's keys (lib/isaac.hpp:1560-1795)."""
        if "projection" in message:
            self.projection = np.asarray(message["projection"], dtype=np.float64).reshape(4, 4)
            self._push_camera()
        if "modelview" in message:
            self.modelview = np.asarray(message["modelview"], dtype=np.float64).reshape(4, 4)
            self._push_camera()
        if "look at" in message:
            self.lookAt = tuple(message["look at"])
            self.updateModelview()
        if "rotation" in message:
            self.rotation = np.asarray(message["rotation"], dtype=np.float64).reshape(3, 3)
            self.updateModelview()
        if "distance" in message:
            self.distance = float(message["distance"])
            self.updateModelview()
        if "transfer points" in message:
            for i, pts in enumerate(message["transfer points"]):
                self.setTransferPoints(i, {int(p["value"]): (p["r"], p["g"], p["b"], p["a"]) for p in pts})
        if "interpolation" in message:
            self.setInterpolation(bool(message["interpolation"]))
        if "render optimization" in message:
            self.setRenderOptimization(bool(message["render optimization"]))
        if "step" in message:
            self.setStep(float(message["step"]))
        if "iso threshold" in message:
            for i, v in enumerate(message["iso threshold"]):
                self.setIsoThreshold(i, v)
        if "functions" in message:
            for i, f in enumerate(message["functions"]):
                self.functions[i] = str(f)
            self.updateFunctions()
        if "weight" in message:
            for i, v in enumerate(message["weight"]):
                self.setWeight(i, v)
        if "background color" in message and len(message["background color"]) == 3:
            self.setBackgroundColor(list(message["background color"]) + [self.backgroundColor[3]])
        if "clipping add" in message:
            c = message["clipping add"]
            self.addClipping(*c["position"], *c["normal"])
        if "clipping remove" in message:
            self.removeClipping(int(message["clipping remove"]))
        keys = {"advection step": "step", "advection weight": "weight", "advection seeding period": "period",
                "advection seeding duration": "duration", "seed points": "seeds"}
        if any(k in message for k in keys):
            a = dict(getattr(self, "advection", dict(step=1.0, weight=0.95, period=1, duration=1, seeds=1000)))
            for k, name in keys.items():
                if k in message:
                    a[name] = message[k]
            if "seed points" in message:
                a["seeds"] = max(int(a["seeds"]), 0)
            self.setAdvection(a["step"], a["weight"], a["period"], a["duration"], a["seeds"])
        if "advection border" in message:
            self.setAdvectionBorder(bool(message["advection border"]))
        if "clipping edit" in message:
            c = message["clipping edit"]
            self.editClipping(int(c["nr"]), *c["position"], *c["normal"])
        if "ao" in message:
            a = message["ao"]
            self.setAmbientOcclusion(bool(a.get("isEnabled", False)), float(a.get("weight", 0.5)))
        if "render mode" in message:
            self.setRenderMode(int(message["render mode"]["mode"]))
        if "dither mode" in message:
            self.setDitherMode(int(message["dither mode"]["mode"]))

    # ------------------------------------------------------------------ per frame
    def _sync_source_pointers(self):
        """A source whose ``update`` hook replaced its ``data`` (another buffer of the
        same shape, e.g. double-buffered inputs) is read from the new memory."""
        for i, s in enumerate(self.volumeSources):
            ptr = s.data.data_ptr()
            if ptr != self._srcPtrs[i]:
                check(self.lib.isaacb_set_source(self.ctx, i, C.c_void_p(ptr)), self.ctx)
                self._srcPtrs[i] = ptr

    def _stream(self):
        return C.c_void_p(_torch().cuda.current_stream().cuda_stream)

    def doVisualization(self, pointer=None, redraw: bool = True, host: bool = True, out=None, timing: bool = False):
        """One frame: the sources' ``update`` hooks, buffer update, draw and readback
        (lib/isaac.hpp:1298-2104 with drawCallBack).

        With ``host`` the frame comes back as an (H, W, 4) uint8 numpy array
        (row 0 = bottom) through one synchronous ``isaacb_frame`` call; else it
        is written to a (H, W, 4) uint8 CUDA tensor and the call stays
        asynchronous.  ``timing`` records ``mergeTime`` / ``kernelTime`` (ms)
        with CUDA events, like the reference's per-phase counters.
        """
        if self.session is not None:
            # the server's messages first, then the frame, then the period message
            # carrying it (lib/isaac.hpp:1345-1800, 2546-2856)
            message, asked = self.session.receive()
            redraw = self.session.apply(message) or asked or redraw
            self.metadata = message.get("metadata")
            frame = self._draw(pointer, redraw, host, out, timing, device_frame=True)
            self.session.send_period(self._frame_dev)
            return frame
        return self._draw(pointer, redraw, host, out, timing)

    def _draw(self, pointer, redraw, host, out, timing, device_frame=False):
        for i, s in enumerate(self.volumeSources):
            s.update(self.sourceWeight[i] != 0 or self.sourceIsoThreshold[i] != 0, pointer)
        for j, p in enumerate(self.particleSources):
            p.update(self.sourceWeight[len(self.volumeSources) + j] != 0, pointer)
        self._sync_source_pointers()
        if not redraw:
            return self._frame
        w, h = self.framebufferSize
        st = self._stream()
        self._exchange_borders()
        if len(self.projections) > 1 or not isinstance(self.compositor, DefaultCompositor):
            return self._multi_pass(host, st)
        if host and not timing and not device_frame:
            if out is None:
                out = np.empty((h, w, 4), dtype=np.uint8)
            check(self.lib.isaacb_frame(self.ctx, st, C.c_void_p(out.ctypes.data)), self.ctx)
            self._frame = out
            return out
        torch = _torch()
        dev = torch.empty((h, w, 4), dtype=torch.uint8, device="cuda") if (host or out is None) else out
        if timing:
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
        check(self.lib.isaacb_update(self.ctx, st), self.ctx)
        if timing:
            e1.record()
        check(self.lib.isaacb_render(self.ctx, st, C.c_void_p(dev.data_ptr())), self.ctx)
        if timing:
            e2.record()
            e2.synchronize()
            self.mergeTime = e0.elapsed_time(e1)
            self.kernelTime = e1.elapsed_time(e2)
        self._frame_dev = dev
        result = dev.cpu().numpy() if host else dev
        self._frame = result
        return result

    def _multi_pass(self, host: bool, st):
        """One render per controller pass (lib/isaac.hpp:2008-2061) with the pass's
        projection and the common modelview, then the compositor on the GPU."""
        torch = _torch()
        w, h = self.framebufferSize
        check(self.lib.isaacb_update(self.ctx, st), self.ctx)
        m = np.ascontiguousarray(self.modelview, dtype=np.float64).reshape(16)
        images = []
        for proj in self.projections:
            pp = np.ascontiguousarray(proj, dtype=np.float64).reshape(16)
            check(self.lib.isaacb_set_camera(self.ctx, pp.ctypes.data_as(_lib._dp), m.ctypes.data_as(_lib._dp)), self.ctx)
            img = torch.empty((h, w, 4), dtype=torch.uint8, device="cuda")
            check(self.lib.isaacb_render(self.ctx, st, C.c_void_p(img.data_ptr())), self.ctx)
            images.append(img)
        self._push_camera()
        frame = self.compositor.compose(images)
        self._frame_dev = frame
        result = frame.cpu().numpy() if host else frame
        self._frame = result
        return result

    def update(self):
        """Buffer update only (merge / per-source bricks), asynchronous; with neighbour
        ranks the advection borders are exchanged first."""
        self._sync_source_pointers()
        self._exchange_borders()
        check(self.lib.isaacb_update(self.ctx, self._stream()), self.ctx)

    def render(self, out=None):
        """Draw only, asynchronous; optionally copies the frame into the CUDA tensor ``out``."""
        ptr = C.c_void_p(out.data_ptr()) if out is not None else None
        check(self.lib.isaacb_render(self.ctx, self._stream(), ptr), self.ctx)

    def minMax(self) -> tuple[np.ndarray, np.ndarray]:
        """"minmax" request (lib/isaac.hpp:1951-2006): per-source min and max after the functor chain."""
        n = self.combinedSourceListSize
        mn = np.zeros(n, dtype=np.float32)
        mx = np.zeros(n, dtype=np.float32)
        check(self.lib.isaacb_minmax(self.ctx, self._stream(), mn.ctypes.data_as(_lib._fp), mx.ctypes.data_as(_lib._fp)), self.ctx)
        return mn, mx

    # ------------------------------------------------------------------ diagnostics
    def gbuffer(self):
        w, h = self.framebufferSize
        depth = np.zeros((h, w), dtype=np.float32)
        normal = np.zeros((h, w, 3), dtype=np.float32)
        ao = np.zeros((h, w), dtype=np.float32)
        check(
            self.lib.isaacb_get_gbuffer(
                self.ctx, self._stream(), C.c_void_p(depth.ctypes.data), C.c_void_p(normal.ctypes.data), C.c_void_p(ao.ctypes.data)
            ),
            self.ctx,
        )
        return depth, normal, ao

    def combinedTextures(self):
        lx, ly, lz = (int(v) for v in self.desc.local_size)
        vol = np.zeros((lz, ly, lx, 4), dtype=np.uint8)
        iso = np.zeros((lz, ly, lx, 4), dtype=np.uint8)
        check(
            self.lib.isaacb_get_combined(self.ctx, self._stream(), C.c_void_p(vol.ctypes.data), C.c_void_p(iso.ctypes.data)),
            self.ctx,
        )
        return vol, iso

    def setCounting(self, on: bool):
        check(self.lib.isaacb_set_counting(self.ctx, int(on)), self.ctx)

    def setTiming(self, on: bool):
        check(self.lib.isaacb_set_timing(self.ctx, int(on)), self.ctx)

    def timings(self) -> dict:
        """Milliseconds per phase of the last update + render (CUDA events on the launch stream)."""
        ms = (C.c_float * _lib.TIMING_SLOTS)()
        check(self.lib.isaacb_get_timing(self.ctx, self._stream(), ms), self.ctx)
        return dict(zip(_lib.TIMING_NAMES, [float(v) for v in ms]))

    def launchCounts(self) -> tuple[int, int]:
        u = C.c_uint32(0)
        r = C.c_uint32(0)
        check(self.lib.isaacb_get_launch_count(self.ctx, C.byref(u), C.byref(r)), self.ctx)
        return int(u.value), int(r.value)

    def counters(self) -> tuple[int, int]:
        v = C.c_uint64(0)
        i = C.c_uint64(0)
        check(self.lib.isaacb_get_counters(self.ctx, self._stream(), C.byref(v), C.byref(i)), self.ctx)
        return int(v.value), int(i.value)


