"""The streaming-server side of ``IsaacVisualization``: frame output and the JSON protocol.

* ``FrameEncoder`` wraps the GPU encoder of ``include/isaac_b200.h``
  (``isaacb_encode_frame``): a device RGBA8 frame becomes the payload message
  ``{"payload": "data:image/jpeg;base64,..."}`` that
  ``IsaacCommunicator::serverSendFrame`` builds on the host with libjpeg and boost
  (lib/isaac/isaac_communicator.hpp:214-290).
* ``IsaacCommunicator`` is the reference's TCP client
  (lib/isaac/isaac_communicator.hpp:44-362): connect, the ``{"uid": n, ...} ``
  message framing with at most ``ISAAC_MAX_DIFFERENCE`` messages ahead of the
  server's ``done`` acknowledgements, the register message re-sent after a
  reconnect, and a reader thread that queues the server's messages.
* The message builders and ``Session`` follow ``IsaacVisualization``: the
  register message (lib/isaac.hpp:833-891), the per-frame handling of requests
  and camera changes (lib/isaac.hpp:1345-1560), the ``send*`` flags the steering
  keys raise (lib/isaac.hpp:1560-1795), the period message (lib/isaac.hpp:2546-2846)
  and the exit message (lib/isaac.hpp:2110-2118).

JSON text is produced by ``json.dumps`` with its default separators (``", "`` and
``": "``, the form of ``json_dumps(..., 0)``), keys in insertion order.
"""

from __future__ import annotations

import copy
import ctypes as C
import json
import math
import socket
import sys
import threading
import time

import numpy as np

from . import _lib
from ._lib import check

# CommunicatorSetting (lib/isaac/isaac_communicator.hpp:38-42)
ReturnAtError, RetryEverySend = 0, 1
# IsaacVisualizationMetaEnum (lib/isaac/isaac_types.hpp)
META_NONE, META_MERGE, META_MASTER = 0, 1, 2
ISAAC_MAX_DIFFERENCE = 4  # lib/isaac/isaac_defines.hpp:23-25
ISAAC_MAX_FUNCTORS = 3  # lib/isaac/isaac_defines.hpp:27-29
PROTOCOL_VERSION = (1, 0)  # lib/isaac/isaac_version.hpp:7-8

# the functor pool in its order, with the names, descriptions and parameter use the
# register message announces (lib/isaac/isaac_functors.hpp:42-208)
FUNCTORS = [
    ("idem", "Does nothing. Keeps the feature dimension.", False),
    ("add", "Summarizes the input with a constant parameter. Keeps the feature dimension.", True),
    ("mul", "Multiplies the input with a constant parameter. Keeps the feature dimension.", True),
    ("length", "Calculates the length of an input. Reduces the feature dimension to 1.", False),
    ("pow", "Calculates the power of the input with a constant exponent. Keeps the feature dimension.", True),
    ("sum", "Calculates the sum of all components. Reduces the feature dimension to 1.", False),
]


def _stream_ptr():
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class FrameEncoder:
    """GPU frame encoder: JPEG (nvJPEG) or raw RGBA, base64 as boost writes it."""

    def __init__(self, quality: int = 90):
        self.lib = _lib.load()
        h = C.c_void_p()
        check(self.lib.isaacb_encoder_create(C.byref(h)))
        self.handle = h
        self.setQuality(quality)

    def setQuality(self, quality: int):
        check(self.lib.isaacb_encoder_set_quality(self.handle, max(int(quality), 0)))

    @property
    def quality(self) -> int:
        q = C.c_uint32()
        check(self.lib.isaacb_encoder_get_quality(self.handle, C.byref(q)))
        return int(q.value)

    def jpeg(self, frame) -> bytes:
        """JPEG bytes of a (H, W, 4) uint8 CUDA frame, rows in memory order."""
        h, w, _ = frame.shape
        ptr, n = C.c_void_p(), C.c_size_t()
        check(self.lib.isaacb_encode_jpeg(self.handle, C.c_void_p(frame.data_ptr()), w, h, _stream_ptr(), C.byref(ptr),
                                          C.byref(n)))
        return C.string_at(ptr.value, n.value)

    def message(self, frame, jpeg: bool = True) -> bytes:
        """The payload message of serverSendFrame for a (H, W, 4) uint8 CUDA frame."""
        h, w, _ = frame.shape
        ptr, n = C.c_void_p(), C.c_size_t()
        check(self.lib.isaacb_encode_frame(self.handle, C.c_void_p(frame.data_ptr()), w, h, int(bool(jpeg)), _stream_ptr(),
                                           C.byref(ptr), C.byref(n)))
        return C.string_at(ptr.value, n.value)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.isaacb_encoder_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def base64_device(data) -> bytes:
    """base64 text of a 1-D uint8 CUDA tensor, computed by the encoder's kernel."""
    import torch

    n = int(data.numel())
    out = torch.empty((n * 8 + 5) // 6, dtype=torch.uint8, device=data.device)
    check(_lib.load().isaacb_base64(C.c_void_p(data.data_ptr()), n, C.c_void_p(out.data_ptr()), _stream_ptr()))
    return bytes(out.cpu().numpy())


class IsaacCommunicator:
    """TCP client of the ISAAC server (lib/isaac/isaac_communicator.hpp:44-362)."""

    def __init__(self, url: str, port: int, jpeg: bool = True):
        self.url = url
        self.port = int(port)
        self.jpeg = bool(jpeg)
        self.id = 0
        self.server_id = 0
        self.sock: socket.socket | None = None
        self.closed = False  # the server refused the protocol: no reconnects
        self.registerMessage: dict | None = None
        self.messageList: list = []
        self._lock = threading.Lock()
        self._reader: threading.Thread | None = None
        self.encoder: FrameEncoder | None = None
        self.jpeg_quality = 90

    # ------------------------------------------------------------ connection
    def serverConnect(self, setting: int = ReturnAtError) -> int:
        """0 on success; -1 unresolvable host, -2 no socket, -3 refused connection
        (ReturnAtError); with RetryEverySend every failure returns 1 instead."""
        try:
            addr = socket.gethostbyname(self.url)
        except OSError:
            if setting == ReturnAtError:
                print(f"Could not resolve {self.url}.", file=sys.stderr)
                return -1
            return 1
        try:
            s = socket.socket(socket.AF_INET, socket.SOCK_STREAM)
        except OSError:
            if setting == ReturnAtError:
                print("Could not create socket.", file=sys.stderr)
                return -2
            return 1
        try:
            s.connect((addr, self.port))
        except OSError:
            s.close()
            if setting == ReturnAtError:
                print(f"Could not connect to {self.url}.", file=sys.stderr)
                return -3
            return 1
        s.setsockopt(socket.IPPROTO_TCP, socket.TCP_NODELAY, 1)
        self.sock = s
        self._reader = threading.Thread(target=self._read_messages, args=(s,), daemon=True)
        self._reader.start()
        return 0

    def serverDisconnect(self):
        if self.sock is not None:
            try:
                self.sock.shutdown(socket.SHUT_RDWR)
            except OSError:
                pass
            self.sock.close()
            self.sock = None

    def close(self):
        self.serverDisconnect()
        if self._reader is not None:
            self._reader.join(timeout=1.0)
            self._reader = None
        if self.encoder is not None:
            self.encoder.close()
            self.encoder = None

    # ------------------------------------------------------------ sending
    def _lost(self):
        """A failed send (ISAAC_HANDLE_EPIPE): the connection counts as lost and
        the next send reconnects."""
        s, self.sock = self.sock, None
        if s is not None:
            s.close()
        if self._reader is not None:
            self._reader.join(timeout=1.0)
            self._reader = None

    def _send(self, data: bytes) -> int:
        try:
            self.sock.sendall(data)
        except OSError:
            self._lost()
            return -1
        return len(data)

    def serverSend(self, content, starting: bool = True, finishing: bool = False) -> int:
        """Send one message part: with ``starting`` the ``{"uid": n`` opener (waiting,
        up to 1 s, while more than ISAAC_MAX_DIFFERENCE messages are unacknowledged);
        then ``content`` (a JSON object's text) with its braces turned into a
        continuation; with ``finishing`` the closing ``} ``.  Returns bytes sent."""
        if self.closed:
            return 0
        if self.sock is None:  # connection lost or never made: retry, then re-register
            if self.serverConnect(RetryEverySend):
                return 0
            if self.registerMessage is not None:
                self.serverSend(json.dumps(self.registerMessage), True, True)
        n = 0
        if starting:
            c = 0
            while self.id > self.server_id + ISAAC_MAX_DIFFERENCE:
                time.sleep(0.001)
                c += 1
                if c > 1000:
                    self.id = self.server_id - 1
                    break
            add = self._send(b'{"uid": %d' % self.id)
            if add < 0:
                return n
            n += add
            self.id += 1
        if content is not None:
            text = content.encode() if isinstance(content, str) else bytes(content)
            add = self._send(b"," + text[1:-1])
            if add < 0:
                return n
            n += add
        if finishing:
            add = self._send(b"} ")
            if add < 0:
                return n
            n += add
        return n

    def serverSendRegister(self, message: dict) -> int:
        self.registerMessage = message
        return self.serverSend(json.dumps(message), True, True)

    def setJpegQuality(self, quality: int):
        self.jpeg_quality = min(int(quality), 100)
        if self.encoder is not None:
            self.encoder.setQuality(self.jpeg_quality)

    def serverSendFrame(self, frame, width: int | None = None, height: int | None = None, depth: int = 4) -> int:
        """Finish the current message with the frame's payload (a (H, W, 4) uint8 CUDA tensor)."""
        if self.encoder is None:
            self.encoder = FrameEncoder(self.jpeg_quality)
        msg = self.encoder.message(frame, self.jpeg)
        return self.serverSend(msg, False, True)

    # ------------------------------------------------------------ receiving
    def getLastMessage(self):
        with self._lock:
            return self.messageList.pop(0) if self.messageList else None

    def setMessage(self, content: dict):
        with self._lock:
            self.messageList.append(content)

    def _read_messages(self, s: socket.socket):
        """Reader thread: one JSON object after another from the stream.  ``fatal
        error`` is printed (``protocol mismatch`` also ends the connection for good),
        ``done`` advances the acknowledged id, anything else is queued."""
        dec = json.JSONDecoder()
        buf = b""
        while True:
            try:
                chunk = s.recv(65536)
            except OSError:
                return
            if not chunk:
                return
            buf += chunk
            while True:
                text_bytes = buf.lstrip()
                if not text_bytes:
                    buf = b""
                    break
                try:
                    text = text_bytes.decode("utf-8")
                except UnicodeDecodeError as e:
                    text = text_bytes[: e.start].decode("utf-8")
                try:
                    obj, end = dec.raw_decode(text)
                except json.JSONDecodeError:
                    buf = text_bytes
                    break
                buf = text_bytes[len(text[:end].encode("utf-8")):]
                if not isinstance(obj, dict):
                    continue
                if "fatal error" in obj:
                    print(f'Fatal error: "{obj["fatal error"]}".', file=sys.stderr)
                    if obj["fatal error"] == "protocol mismatch":
                        self.closed = True
                        try:
                            s.close()
                        except OSError:
                            pass
                        return
                elif "done" in obj:
                    try:
                        done = int(obj["done"])
                    except (TypeError, ValueError):
                        done = 0
                    if done > self.server_id:
                        self.server_id = done
                else:
                    self.setMessage(obj)


# ---------------------------------------------------------------------------- messages
def merge_json(result: dict, candidate: dict) -> None:
    """mergeJSON (lib/isaac/isaac_helper.hpp:173-226): metadata arrays are extended,
    other metadata values and every other key take the candidate's value."""
    mc, mr = candidate.get("metadata"), result.get("metadata")
    if isinstance(mc, dict) and isinstance(mr, dict):
        for k, v in mc.items():
            if isinstance(mr.get(k), list) and isinstance(v, list):
                mr[k].extend(v)
            else:
                mr[k] = v
    for k, v in candidate.items():
        if k == "metadata" and "metadata" in result:
            continue
        result[k] = v


def _flat(m) -> list:
    return [float(v) for v in np.asarray(m, dtype=np.float64).reshape(-1)]


def register_message(viz, nodes: int = 1) -> dict:
    """The register message (lib/isaac.hpp:833-891)."""
    fb = viz.compositor.size(viz.framebufferSize)
    sources = [{"name": s.getName(), "feature dimension": int(s.featureDim)} for s in viz.volumeSources]
    sources += [{"name": p.getName(), "feature dimension": int(p.featureDim)} for p in viz.particleSources]
    scaled = [int(g * s) for g, s in zip(viz.globalSize, viz.scale)]
    return {
        "type": "register",
        "name": viz.name,
        "nodes": int(nodes),
        "framebuffer width": int(fb[0]),
        "framebuffer height": int(fb[1]),
        "max functors": ISAAC_MAX_FUNCTORS,
        "functors": [{"name": n, "description": d, "uses parameter": u} for n, d, u in FUNCTORS],
        "projection count": len(viz.projections),
        "projection": sum((_flat(p) for p in viz.projections), []),
        "position": [float(v) for v in viz.lookAt],
        "rotation": _flat(viz.rotation),
        "distance": float(viz.distance),
        "sources": sources,
        "interpolation": bool(viz.interpolation),
        "step": float(viz.step),
        "dimension": 3,
        "width": scaled[0],
        "height": scaled[1],
        "depth": scaled[2],
        "protocol": list(PROTOCOL_VERSION),
        "ao isEnabled": bool(viz.ambientOcclusion["isEnabled"]),
        "ao weight": float(viz.ambientOcclusion["weight"]),
    }


# requests a client can send, and the send flags each raises (lib/isaac.hpp:1369-1444)
_REQUESTS = {
    "rotation": ["rotation"],
    "position": ["position"],
    "distance": ["distance"],
    "projection": ["projection"],
    "transfer": ["transfer"],
    "interpolation": ["interpolation"],
    "step": ["step"],
    "iso threshold": ["iso threshold"],
    "functions": ["functions"],
    "weight": ["weight"],
    "background color": ["background color"],
    "clipping": ["clipping"],
    "controller": ["controller"],
    "init": ["init"],
    "ao": ["ao"],
    "start observing": [
        "transfer", "functions", "weight", "iso threshold", "clipping", "controller", "interpolation",
        "render optimization", "step", "seed points", "advection step", "advection weight",
        "advection seeding period", "advection seeding duration", "advection on pause", "advection border",
        "background color", "ao", "render mode", "dither mode",
    ],
}

# steering keys and the send flag each raises when applied (lib/isaac.hpp:1590-1795)
_STEER_FLAGS = {
    "transfer points": "transfer",
    "interpolation": "interpolation",
    "render optimization": "render optimization",
    "step": "step",
    "seed points": "seed points",
    "advection step": "advection step",
    "advection weight": "advection weight",
    "advection seeding period": "advection seeding period",
    "advection seeding duration": "advection seeding duration",
    "advection on pause": "advection on pause",
    "advection border": "advection border",
    "iso threshold": "iso threshold",
    "functions": "functions",
    "weight": "weight",
    "background color": "background color",
    "clipping add": "clipping",
    "clipping remove": "clipping",
    "clipping edit": "clipping",
    "ao": "ao",
    "render mode": "render mode",
    "dither mode": "dither mode",
}


def rotation_about(axis, degrees: float) -> np.ndarray:
    """The rotation by ``degrees`` about ``axis`` (normalised), column-major [col][row]:
    Rodrigues' formula R = cos a I + sin a [u]x + (1 - cos a) u u^T, the matrix
    glm::rotate builds (lib/isaac.hpp:1478-1491)."""
    u = np.asarray(axis, dtype=np.float64)
    u = u / math.sqrt(float(u @ u))
    a = math.radians(float(degrees))
    c, s = math.cos(a), math.sin(a)
    k = np.array([[0.0, -u[2], u[1]], [u[2], 0.0, -u[0]], [-u[1], u[0], 0.0]])
    r = c * np.eye(3) + s * k + (1.0 - c) * np.outer(u, u)  # [row][col]
    return r.T.copy()


def _cm3(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Product of column-major [col][row] 3x3 matrices, column-major."""
    return (a.T @ b.T).T


class Session:
    """The per-frame protocol state of one IsaacVisualization on the master rank."""

    def __init__(self, viz, communicator: IsaacCommunicator):
        self.viz = viz
        self.comm = communicator
        self.metaNr = 0
        self.flags: set[str] = set()
        self.initRoot: dict | None = None
        self.sendInit = False
        self.metaRoot: dict = {}

    # ------------------------------------------------------------ lifecycle
    def init(self, setting: int = ReturnAtError) -> int:
        """init (lib/isaac.hpp:1276-1295): connect and register; -1 on failure."""
        if self.comm.serverConnect(setting) < 0:
            return -1
        self.initRoot = register_message(self.viz)
        self.comm.serverSendRegister(self.initRoot)
        self.metaRoot = {}
        return 0

    def exit(self):
        """The exit message of the destructor (lib/isaac.hpp:2110-2118)."""
        self.comm.serverSend(json.dumps({"type": "exit"}), True, True)

    # ------------------------------------------------------------ incoming
    def receive(self) -> tuple[dict, bool]:
        """Drain the server's messages: requests raise send flags, camera keys
        (rotation / position / distance, absolute or relative, rotation axis) change
        the modelview, the controller sees each message; the rest is merged and
        returned with whether anything asks for a redraw (lib/isaac.hpp:1350-1557)."""
        viz = self.viz
        self.flags = set()
        message: dict = {}
        add_modelview = False
        redraw = False
        ctrl = viz.controller
        while True:
            last = self.comm.getLastMessage()
            if last is None:
                break
            req = last.get("request")
            if isinstance(req, str):
                self.flags.update(_REQUESTS.get(req, []))
            js = last.get("rotation absolute")
            if isinstance(js, list) and len(js) == 9:
                viz.rotation = np.asarray(js, dtype=np.float64).reshape(3, 3)
                add_modelview = True
                self.flags.add("rotation")
                del last["rotation absolute"]
            js = last.get("rotation relative")
            if isinstance(js, list) and len(js) == 9:
                viz.rotation = _cm3(np.asarray(js, dtype=np.float64).reshape(3, 3), viz.rotation)
                add_modelview = True
                self.flags.add("rotation")
                del last["rotation relative"]
            js = last.get("rotation axis")
            if isinstance(js, list) and len(js) == 4:
                viz.rotation = _cm3(rotation_about(js[:3], js[3]), viz.rotation)
                add_modelview = True
                self.flags.add("rotation")
                del last["rotation axis"]
            js = last.get("position absolute")
            if isinstance(js, list) and len(js) == 3:
                viz.lookAt = tuple(float(v) for v in js)
                add_modelview = True
                self.flags.add("position")
                del last["position absolute"]
            js = last.get("position relative")
            if isinstance(js, list) and len(js) == 3:
                # lookAt += transpose(rotation) * t; [col][row] storage is that transpose
                t = np.asarray(js, dtype=np.float64)
                viz.lookAt = tuple(np.asarray(viz.lookAt, dtype=np.float64) + np.asarray(viz.rotation) @ t)
                add_modelview = True
                self.flags.add("position")
                del last["position relative"]
            if "distance absolute" in last:
                viz.distance = float(last.pop("distance absolute"))
                add_modelview = True
                self.flags.add("distance")
            if "distance relative" in last:
                viz.distance += float(last.pop("distance relative"))
                add_modelview = True
                self.flags.add("distance")
            handle = getattr(ctrl, "handleMessage", None)
            if handle is not None and handle(last):
                redraw = True
                self.flags.add("projection")
                viz.projections = [np.asarray(m, dtype=np.float64) for m in ctrl.projections(viz.framebufferSize)]
                viz.projection = viz.projections[0]
                viz._push_camera()
            merge_json(message, last)
        if add_modelview:
            redraw = True
            viz.updateModelview()
        return message, redraw

    def apply(self, message: dict) -> bool:
        """Apply the merged message's steering keys; returns whether to redraw."""
        viz = self.viz
        redraw = False
        req = message.get("request")
        if req == "redraw":
            redraw = True
        if req == "minmax":
            self.flags.add("minmax")
        proj = message.get("projection")
        if isinstance(proj, list) and len(proj) == 16 * len(viz.projections):
            viz.projections = [np.asarray(proj[16 * i: 16 * i + 16], dtype=np.float64).reshape(4, 4)
                               for i in range(len(viz.projections))]
            viz.projection = viz.projections[0]
            viz._push_camera()
            self.flags.add("projection")
            redraw = True
        steer = {k: v for k, v in message.items() if k not in ("projection", "modelview", "request", "metadata")}
        for k in steer:
            if k in _STEER_FLAGS:
                self.flags.add(_STEER_FLAGS[k])
                redraw = True
        if steer:
            viz.steer(steer)
        return redraw

    # ------------------------------------------------------------ outgoing
    def _set_init(self, key, value):
        if self.initRoot is not None:
            self.initRoot[key] = copy.deepcopy(value)
        self.sendInit = True

    def period_message(self) -> dict:
        """The period message of this frame (lib/isaac.hpp:2549-2846)."""
        viz, f = self.viz, self.flags
        root: dict = {"metadata": self.metaRoot, "type": "period", "meta nr": self.metaNr}
        self.sendInit = "init" in f
        if "projection" in f:
            root["projection"] = sum((_flat(p) for p in viz.projections), [])
            self._set_init("projection", root["projection"])
        if "position" in f:
            root["position"] = [float(v) for v in viz.lookAt]
            self._set_init("position", root["position"])
        if "rotation" in f:
            root["rotation"] = _flat(viz.rotation)
            self._set_init("rotation", root["rotation"])
        if "distance" in f:
            root["distance"] = float(viz.distance)
            self._set_init("distance", root["distance"])
        if "transfer" in f:
            arrays = []
            for i in range(viz.combinedSourceListSize):
                lut = np.asarray(viz.getTransfer(i), dtype=np.float32)
                arrays.append((lut * np.float32(255.0)).astype(np.uint32).tolist())
            root["transfer array"] = arrays
            root["transfer points"] = [
                [{"value": int(k), "r": float(c[0]), "g": float(c[1]), "b": float(c[2]), "a": float(c[3])}
                 for k, c in sorted(viz.transferDescription[i].items())]
                for i in range(viz.combinedSourceListSize)
            ]
        if "functions" in f:
            root["functions"] = [{"source": viz.functions[i], "error": int(viz.functionErrors[i])}
                                 for i in range(viz.combinedSourceListSize)]
        if "weight" in f:
            root["weight"] = [float(v) for v in viz.sourceWeight]
        if "interpolation" in f:
            root["interpolation"] = bool(viz.interpolation)
            self._set_init("interpolation", root["interpolation"])
        if "render optimization" in f:
            root["render optimization"] = bool(viz.renderOptimization)
            self._set_init("render optimization", root["render optimization"])
        if "step" in f:
            root["step"] = float(viz.step)
            self._set_init("step", root["step"])
        adv = dict(getattr(viz, "advection", dict(step=1.0, weight=0.95, period=1, duration=1, seeds=1000)))
        for flag, val in (
            ("seed points", int(adv["seeds"])),
            ("advection step", float(adv["step"])),
            ("advection weight", float(adv["weight"])),
            ("advection seeding period", int(adv["period"])),
            ("advection seeding duration", int(adv["duration"])),
            ("advection on pause", bool(getattr(viz, "advectionOnPause", False))),
            ("advection border", bool(getattr(viz, "advectionBorder", True))),
        ):
            if flag in f:
                root[flag] = val
                self._set_init(flag, val)
        if "iso threshold" in f:
            root["iso threshold"] = [float(v) for v in viz.sourceIsoThreshold[: len(viz.volumeSources)]]
        if "minmax" in f:
            mn, mx = viz.minMax()
            root["minmax"] = [{"min": float(a), "max": float(b)} for a, b in zip(mn, mx)]
        if "background color" in f:
            root["background color"] = [float(v) for v in viz.backgroundColor[:3]]
            self._set_init("background color", root["background color"])
        if "clipping" in f:
            root["clipping"] = [{"position": [float(v) for v in c[0:3]], "normal": [float(v) for v in c[3:6]]}
                                for c in viz.clipping]
        if "ao" in f:
            root["ao isEnabled"] = bool(viz.ambientOcclusion["isEnabled"])
            root["ao weight"] = float(viz.ambientOcclusion["weight"])
            self._set_init("ao isEnabled", root["ao isEnabled"])
            self._set_init("ao weight", root["ao weight"])
        if "render mode" in f:
            root["render mode"] = int(viz.renderMode)
            self._set_init("render mode", root["render mode"])
        if "dither mode" in f:
            root["dither mode"] = int(viz.ditherMode)
            self._set_init("dither mode", root["dither mode"])
        feedback = getattr(viz.controller, "sendFeedback", None)
        if feedback is not None:
            feedback(root, "controller" in f)
        if self.sendInit and self.initRoot is not None:
            root["init"] = self.initRoot
        return root

    def send_period(self, frame) -> None:
        """Send the period message, finished by the frame's payload (or closed
        without one when there is no frame)."""
        self.comm.serverSend(json.dumps(self.period_message()), True, False)
        if frame is not None:
            self.comm.serverSendFrame(frame)
        else:
            self.comm.serverSend(None, False, True)
        self.metaNr += 1
        self.metaRoot = {}
