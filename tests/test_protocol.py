"""The server protocol on the host (no GPU): IsaacCommunicator's framing, the done
window, the reader thread, reconnects, and the Session's handling of requests,
camera messages and steering, against a fake server on 127.0.0.1.  Expected
bytes and keys follow lib/isaac/isaac_communicator.hpp:125-362 and
lib/isaac.hpp:833-891, 1345-1800, 2546-2856."""

import math
import socket
import time

import numpy as np
import pytest

from fake_server import FakeServer
from isaac_b200 import protocol as P
from isaac_b200.controllers import DefaultCompositor, DefaultController, StereoController, perspective
from isaac_b200.visualization import modelview


class _Src:
    def __init__(self, name, dim):
        self.name, self.featureDim = name, dim

    def getName(self):
        return self.name


class FakeViz:
    """The attributes and methods of IsaacVisualization that Session uses."""

    def __init__(self, controller=DefaultController):
        self.name = "fake"
        self.framebufferSize = (64, 48)
        self.compositor = DefaultCompositor()
        self.volumeSources = [_Src("density", 1), _Src("field", 3)]
        self.particleSources = [_Src("electrons", 1)]
        self.globalSize = (32, 16, 8)
        self.scale = (1.0, 2.0, 1.5)
        self.controller = controller
        self.projections = [np.asarray(m) for m in controller.projections(self.framebufferSize)]
        self.projection = self.projections[0]
        self.lookAt = (0.0, 0.0, 0.0)
        self.rotation = np.eye(3)
        self.distance = -4.5
        self.modelview = modelview(self.lookAt, self.rotation, self.distance)
        self.interpolation = False
        self.renderOptimization = True
        self.step = 0.5
        self.ambientOcclusion = {"isEnabled": False, "weight": 0.5}
        self.combinedSourceListSize = 3
        self.transferDescription = [{0: (0, 0, 0, 0), 1024: (1, 1, 1, 1)} for _ in range(3)]
        self.functions = ["idem", "length", "idem"]
        self.functionErrors = [0, 0, 0]
        self.sourceWeight = [2.0, 2.0, 2.0]
        self.sourceIsoThreshold = [0.0, 0.0, 0.0]
        self.backgroundColor = [0.0, 0.0, 0.0, 1.0]
        self.clipping = []
        self.renderMode = 0
        self.ditherMode = 1
        self.steered = []
        self.pushes = 0

    def steer(self, message):
        self.steered.append(dict(message))
        if "step" in message:
            self.step = float(message["step"])
        if "weight" in message:
            self.sourceWeight = [float(v) for v in message["weight"]]

    def updateModelview(self):
        self.modelview = modelview(self.lookAt, self.rotation, self.distance)
        self._push_camera()

    def _push_camera(self):
        self.pushes += 1

    def getTransfer(self, i):
        return np.linspace(0, 1, 1024 * 4, dtype=np.float32).reshape(1024, 4)

    def minMax(self):
        return np.array([0.0, 1.0, 2.0], np.float32), np.array([1.0, 2.0, 3.0], np.float32)


@pytest.fixture
def server():
    s = FakeServer()
    yield s
    s.close()


def _wait_queue(comm, n, timeout=5.0):
    end = time.time() + timeout
    while len(comm.messageList) < n and time.time() < end:
        time.sleep(0.01)
    assert len(comm.messageList) >= n


def test_register_message_and_framing(server):
    viz = FakeViz()
    comm = P.IsaacCommunicator("127.0.0.1", server.port)
    sess = P.Session(viz, comm)
    assert sess.init() == 0
    reg = server.wait_messages(1)[0]
    # the opener {"uid": n, then the JSON object with its brace turned into a comma
    assert server.raw[0].startswith(b'{"uid": 0,"type": "register", "name": "fake"')
    assert list(reg) == ["uid", "type", "name", "nodes", "framebuffer width", "framebuffer height", "max functors",
                         "functors", "projection count", "projection", "position", "rotation", "distance", "sources",
                         "interpolation", "step", "dimension", "width", "height", "depth", "protocol", "ao isEnabled",
                         "ao weight"]
    assert reg["uid"] == 0 and reg["nodes"] == 1 and reg["max functors"] == 3
    assert [f["name"] for f in reg["functors"]] == ["idem", "add", "mul", "length", "pow", "sum"]
    assert [f["uses parameter"] for f in reg["functors"]] == [False, True, True, False, True, False]
    assert reg["sources"] == [{"name": "density", "feature dimension": 1}, {"name": "field", "feature dimension": 3},
                              {"name": "electrons", "feature dimension": 1}]
    assert (reg["width"], reg["height"], reg["depth"]) == (32, 32, 12)  # globalSize * scale
    assert reg["projection count"] == 1
    assert np.allclose(reg["projection"], perspective(45.0, 64 / 48, 0.002, 100.0).reshape(16))
    assert reg["protocol"] == [1, 0]
    # a period message without a frame: opened, then closed by a bare "} "
    sess.send_period(None)
    msgs = server.wait_messages(2)
    assert msgs[1] == {"uid": 1, "metadata": {}, "type": "period", "meta nr": 0}
    assert server.raw[1] == b'{"uid": 1,"metadata": {}, "type": "period", "meta nr": 0}'
    comm.close()


def test_connect_failure_codes():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()  # nothing listens there
    comm = P.IsaacCommunicator("127.0.0.1", port)
    assert comm.serverConnect(P.ReturnAtError) == -3
    assert comm.serverConnect(P.RetryEverySend) == 1
    # a send without a connection retries and sends nothing
    assert comm.serverSend('{"type": "x"}') == 0


def test_done_window_blocks_then_resets():
    srv = FakeServer(ack=False)
    try:
        comm = P.IsaacCommunicator("127.0.0.1", srv.port)
        assert comm.serverConnect() == 0
        t0 = time.time()
        for _ in range(5):  # ids 0..4: within ISAAC_MAX_DIFFERENCE of server id 0
            comm.serverSend('{"a": 1}', True, True)
        assert time.time() - t0 < 0.5
        t0 = time.time()
        comm.serverSend('{"a": 2}', True, True)  # id 5 > 0 + 4: waits 1 s, then id = server_id - 1
        assert time.time() - t0 >= 0.9
        msgs = srv.wait_messages(6)
        assert [m["uid"] for m in msgs] == [0, 1, 2, 3, 4, -1]
        # an acknowledgement opens the window again
        srv.send({"done": 20})
        end = time.time() + 5
        while comm.server_id != 20 and time.time() < end:
            time.sleep(0.01)
        assert comm.server_id == 20
        t0 = time.time()
        comm.serverSend('{"a": 3}', True, True)
        assert time.time() - t0 < 0.5
        comm.close()
    finally:
        srv.close()


def test_reader_queues_messages_in_order(server):
    comm = P.IsaacCommunicator("127.0.0.1", server.port)
    assert comm.serverConnect() == 0
    server.wait_connections(1)
    server.send('{"request": "rotation"} {"done": 3}{"step": 0.25}')
    server.send('{"weight": [1.0,')
    time.sleep(0.05)
    server.send(' 2.0]} ')
    _wait_queue(comm, 3)
    assert comm.getLastMessage() == {"request": "rotation"}
    assert comm.getLastMessage() == {"step": 0.25}
    assert comm.getLastMessage() == {"weight": [1.0, 2.0]}
    assert comm.getLastMessage() is None
    assert comm.server_id == 3
    comm.close()


def test_protocol_mismatch_closes_for_good(server, capsys):
    comm = P.IsaacCommunicator("127.0.0.1", server.port)
    assert comm.serverConnect() == 0
    server.wait_connections(1)
    server.send({"fatal error": "protocol mismatch"})
    end = time.time() + 5
    while not comm.closed and time.time() < end:
        time.sleep(0.01)
    assert comm.closed
    assert comm.serverSend('{"a": 1}') == 0
    assert "protocol mismatch" in capsys.readouterr().err


def test_reconnect_resends_register(server):
    viz = FakeViz()
    comm = P.IsaacCommunicator("127.0.0.1", server.port)
    sess = P.Session(viz, comm)
    assert sess.init() == 0
    server.wait_messages(1)
    server.drop()
    end = time.time() + 10
    while server.connections < 2 and time.time() < end:
        comm.serverSend('{"type": "ping"}', True, True)
        time.sleep(0.05)
    assert server.connections == 2
    end = time.time() + 5
    while 2 not in server.connection_of and time.time() < end:
        time.sleep(0.01)
    # the first message of the new connection is the register message again
    first_new = server.messages[server.connection_of.index(2)]
    assert first_new["type"] == "register" and first_new["name"] == "fake"
    comm.close()


def test_rotation_about_is_rodrigues():
    R = P.rotation_about([0, 2, 0], 90.0).T  # column-major storage -> math matrix
    assert np.allclose(R @ R.T, np.eye(3)) and math.isclose(np.linalg.det(R), 1.0)
    assert np.allclose(R @ [1, 0, 0], [0, 0, -1])
    assert np.allclose(R @ [0, 1, 0], [0, 1, 0])
    r2 = P.rotation_about([1, 1, 1], 120.0).T  # cyclic permutation x -> y -> z
    assert np.allclose(r2 @ [1, 0, 0], [0, 1, 0])


def test_merge_json():
    a = {"metadata": {"list": [1], "v": 1}, "step": 0.5}
    P.merge_json(a, {"metadata": {"list": [2], "v": 2, "w": 3}, "step": 0.25, "weight": [1]})
    assert a == {"metadata": {"list": [1, 2], "v": 2, "w": 3}, "step": 0.25, "weight": [1]}
    b = {}
    P.merge_json(b, {"metadata": {"x": 1}})
    assert b == {"metadata": {"x": 1}}


def test_session_camera_requests_and_steering(server):
    viz = FakeViz()
    comm = P.IsaacCommunicator("127.0.0.1", server.port)
    sess = P.Session(viz, comm)
    assert sess.init() == 0
    server.wait_messages(1)
    rot = P.rotation_about([0, 1, 0], 30.0)
    server.send({"rotation absolute": rot.reshape(9).tolist()})
    server.send({"position relative": [1.0, 0.0, 0.0], "distance relative": -0.5})
    server.send({"request": "rotation"})
    server.send({"step": 0.25, "weight": [1.0, 2.0, 3.0], "metadata": {"note": [1]}})
    _wait_queue(comm, 4)
    message, redraw = sess.receive()
    assert redraw
    assert np.allclose(viz.rotation, rot)
    # position relative: lookAt += transpose(rotation) * t
    assert np.allclose(viz.lookAt, rot @ np.array([1.0, 0.0, 0.0]))
    assert viz.distance == -5.0
    assert np.allclose(viz.modelview, modelview(viz.lookAt, viz.rotation, viz.distance))
    assert {"rotation", "position", "distance"} <= sess.flags
    assert message["metadata"] == {"note": [1]}
    assert sess.apply(message)
    assert viz.step == 0.25 and viz.sourceWeight == [1.0, 2.0, 3.0]
    assert {"step", "weight"} <= sess.flags
    period = sess.period_message()
    assert list(period)[:3] == ["metadata", "type", "meta nr"]
    assert period["rotation"] == rot.reshape(9).tolist()
    assert period["distance"] == -5.0 and period["step"] == 0.25 and period["weight"] == [1.0, 2.0, 3.0]
    # camera and step changes are also written into the init object, which goes along
    assert period["init"]["step"] == 0.25 and period["init"]["distance"] == -5.0
    assert period["init"]["type"] == "register"
    comm.close()


def test_start_observing_sends_state(server):
    viz = FakeViz()
    comm = P.IsaacCommunicator("127.0.0.1", server.port)
    sess = P.Session(viz, comm)
    assert sess.init() == 0
    server.wait_messages(1)
    server.send({"request": "start observing"})
    server.send({"request": "minmax"})
    _wait_queue(comm, 2)
    message, _ = sess.receive()
    sess.apply(message)
    period = sess.period_message()
    for k in ("transfer array", "transfer points", "functions", "weight", "interpolation", "render optimization", "step",
              "seed points", "advection step", "advection weight", "advection seeding period",
              "advection seeding duration", "iso threshold", "minmax", "background color", "clipping", "ao isEnabled",
              "ao weight", "render mode", "dither mode", "init"):
        assert k in period, k
    assert len(period["transfer array"]) == 3 and len(period["transfer array"][0]) == 1024
    assert period["transfer array"][0][1] == [int(np.float32(v) * np.float32(255)) for v in viz.getTransfer(0)[1]]
    assert period["transfer points"][0] == [{"value": 0, "r": 0.0, "g": 0.0, "b": 0.0, "a": 0.0},
                                            {"value": 1024, "r": 1.0, "g": 1.0, "b": 1.0, "a": 1.0}]
    assert period["functions"][1] == {"source": "length", "error": 0}
    assert period["iso threshold"] == [0.0, 0.0]  # volume (and field) sources only
    assert period["minmax"][2] == {"min": 2.0, "max": 3.0}
    sess.send_period(None)
    msgs = server.wait_messages(2)
    assert msgs[1]["type"] == "period" and msgs[1]["uid"] == 1 and "transfer array" in msgs[1]
    comm.close()


def test_stereo_controller_messages(server):
    ctrl = StereoController(0.06)
    viz = FakeViz(controller=ctrl)
    comm = P.IsaacCommunicator("127.0.0.1", server.port)
    sess = P.Session(viz, comm)
    assert sess.init() == 0
    server.wait_messages(1)
    assert len(viz.projections) == 2
    server.send({"eye distance": 0.1})
    _wait_queue(comm, 1)
    message, redraw = sess.receive()
    assert redraw and "eye distance" not in message and "projection" in sess.flags
    assert ctrl.eyeDistance == 0.1
    expect = ctrl.projections(viz.framebufferSize)
    assert all(np.array_equal(a, b) for a, b in zip(viz.projections, expect))
    period = sess.period_message()
    assert period["eye distance"] == float(np.float32(0.1))
    assert len(period["projection"]) == 32
    # reported once; a "controller" request sends it again
    assert "eye distance" not in sess.period_message()
    sess.flags = {"controller"}
    assert "eye distance" in sess.period_message()
    comm.close()
