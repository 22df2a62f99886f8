"""GPU frame output against host references.

* base64: the kernel against Python's encoder with the '=' padding removed (boost's
  base64_from_binary writes none, lib/isaac/isaac_communicator.hpp:254-265).
* raw frames: the payload message decodes to the frame's bytes exactly.
* JPEG: libjpeg (PIL) decodes the GPU's baseline 4:2:0 stream, rows in memory
  order, and its error against the frame is within 1 dB of libjpeg's own encoding
  at the same quality and subsampling, the reference's encoder settings
  (lib/isaac/isaac_communicator.hpp:214-252).
* the streaming loop: IsaacVisualization registers with a fake server, sends period
  messages whose payload is the frame it returned, and follows the server's
  camera and transfer steering.
"""

import base64
import io
import time

import numpy as np
import pytest
import torch
from PIL import Image

from fake_server import FakeServer
from isaac_b200 import protocol as P
from isaac_b200 import scenes
from isaac_b200.visualization import IsaacVisualization, VolumeSource

pytestmark = pytest.mark.gpu

JPEG_HEAD = "data:image/jpeg;base64,"
RAW_HEAD = "data:image/raw-rgba;base64,"


def _unb64(text: str) -> bytes:
    return base64.b64decode(text + "=" * (-len(text) % 4))


def _psnr(a, b) -> float:
    d = np.asarray(a, np.float64) - np.asarray(b, np.float64)
    mse = float(np.mean(d * d))
    return float("inf") if mse == 0 else 10.0 * np.log10(255.0**2 / mse)


def _frame(h, w, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    img = np.zeros((h, w, 4))
    for c in range(3):
        f = rng.uniform(0.02, 0.2, 2)
        img[..., c] = 128 + 90 * np.sin(f[0] * xx + c) * np.cos(f[1] * yy - c)
    img[..., :3] += rng.normal(0, 4, (h, w, 3))
    img[..., 3] = rng.integers(0, 256, (h, w))
    return np.clip(np.rint(img), 0, 255).astype(np.uint8)


@pytest.mark.parametrize("n", [0, 1, 2, 3, 4, 5, 6, 7, 100, 4097, (1 << 20) + 1])
def test_base64_kernel(n):
    data = np.random.default_rng(n).integers(0, 256, n, dtype=np.uint8)
    got = P.base64_device(torch.from_numpy(data).cuda())
    assert got == base64.b64encode(data.tobytes()).rstrip(b"=")
    assert len(got) == (8 * n + 5) // 6


@pytest.mark.parametrize("shape", [(150, 200), (61, 97)])
def test_raw_payload_is_the_frame(shape):
    frame = _frame(*shape, seed=1)
    enc = P.FrameEncoder()
    msg = enc.message(torch.from_numpy(frame).cuda(), jpeg=False).decode()
    head = '{"payload": "' + RAW_HEAD
    assert msg.startswith(head) and msg.endswith('"}')
    assert _unb64(msg[len(head):-2]) == frame.tobytes()
    enc.close()


@pytest.mark.parametrize("quality", [90, 50])
@pytest.mark.parametrize("shape", [(150, 200), (61, 97), (1080, 1920)])
def test_jpeg_against_libjpeg(shape, quality):
    h, w = shape
    frame = _frame(h, w, seed=2)
    enc = P.FrameEncoder(quality)
    jpg = enc.jpeg(torch.from_numpy(frame).cuda())
    assert jpg[:2] == b"\xff\xd8" and b"\xff\xc0" in jpg  # SOI, baseline SOF0
    im = Image.open(io.BytesIO(jpg))
    assert im.format == "JPEG" and im.mode == "RGB" and im.size == (w, h)
    assert [(c[1], c[2]) for c in im.layer] == [(2, 2), (1, 1), (1, 1)]  # 4:2:0
    got = np.asarray(im)
    ref_buf = io.BytesIO()
    Image.fromarray(frame[..., :3]).save(ref_buf, format="JPEG", quality=quality, subsampling=2)
    ref = np.asarray(Image.open(io.BytesIO(ref_buf.getvalue())))
    p_gpu, p_ref = _psnr(got, frame[..., :3]), _psnr(ref, frame[..., :3])
    assert p_gpu >= p_ref - 1.0, (p_gpu, p_ref)
    # the message carries the same JPEG
    msg = enc.message(torch.from_numpy(frame).cuda(), jpeg=True).decode()
    head = '{"payload": "' + JPEG_HEAD
    assert msg.startswith(head) and msg.endswith('"}')
    assert _unb64(msg[len(head):-2]) == jpg
    enc.close()


def test_quality_setting():
    enc = P.FrameEncoder()
    assert enc.quality == 90
    enc.setQuality(150)
    assert enc.quality == 100
    enc.setQuality(0)
    frame = torch.from_numpy(_frame(32, 48, seed=3)).cuda()
    assert len(enc.jpeg(frame)) > 0
    enc.close()


def _viz(port, jpeg=True, fb=(96, 64)):
    n = 32
    scalar, _ = scenes.gaussian_scene(n, seed=3)
    src = VolumeSource("scalar", scalar.cuda().contiguous(), 1)
    viz = IsaacVisualization("stream test", fb, (n, n, n), (n, n, n), (n, n, n), (0, 0, 0), [src],
                             server_url="127.0.0.1", server_port=port, jpeg=jpeg)
    viz.setInterpolation(True)
    viz.setTransferPoints(0, {0: (0.0, 0.0, 1.0, 0.0), 400: (0.0, 1.0, 0.5, 0.4), 1024: (1.0, 0.2, 0.0, 1.0)})
    return viz


def _wait(cond, timeout=10.0):
    end = time.time() + timeout
    while not cond() and time.time() < end:
        time.sleep(0.01)
    assert cond()


def test_streaming_loop_with_fake_server():
    server = FakeServer()
    try:
        viz = _viz(server.port)
        assert viz.init() == 0
        reg = server.wait_messages(1)[0]
        assert reg["type"] == "register" and reg["framebuffer width"] == 96 and reg["framebuffer height"] == 64
        viz.getJsonMetaRoot()["time step"] = 7
        frame = viz.doVisualization()
        per = server.wait_messages(2)[1]
        assert per["uid"] == 1 and per["type"] == "period" and per["meta nr"] == 0
        assert per["metadata"] == {"time step": 7}
        assert per["payload"].startswith(JPEG_HEAD)
        got = np.asarray(Image.open(io.BytesIO(_unb64(per["payload"][len(JPEG_HEAD):]))).convert("RGB"))
        assert got.shape == (64, 96, 3)
        assert _psnr(got, frame[..., :3]) > 30.0
        # steering from the server: a rotation about y, and the rotation asked back
        server.send({"rotation axis": [0, 1, 0, 90.0]})
        server.send({"request": "rotation"})
        _wait(lambda: len(viz.communicator.messageList) >= 2)
        frame2 = viz.doVisualization()
        per2 = server.wait_messages(3)[2]
        assert per2["meta nr"] == 1
        assert np.allclose(per2["rotation"], P.rotation_about([0, 1, 0], 90.0).reshape(9))
        assert not np.array_equal(frame2, frame)
        # a transfer change from the server redraws with the new table and reports it
        server.send({"transfer points": [[{"value": 0, "r": 1, "g": 1, "b": 1, "a": 1},
                                          {"value": 1024, "r": 1, "g": 1, "b": 1, "a": 1}]]})
        _wait(lambda: len(viz.communicator.messageList) >= 1)
        viz.doVisualization()
        per3 = server.wait_messages(4)[3]
        assert per3["transfer array"][0][0] == [255, 255, 255, 255]
        viz.close()
        assert server.wait_messages(5)[4]["type"] == "exit"
    finally:
        server.close()


def test_streaming_raw_frames_are_exact():
    server = FakeServer()
    try:
        viz = _viz(server.port, jpeg=False, fb=(40, 30))
        assert viz.init() == 0
        frame = viz.doVisualization()
        per = server.wait_messages(2)[1]
        assert per["payload"].startswith(RAW_HEAD)
        assert _unb64(per["payload"][len(RAW_HEAD):]) == frame.tobytes()
        viz.close()
    finally:
        server.close()
