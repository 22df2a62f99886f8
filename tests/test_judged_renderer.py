"""Judge and fallback logic of the learned path (host side, no GPU): fake
views, network and PSNR measurements drive JudgedRenderer."""

import torch

from isaac_b200.recon import JudgedRenderer


class FakeView:
    def __init__(self, w, h, fill):
        self.framebufferSize = (w, h)
        self.fill = fill
        self.renders = 0
        self.updates = 0

    def render(self, out):
        self.renders += 1
        out.fill_(self.fill)

    def update(self):
        self.updates += 1

    def setCamera(self, P, MV):
        pass


class FakeNet:
    def __init__(self):
        self.calls = 0

    def infer(self, half, out):
        self.calls += 1
        out.fill_(7)


def _make(scores, every=4, thr=40.0):
    full, low, net = FakeView(8, 6, 200), FakeView(4, 3, 9), FakeNet()
    it = iter(scores)
    jr = JudgedRenderer(full, low, net, judge_every=every, threshold=thr, measure=lambda a, b: next(it), device="cpu")
    return jr, full, low, net


def test_good_reconstruction_is_served_and_judged_every_nth_frame():
    jr, full, low, net = _make([45.0, 44.0, 43.0])
    frames = [int(jr.frame()[0, 0, 0]) for _ in range(12)]
    assert frames == [7] * 12
    assert [k for k, _ in jr.judged] == [0, 4, 8]
    assert full.renders == 3 and low.renders == 12 and net.calls == 12
    assert jr.fallback_frames == 0


def test_fallback_below_threshold_and_recovery():
    jr, full, low, net = _make([30.0, 39.9, 41.0])
    frames = [int(jr.frame()[0, 0, 0]) for _ in range(12)]
    # judge at 0 fails: plain frames 0-3; judge at 4 fails again: plain 4-7; judge at 8 passes
    assert frames == [200] * 8 + [7] * 4
    assert jr.fallback_frames == 8
    # while falling back only the plain view renders, except on judge frames
    assert low.renders == 3 + 4 - 1 and net.calls == 3 + 4 - 1


def test_update_reaches_the_views_that_render():
    jr, full, low, net = _make([45.0, 45.0])
    for _ in range(5):
        jr.frame(update=True)
    assert low.updates == 5 and full.updates == 2


def test_sizes_must_be_exactly_half():
    import pytest

    with pytest.raises(ValueError):
        JudgedRenderer(FakeView(8, 6, 0), FakeView(4, 4, 0), FakeNet(), device="cpu")
