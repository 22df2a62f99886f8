"""Learned frame reconstructor: Python side of ``isaacb_recon_*``.

A 4-level convolutional U-Net rebuilds the full-size frame from a half-size
render taken at twice the ray step.  The network trains and runs on the GPU
in the library's own tcgen05 kernels; this module holds the weights file
format, the training loop's host side and the judged renderer that falls back
to the plain full-size render when the reconstruction's PSNR against it drops
below a threshold.
"""

from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import check

WEIGHTS = Path(__file__).resolve().parent / "data" / "recon_unet.f32"
# trained on pairs of the combined (pre-classified RGBA8) renderer
WEIGHTS_COMBINED = Path(__file__).resolve().parent / "data" / "recon_unet_combined.f32"


def weights_for(renderer: str) -> Path:
    """The trained weights for half-size frames of the given renderer ("per_source" or "combined")."""
    return WEIGHTS_COMBINED if renderer == "combined" else WEIGHTS


def _torch():
    import torch

    return torch


def _stream():
    return C.c_void_p(_torch().cuda.current_stream().cuda_stream)


def psnr_from_sq(sq: float, nbytes: int) -> float:
    mse = sq / max(nbytes, 1)
    return float("inf") if mse == 0 else 10.0 * math.log10(255.0**2 / mse)


class Reconstructor:
    """The network with buffers for ``max_batch`` half-size inputs of max_h x max_w."""

    def __init__(self, max_batch: int, max_h: int, max_w: int, seed: int = 1):
        self.lib = _lib.load()
        h = C.c_void_p()
        check(self.lib.isaacb_recon_create(max_batch, max_h, max_w, seed, C.byref(h)))
        self.handle = h
        self.n_params = int(self.lib.isaacb_recon_param_count())
        torch = _torch()
        self._loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        self._sq = torch.zeros(1, dtype=torch.int64, device="cuda")

    def close(self):
        if getattr(self, "handle", None):
            self.lib.isaacb_recon_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ parameters
    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        check(self.lib.isaacb_recon_get_params(self.handle, out.ctypes.data_as(_lib._fp)))
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.n_params
        check(self.lib.isaacb_recon_set_params(self.handle, p.ctypes.data_as(_lib._fp)))

    def save(self, path: Path = WEIGHTS):
        path = Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        self.params().tofile(path)

    def load(self, path: Path = WEIGHTS):
        self.set_params(np.fromfile(path, dtype=np.float32))

    # ------------------------------------------------------------------ training
    def train_step(self, low, high, index, lr: float):
        """One Adam step; ``low`` (N,h,w,4) and ``high`` (N,2h,2w,4) uint8 CUDA tensors,
        ``index`` an int32 CUDA tensor of the batch's pairs.  Returns the loss as a CUDA tensor."""
        n, h, w, _ = low.shape
        check(
            self.lib.isaacb_recon_train_step(
                self.handle, C.c_void_p(low.data_ptr()), C.c_void_p(high.data_ptr()), C.c_void_p(index.data_ptr()),
                int(index.numel()), h, w, float(lr), C.c_void_p(self._loss.data_ptr()), None, _stream(),
            )
        )
        return self._loss

    def gradients(self, low, high, index=None):
        """Loss gradient with respect to the parameters (no update), as a numpy array."""
        n, h, w, _ = low.shape
        g = np.empty(self.n_params, np.float32)
        check(
            self.lib.isaacb_recon_train_step(
                self.handle, C.c_void_p(low.data_ptr()), C.c_void_p(high.data_ptr()),
                None if index is None else C.c_void_p(index.data_ptr()), n if index is None else int(index.numel()),
                h, w, 0.0, C.c_void_p(self._loss.data_ptr()), g.ctypes.data_as(_lib._fp), _stream(),
            )
        )
        return g, float(self._loss.item())

    # ------------------------------------------------------------------ inference
    def infer(self, low, out=None):
        """Full-size RGBA8 frame (2h, 2w, 4) from a half-size (h, w, 4) CUDA tensor."""
        torch = _torch()
        h, w, _ = low.shape
        if out is None:
            out = torch.empty((2 * h, 2 * w, 4), dtype=torch.uint8, device="cuda")
        check(self.lib.isaacb_recon_infer(self.handle, C.c_void_p(low.data_ptr()), h, w, C.c_void_p(out.data_ptr()), _stream()))
        return out

    def error_flag(self) -> int:
        """Reads and clears the flag a bounded wait in the kernels raises when it gives up."""
        f = C.c_int32()
        check(self.lib.isaacb_recon_error(self.handle, C.byref(f)))
        return int(f.value)

    def arm_wait_check(self, budget_us: int):
        """The next inference or training step's first convolution checks the failure path:
        a wait of ``budget_us`` on a barrier nothing arrives at, which raises the flag."""
        check(self.lib.isaacb_recon_arm_wait_check(self.handle, int(budget_us)))


def bilinear2(low, out=None):
    """The method without the network: bilinear x2 of a half-size (h, w, 4) CUDA frame."""
    torch = _torch()
    h, w, _ = low.shape
    if out is None:
        out = torch.empty((2 * h, 2 * w, 4), dtype=torch.uint8, device="cuda")
    check(_lib.load().isaacb_upsample_bilinear2(C.c_void_p(low.data_ptr()), h, w, C.c_void_p(out.data_ptr()), _stream()))
    return out


def psnr(a, b, acc=None) -> float:
    """PSNR (dB) of two RGBA8 CUDA images, reduced on the GPU."""
    torch = _torch()
    if acc is None:
        acc = torch.zeros(1, dtype=torch.int64, device="cuda")
    else:
        acc.zero_()
    check(_lib.load().isaacb_image_sq_error(C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), a.numel(),
                                            C.c_void_p(acc.data_ptr()), _stream()))
    return psnr_from_sq(float(acc.item()), a.numel())


class JudgedRenderer:
    """The learned path with the plain renderer as its judge and fallback.

    Every frame renders the half-size view (``low_viz``, twice the ray step)
    and reconstructs the full-size frame.  Every ``judge_every``-th frame,
    the first included, the plain full-size frame (``full_viz``) is rendered
    too and the reconstruction's PSNR against it measured on the GPU.  Below
    ``threshold`` dB the plain frame is served, and plain frames keep being
    served until a later judge frame measures the reconstruction at or above
    the threshold again.  Both visualizations must show the same sources,
    transfer functions and camera."""

    def __init__(self, full_viz, low_viz, net, judge_every: int = 16, threshold: float = 40.0, measure=None, device="cuda"):
        torch = _torch()
        self.full_viz, self.low_viz, self.net = full_viz, low_viz, net
        self.judge_every, self.threshold = judge_every, threshold
        W, H = full_viz.framebufferSize
        w, h = low_viz.framebufferSize
        if (W, H) != (2 * w, 2 * h):
            raise ValueError("the half-size view must be exactly half the full size")
        self.half = torch.empty((h, w, 4), dtype=torch.uint8, device=device)
        self.rec = torch.empty((H, W, 4), dtype=torch.uint8, device=device)
        self.full = torch.empty((H, W, 4), dtype=torch.uint8, device=device)
        self._acc = torch.zeros(1, dtype=torch.int64, device=device)
        # PSNR (dB) of the reconstruction against the plain frame
        self.measure = measure or (lambda a, b: psnr(a, b, self._acc))
        self.count = 0
        self.fallback = False
        self.judged = []  # (frame number, PSNR dB)
        self.fallback_frames = 0
        # a judge frame's plain render does not depend on the half-size render or the
        # network: it runs on a side stream beside them and fills their idle SMs
        self._side = torch.cuda.Stream(device=device) if torch.device(device).type == "cuda" else None

    def setCamera(self, projection, modelview):
        self.full_viz.setCamera(projection, modelview)
        self.low_viz.setCamera(projection, modelview)

    def frame(self, update: bool = False):
        """The frame to show, an (H, W, 4) uint8 CUDA tensor (row 0 = bottom)."""
        k = self.count
        self.count += 1
        judge = k % self.judge_every == 0
        if self.fallback and not judge:
            self.fallback_frames += 1
            if update:
                self.full_viz.update()
            self.full_viz.render(self.full)
            return self.full
        torch = _torch()
        side = self._side if judge else None
        if side is not None:
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(side):
                if update:
                    self.full_viz.update()
                self.full_viz.render(self.full)
        if update:
            self.low_viz.update()
        self.low_viz.render(self.half)
        self.net.infer(self.half, self.rec)
        if not judge:
            return self.rec
        if side is not None:
            torch.cuda.current_stream().wait_stream(side)
        else:
            if update:
                self.full_viz.update()
            self.full_viz.render(self.full)
        p = self.measure(self.rec, self.full)
        self.judged.append((k, p))
        self.fallback = p < self.threshold
        if self.fallback:
            self.fallback_frames += 1
            return self.full
        return self.rec

    def autotune_step(self, cameras, steps=(1.0, 1.25, 1.5, 2.0), margin_db: float = 3.0, repeat: int = 3) -> dict:
        """Step schedule of the half-size render, picked by measurement under the judge's
        quality constraint.  For every candidate step (cells) the half-size render plus the
        network is timed (CUDA events, ``repeat`` passes over ``cameras``) and its PSNR
        against the plain full-size frame measured on each camera.  A candidate qualifies
        when every camera is at or above ``threshold + margin_db``; the fastest qualifying
        one is set on the half-size view (the first candidate when none qualifies) and the
        report returned.  The plain frames are the judge's own, so the choice keeps the
        learned path above the fallback threshold on these views."""
        torch = _torch()
        fulls = []
        for P, MV in cameras:
            self.full_viz.setCamera(P, MV)
            f = torch.empty_like(self.full)
            self.full_viz.render(f)
            fulls.append(f)
        results = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for st in steps:
            self.low_viz.setStep(st)
            ps = []
            for (P, MV), f in zip(cameras, fulls):
                self.low_viz.setCamera(P, MV)
                self.low_viz.render(self.half)
                self.net.infer(self.half, self.rec)
                ps.append(self.measure(self.rec, f))
            torch.cuda.synchronize()
            e0.record()
            for _ in range(repeat):
                for P, MV in cameras:
                    self.low_viz.setCamera(P, MV)
                    self.low_viz.render(self.half)
                    self.net.infer(self.half, self.rec)
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1) / (repeat * len(cameras))
            # an identical frame has infinite PSNR; the report keeps JSON-safe numbers (None)
            fin = [x for x in ps if x != float("inf")]
            results.append({"step": st, "ms": ms, "psnr_min": min(fin) if fin else None,
                            "psnr_mean": sum(fin) / len(fin) if fin else None, "identical_views": len(ps) - len(fin),
                            "qualifies": min(ps) >= self.threshold + margin_db})
        ok = [r for r in results if r["qualifies"]]
        best = min(ok, key=lambda r: r["ms"]) if ok else results[0]
        self.low_viz.setStep(best["step"])
        return {"chosen_step": best["step"], "margin_db": margin_db, "candidates": results}


# (ksize, stride, pad, c_in, c_out, output level) of the network's convolutions
LAYER_SHAPES = [
    (3, 1, 1, 8, 32, 0), (3, 1, 1, 32, 32, 0), (3, 2, 1, 32, 64, 1), (3, 1, 1, 64, 64, 1), (3, 2, 1, 64, 96, 2),
    (2, 2, 0, 96, 128, 3), (1, 1, 0, 224, 96, 2), (1, 1, 0, 160, 64, 1), (1, 1, 0, 96, 32, 0), (3, 1, 1, 32, 32, 0),
    (1, 1, 0, 32, 16, 0),
]


def level_sizes(h: int, w: int):
    def o(n, k, s, p):
        return (n + 2 * p - k) // s + 1

    hs, ws = [h], [w]
    for k, s, p in ((3, 2, 1), (3, 2, 1), (2, 2, 0)):
        hs.append(o(hs[-1], k, s, p))
        ws.append(o(ws[-1], k, s, p))
    return hs, ws


def inference_flops(h: int, w: int) -> float:
    """Multiply-adds x 2 of one inference on an h x w half-size frame (the convolutions)."""
    hs, ws = level_sizes(h, w)
    return float(sum(2 * k * k * ci * co * hs[l] * ws[l] for k, s, p, ci, co, l in LAYER_SHAPES))


def _main(argv=None):
    """``python -m isaac_b200.recon [--height H --width W --repeat N --weights F]``:
    inference on a seeded random half-size frame, N times (used for profiling)."""
    import argparse

    torch = _torch()
    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--height", type=int, default=540)
    ap.add_argument("--width", type=int, default=960)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--weights", default=str(WEIGHTS))
    ap.add_argument("--producer", default="tma", choices=["tma", "cp_async"],
                    help="input staging of the row-tile convolutions")
    a = ap.parse_args(argv)
    check(_lib.load().isaacb_conv_set_producer(1 if a.producer == "tma" else 0))
    net = Reconstructor(1, a.height, a.width, seed=1)
    if Path(a.weights).exists():
        net.load(Path(a.weights))
    g = torch.Generator(device="cuda").manual_seed(1)
    low = torch.randint(0, 256, (a.height, a.width, 4), dtype=torch.uint8, device="cuda", generator=g)
    out = torch.empty((2 * a.height, 2 * a.width, 4), dtype=torch.uint8, device="cuda")
    net.infer(low, out)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(a.repeat):
        net.infer(low, out)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(a.repeat, 1)
    print(f"ok error_flag={net.error_flag()} ms_per_inference={ms:.4f} "
          f"tflops={inference_flops(a.height, a.width) / (ms * 1e-3) / 1e12:.1f}")
    return 0


if __name__ == "__main__":
    raise SystemExit(_main())
