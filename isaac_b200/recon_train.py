"""Training pairs and training of the learned frame reconstructor.

The plain renderer makes its own training data: the four-source spectral
scene (seeds 6-9, slopes -5/3, -2, -3, -11/3) stored as BF16 bricks, advected
by 0.05 box per timestep, rendered from seeded random cameras with seeded
random 4-8 point transfer functions at full size (step 0.5) and half size
(step 1.0).  Aligned crops of each frame pair (a half-size crop of c x c and
the full-size crop of 2c x 2c at twice its origin) are the training pairs.

    python -m isaac_b200.recon_train --pairs 20000 --timesteps 64 --steps 4000 [--renderer combined]
    python -m isaac_b200.recon_train --error-budget --eval-views 12 [--renderer combined]

writes the FP32 weights to isaac_b200/data/recon_unet.f32 (per-source renderer)
or recon_unet_combined.f32 (combined renderer), the defaults the judged renderer
loads, and prints one JSON line with the losses and the held-out PSNRs of the
reconstruction and of bilinear upsampling.
"""

from __future__ import annotations

import argparse
import json
import math
import time
from pathlib import Path

import numpy as np

from . import scenes
from .recon import Reconstructor, bilinear2, psnr, weights_for

SEEDS = (6, 7, 8, 9)
SLOPES = (-5.0 / 3.0, -2.0, -3.0, -11.0 / 3.0)


def random_transfer(rng: np.random.Generator, sharp: float = 0.35) -> dict:
    """4-8 control points over [0, 1024]; colours uniform, alpha mostly low so
    the volume stays translucent, with an occasional opaque band.  With
    probability ``sharp`` a near-iso function instead: low alpha except one narrow
    opaque band (4-40 keys wide) around a random key, which renders as thin
    surfaces and sharp edges, where a half-size frame loses the most."""
    if rng.random() < sharp:
        k = int(rng.integers(60, 964))
        wd = int(rng.integers(2, 21))
        lo = (float(rng.random()), float(rng.random()), float(rng.random()), float(rng.uniform(0.0, 0.08)))
        hi = (float(rng.random()), float(rng.random()), float(rng.random()), float(rng.uniform(0.7, 1.0)))
        return {0: lo, k - wd: lo, k: hi, k + wd: lo, 1024: lo}
    n = int(rng.integers(4, 9))
    keys = np.sort(rng.choice(np.arange(1, 1024), size=n - 2, replace=False))
    keys = [0] + [int(k) for k in keys] + [1024]
    pts = {}
    for k in keys:
        a = float(rng.uniform(0.0, 0.35)) if rng.random() > 0.15 else float(rng.uniform(0.6, 1.0))
        pts[k] = (float(rng.random()), float(rng.random()), float(rng.random()), a)
    return pts


def random_camera(w: int, h: int, rng: np.random.Generator):
    seed = int(rng.integers(0, 2**31 - 1))
    dist = float(rng.uniform(1.8, 3.2))
    return scenes.camera(w, h, seed=seed, distance=dist)


class PairRenderer:
    """A full-size and a half-size view of the same four sources.

    ``renderer``: "per_source" draws with the per-source renderer from BF16 bricks
    (transfer functions applied per sample); "combined" with the default renderer
    from the merged RGBA8 texture (transfer functions baked in by the merge, so a
    transfer-function change re-merges).  ``step`` is the full-size ray step; the
    half-size view marches at twice it.  Both visualizations read the same device
    fields, which ``set_timestep`` overwrites in place."""

    def __init__(self, size: int = 512, width: int = 1920, height: int = 1080, step: float = 0.5, shift: float = 0.05,
                 renderer: str = "per_source"):
        import torch

        from . import IsaacVisualization, VolumeSource

        if renderer not in ("per_source", "combined"):
            raise ValueError(f"renderer must be per_source or combined, not {renderer!r}")
        self.size, self.width, self.height, self.step, self.shift = size, width, height, step, shift
        self.renderer = renderer
        self.fields = [torch.empty((size, size, size), dtype=torch.float32, device="cuda") for _ in SEEDS]
        vols = [VolumeSource(f"src{i}", f, feature_dim=1, persistent=True) for i, f in enumerate(self.fields)]
        n = (size, size, size)
        self.full = IsaacVisualization("full", (width, height), n, n, (1, 1, 1), (0, 0, 0), vols, [])
        self.low = IsaacVisualization("half", (width // 2, height // 2), n, n, (1, 1, 1), (0, 0, 0), vols, [])
        self._keep = vols
        for v, st in ((self.full, step), (self.low, 2 * step)):
            if renderer == "per_source":
                v.setRenderOptimization(False)
                for i in range(len(SEEDS)):
                    v.setStorage(i, 1)  # BF16 bricks
            v.setInterpolation(True)
            v.setStep(st)
        self.timestep = None
        self.dirty = True

    def set_timestep(self, t: int):
        import torch

        fields = scenes.precision_scene(self.size, seeds=SEEDS, slopes=SLOPES, device="cuda", shift=t * self.shift)
        for d, f in zip(self.fields, fields):
            d.copy_(f)
        del fields
        torch.cuda.synchronize()
        self.timestep = t
        self.dirty = True

    def set_view(self, P, MV, transfers):
        for v in (self.full, self.low):
            for i, tf in enumerate(transfers):
                v.setTransferPoints(i, tf)
            v.updateTransfer()
            v.setCamera(P, MV)
        if self.renderer == "combined":
            self.dirty = True  # the merged texture holds the transfer functions

    def render(self, full_out, low_out, update: bool = True):
        """Both frames into (H, W, 4) / (H/2, W/2, 4) uint8 CUDA tensors."""
        if update or self.dirty:
            self.full.update()
            self.low.update()
            self.dirty = False
        self.full.render(full_out)
        self.low.render(low_out)


def make_pairs(pr: PairRenderer, pairs: int, timesteps: int, crop: int, seed: int, log=print):
    """``pairs`` aligned crops from frames over ``timesteps`` timesteps; returns
    (low (N, crop, crop, 4), high (N, 2crop, 2crop, 4)) uint8 CUDA tensors."""
    import torch

    rng = np.random.default_rng(seed)
    W, H = pr.width, pr.height
    per_frame = 40
    frames = max(timesteps, (pairs + per_frame - 1) // per_frame)
    low = torch.empty((pairs, crop, crop, 4), dtype=torch.uint8, device="cuda")
    high = torch.empty((pairs, 2 * crop, 2 * crop, 4), dtype=torch.uint8, device="cuda")
    full = torch.empty((H, W, 4), dtype=torch.uint8, device="cuda")
    half = torch.empty((H // 2, W // 2, 4), dtype=torch.uint8, device="cuda")
    k = 0
    t0 = time.time()
    for f in range(frames):
        t = f * timesteps // frames
        if pr.timestep != t:
            pr.set_timestep(t)
        P, MV = random_camera(W, H, rng)
        pr.set_view(P, MV, [random_transfer(rng) for _ in SEEDS])
        pr.render(full, half, update=False)
        take = min(per_frame, pairs - k)
        if take <= 0:
            break
        ys = rng.integers(0, H // 2 - crop + 1, take)
        xs = rng.integers(0, W // 2 - crop + 1, take)
        for y, x in zip(ys, xs):
            low[k] = half[y : y + crop, x : x + crop]
            high[k] = full[2 * y : 2 * y + 2 * crop, 2 * x : 2 * x + 2 * crop]
            k += 1
    torch.cuda.synchronize()
    log(f"pairs: {k} crops from {frames} frame pairs over {timesteps} timesteps in {time.time() - t0:.1f} s")
    return low[:k], high[:k]


def train(net: Reconstructor, low, high, steps: int, batch: int, lr: float, seed: int, log=print):
    """Adam with a cosine learning-rate decay to lr/20; returns the loss history (every 100 steps)."""
    import torch

    rng = np.random.default_rng(seed)
    n = low.shape[0]
    hist = []
    acc = torch.zeros(1, device="cuda")
    t0 = time.time()
    for s in range(steps):
        idx = torch.from_numpy(rng.integers(0, n, batch).astype(np.int32)).cuda(non_blocking=True)
        rate = lr * (0.05 + 0.95 * 0.5 * (1.0 + math.cos(math.pi * s / steps)))
        acc += net.train_step(low, high, idx, rate)
        if (s + 1) % 100 == 0:
            hist.append(float(acc.item()) / 100)
            acc.zero_()
            if (s + 1) % 1000 == 0:
                log(f"step {s + 1}: loss {hist[-1]:.3e} ({time.time() - t0:.1f} s)")
    torch.cuda.synchronize()
    return hist, time.time() - t0


def evaluate(pr: PairRenderer, net: Reconstructor, views: int, seed: int, timesteps: int):
    """Held-out full frames: PSNR (dB) of the reconstruction and of bilinear x2
    against the plain full-size render, per view."""
    import torch

    rng = np.random.default_rng(seed)
    W, H = pr.width, pr.height
    full = torch.empty((H, W, 4), dtype=torch.uint8, device="cuda")
    half = torch.empty((H // 2, W // 2, 4), dtype=torch.uint8, device="cuda")
    out = torch.empty_like(full)
    rec, bil = [], []
    for v in range(views):
        t = int(rng.integers(0, timesteps))
        if pr.timestep != t:
            pr.set_timestep(t)
        P, MV = random_camera(W, H, rng)
        pr.set_view(P, MV, [random_transfer(rng) for _ in SEEDS])
        pr.render(full, half, update=False)
        net.infer(half, out)
        rec.append(psnr(out, full))
        bil.append(psnr(bilinear2(half, out), full))
    return rec, bil


def error_budget(pr: PairRenderer, net: Reconstructor, views: int, seed: int, timesteps: int) -> dict:
    """Where the learned path's error comes from, per held-out view, as PSNR (dB)
    against the plain full-size step render:

    * ``reconstruction`` / ``bilinear``: the network and bilinear x2 on the half-size
      frame at twice the step (the learned path and the method without the network);
    * ``bilinear_half_step``: bilinear x2 on a half-size frame at the full-size step
      (the error of the half-size ray grid alone);
    * ``reconstruction_half_step``: the network on that frame;
    * ``full_double_step``: the full-size frame at twice the step (the error of the
      longer step alone).

    Returns the per-view rows and their means."""
    import torch

    rng = np.random.default_rng(seed)
    W, H = pr.width, pr.height
    full = torch.empty((H, W, 4), dtype=torch.uint8, device="cuda")
    full2 = torch.empty_like(full)
    half = torch.empty((H // 2, W // 2, 4), dtype=torch.uint8, device="cuda")
    half1 = torch.empty_like(half)
    out = torch.empty_like(full)
    rows = []
    for _ in range(views):
        t = int(rng.integers(0, timesteps))
        if pr.timestep != t:
            pr.set_timestep(t)
        P, MV = random_camera(W, H, rng)
        pr.set_view(P, MV, [random_transfer(rng) for _ in SEEDS])
        pr.render(full, half, update=False)
        net.infer(half, out)
        r = {"reconstruction": psnr(out, full), "bilinear": psnr(bilinear2(half, out), full)}
        pr.low.setStep(pr.step)
        pr.full.setStep(2 * pr.step)
        try:
            pr.render(full2, half1, update=False)
        finally:
            pr.low.setStep(2 * pr.step)
            pr.full.setStep(pr.step)
        r["bilinear_half_step"] = psnr(bilinear2(half1, out), full)
        net.infer(half1, out)
        r["reconstruction_half_step"] = psnr(out, full)
        r["full_double_step"] = psnr(full2, full)
        rows.append(r)
    means = {k: float(np.mean([r[k] for r in rows])) for k in rows[0]}
    return {"views": rows, "mean": means}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--pairs", type=int, default=20000)
    ap.add_argument("--timesteps", type=int, default=64)
    ap.add_argument("--crop", type=int, default=128, help="half-size crop edge")
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--eval-views", type=int, default=16)
    ap.add_argument("--renderer", default="per_source", choices=["per_source", "combined"])
    ap.add_argument("--out", default=None, help="weights file (default: the renderer's)")
    ap.add_argument("--error-budget", action="store_true",
                    help="no training: split the committed network's held-out error into its sources (error_budget)")
    a = ap.parse_args(argv)
    a.out = a.out or str(weights_for(a.renderer))
    if a.error_budget:
        pr = PairRenderer(a.size, a.width, a.height, renderer=a.renderer)
        net = Reconstructor(1, a.height // 2, a.width // 2, seed=a.seed)
        net.load(Path(a.out))
        eb = error_budget(pr, net, a.eval_views, a.seed + 4241, a.timesteps)
        print(json.dumps({"renderer": a.renderer, "size": a.size, "frame": [a.width, a.height], "views": a.eval_views,
                          "psnr_db_mean": eb["mean"]}), flush=True)
        return 0

    pr = PairRenderer(a.size, a.width, a.height, renderer=a.renderer)
    low, high = make_pairs(pr, a.pairs, a.timesteps, a.crop, a.seed)
    net = Reconstructor(a.batch, a.crop, a.crop, seed=a.seed)
    hist, secs = train(net, low, high, a.steps, a.batch, a.lr, a.seed + 1)
    del low, high
    net.save(Path(a.out))
    infer_net = Reconstructor(1, a.height // 2, a.width // 2, seed=a.seed)
    infer_net.load(Path(a.out))
    # held-out views: another camera and transfer-function stream, timesteps between the trained ones
    rec, bil = evaluate(pr, infer_net, a.eval_views, a.seed + 1000, a.timesteps)
    line = {
        "renderer": a.renderer, "pairs": a.pairs, "timesteps": a.timesteps, "crop": a.crop, "steps": a.steps,
        "batch": a.batch,
        "train_seconds": secs, "loss_first": hist[0] if hist else None, "loss_last": hist[-1] if hist else None,
        "psnr_recon_db": {"mean": float(np.mean(rec)), "min": float(np.min(rec))},
        "psnr_bilinear_db": {"mean": float(np.mean(bil)), "min": float(np.min(bil))},
        "gain_db_mean": float(np.mean(np.array(rec) - np.array(bil))),
        "error_flag": infer_net.error_flag() | net.error_flag(),
        "weights": a.out,
    }
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
