"""Ray-march speed against the viewing angle, a diagnostic for the brick layouts.

``python -m isaac_b200.sweep`` renders the same 4 x 512^3 spectral sources from an
orbit of cameras (yaw 0-90 degrees) with the per-source renderer (BF16 bricks,
1920x1080 at step 0.5 and 960x540 at step 1.0, as the learned path uses) and with
the combined renderer (1920x1080, step 0.5), and prints one JSON line per view:
milliseconds per frame (CUDA events, 5 frames after 2 untimed ones), samples per
frame (the kernels' own count) and millions of samples per millisecond.  The
samples hardly change with the angle, so the rate shows how the access pattern of
each layout depends on the view direction.
"""

from __future__ import annotations

import argparse
import json
import math


def _time(viz, buf, repeat=5):
    import torch

    viz.setCounting(True)
    viz.render(buf)
    samples = viz.counters()[0]
    viz.setCounting(False)
    for _ in range(2):
        viz.render(buf)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(repeat):
        viz.render(buf)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / repeat
    return round(ms, 3), int(samples), round(samples / ms / 1e6, 1)


def main(argv=None) -> int:
    import torch

    from . import scenes
    from .recon_train import PairRenderer
    from .visualization import IsaacVisualization, VolumeSource

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--yaws", default="0,10,20,30,45,60,75,90", help="degrees")
    ap.add_argument("--pitch", type=float, default=0.35, help="radians")
    args = ap.parse_args(argv)
    W, H = 1920, 1080
    n = args.size
    pr = PairRenderer(n, W, H)
    pr.set_timestep(0)
    tfs = [scenes.transfer_4point(0.7 * i) for i in range(4)]
    pr.set_view(*scenes.orbit_camera(W, H, yaw=0.0, pitch=args.pitch, distance=2.4), tfs)
    pr.full.update()
    pr.low.update()
    fields = scenes.precision_scene(n, device="cuda")
    comb = IsaacVisualization("combined", (W, H), (n, n, n), (n, n, n), (1, 1, 1), (0, 0, 0),
                              [VolumeSource(f"s{i}", f.contiguous(), 1) for i, f in enumerate(fields)])
    comb.setInterpolation(True)
    for i in range(4):
        comb.setTransferPoints(i, tfs[i])
    comb.update()
    full = torch.empty((H, W, 4), dtype=torch.uint8, device="cuda")
    half = torch.empty((H // 2, W // 2, 4), dtype=torch.uint8, device="cuda")
    for deg in (float(v) for v in args.yaws.split(",")):
        P, MV = scenes.orbit_camera(W, H, yaw=math.radians(deg), pitch=args.pitch, distance=2.4)
        line = {"yaw_deg": deg, "pitch_rad": args.pitch, "fields": "[ms, samples, Msamples/ms]"}
        pr.low.setCamera(P, MV)
        line["per_source_half"] = _time(pr.low, half)
        pr.full.setCamera(P, MV)
        line["per_source_full"] = _time(pr.full, full)
        comb.setCamera(P, MV)
        line["combined_full"] = _time(comb, full)
        print(json.dumps(line), flush=True)
    comb.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
