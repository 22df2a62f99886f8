"""Storage precision of the per-source renderer against the FP64 CPU ray-marcher.

Four spectral sources (slopes -5/3, -2, -3, -11/3) are rendered by the GPU from
FP32, BF16 and FP16 bricks; interpolation and compositing stay FP32.  The
reference image is the FP64 instantiation of the oracle on the original FP32
data.  Set ISAACB_REPORT to a file path to record the error table as JSON."""

import json
import math
import os

import numpy as np
import pytest

from harness import Scene, build_gpu, build_oracle, image_diff
from isaac_b200 import scenes

pytestmark = pytest.mark.gpu


def _psnr(a, b):
    mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    return float("inf") if mse == 0 else 10 * math.log10(255.0**2 / mse)


def _scene(n=64, fb=(160, 120), optimized=False):
    fields = scenes.precision_scene(n)
    s = Scene(n=(n, n, n), fb=fb, volumes=[(f.numpy(), True) for f in fields])
    s.transfer = [scenes.transfer_4point(0.7 * i) for i in range(4)]
    s.optimized = optimized
    return s


def test_storage_precision_vs_fp64():
    base = _scene()
    ref64 = build_oracle(base, f64=True).frame()
    ref32 = build_oracle(base).frame()
    rows = {"oracle_fp32": dict(image_diff(ref32, ref64), psnr_db=_psnr(ref32, ref64))}
    for dtype, name in [(0, "fp32"), (1, "bf16"), (2, "fp16")]:
        s = _scene()
        s.storage = [dtype] * 4
        got = build_gpu(s).doVisualization()
        rows[name] = dict(image_diff(got, ref64), psnr_db=_psnr(got, ref64))
    # combined renderer (RGBA8 pre-classification) against the FP64 combined march
    comb = _scene(optimized=True)
    ref64c = build_oracle(comb, f64=True).frame()
    ref32c = build_oracle(comb).frame()
    rows["oracle_fp32_combined"] = dict(image_diff(ref32c, ref64c), psnr_db=_psnr(ref32c, ref64c))
    gotc = build_gpu(comb).doVisualization()
    rows["combined_rgba8"] = dict(image_diff(gotc, ref64c), psnr_db=_psnr(gotc, ref64c))
    print(json.dumps(rows, indent=1))
    if os.environ.get("ISAACB_REPORT"):
        with open(os.environ["ISAACB_REPORT"], "w") as f:
            json.dump(rows, f, indent=1)
    # the GPU's FP32 error against FP64 is that of the FP32 restatement itself
    assert rows["fp32"]["mean"] <= rows["oracle_fp32"]["mean"] * 1.5 + 0.01
    assert rows["fp32"]["max"] <= rows["oracle_fp32"]["max"] + 1
    assert rows["combined_rgba8"]["mean"] <= rows["oracle_fp32_combined"]["mean"] * 1.5 + 0.01
    assert rows["combined_rgba8"]["max"] <= rows["oracle_fp32_combined"]["max"] + 1
    # reduced storage precision costs little behind the 1024-entry transfer-function lookup
    assert rows["bf16"]["psnr_db"] > 40 and rows["fp16"]["psnr_db"] > 45
