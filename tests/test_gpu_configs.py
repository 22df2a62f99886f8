"""Parity at the full sizes of the benchmark configurations, through the C ABI, and
the error of each configuration against the FP64 CPU ray-marcher.

Each scene is the benchmark's own (``bench.build_scene``, generated on the GPU from
the same seeds) and is compared with the CPU oracle:

* 8-Gaussian scene: 128^3 scalar + curl (chain ``length``) -> 512x512;
* full-feature scene: 3 x 256^3 sources (lognormal density under ``mul(2),add(1)``,
  its gradient under ``length``, an iso scalar), 1M particles, two clipping planes,
  SSAO -> 1920x1080;
* precision scene: 4 x 512^3 spectral sources -> 1920x1080, with the combined
  renderer over the whole frame and with the per-source renderer on FP32, BF16 and
  FP16 bricks over five bands of rows spread over the frame (the CPU march of four
  sources costs about a minute per full frame).

Parity bars: merged textures and min/max bit-exact; RGBA8 frames within 1 LSB per
channel on >= 99.9 % of pixels and <= 3 LSB anywhere; ray-march iteration counts
within 0.05 % of the oracle's.

Error table: every frame is also compared with the FP64 instantiation of the
oracle on the same FP32 inputs (per-source rows: on the unrounded sources, so the
storage rounding is part of the error).  Per row: max, mean and 99.9th-percentile
absolute error per channel (LSB) and PSNR.  Set ISAACB_REPORT to a file path to
write the table as JSON.
"""

import dataclasses
import json
import math
import os

import numpy as np
import pytest
import torch

from harness import assert_image_parity, build_gpu, build_oracle, config_scene

pytestmark = pytest.mark.gpu

# five bands of 24 rows, spread from the bottom to the top of a 1080-row frame
BANDS = [(60, 84), (300, 324), (528, 552), (756, 780), (996, 1020)]

TABLE = {}


def _rows(img, bands):
    return np.concatenate([img[r0:r1] for r0, r1 in bands], axis=0)


def error_row(img: np.ndarray, ref64: np.ndarray) -> dict:
    d = np.abs(img.astype(np.int16) - ref64.astype(np.int16)).astype(np.float64)
    mse = float(np.mean(d * d))
    return {
        "max": int(d.max()),
        "mean": float(d.mean()),
        "p99_9": float(np.percentile(d, 99.9)),
        "psnr_db": float("inf") if mse == 0 else 10 * math.log10(255.0**2 / mse),
    }


# Per-row bounds on the GPU frame against FP64 (max LSB, mean LSB, min PSNR dB), set from
# the measured table with margin.  The full-feature row is dominated by threshold
# decisions -- iso hits at local maxima of the field near the threshold, particle
# silhouettes and the SSAO depth comparisons they feed -- that FP32 and FP64 arithmetic
# take differently at a few hundred pixels; the FP32 oracle shows the same error.
BOUNDS = {
    "gaussian_128_512px_combined": (3, 0.02, 60.0),
    "full_feature_256_1080p_combined": (255, 0.6, 33.0),
    "precision_512_1080p_combined": (3, 0.02, 60.0),
    "precision_512_1080p_per_source_f32": (3, 0.02, 60.0),
    "precision_512_1080p_per_source_bf16": (3, 0.03, 60.0),
    "precision_512_1080p_per_source_f16": (3, 0.02, 60.0),
}


def _record(name, got, ref32, ref64, **extra):
    row = {"gpu": error_row(got, ref64), "oracle_fp32": error_row(ref32, ref64)}
    row.update(extra)
    TABLE[name] = row
    mx, mean, psnr = BOUNDS[name]
    g = row["gpu"]
    assert g["max"] <= mx and g["mean"] <= mean and g["psnr_db"] >= psnr, (name, row)
    return row


def _counts_close(got: int, ref: int):
    assert abs(got - ref) <= max(2, ref // 2000), (got, ref)


def _minmax_exact(viz, o):
    gmn, gmx = viz.minMax()
    rmn, rmx = o.minmax()
    assert gmn.tobytes() == rmn.tobytes() and gmx.tobytes() == rmx.tobytes(), (gmn, rmn, gmx, rmx)


def _close(viz):
    viz.close()
    torch.cuda.empty_cache()


def _fp32_error_bounds(row):
    """The GPU computes in FP32 like the FP32 oracle and stays within 1 LSB of it, so
    its error against FP64 is the FP32 restatement's own, give or take that LSB."""
    g, o = row["gpu"], row["oracle_fp32"]
    assert g["max"] <= o["max"] + 1, row
    assert g["mean"] <= o["mean"] * 1.25 + 0.01, row
    assert g["p99_9"] <= o["p99_9"] + 1, row


# --------------------------------------------------------------------- 8-Gaussian scene, 512x512
def test_gaussian_128_at_512px():
    s = config_scene("gaussian")
    o = build_oracle(s)
    o.update()
    rv, ri = o.combined()
    ref = o.render()
    rs = o.samples()
    viz = build_gpu(s)
    viz.update()
    gv, gi = viz.combinedTextures()
    assert np.array_equal(gv, rv) and np.array_equal(gi, ri)
    viz.setCounting(True)
    got = viz.doVisualization()
    assert_image_parity(got, ref)
    _counts_close(viz.counters()[0], rs[0])
    _minmax_exact(viz, o)
    _close(viz)
    ref64 = build_oracle(s, f64=True).frame()
    _fp32_error_bounds(_record("gaussian_128_512px_combined", got, ref, ref64, pixels="all"))


# --------------------------------------------------------------------- full-feature scene, 1080p
def test_full_feature_256_at_1080p():
    s = config_scene("full")
    o = build_oracle(s)
    o.update()
    rv, ri = o.combined()
    ref = o.render()
    rs = o.samples()
    rd, _, rao = o.gbuffer()
    viz = build_gpu(s)
    viz.update()
    gv, gi = viz.combinedTextures()
    assert np.array_equal(gv, rv) and np.array_equal(gi, ri)
    viz.setCounting(True)
    got = viz.doVisualization()
    assert_image_parity(got, ref)
    gvs, gis = viz.counters()
    _counts_close(gvs, rs[0])
    _counts_close(gis, rs[1])
    gd, _, gao = viz.gbuffer()
    hit = rd < 1e30
    ghit = gd < 1e30
    assert hit.mean() > 0.05  # particles and the iso surface cover part of the frame
    # a silhouette pixel may hit on one side only where a ray grazes a sphere or the
    # iso threshold within rounding
    assert (ghit != hit).mean() <= 0.001
    both = hit & ghit
    assert np.allclose(gd[both], rd[both], rtol=1e-4, atol=1e-4)
    # AO counts depth comparisons over 49 taps: a tap flips only where two depths are
    # within rounding of each other
    assert (gao == rao).mean() >= 0.999 and np.abs(gao - rao).max() <= 2.0 / 42.0 + 1e-6
    _minmax_exact(viz, o)  # three volume sources and the particle attribute
    _close(viz)
    ref64 = build_oracle(s, f64=True).frame()
    _fp32_error_bounds(_record("full_feature_256_1080p_combined", got, ref, ref64, pixels="all"))


# --------------------------------------------------------------------- precision scene, 4 x 512^3, 1080p
@pytest.fixture(scope="module")
def precision_scene():
    return config_scene("precision")


def test_precision_512_combined(precision_scene):
    s = precision_scene
    o = build_oracle(s)
    o.update()
    rv, ri = o.combined()
    viz = build_gpu(s)
    viz.update()
    gv, gi = viz.combinedTextures()
    assert np.array_equal(gv, rv) and np.array_equal(gi, ri)
    del gv, gi, rv, ri
    _minmax_exact(viz, o)
    ref = o.render()
    rs = o.samples()
    viz.setCounting(True)
    got = viz.doVisualization()
    assert_image_parity(got, ref)
    _counts_close(viz.counters()[0], rs[0])
    _close(viz)
    o.close()
    o64 = build_oracle(s, f64=True)
    ref64 = o64.frame()
    o64.close()
    _fp32_error_bounds(_record("precision_512_1080p_combined", got, ref, ref64, pixels="all"))


@pytest.fixture(scope="module")
def per_source_fp64(precision_scene):
    """The FP64 per-source march over the unrounded FP32 sources, on the bands."""
    s = dataclasses.replace(precision_scene, optimized=False, storage=[])
    o = build_oracle(s, f64=True)
    o.update()
    ref = np.zeros((s.fb[1], s.fb[0], 4), dtype=np.uint8)
    for r0, r1 in BANDS:
        ref[r0:r1] = o.render(rows=(r0, r1))[r0:r1]
    o.close()
    return ref


@pytest.mark.parametrize("dtype", ["f32", "bf16", "f16"])
def test_precision_512_per_source(precision_scene, per_source_fp64, dtype):
    s = dataclasses.replace(precision_scene, optimized=False, storage=[{"f32": 0, "bf16": 1, "f16": 2}[dtype]] * 4)
    o = build_oracle(s)
    o.update()
    viz = build_gpu(s)
    got = viz.doVisualization()
    _close(viz)
    ref = np.zeros_like(got)
    for r0, r1 in BANDS:
        ref[r0:r1] = o.render(rows=(r0, r1))[r0:r1]
        assert_image_parity(got[r0:r1], ref[r0:r1])
    o.close()
    row = _record(f"precision_512_1080p_per_source_{dtype}", _rows(got, BANDS), _rows(ref, BANDS),
                  _rows(per_source_fp64, BANDS), pixels=f"rows {BANDS}")
    if dtype == "f32":
        _fp32_error_bounds(row)
    else:
        # the storage rounding dominates; the FP32 oracle on the rounded sources shows
        # the same error, so the GPU adds nothing to it
        _fp32_error_bounds(row)
        assert row["gpu"]["psnr_db"] >= 40.0, row


def test_zz_error_table():
    """Writes the table (ISAACB_REPORT) once every configuration above has run."""
    print(json.dumps(TABLE, indent=1))
    if os.environ.get("ISAACB_REPORT"):
        with open(os.environ["ISAACB_REPORT"], "w") as f:
            json.dump(TABLE, f, indent=1)
    if len(TABLE) < 6:
        pytest.skip(f"only {sorted(TABLE)} ran")


# --------------------------------------------------------------------- batching, 16 views x 4 timesteps of 4 x 512^3
def test_batch_16_views_at_config_size():
    """The batching configuration at full size: 16 views of uneven resolution over 4
    advected timesteps of the four 512^3 sources, in one persistent launch and as a
    captured graph.  Every view equals the single-view render of its timestep's context
    bit for bit, and a 256x256 view is within the parity bar of the oracle."""
    import argparse

    import bench
    from isaac_b200 import scenes
    from isaac_b200.batch import IsaacBatch

    args = argparse.Namespace(scene="batch", size=512, sources=4, width=1920, height=1080, timesteps=4, shift=0.05,
                              renderer="combined", dtype="f32", learned_renderer="per_source", ao_samples=0,
                              ao_radius=8.0)
    small = bench._small(args)
    steps_sc = bench.build_batch_scenes(args, "cuda")
    vis = [bench.make_viz(small, sc) for sc in steps_sc]
    views = scenes.batch_views(timesteps=args.timesteps)
    batch = IsaacBatch(vis, views)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        batch.render(update=True)
        batch.capture(update=True)
        batch.launchGraph()
    stream.synchronize()
    for i, (t, w, h, P, MV) in enumerate(views):
        single = bench.make_viz(argparse.Namespace(**{**vars(small), "width": w, "height": h}), steps_sc[t])
        single.setCamera(P, MV)
        ref = single.doVisualization()
        assert np.array_equal(batch.frames[i].cpu().numpy(), ref), i
        if i == 0:
            # the oracle on the same timestep's sources, 256x256
            from harness import Scene

            s = Scene(n=(512, 512, 512), fb=(w, h), volumes=[(f.cpu().numpy(), True) for f, _ in steps_sc[t].volumes])
            s.transfer = list(steps_sc[t].transfer)
            s.P, s.MV = P, MV
            o = build_oracle(s)
            assert_image_parity(ref, o.frame())
            o.close()
        single.close()
    batch.close()
    for v in vis:
        v.close()


# --------------------------------------------------------------------- learned reconstruction at 1920x1080
@pytest.mark.parametrize("renderer", ["per_source", "combined"])
def test_learned_path_at_config_size(renderer):
    """The learned configuration at full size: the four 512^3 sources, 960x540 at step
    1.0 reconstructed to 1920x1080 by the committed network, judged against the plain
    1920x1080 step-0.5 render on an orbit of cameras: every frame at or above 40 dB (no
    fallback) and the network at least as close as bilinear x2 on average."""
    import math

    from isaac_b200 import recon, scenes
    from isaac_b200.recon_train import PairRenderer

    W, H = 1920, 1080
    pr = PairRenderer(512, W, H, renderer=renderer)
    pr.set_timestep(0)
    tfs = [scenes.transfer_4point(0.7 * i) for i in range(4)]
    cams = [scenes.orbit_camera(W, H, yaw=2 * math.pi * k / 8.0, pitch=0.35, distance=2.4) for k in range(8)]
    pr.set_view(*cams[0], tfs)
    pr.full.update()
    pr.low.update()
    net = recon.Reconstructor(1, H // 2, W // 2, seed=1)
    net.load(recon.weights_for(renderer))
    jr = recon.JudgedRenderer(pr.full, pr.low, net, judge_every=1, threshold=40.0)
    tmp = torch.empty((H, W, 4), dtype=torch.uint8, device="cuda")
    gains = []
    for P, MV in cams:
        jr.setCamera(P, MV)
        jr.frame()
        p_rec = jr.judged[-1][1]
        gains.append(p_rec - recon.psnr(recon.bilinear2(jr.half, tmp), jr.full))
        assert p_rec >= 40.0, jr.judged
    assert jr.fallback_frames == 0
    assert float(np.mean(gains)) > 0.0, gains
    assert net.error_flag() == 0
    net.close()
    for v in (pr.full, pr.low):
        v.close()
