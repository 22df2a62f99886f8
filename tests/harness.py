"""Builds the same scene for the product (CUDA, through the C ABI) and for the
CPU oracle, and compares their outputs.  Test infrastructure."""

from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field

import numpy as np
import torch

from isaac_b200 import scenes
from oracle import oracle as O


@dataclass
class Scene:
    n: tuple = (32, 32, 32)  # local size (x, y, z)
    global_n: tuple | None = None  # global size; None: the local size
    position: tuple = (0, 0, 0)  # of the local box inside the global volume
    fb: tuple = (64, 48)
    volumes: list = field(default_factory=list)  # list of (array (Z,Y,X[,C]) float32, persistent)
    particles: list = field(default_factory=list)  # list of (offsets, pos, attr, radii or None, const radius)
    particle_cells: tuple = (8, 8, 8)
    functions: list = field(default_factory=list)  # per combined source
    transfer: list = field(default_factory=list)  # per combined source: dict or None
    weights: list = field(default_factory=list)
    iso: list = field(default_factory=list)
    step: float = 0.5
    interpolation: bool = True
    clips: list = field(default_factory=list)
    ao: tuple = (False, 0.5, False)
    render_mode: int = 0
    dither_mode: int = 1
    background: tuple = (0.0, 0.0, 0.0, 0.0)
    camera_seed: int = 1
    camera_distance: float = 2.5
    optimized: bool = True
    storage: list = field(default_factory=list)  # per volume source: 0 f32, 1 bf16, 2 f16
    scale: tuple = (1.0, 1.0, 1.0)
    transfer_size: int = 1024
    P: object = None  # explicit projection and modelview; None: scenes.camera(camera_seed)
    MV: object = None
    guard: list = field(default_factory=list)  # per volume source: guard cells per side (arrays include them)


def gaussian_pair(n=32, fb=(64, 48), seed=1, **kw) -> Scene:
    sc, curl = scenes.gaussian_scene(n, seed)
    s = Scene(n=(n, n, n), fb=fb, volumes=[(sc.numpy(), True), (curl.numpy(), True)])
    s.functions = ["idem", "length"]
    s.transfer = [scenes.transfer_4point(0.3), scenes.transfer_4point(1.7)]
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def round_storage(a: np.ndarray, dtype: int) -> np.ndarray:
    """Round float32 data to bf16 / fp16 (round to nearest even) and back."""
    if dtype == 2:
        return a.astype(np.float16).astype(np.float32)
    if dtype == 1:
        u = a.astype(np.float32).view(np.uint32).astype(np.uint64)
        lsb = (u >> 16) & 1
        u = ((u + 0x7FFF + lsb) & 0xFFFF0000).astype(np.uint32)
        return u.view(np.float32)
    return a


def build_oracle(s: Scene, f64: bool = False) -> O.Oracle:
    nvol = len(s.volumes)
    fdims = [1 if v.ndim == 3 else v.shape[-1] for v, _ in s.volumes] + [
        (1 if p[2].ndim == 1 else p[2].shape[-1]) for p in s.particles
    ]
    pers = [int(p) for _, p in s.volumes] + [1] * len(s.particles)
    guard = [s.guard[i] if i < len(s.guard) else 0 for i in range(nvol)] + [0] * len(s.particles)
    o = O.Oracle(
        s.fb, s.global_n or s.n, s.n, s.particle_cells, s.position, s.scale, fdims, pers, nvol,
        transfer_size=s.transfer_size, f64=f64, guard=guard
    )
    for i, (v, _) in enumerate(s.volumes):
        dt = s.storage[i] if i < len(s.storage) else 0
        o.set_source(i, round_storage(v, dt) if (not s.optimized and _ and dt) else v)
        if not s.optimized and dt:
            o.set_storage(i, dt)
    for j, p in enumerate(s.particles):
        off, pos, attr, radii, cr = p
        o.set_particles(nvol + j, off, pos, attr, radii, cr)
    _apply_settings(s, o, oracle=True)
    return o


def build_gpu(s: Scene):
    from isaac_b200 import IsaacVisualization, ParticleSource, VolumeSource

    vols = []
    for i, (v, pers) in enumerate(s.volumes):
        t = torch.from_numpy(np.ascontiguousarray(v)).cuda()
        vols.append(VolumeSource(f"src{i}", t, feature_dim=1 if v.ndim == 3 else v.shape[-1], persistent=pers,
                                 guard_size=s.guard[i] if i < len(s.guard) else 0))
    parts = []
    for j, p in enumerate(s.particles):
        off, pos, attr, radii, cr = p
        parts.append(
            ParticleSource(
                f"part{j}",
                torch.from_numpy(np.ascontiguousarray(off.astype(np.int32))).cuda(),
                torch.from_numpy(np.ascontiguousarray(pos)).cuda(),
                torch.from_numpy(np.ascontiguousarray(attr)).cuda(),
                None if radii is None else torch.from_numpy(np.ascontiguousarray(radii)).cuda(),
                cr,
            )
        )
    viz = IsaacVisualization(
        "test", s.fb, s.global_n or s.n, s.n, s.particle_cells, s.position, vols, parts, scale=s.scale,
        transfer_size=s.transfer_size
    )
    viz._keep = (vols, parts)
    _apply_settings(s, viz, oracle=False)
    return viz


def _apply_settings(s: Scene, t, oracle: bool):
    n = len(s.volumes) + len(s.particles)
    if s.P is not None:
        P, MV = s.P, s.MV
    else:
        P, MV = scenes.camera(s.fb[0], s.fb[1], seed=s.camera_seed, distance=s.camera_distance)
    if oracle:
        for i in range(n):
            if i < len(s.functions) and s.functions[i]:
                t.set_functions(i, s.functions[i])
            if i < len(s.transfer) and s.transfer[i]:
                t.set_transfer(i, s.transfer[i])
            if i < len(s.weights):
                t.set_weight(i, s.weights[i])
            if i < len(s.iso):
                t.set_iso(i, s.iso[i])
        t.set_step(s.step)
        t.set_interpolation(s.interpolation)
        t.set_optimized(s.optimized)
        for c in s.clips:
            t.add_clipping(*c)
        t.set_ao(*s.ao)
        t.set_render_mode(s.render_mode)
        t.set_dither_mode(s.dither_mode)
        t.set_background(s.background)
        t.set_camera(P, MV)
    else:
        for i in range(n):
            if i < len(s.functions) and s.functions[i]:
                t.functions[i] = s.functions[i]
            if i < len(s.transfer) and s.transfer[i]:
                t.setTransferPoints(i, s.transfer[i])
            if i < len(s.weights):
                t.setWeight(i, s.weights[i])
            if i < len(s.iso):
                t.setIsoThreshold(i, s.iso[i])
        t.updateFunctions()
        t.setStep(s.step)
        t.setInterpolation(s.interpolation)
        t.setRenderOptimization(s.optimized)
        for i in range(len(s.volumes)):
            if i < len(s.storage):
                t.setStorage(i, s.storage[i])
        for c in s.clips:
            t.addClipping(*c)
        t.setAmbientOcclusion(*s.ao)
        t.setRenderMode(s.render_mode)
        t.setDitherMode(s.dither_mode)
        t.setBackgroundColor(s.background)
        t.setCamera(P, MV)


def config_scene(scene: str, renderer: str = "combined", dtype: str = "f32") -> Scene:
    """The benchmark's own scene of one configuration (``bench.build_scene``), generated
    on the GPU from the same seeds, as a harness Scene with float32 host arrays.

    ``scene``: "gaussian" (128^3 scalar + curl -> 512x512), "full" (3 x 256^3 sources,
    1M particles, iso, 2 clipping planes, SSAO -> 1920x1080) or "precision" (4 x 512^3
    spectral sources -> 1920x1080)."""
    import argparse

    import bench

    args = argparse.Namespace(scene=scene, size=512, sources=4, width=1920, height=1080, renderer=renderer,
                              dtype=dtype)
    bench.apply_scene_defaults(args)
    sc = bench.build_scene(args, "cuda")
    n = args.size
    s = Scene(n=(n, n, n), fb=(args.width, args.height))
    s.volumes = [(t.cpu().numpy(), True) for t, _ in sc.volumes]
    if sc.particles is not None:
        off, pos, attr, radius, cells = sc.particles
        s.particles = [(off.cpu().numpy(), pos.cpu().numpy(), attr.cpu().numpy(), None, radius)]
        s.particle_cells = tuple(cells)
    s.functions = list(sc.functions)
    s.transfer = list(sc.transfer)
    s.iso = list(sc.iso)
    s.clips = list(sc.clips)
    s.ao = (bool(sc.ao), 0.5, False)
    s.P, s.MV = sc.P, sc.MV
    if renderer == "per_source":
        s.optimized = False
        s.storage = [{"f32": 0, "bf16": 1, "f16": 2}[dtype]] * len(s.volumes)
    del sc
    return s


def image_diff(a: np.ndarray, b: np.ndarray) -> dict:
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    per_px = d.max(axis=-1)
    return {
        "max": int(d.max()) if d.size else 0,
        "frac_le1": float((per_px <= 1).mean()) if per_px.size else 1.0,
        "frac_exact": float((per_px == 0).mean()) if per_px.size else 1.0,
        "mean": float(d.mean()) if d.size else 0.0,
    }


def assert_image_parity(gpu: np.ndarray, ref: np.ndarray, frac: float = 0.999, max_lsb: int = 3):
    """RGBA8 parity bar: <=1 LSB per channel on >= 99.9 % of pixels and <= 3 LSB anywhere."""
    st = image_diff(gpu, ref)
    assert st["frac_le1"] >= frac and st["max"] <= max_lsb, st
    return st
