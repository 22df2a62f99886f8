"""Seeded synthetic scenes for the parity tests and the benchmark.

The reference ships no data sets; these generators produce inputs with the
shapes, sizes and value ranges of the benchmark configurations:

* ``gaussian_scene`` -- a float32 scalar field, the sum of 8 Gaussians
  (centres U[0,1]^3, sigma U[0.05,0.15], amplitudes U[0.5,1]) at cell
  centres, rescaled to [0,1], plus the float32x3 curl of psi*z_hat,
  (d psi/dy, -d psi/dx, 0), divided by its largest length.
* ``spectral_field`` -- a Gaussian random field with power spectrum k^slope
  (FFT of seeded white noise), used for the lognormal density, its gradient
  and the iso-surface scalar, and for the four-source precision scene.
* ``particles_uniform`` -- particles uniform in the box with Maxwellian
  velocities, binned into a cell list (counting sort).
* ``camera`` -- explicit projection (45 degrees, in degrees) and an orbit
  modelview at a given distance.

Everything is generated with torch on the requested device from a seeded
generator, so a test can build the same float32 arrays on the CPU for the
oracle and copy them to the GPU for the kernels.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from .visualization import _cm_mul, perspective


def _gen(seed: int, device="cpu") -> torch.Generator:
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return g


def gaussian_scene(n: int, seed: int = 1, device="cpu"):
    """Scalar (n,n,n) and curl (n,n,n,3) float32 fields of the 8-Gaussian scene."""
    g = _gen(seed, "cpu")
    c = torch.rand(8, 3, generator=g, dtype=torch.float64)
    sig = 0.05 + 0.10 * torch.rand(8, generator=g, dtype=torch.float64)
    amp = 0.5 + 0.5 * torch.rand(8, generator=g, dtype=torch.float64)
    x = (torch.arange(n, dtype=torch.float64, device=device) + 0.5) / n
    Z, Y, X = torch.meshgrid(x, x, x, indexing="ij")
    phi = torch.zeros_like(X)
    dpx = torch.zeros_like(X)
    dpy = torch.zeros_like(X)
    for i in range(8):
        cx, cy, cz = (float(v) for v in c[i])
        s2 = float(sig[i]) ** 2
        e = float(amp[i]) * torch.exp(-((X - cx) ** 2 + (Y - cy) ** 2 + (Z - cz) ** 2) / (2 * s2))
        phi += e
        dpx += e * (-(X - cx) / s2)
        dpy += e * (-(Y - cy) / s2)
    scalar = (phi - phi.min()) / (phi.max() - phi.min())
    curl = torch.stack([dpy, -dpx, torch.zeros_like(dpx)], dim=-1)
    curl = curl / torch.linalg.vector_norm(curl, dim=-1).max()
    return scalar.to(torch.float32).contiguous(), curl.to(torch.float32).contiguous()


def spectral_field(n: int, slope: float, seed: int, device="cpu", shift: float = 0.0) -> torch.Tensor:
    """Zero-mean, unit-variance Gaussian random field on n^3 with P(k) ~ k^slope (float32).

    ``shift`` advects the periodic field along x (the fastest axis) by that
    fraction of the box, as a phase shift of every Fourier mode."""
    g = _gen(seed, device)
    noise = torch.randn((n, n, n), generator=g, device=device, dtype=torch.float32)
    f = torch.fft.rfftn(noise)
    kx = torch.fft.fftfreq(n, device=device)
    kz = torch.fft.rfftfreq(n, device=device)
    KX, KY, KZ = torch.meshgrid(kx, kx, kz, indexing="ij")
    k = torch.sqrt(KX * KX + KY * KY + KZ * KZ)
    amp = torch.where(k > 0, k.clamp_min(1e-12) ** (slope / 2.0), torch.zeros_like(k))
    if shift:
        # f(x - s) <-> F(k) exp(-2 pi i k s), s in cells along the last axis
        amp = amp * torch.exp(torch.complex(torch.zeros_like(KZ), -2.0 * math.pi * KZ * (shift * n)))
    field = torch.fft.irfftn(f * amp, s=(n, n, n))
    field = (field - field.mean()) / field.std()
    return field.to(torch.float32).contiguous()


def unit_range(f: torch.Tensor) -> torch.Tensor:
    lo, hi = f.min(), f.max()
    return ((f - lo) / (hi - lo)).to(torch.float32).contiguous()


def density_gradient_scene(n: int, seeds=(2, 3, 4), device="cpu"):
    """Three sources of the full-feature scene.

    * lognormal density rho = exp(g), stored as (log rho - min)/(2 range) in [0, 0.5],
      so that the chain "mul(2),add(1)" -- which the reference parser reads as
      mul(2), the part after the comma being ignored -- maps it onto [0, 1];
    * E = grad g (float32x3), divided by its largest length, chain "length";
    * a second spectral scalar in [0,1], chain "idem", whose transfer-function
      alpha steps at its 90th percentile (the iso surface).
    """
    g = spectral_field(n, -5.0 / 3.0, seeds[0], device)
    dens = ((g - g.min()) / (2 * (g.max() - g.min()))).to(torch.float32).contiguous()
    gx = (torch.roll(g, -1, 2) - torch.roll(g, 1, 2)) * 0.5
    gy = (torch.roll(g, -1, 1) - torch.roll(g, 1, 1)) * 0.5
    gz = (torch.roll(g, -1, 0) - torch.roll(g, 1, 0)) * 0.5
    E = torch.stack([gx, gy, gz], dim=-1)
    E = (E / torch.linalg.vector_norm(E, dim=-1).max()).to(torch.float32).contiguous()
    s = unit_range(spectral_field(n, -2.0, seeds[2], device))
    p90 = float(torch.quantile(s.flatten()[:: max(1, s.numel() // (1 << 22))].double(), 0.9))
    return dens, E, s, p90


def precision_scene(
    n: int, seeds=(6, 7, 8, 9), slopes=(-5.0 / 3.0, -2.0, -3.0, -11.0 / 3.0), device="cpu", shift: float = 0.0
):
    """Four scalar spectral fields in [0,1] (advected by ``shift`` of the box along x)."""
    return [unit_range(spectral_field(n, s, sd, device, shift)) for sd, s in zip(seeds, slopes)]


# the batching workload: 16 views of uneven resolution over 4 timesteps
BATCH_RESOLUTIONS = [(256, 256)] * 4 + [(1280, 720)] * 4 + [(1920, 1080)] * 4 + [(2048, 1152)] * 4


def batch_views(resolutions=None, timesteps: int = 4, seed0: int = 100, distance: float = 2.5):
    """(timestep, width, height, projection, modelview) per view: view i shows
    timestep i mod ``timesteps`` from a seeded camera on the orbit sphere."""
    res = BATCH_RESOLUTIONS if resolutions is None else resolutions
    out = []
    for i, (w, h) in enumerate(res):
        P, MV = camera(w, h, seed=seed0 + i, distance=distance)
        out.append((i % timesteps, w, h, P, MV))
    return out


def particles_uniform(count: int, cells, seed: int = 5, device="cpu"):
    """``count`` particles uniform in a box of ``cells`` (x,y,z) particle cells with
    N(0,1)^3 velocities; returns (offsets, positions, attributes) as a cell list
    sorted by cell (x fastest), positions relative to their cell, attributes = v / max|v|."""
    g = _gen(seed, device)
    cx, cy, cz = (int(v) for v in cells)
    p = torch.rand((count, 3), generator=g, device=device, dtype=torch.float32)
    p = p * torch.tensor([cx, cy, cz], device=device, dtype=torch.float32)
    v = torch.randn((count, 3), generator=g, device=device, dtype=torch.float32)
    v = v / torch.linalg.vector_norm(v, dim=-1).max()
    cell = torch.floor(p).to(torch.int64)
    cell[:, 0].clamp_(0, cx - 1)
    cell[:, 1].clamp_(0, cy - 1)
    cell[:, 2].clamp_(0, cz - 1)
    idx = cell[:, 0] + cell[:, 1] * cx + cell[:, 2] * cx * cy
    order = torch.argsort(idx, stable=True)
    idx = idx[order]
    rel = (p - cell.to(torch.float32))[order].contiguous()
    attr = v[order].contiguous()
    counts = torch.bincount(idx, minlength=cx * cy * cz)
    offsets = torch.zeros(cx * cy * cz + 1, dtype=torch.int64, device=device)
    offsets[1:] = torch.cumsum(counts, 0)
    return offsets.to(torch.int32).contiguous(), rel, attr


def rotation_y(angle: float) -> np.ndarray:
    """3x3 rotation about y, column-major [col][row]."""
    c, s = math.cos(angle), math.sin(angle)
    row_major = np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]], dtype=np.float64)
    return row_major.T.copy()


def rotation_x(angle: float) -> np.ndarray:
    c, s = math.cos(angle), math.sin(angle)
    row_major = np.array([[1, 0, 0], [0, c, -s], [0, s, c]], dtype=np.float64)
    return row_major.T.copy()


def camera(width: int, height: int, seed: int = 1, distance: float = 2.5, fov_degrees: float = 45.0, tilt: float | None = None):
    """Projection (fov in degrees) and modelview orbiting the volume centre at ``distance``
    with a seeded rotation about y (and a seeded tilt about x unless ``tilt`` is given)."""
    rng = np.random.default_rng(seed)
    yaw = float(rng.uniform(0, 2 * math.pi))
    pitch = float(rng.uniform(-0.6, 0.6)) if tilt is None else float(tilt)
    P = perspective(math.radians(fov_degrees), width / height, 0.002, 100.0)
    rot = _cm_mul(rotation_x(pitch), rotation_y(yaw))
    R = np.eye(4)
    R[0:3, 0:3] = rot
    D = np.eye(4)
    D[3][2] = -distance
    MV = _cm_mul(D, R)
    return P, MV


def orbit_camera(width: int, height: int, yaw: float, pitch: float = 0.3, distance: float = 2.5, fov_degrees: float = 45.0):
    """Projection and modelview of a camera orbiting the volume centre (angles in radians)."""
    P = perspective(math.radians(fov_degrees), width / height, 0.002, 100.0)
    rot = _cm_mul(rotation_x(pitch), rotation_y(yaw))
    R = np.eye(4)
    R[0:3, 0:3] = rot
    D = np.eye(4)
    D[3][2] = -distance
    return P, _cm_mul(D, R)


def transfer_4point(hue: float = 0.0):
    """A 4-point piecewise-linear RGBA transfer function (keys in 0..1024)."""
    h = hue
    c1 = (0.9 * abs(math.cos(h)), 0.5 * abs(math.sin(h)) + 0.2, 0.3, 0.0)
    c2 = (0.2, 0.8 * abs(math.cos(h + 1.0)), 0.9 * abs(math.sin(h + 1.0)), 0.35)
    c3 = (1.0, 0.9, 0.5 * abs(math.cos(h + 2.0)), 0.9)
    return {0: (0.0, 0.0, 0.0, 0.0), 300: c1, 700: c2, 1024: c3}
