"""The C++ front end (include/isaac_b200.hpp) used as a simulation would use it:
compiled with nvcc into tests/cpp/frontend_example.cu, fed a seeded scene, and
checked against the CPU oracle (frame within the parity bar, min/max bit-exact).
With a field source (the reference's FieldSourceList), the vector source is
advected and the third frame is compared."""

import os
import shutil
import subprocess

import numpy as np
import pytest

from harness import Scene, assert_image_parity, build_oracle
from isaac_b200 import build as B
from isaac_b200 import scenes

pytestmark = pytest.mark.gpu


def _compile(tmp):
    exe = os.path.join(tmp, "frontend_example")
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    lib = str(B.OUT_DIR)
    cmd = [nvcc, "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-I", str(B.ROOT / "include"),
           str(B.ROOT / "tests" / "cpp" / "frontend_example.cu"), "-L", lib, "-lisaac_b200",
           "-Xlinker", f"-rpath={lib}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


@pytest.mark.parametrize("field", [False, True], ids=["volume_sources", "field_source"])
def test_cpp_frontend_matches_oracle(tmp_path, field):
    B.build()
    n, W, H = 32, 64, 48
    cells = (8, 8, 8)
    scalar, curl = scenes.gaussian_scene(n, seed=3)
    off, pos, attr = scenes.particles_uniform(700, cells, seed=4)
    P, MV = scenes.camera(W, H, seed=5)
    scene_file = tmp_path / "scene.bin"
    with open(scene_file, "wb") as f:
        np.array([n, W, H, *cells], dtype=np.int32).tofile(f)
        np.ascontiguousarray(P, dtype=np.float64).tofile(f)
        np.ascontiguousarray(MV, dtype=np.float64).tofile(f)
        scalar.numpy().tofile(f)
        curl.numpy().tofile(f)
        off.numpy().astype(np.uint32).tofile(f)
        pos.numpy().tofile(f)
        attr.numpy().tofile(f)
    exe = _compile(str(tmp_path))
    out_file = tmp_path / "out.bin"
    r = subprocess.run([exe, str(scene_file), str(out_file)] + (["--field"] if field else []), capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = np.fromfile(out_file, dtype=np.uint8)
    frame = raw[: W * H * 4].reshape(H, W, 4)
    mm = raw[W * H * 4:].view(np.float32)
    gmn, gmx = mm[:3], mm[3:]

    s = Scene(n=(n, n, n), fb=(W, H), volumes=[(scalar.numpy(), True), (curl.numpy(), True)])
    s.particle_cells = cells
    s.particles = [(off.numpy(), pos.numpy(), attr.numpy(), np.full(len(pos), 0.45, np.float32), 0.0)]
    s.functions = ["idem", "length", "length"]
    s.transfer = [
        {0: (0, 0, 0, 0), 300: (0.8, 0.3, 0.2, 0.1), 700: (0.2, 0.7, 0.9, 0.4), 1024: (1, 1, 0.5, 0.9)},
        {0: (0, 0, 0, 0), 1024: (0.3, 0.9, 0.4, 0.6)},
        {0: (0.1, 0.9, 0.1, 1), 1024: (0.9, 0.1, 0.1, 1)},
    ]
    s.iso = [0.45, 0.0]
    o = build_oracle(s)
    o.set_camera(P, MV)
    if field:
        o.set_field(1)
        o.set_advection(1.0, 0.95, 1, 1, 40)
        for _ in range(2):
            o.frame()
    ref = o.frame()
    assert_image_parity(frame, ref)
    rmn, rmx = o.minmax()
    assert gmn.tobytes() == rmn.tobytes() and gmx.tobytes() == rmx.tobytes()
