"""Build recipe of the native library ``isaac_b200/_build/libisaac_b200.so``.

The library is plain CUDA C++ behind a C ABI (``include/isaac_b200.h``); it is
compiled with ``nvcc`` for sm_100a only.  Device code is compiled with
``--fmad=false`` so that plain float expressions round like the reference's CPU
backend; kernels that accept a fused multiply-add call ``fmaf`` explicitly.
Host code is compiled with ``-ffp-contract=off`` for the same reason (the
camera inverse and the transfer tables are formed on the host).
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_build"
LIB = OUT_DIR / "libisaac_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--fmad=false",
    "-Xcompiler",
    "-fPIC,-ffp-contract=off,-O2",
    "-I",
    str(ROOT / "include"),
]
SOURCES = [
    "api.cu",
    "kernels_merge.cu",
    "kernels_minmax.cu",
    "kernels_render.cu",
    "kernels_legacy.cu",
    "minmax_static.cu",
    "kernels_batch.cu",
    "recon_gemm.cu",
    "recon.cu",
    "composite.cu",
    "encode.cu",
]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build isaac_b200")
    return exe


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> Path:
    """Compile every CUDA source and link the shared library; returns its path."""
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "isaac_b200.h"]
    objs = []
    jobs = []
    for src in SOURCES:
        s = CSRC / src
        o = OUT_DIR / (s.stem + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers + [Path(__file__)]):
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(s), "-o", str(o)]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    failures = []
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, r in ex.map(run, jobs):
            if r.returncode != 0:
                failures.append((cmd, r.stderr))
            elif verbose or ptxas_info:
                sys.stdout.write(r.stderr)
    if failures:
        msg = "\n".join(" ".join(c) + "\n" + e for c, e in failures)
        raise RuntimeError("nvcc failed:\n" + msg)
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart", "-lnvjpeg"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stderr)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
