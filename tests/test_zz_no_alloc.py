"""isaacb_minmax_noalloc: the min/max entry point for callers that cannot call
cudaMalloc (a simulation that keeps nearly all device memory for its own heap,
or a loop that must not take cudaMalloc's device synchronisation).  It must give
exactly what the context-based isaacb_minmax gives, call after call, although
every call shares one static scratch array.

This file is collected last on purpose (tests/test_zz_*), so a run that stops at
the first failure has run every other test first."""

import ctypes as C

import numpy as np
import pytest
import torch

from isaac_b200 import _lib, scenes

pytestmark = pytest.mark.gpu


def _parse(chain: str):
    lib = _lib.load()
    bc = (C.c_int32 * 3)()
    pr = (C.c_float * 12)()
    err = C.c_int32(0)
    assert lib.isaacb_parse_chain(chain.encode(), bc, pr, C.byref(err)) == _lib.OK
    return bc, pr


def _noalloc(src: torch.Tensor, size, fdim: int, chain: str) -> np.ndarray:
    lib = _lib.load()
    bc, pr = _parse(chain)
    out = torch.full((2,), float("nan"), dtype=torch.float32, device="cuda")
    sz = (C.c_uint32 * 3)(*size)
    st = lib.isaacb_minmax_noalloc(
        C.c_void_p(src.data_ptr()), sz, fdim, bc, pr, C.c_void_p(out.data_ptr()),
        C.c_void_p(torch.cuda.current_stream().cuda_stream),
    )
    assert st == _lib.OK, lib.isaacb_last_error(None)
    return out.cpu().numpy()


def _with_context(vols, chains):
    from isaac_b200 import IsaacVisualization, VolumeSource

    n = vols[0].shape[0]
    srcs = [VolumeSource(f"s{i}", v, feature_dim=(v.shape[-1] if v.dim() == 4 else 1)) for i, v in enumerate(vols)]
    viz = IsaacVisualization("ref", (16, 16), (n, n, n), (n, n, n), (1, 1, 1), (0, 0, 0), srcs)
    viz.functions = list(chains)
    viz.updateFunctions()
    mn, mx = viz.minMax()
    viz.close()
    return mn, mx


def test_noalloc_matches_context_minmax_on_consecutive_calls():
    n = 48
    scalar, curl = scenes.gaussian_scene(n, seed=5)
    a = (scalar * 3.0 - 1.0).contiguous().cuda()
    a.view(-1)[1234] = -0.0
    b = curl.cuda()
    chains = ["mul(2)|add(-0.5)", "length|mul(3)"]
    mn, mx = _with_context([a, b], chains)
    # two calls in a row share the static scratch; the second must not see the first's leftovers
    r1 = _noalloc(a, (n, n, n), 1, chains[0])
    r2 = _noalloc(b, (n, n, n), 3, chains[1])
    torch.cuda.synchronize()
    assert r1[0].tobytes() == mn[0].tobytes() and r1[1].tobytes() == mx[0].tobytes()
    assert r2[0].tobytes() == mn[1].tobytes() and r2[1].tobytes() == mx[1].tobytes()
    # a smaller source after a larger one reads only its own columns
    small = a[:20, :20, :20].contiguous()
    mn_s, mx_s = _with_context([small], ["idem"])
    r3 = _noalloc(small, (20, 20, 20), 1, "idem")
    torch.cuda.synchronize()
    assert r3[0].tobytes() == mn_s[0].tobytes() and r3[1].tobytes() == mx_s[0].tobytes()


def test_noalloc_signed_zero_in_column_order():
    """The reference scans each (x,y) column over z, then the columns in order, keeping
    the earlier value on ties.  With +0 at (column 5, z 0) and -0 at (column 0, z 1) the
    column order meets -0 first, while a scan in memory order would meet +0 first."""
    n = 16
    rng = np.random.default_rng(11)
    neg = -rng.uniform(0.1, 1.0, (n, n, n)).astype(np.float32)  # (z, y, x), all < 0
    neg[0, 0, 5] = 0.0
    neg[1, 0, 0] = -0.0
    pos = -neg  # all > 0; -0 at (column 5, z 0), +0 at (column 0, z 1)
    a = torch.from_numpy(neg).cuda()
    b = torch.from_numpy(pos).cuda()
    mn, mx = _with_context([a, b], ["idem", "idem"])
    ra = _noalloc(a, (n, n, n), 1, "idem")
    rb = _noalloc(b, (n, n, n), 1, "idem")
    torch.cuda.synchronize()
    assert ra[1].tobytes() == mx[0].tobytes() == np.float32(-0.0).tobytes()
    assert rb[0].tobytes() == mn[1].tobytes() == np.float32(0.0).tobytes()
    assert ra[0].tobytes() == mn[0].tobytes() and rb[1].tobytes() == mx[1].tobytes()


def test_noalloc_rejects_sources_beyond_the_static_scratch():
    lib = _lib.load()
    bc, pr = _parse("idem")
    dummy = torch.zeros(4, device="cuda")
    out = torch.zeros(2, device="cuda")
    sz = (C.c_uint32 * 3)(1024, 257, 1)  # 263168 columns > 262144
    st = lib.isaacb_minmax_noalloc(C.c_void_p(dummy.data_ptr()), sz, 1, bc, pr, C.c_void_p(out.data_ptr()), None)
    assert st == _lib.INVALID_ARG
    assert b"static scratch" in lib.isaacb_last_error(None)
    deep = (C.c_uint32 * 3)(1, 1, (1 << 20) + 1)
    st = lib.isaacb_minmax_noalloc(C.c_void_p(dummy.data_ptr()), deep, 1, bc, pr, C.c_void_p(out.data_ptr()), None)
    assert st == _lib.INVALID_ARG
    assert b"z planes" in lib.isaacb_last_error(None)
