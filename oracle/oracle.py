"""ctypes wrapper of the CPU oracle (``oracle/isaac_oracle.cpp``).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg, never by the product package.  Parity status:
unpinned (see the header of isaac_oracle.cpp).
"""

from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "build" / "liboracle.so"

_P = C.c_void_p
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)

SIG = {
    "or_create": (_P, [C.c_int, C.c_int, C.c_int, _ip, _ip, _ip, _ip, _fp, C.c_int, C.c_int, C.c_int, _ip, _ip, _ip]),
    "or_destroy": (None, [_P]),
    "or_set_source": (None, [_P, C.c_int, _fp]),
    "or_set_storage": (None, [_P, C.c_int, C.c_int]),
    "or_set_particles": (None, [_P, C.c_int, _u32p, _fp, _fp, _fp, C.c_float]),
    "or_set_functions": (C.c_int, [_P, C.c_int, C.c_char_p]),
    "or_get_chain": (None, [_P, C.c_int, _ip, _fp]),
    "or_set_transfer": (None, [_P, C.c_int, C.c_int, _u32p, _fp]),
    "or_get_lut": (None, [_P, C.c_int, _fp]),
    "or_set_weight": (None, [_P, C.c_int, C.c_float]),
    "or_set_iso": (None, [_P, C.c_int, C.c_float]),
    "or_set_step": (None, [_P, C.c_float]),
    "or_set_interpolation": (None, [_P, C.c_int]),
    "or_set_optimized": (None, [_P, C.c_int]),
    "or_add_clipping": (C.c_int, [_P] + [C.c_float] * 6),
    "or_edit_clipping": (C.c_int, [_P, C.c_int] + [C.c_float] * 6),
    "or_remove_clipping": (None, [_P, C.c_int]),
    "or_set_ao": (None, [_P, C.c_int, C.c_float, C.c_int]),
    "or_set_render_mode": (None, [_P, C.c_int]),
    "or_set_dither_mode": (None, [_P, C.c_int]),
    "or_set_background": (None, [_P, _fp]),
    "or_set_camera": (None, [_P, _dp, _dp]),
    "or_set_framebuffer": (None, [_P, C.c_int, C.c_int]),
    "or_set_field": (None, [_P, C.c_int, C.c_int]),
    "or_set_advection": (None, [_P, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int]),
    "or_get_advection": (None, [_P, C.c_int, _u8p]),
    "or_advect": (None, [_P]),
    "or_pack_guard": (None, [_P, C.c_int, C.c_int, _u8p]),
    "or_unpack_guard": (None, [_P, C.c_int, C.c_int, _u8p]),
    "or_clear_advection": (None, [_P]),
    "or_get_noise": (None, [_P, _fp]),
    "or_update": (None, [_P]),
    "or_render": (None, [_P, _u8p, C.c_int, C.c_int]),
    "or_minmax": (None, [_P, _fp, _fp]),
    "or_get_combined": (None, [_P, _u8p, _u8p]),
    "or_get_gbuffer": (None, [_P, _fp, _fp, _fp]),
    "or_get_inverse_mvp": (None, [_P, _fp]),
    "or_volume_samples": (C.c_ulonglong, [_P]),
    "or_iso_samples": (C.c_ulonglong, [_P]),
    "or_parse_chain": (C.c_int, [C.c_char_p, _ip, _fp]),
    "or_apply_chain": (C.c_float, [_fp, C.c_int, _ip, _fp]),
    "or_dither": (None, [C.c_int, C.c_int, C.c_int, C.c_int, _fp, _u8p]),
    "or_halton": (C.c_float, [C.c_uint, C.c_uint]),
    "or_hsva": (None, [C.c_float, C.c_float, C.c_float, C.c_float, _fp]),
    "or_inverse": (None, [_fp, _fp]),
    "or_round_bf16": (C.c_float, [C.c_float]),
    "or_round_fp16": (C.c_float, [C.c_float]),
    "or_num_threads": (C.c_int, []),
}

_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        for name, (res, args) in SIG.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _iarr(v):
    return (C.c_int * len(v))(*[int(x) for x in v])


def direction_of(index: int) -> tuple:
    """indexToDirection (lib/isaac/isaac_types.hpp:133-143): base-3 digits x, y, z, 2 -> -1."""
    d = []
    for _ in range(3):
        m = index % 3
        d.append(-1 if m == 2 else m)
        index //= 3
    return tuple(d)


def mirrored(index: int) -> int:
    """toMirroredIndex (lib/isaac/isaac_types.hpp:158-161)."""
    return sum((2 if -v == -1 else -v) * 3**a for a, v in enumerate(direction_of(index)))


class Oracle:
    """One oracle context; mirrors the product's setters (test infrastructure)."""

    def __init__(
        self,
        framebuffer,
        global_size,
        local_size,
        local_particle_size,
        position,
        scale,
        feature_dims,
        persistent,
        n_volume,
        transfer_size=1024,
        f64=False,
        guard=None,
    ):
        self.lib = load()
        self.W, self.H = (int(v) for v in framebuffer)
        self.local_size = tuple(int(v) for v in local_size)
        self.scale = tuple(float(v) for v in scale)
        n = len(feature_dims)
        self.n = n
        self.n_volume = n_volume
        self._keep = []
        self.ctx = self.lib.or_create(
            int(f64),
            self.W,
            self.H,
            _iarr(global_size),
            _iarr(local_size),
            _iarr(local_particle_size),
            _iarr(position),
            (C.c_float * 3)(*[float(x) for x in scale]),
            int(transfer_size),
            int(n_volume),
            int(n - n_volume),
            _iarr(feature_dims),
            _iarr([int(p) for p in persistent]),
            _iarr(list(guard) if guard is not None else [0] * n),
        )
        if not self.ctx:
            raise ValueError("oracle: bad configuration")

    def close(self):
        if self.ctx:
            self.lib.or_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_source(self, s: int, data: np.ndarray):
        a = np.ascontiguousarray(data, dtype=np.float32)
        self._keep.append(a)
        self.lib.or_set_source(self.ctx, s, _ptr(a, _fp))

    def set_storage(self, s: int, dtype: int):
        self.lib.or_set_storage(self.ctx, s, int(dtype))

    def set_particles(self, s: int, offsets, positions, attributes, radii=None, const_radius=0.5):
        o = np.ascontiguousarray(offsets, dtype=np.uint32)
        p = np.ascontiguousarray(positions, dtype=np.float32)
        a = np.ascontiguousarray(attributes, dtype=np.float32)
        r = None if radii is None else np.ascontiguousarray(radii, dtype=np.float32)
        self._keep += [o, p, a, r]
        self.lib.or_set_particles(
            self.ctx, s, _ptr(o, _u32p), _ptr(p, _fp), _ptr(a, _fp), None if r is None else _ptr(r, _fp), float(const_radius)
        )

    def set_functions(self, s: int, text: str) -> int:
        return self.lib.or_set_functions(self.ctx, s, text.encode())

    def set_transfer(self, s: int, points: dict):
        keys = np.array(list(points.keys()), dtype=np.uint32)
        rgba = np.array([c for v in points.values() for c in v], dtype=np.float32)
        self.lib.or_set_transfer(self.ctx, s, len(keys), _ptr(keys, _u32p), _ptr(rgba, _fp))

    def lut(self, s: int, ts: int = 1024) -> np.ndarray:
        out = np.zeros((ts, 4), dtype=np.float32)
        self.lib.or_get_lut(self.ctx, s, _ptr(out, _fp))
        return out

    def set_weight(self, s, w):
        self.lib.or_set_weight(self.ctx, s, float(w))

    def set_iso(self, s, v):
        self.lib.or_set_iso(self.ctx, s, float(v))

    def set_step(self, v):
        self.lib.or_set_step(self.ctx, float(v))

    def set_interpolation(self, on):
        self.lib.or_set_interpolation(self.ctx, int(on))

    def set_optimized(self, on):
        self.lib.or_set_optimized(self.ctx, int(on))

    def add_clipping(self, px, py, pz, nx, ny, nz) -> bool:
        return bool(self.lib.or_add_clipping(self.ctx, px, py, pz, nx, ny, nz))

    def edit_clipping(self, nr, px, py, pz, nx, ny, nz) -> bool:
        return bool(self.lib.or_edit_clipping(self.ctx, nr, px, py, pz, nx, ny, nz))

    def remove_clipping(self, nr):
        self.lib.or_remove_clipping(self.ctx, nr)

    def set_ao(self, enabled, weight=0.5, filt=False):
        self.lib.or_set_ao(self.ctx, int(enabled), float(weight), int(filt))

    def set_render_mode(self, m):
        self.lib.or_set_render_mode(self.ctx, int(m))

    def set_dither_mode(self, m):
        self.lib.or_set_dither_mode(self.ctx, int(m))

    def set_background(self, rgba):
        a = np.array(rgba, dtype=np.float32)
        self.lib.or_set_background(self.ctx, _ptr(a, _fp))

    def set_camera(self, P, MV):
        p = np.ascontiguousarray(P, dtype=np.float64).reshape(16)
        m = np.ascontiguousarray(MV, dtype=np.float64).reshape(16)
        self.lib.or_set_camera(self.ctx, _ptr(p, _dp), _ptr(m, _dp))

    def set_field(self, src: int, enabled: bool = True):
        """Mark volume source ``src`` (featureDim 3, after every plain volume source) as an advected field."""
        self.lib.or_set_field(self.ctx, int(src), int(enabled))

    def set_advection(self, step_factor=1.0, history_weight=0.95, seeding_period=1, seeding_time=1, seed_points=1000):
        self.lib.or_set_advection(self.ctx, float(step_factor), float(history_weight), int(seeding_period),
                                  int(seeding_time), int(seed_points))

    def advection(self, src: int) -> np.ndarray:
        lx, ly, lz = self.local_size
        out = np.zeros((lz, ly, lx), dtype=np.uint8)
        self.lib.or_get_advection(self.ctx, int(src), _ptr(out, _u8p))
        return out

    # ----- advection guard slabs between ranks (SyncToOwnGuard / SyncFromNeighbourGuard)
    def advect(self):
        """The advection step alone; the next update() merges without advecting again."""
        self.lib.or_advect(self.ctx)

    def guard_slab(self, direction: int) -> tuple:
        """(x, y, z) extent of the guard slab of neighbour index ``direction``."""
        e = []
        for a in range(3):
            d = direction_of(direction)[a]
            g = int(np.ceil(np.float32(4.0) / np.float32(self.scale[a])))
            e.append(g if d != 0 else self.local_size[a])
        return tuple(e)

    def pack_guard(self, src: int, direction: int) -> np.ndarray:
        out = np.zeros(int(np.prod(self.guard_slab(direction))), dtype=np.uint8)
        self.lib.or_pack_guard(self.ctx, int(src), int(direction), _ptr(out, _u8p))
        return out

    def unpack_guard(self, src: int, direction: int, data: np.ndarray):
        data = np.ascontiguousarray(data, dtype=np.uint8).reshape(-1)
        assert data.size == int(np.prod(self.guard_slab(direction)))
        self.lib.or_unpack_guard(self.ctx, int(src), int(direction), _ptr(data, _u8p))

    def clear_advection(self):
        self.lib.or_clear_advection(self.ctx)

    def noise(self) -> np.ndarray:
        lx, ly, lz = self.local_size
        out = np.zeros((lz, ly, lx), dtype=np.float32)
        self.lib.or_get_noise(self.ctx, _ptr(out, _fp))
        return out

    def set_framebuffer(self, w: int, h: int):
        self.lib.or_set_framebuffer(self.ctx, int(w), int(h))
        self.W, self.H = int(w), int(h)

    def update(self):
        self.lib.or_update(self.ctx)

    def render(self, rows=None) -> np.ndarray:
        out = np.zeros((self.H, self.W, 4), dtype=np.uint8)
        r0, r1 = (0, self.H) if rows is None else rows
        self.lib.or_render(self.ctx, _ptr(out, _u8p), int(r0), int(r1))
        return out

    def frame(self) -> np.ndarray:
        self.update()
        return self.render()

    def minmax(self):
        mn = np.zeros(self.n, dtype=np.float32)
        mx = np.zeros(self.n, dtype=np.float32)
        self.lib.or_minmax(self.ctx, _ptr(mn, _fp), _ptr(mx, _fp))
        return mn, mx

    def combined(self):
        lx, ly, lz = self.local_size
        vol = np.zeros((lz, ly, lx, 4), dtype=np.uint8)
        iso = np.zeros((lz, ly, lx, 4), dtype=np.uint8)
        self.lib.or_get_combined(self.ctx, _ptr(vol, _u8p), _ptr(iso, _u8p))
        return vol, iso

    def gbuffer(self):
        depth = np.zeros((self.H, self.W), dtype=np.float32)
        normal = np.zeros((self.H, self.W, 3), dtype=np.float32)
        ao = np.zeros((self.H, self.W), dtype=np.float32)
        self.lib.or_get_gbuffer(self.ctx, _ptr(depth, _fp), _ptr(normal, _fp), _ptr(ao, _fp))
        return depth, normal, ao

    def inverse_mvp(self):
        out = np.zeros(16, dtype=np.float32)
        self.lib.or_get_inverse_mvp(self.ctx, _ptr(out, _fp))
        return out

    def samples(self):
        return int(self.lib.or_volume_samples(self.ctx)), int(self.lib.or_iso_samples(self.ctx))


# ---- stand-alone known-answer helpers
def parse_chain(text: str):
    lib = load()
    bc = (C.c_int * 3)()
    pr = (C.c_float * 12)()
    err = lib.or_parse_chain(text.encode(), bc, pr)
    return err, list(bc), list(pr)


def apply_chain(values, bytecode, params) -> float:
    lib = load()
    v = (C.c_float * 4)(*([float(x) for x in values] + [0.0] * (4 - len(values))))
    return float(lib.or_apply_chain(v, len(values), (C.c_int * 3)(*bytecode), (C.c_float * 12)(*params)))


def dither(mode, x, y, z, rgba):
    lib = load()
    out = (C.c_uint8 * 4)()
    lib.or_dither(mode, x, y, z, (C.c_float * 4)(*rgba), out)
    return list(out)


def halton(index, base):
    return float(load().or_halton(index, base))


def hsva(h, s, v, a):
    out = (C.c_float * 4)()
    load().or_hsva(h, s, v, a, out)
    return list(out)


def num_threads() -> int:
    return int(load().or_num_threads())
