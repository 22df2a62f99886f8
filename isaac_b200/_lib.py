"""ctypes binding of the C ABI in ``include/isaac_b200.h``.

The shared library is built in-tree (``isaac_b200/_build/libisaac_b200.so``)
by ``isaac_b200.build``.  There is no fallback: if the library is missing the
import fails loudly.
"""

from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

from . import build as _build

HEADER = _build.ROOT / "include" / "isaac_b200.h"

MAX_SOURCES = 16
MAX_FUNCTORS = 3
MAX_CLIPPING = 16

OK = 0
INVALID_ARG = 1
PARSE_ERROR = 2
CUDA_ERROR = 3
TIMEOUT = 4
OOM = 5
NOT_READY = 6
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "PARSE_ERROR", 3: "CUDA_ERROR", 4: "TIMEOUT", 5: "OOM", 6: "NOT_READY"}

F32, BF16, F16 = 0, 1, 2
RENDERER_COMBINED, RENDERER_PER_SOURCE = 0, 1
TIMING_SLOTS = 5
TIMING_NAMES = ("update", "clear_particles", "iso", "ssao", "shade_volume")


class Desc(C.Structure):
    _fields_ = [
        ("framebuffer", C.c_uint32 * 2),
        ("global_size", C.c_uint32 * 3),
        ("local_size", C.c_uint32 * 3),
        ("local_particle_size", C.c_uint32 * 3),
        ("position", C.c_int32 * 3),
        ("scale", C.c_float * 3),
        ("transfer_size", C.c_uint32),
        ("n_volume_sources", C.c_uint32),
        ("n_particle_sources", C.c_uint32),
        ("feature_dim", C.c_uint32 * MAX_SOURCES),
        ("persistent", C.c_uint32 * MAX_SOURCES),
        ("guard_size", C.c_uint32 * MAX_SOURCES),
    ]


class View(C.Structure):
    """``isaacb_view``: one camera of a batch, rendered into ``rgba_dev``."""

    _fields_ = [
        ("ctx_index", C.c_uint32),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("reserved", C.c_uint32),
        ("projection", C.c_double * 16),
        ("modelview", C.c_double * 16),
        ("rgba_dev", C.c_void_p),
    ]


class BatchConfig(C.Structure):
    """``isaacb_batch_config``: tile shape, CTAs per SM and empty-brick skipping."""

    _fields_ = [
        ("tile_w", C.c_uint32),
        ("tile_h", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("skip_empty", C.c_int32),
    ]


class ConvArgs(C.Structure):
    """``isaacb_conv_args``: one tensor-core convolution (forward, input- or weight-gradient)."""

    _fields_ = [
        ("x", C.c_void_p),
        ("w", C.c_void_p),
        ("bias", C.c_void_p),
        ("y", C.c_void_p),
        ("y_f32", C.c_void_p),
        ("mask", C.c_void_p),
        ("dy", C.c_void_p),
        ("dw", C.c_void_p),
        ("error_flag", C.c_void_p),
        ("batch", C.c_uint32),
        ("in_h", C.c_uint32),
        ("in_w", C.c_uint32),
        ("c_in", C.c_uint32),
        ("out_h", C.c_uint32),
        ("out_w", C.c_uint32),
        ("c_out", C.c_uint32),
        ("ksize", C.c_uint32),
        ("stride", C.c_uint32),
        ("pad", C.c_uint32),
        ("transposed", C.c_int32),
        ("relu", C.c_int32),
        ("accumulate", C.c_int32),
        ("wait_check_us", C.c_uint32),
    ]


class IsaacError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_P = C.c_void_p
_u32 = C.c_uint32
_i32 = C.c_int32
_f = C.c_float
_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)
_u64p = C.POINTER(C.c_uint64)

# name -> (restype, argtypes)
SIGNATURES = {
    "isaacb_create": (_i32, [C.POINTER(Desc), C.POINTER(_P)]),
    "isaacb_destroy": (_i32, [_P]),
    "isaacb_last_error": (C.c_char_p, [_P]),
    "isaacb_set_source": (_i32, [_P, _u32, _P]),
    "isaacb_set_particles": (_i32, [_P, _u32, _P, _P, _P, _P, _f]),
    "isaacb_set_functions": (_i32, [_P, _u32, C.c_char_p, _i32p]),
    "isaacb_parse_chain": (_i32, [C.c_char_p, _i32p, _fp, _i32p]),
    "isaacb_set_transfer": (_i32, [_P, _u32, _u32, _u32p, _fp]),
    "isaacb_get_transfer": (_i32, [_P, _u32, _fp]),
    "isaacb_set_weight": (_i32, [_P, _u32, _f]),
    "isaacb_set_iso_threshold": (_i32, [_P, _u32, _f]),
    "isaacb_set_step": (_i32, [_P, _f]),
    "isaacb_set_interpolation": (_i32, [_P, _i32]),
    "isaacb_set_renderer": (_i32, [_P, _i32]),
    "isaacb_set_ao": (_i32, [_P, _i32, _f, _i32]),
    "isaacb_set_ao_pattern": (_i32, [_P, _u32, _f]),
    "isaacb_get_ao_pattern": (_i32, [_P, _P, _P]),
    "isaacb_set_render_mode": (_i32, [_P, _i32]),
    "isaacb_set_dither_mode": (_i32, [_P, _i32]),
    "isaacb_set_storage": (_i32, [_P, _u32, _i32]),
    "isaacb_set_slot_order": (_i32, [_P, _i32]),
    "isaacb_set_background": (_i32, [_P, _fp]),
    "isaacb_add_clipping": (_i32, [_P, _fp, _fp]),
    "isaacb_edit_clipping": (_i32, [_P, _u32, _fp, _fp]),
    "isaacb_remove_clipping": (_i32, [_P, _u32]),
    "isaacb_set_camera": (_i32, [_P, _dp, _dp]),
    "isaacb_update": (_i32, [_P, _P]),
    "isaacb_render": (_i32, [_P, _P, _P]),
    "isaacb_frame": (_i32, [_P, _P, _P]),
    "isaacb_framebuffer": (_i32, [_P, C.POINTER(_P)]),
    "isaacb_minmax": (_i32, [_P, _P, _fp, _fp]),
    "isaacb_get_gbuffer": (_i32, [_P, _P, _P, _P, _P]),
    "isaacb_get_combined": (_i32, [_P, _P, _P, _P]),
    "isaacb_set_counting": (_i32, [_P, _i32]),
    "isaacb_get_counters": (_i32, [_P, _P, _u64p, _u64p]),
    "isaacb_get_launch_count": (_i32, [_P, _u32p, _u32p]),
    "isaacb_set_timing": (_i32, [_P, _i32]),
    "isaacb_get_timing": (_i32, [_P, _P, _fp]),
    "isaacb_minmax_noalloc": (_i32, [_P, _u32p, _u32, _i32p, _fp, _P, _P]),
    "isaacb_batch_create": (_i32, [C.POINTER(_P), _u32, C.POINTER(View), _u32, C.POINTER(_P)]),
    "isaacb_batch_destroy": (_i32, [_P]),
    "isaacb_batch_set_config": (_i32, [_P, C.POINTER(BatchConfig)]),
    "isaacb_batch_get_config": (_i32, [_P, C.POINTER(BatchConfig)]),
    "isaacb_batch_set_camera": (_i32, [_P, _u32, _dp, _dp]),
    "isaacb_batch_render": (_i32, [_P, _P, _i32]),
    "isaacb_batch_capture": (_i32, [_P, _P, _i32]),
    "isaacb_batch_launch_graph": (_i32, [_P, _P]),
    "isaacb_batch_autotune": (_i32, [_P, _P, C.POINTER(BatchConfig), _fp]),
    "isaacb_batch_set_counting": (_i32, [_P, _i32]),
    "isaacb_batch_get_samples": (_i32, [_P, _P, _u64p]),
    "isaacb_batch_get_launch_count": (_i32, [_P, _u32p]),
    "isaacb_conv_forward": (_i32, [C.POINTER(ConvArgs), _P]),
    "isaacb_conv_wgrad": (_i32, [C.POINTER(ConvArgs), _P]),
    "isaacb_recon_param_count": (_u32, []),
    "isaacb_recon_create": (_i32, [_u32, _u32, _u32, C.c_uint64, C.POINTER(_P)]),
    "isaacb_recon_destroy": (_i32, [_P]),
    "isaacb_recon_get_params": (_i32, [_P, _fp]),
    "isaacb_recon_set_params": (_i32, [_P, _fp]),
    "isaacb_recon_train_step": (_i32, [_P, _P, _P, _P, _u32, _u32, _u32, _f, _P, _P, _P]),
    "isaacb_recon_infer": (_i32, [_P, _P, _u32, _u32, _P, _P]),
    "isaacb_recon_error": (_i32, [_P, _i32p]),
    "isaacb_recon_arm_wait_check": (_i32, [_P, _u32]),
    "isaacb_conv_set_producer": (_i32, [_i32]),
    "isaacb_upsample_bilinear2": (_i32, [_P, _u32, _u32, _P, _P]),
    "isaacb_image_sq_error": (_i32, [_P, _P, C.c_uint64, _P, _P]),
    "isaacb_composite": (_i32, [_i32, _P, _P, _u32, _u32, _u32, _u32, _P, _P]),
    "isaacb_set_field_source": (_i32, [_P, _u32, _i32]),
    "isaacb_set_advection": (_i32, [_P, _f, _f, _i32, _i32, _i32]),
    "isaacb_get_advection": (_i32, [_P, _P, _u32, _P]),
    "isaacb_get_noise": (_i32, [_P, _P, _fp]),
    "isaacb_advect": (_i32, [_P, _P]),
    "isaacb_advection_guard": (_i32, [_P, _u32p]),
    "isaacb_pack_guard": (_i32, [_P, _u32, _u32, _P, _P]),
    "isaacb_unpack_guard": (_i32, [_P, _u32, _u32, _P, _P]),
    "isaacb_clear_advection": (_i32, [_P, _P]),
    "isaacb_encoder_create": (_i32, [C.POINTER(_P)]),
    "isaacb_encoder_destroy": (_i32, [_P]),
    "isaacb_encoder_set_quality": (_i32, [_P, _u32]),
    "isaacb_encoder_get_quality": (_i32, [_P, _u32p]),
    "isaacb_encode_jpeg": (_i32, [_P, _P, _u32, _u32, _P, C.POINTER(_P), C.POINTER(C.c_size_t)]),
    "isaacb_encode_frame": (_i32, [_P, _P, _u32, _u32, _i32, _P, C.POINTER(_P), C.POINTER(C.c_size_t)]),
    "isaacb_base64": (_i32, [_P, C.c_size_t, _P, _P]),
    "isaacb_blend_ordered": (_i32, [C.POINTER(_P), _u32, _i32p, _u32, _P, _P, _P]),
}


def header_symbols() -> list[str]:
    """Every ``isaacb_*`` function declared in include/isaac_b200.h."""
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(isaacb_[a-z_0-9]+)\s*\(", text)))


_lib = None


def load(build_if_missing: bool = True) -> C.CDLL:
    """Load the native library (building it first when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not path.exists():
        if not build_if_missing:
            raise ImportError(f"isaac_b200 native library missing: {path}")
        _build.build()
    lib = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, ctx=None) -> int:
    if status not in (OK,):
        msg = load().isaacb_last_error(ctx)
        raise IsaacError(status, msg.decode() if msg else "")
    return status


def lib_path() -> Path:
    return _build.LIB
