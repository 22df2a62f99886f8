"""The C-ABI library loads on a machine without a GPU, exports every symbol the
header declares, and its host-only parser agrees with the oracle."""

import ctypes as C

import numpy as np
import pytest

from isaac_b200 import _lib
from oracle import oracle as O


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    declared = _lib.header_symbols()
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared) == set(_lib.SIGNATURES), "ctypes signatures out of date"


def _product_parse(text: str):
    lib = _lib.load()
    bc = (C.c_int32 * 3)()
    pr = (C.c_float * 12)()
    err = C.c_int32(0)
    st = lib.isaacb_parse_chain(text.encode(), bc, pr, C.byref(err))
    assert st in (_lib.OK, _lib.PARSE_ERROR)
    assert (st == _lib.OK) == (err.value == 0)
    return err.value, list(bc), list(pr)


CASES = [
    "idem", "mul(2)|add(1)", "mul(2),add(1)", "length|mul(2)|add(-1)", "idem|idem|idem|idem", "mul(2", "mul(1,2,3,4,5)",
    "foo", "mul(x)|add(1)", "mul(1e50)", " mul ( 2 ) | sum ", "mul()", "mul(1,2)", "", "idem|", "pow(2)|length|sum",
    "add(0x1p3)", "mul(inf)", "add(nan)", "mul(1e-50)", "mul(2)xyz", "sum|sum|sum", "|", "((", "mul)(2",
]


@pytest.mark.parametrize("text", CASES)
def test_parser_matches_oracle(text):
    e1, b1, p1 = _product_parse(text)
    e2, b2, p2 = O.parse_chain(text)
    assert e1 == e2 and b1 == b2
    assert np.array_equal(np.array(p1, dtype=np.float32), np.array(p2, dtype=np.float32), equal_nan=True)


def test_parser_fuzz_matches_oracle():
    rng = np.random.default_rng(11)
    alphabet = list("idemaulngthpowsr()|,.0123456789-+e ")
    for _ in range(3000):
        text = "".join(rng.choice(alphabet, size=int(rng.integers(0, 24))))
        e1, b1, p1 = _product_parse(text)
        e2, b2, p2 = O.parse_chain(text)
        assert (e1, b1) == (e2, b2), text
        assert np.array_equal(np.array(p1, dtype=np.float32), np.array(p2, dtype=np.float32), equal_nan=True), text


def test_create_rejects_bad_descriptors_without_gpu():
    lib = _lib.load()
    d = _lib.Desc()
    ctx = C.c_void_p()
    st = lib.isaacb_create(C.byref(d), C.byref(ctx))  # zero sources
    assert st == _lib.INVALID_ARG
    assert b"sources" in lib.isaacb_last_error(None)
    d.n_volume_sources = 1
    d.framebuffer[:] = (16, 16)
    d.local_size[:] = (8, 8, 8)
    d.global_size[:] = (8, 8, 8)
    d.scale[:] = (1, 1, 1)
    d.transfer_size = 1024
    d.feature_dim[0] = 5
    assert lib.isaacb_create(C.byref(d), C.byref(ctx)) == _lib.INVALID_ARG
    d.feature_dim[0] = 1
    d.guard_size[0] = 65  # guard cells: 0..64 per side
    assert lib.isaacb_create(C.byref(d), C.byref(ctx)) == _lib.INVALID_ARG
    assert b"guard_size" in lib.isaacb_last_error(None)
    d.guard_size[0] = 0
    d.n_particle_sources = 1
    d.local_particle_size[:] = (2, 2, 2)
    d.feature_dim[1] = 1
    d.guard_size[1] = 1  # particle sources have no guard
    assert lib.isaacb_create(C.byref(d), C.byref(ctx)) == _lib.INVALID_ARG


def test_batch_rejects_bad_arguments_without_gpu():
    lib = _lib.load()
    out = C.c_void_p()
    views = (_lib.View * 1)()
    ctxs = (C.c_void_p * 1)()
    assert lib.isaacb_batch_create(None, 1, views, 1, C.byref(out)) == _lib.INVALID_ARG
    assert lib.isaacb_batch_create(ctxs, 0, views, 1, C.byref(out)) == _lib.INVALID_ARG
    assert lib.isaacb_batch_create(ctxs, 1, views, 1, C.byref(out)) == _lib.INVALID_ARG  # null context
    assert b"null context" in lib.isaacb_last_error(None)
    assert lib.isaacb_batch_destroy(None) == _lib.OK
    assert lib.isaacb_batch_render(None, None, 0) == _lib.INVALID_ARG
    assert lib.isaacb_batch_launch_graph(None, None) == _lib.NOT_READY
    assert lib.isaacb_batch_set_config(None, None) == _lib.INVALID_ARG
    assert lib.isaacb_batch_get_launch_count(None, None) == _lib.INVALID_ARG


def test_encoder_rejects_bad_arguments_without_gpu():
    lib = _lib.load()
    ptr, n = C.c_void_p(), C.c_size_t()
    assert lib.isaacb_encoder_create(None) == _lib.INVALID_ARG
    assert lib.isaacb_encoder_destroy(None) == _lib.OK
    assert lib.isaacb_encoder_set_quality(None, 90) == _lib.INVALID_ARG
    assert lib.isaacb_encoder_get_quality(None, None) == _lib.INVALID_ARG
    assert lib.isaacb_encode_jpeg(None, None, 16, 16, None, C.byref(ptr), C.byref(n)) == _lib.INVALID_ARG
    assert lib.isaacb_encode_frame(None, None, 16, 16, 1, None, C.byref(ptr), C.byref(n)) == _lib.INVALID_ARG
    assert b"isaacb_encode_frame" in lib.isaacb_last_error(None)
    assert lib.isaacb_base64(None, 5, None, None) == _lib.INVALID_ARG
    assert lib.isaacb_base64(None, 0, None, None) == _lib.OK


def test_blend_rejects_bad_arguments_without_gpu():
    lib = _lib.load()
    ptrs = (C.c_void_p * 2)(16, 32)
    bad = (C.c_int32 * 2)(0, 0)  # not a permutation
    assert lib.isaacb_blend_ordered(ptrs, 2, bad, 4, None, C.c_void_p(64), None) == _lib.INVALID_ARG
    assert b"permutation" in lib.isaacb_last_error(None)
    assert lib.isaacb_blend_ordered(ptrs, 0, bad, 4, None, C.c_void_p(64), None) == _lib.INVALID_ARG
    assert lib.isaacb_blend_ordered(ptrs, 65, bad, 4, None, C.c_void_p(64), None) == _lib.INVALID_ARG


def test_parser_token_fuzz_matches_oracle():
    """Strings built from whole tokens reach the argument lists and the functor limit
    far more often than single characters do."""
    rng = np.random.default_rng(12)
    tokens = ["idem", "add", "mul", "length", "pow", "sum", "foo", "(", ")", ",", "|", " ", "2", "-1.5", "1e40",
              "1e-45", "x", "nan", "0x10", ""]
    for _ in range(5000):
        text = "".join(rng.choice(tokens, size=int(rng.integers(0, 14))))
        e1, b1, p1 = _product_parse(text)
        e2, b2, p2 = O.parse_chain(text)
        assert (e1, b1) == (e2, b2), text
        assert np.array_equal(np.array(p1, dtype=np.float32), np.array(p2, dtype=np.float32), equal_nan=True), text
