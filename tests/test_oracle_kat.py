"""Known-answer tests of the CPU oracle, derived by hand from the reference text.

The reference has no tests or golden vectors; these values follow from reading
lib/isaac.hpp:1079-1266 (parser, transfer tables), lib/isaac/isaac_functors.hpp,
lib/isaac/isaac_dither_kernel.hpp:7-329, lib/isaac/isaac_helper.hpp:57-264.
"""

import math

import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize(
    "text,err,bc,p0,p1",
    [
        ("idem", 0, [0, 0, 0], [0, 0, 0, 0], [0, 0, 0, 0]),
        ("mul(2)|add(1)", 0, [2, 1, 0], [2, 2, 2, 2], [1, 1, 1, 1]),
        # the parser splits on '|': everything after the first ')' of a token is ignored
        ("mul(2),add(1)", 0, [2, 0, 0], [2, 2, 2, 2], [0, 0, 0, 0]),
        ("idem|idem|idem|idem", 1, [0, 0, 0], [0, 0, 0, 0], [0, 0, 0, 0]),
        ("mul(2", -1, [0, 0, 0], [0, 0, 0, 0], [0, 0, 0, 0]),
        ("mul(1,2,3,4,5)", 2, [2, 0, 0], [1, 2, 3, 4], [0, 0, 0, 0]),
        ("foo", -2, [0, 0, 0], [0, 0, 0, 0], [0, 0, 0, 0]),
        ("mul(x)|add(1)", -2, [2, 1, 0], [0, 0, 0, 0], [1, 1, 1, 1]),
        ("mul(1e50)", -2, [2, 0, 0], [0, 0, 0, 0], [0, 0, 0, 0]),
        (" mul ( 2 ) | sum ", 0, [2, 5, 0], [2, 2, 2, 2], [0, 0, 0, 0]),
        ("mul()", 0, [2, 0, 0], [0, 0, 0, 0], [0, 0, 0, 0]),
        ("mul(1,2)", 0, [2, 0, 0], [1, 2, 2, 2], [0, 0, 0, 0]),
        ("", -2, [0, 0, 0], [0, 0, 0, 0], [0, 0, 0, 0]),
        ("idem|", -2, [0, 0, 0], [0, 0, 0, 0], [0, 0, 0, 0]),
        ("pow(2)|length|sum", 0, [4, 3, 5], [2, 2, 2, 2], [0, 0, 0, 0]),
        ("mul(2)xyz", 0, [2, 0, 0], [2, 2, 2, 2], [0, 0, 0, 0]),
    ],
)
def test_parser_known_answers(text, err, bc, p0, p1):
    e, b, p = O.parse_chain(text)
    assert e == err
    assert b == bc
    assert p[0:4] == pytest.approx(p0)
    assert p[4:8] == pytest.approx(p1)


def _chain(text):
    e, b, p = O.parse_chain(text)
    return b, p


@pytest.mark.parametrize(
    "text,values,expected",
    [
        ("mul(2)|add(1)", [3.0], 7.0),
        ("mul(2),add(1)", [3.0], 6.0),
        ("length", [3.0, 4.0], 5.0),
        ("length", [3.0, 4.0, 12.0], 13.0),
        ("sum", [1.0, 2.0, 3.0], 6.0),
        ("length|mul(2)", [3.0, 4.0, 0.0], 10.0),
        ("add(1,2,3)", [1.0, 1.0, 1.0], 2.0),  # the chain result is the x component
        ("idem", [0.25, 7.0, 9.0], 0.25),
        ("pow(2)", [3.0], 9.0),
        ("mul(-1)|length", [-2.0], 2.0),
    ],
)
def test_chain_known_answers(text, values, expected):
    b, p = _chain(text)
    assert O.apply_chain(values, b, p) == pytest.approx(expected, rel=1e-6)


def test_dither_mode1_mask():
    # mask (isaac_dither_kernel.hpp:25-29): index x%4 + (y%4)*4 + (z%4)*16, value/64
    assert O.dither(1, 0, 0, 0, [0.5, 0.5, 0.5, 0.5]) == [128] * 4  # fract .5 > 17/64
    assert O.dither(1, 1, 0, 0, [0.5, 0.5, 0.5, 0.5]) == [127] * 4  # fract .5 < 46/64
    assert O.dither(1, 3, 3, 3, [0.5] * 4) == [128] * 4  # mask[63] = 16 -> .25 < .5
    assert O.dither(1, 3, 0, 0, [0.5] * 4) == [128] * 4  # mask[3] = 1 -> 1/64


def test_dither_values():
    m1 = [17, 46, 55, 1, 57, 7, 38, 31, 9, 52, 2, 54, 36, 26, 19, 44, 53, 20, 47, 22, 29, 60, 62, 12, 45, 14, 26,
          33, 8, 39, 11, 63, 13, 56, 6, 50, 40, 32, 23, 48, 21, 42, 51, 5, 61, 3, 34, 27, 41, 10, 30, 37, 4, 35, 15,
          59, 49, 24, 43, 18, 25, 64, 58, 16]
    rng = np.random.default_rng(0)
    for _ in range(200):
        x, y, z = (int(v) for v in rng.integers(0, 50, 3))
        c = rng.uniform(0, 1, 4).astype(np.float32)
        d = np.float32(m1[x % 4 + (y % 4) * 4 + (z % 4) * 16]) / np.float32(64)
        s = c * np.float32(255)
        exp = [min(255, int(v) + (1 if (v - math.floor(v)) > d else 0)) for v in s]
        assert O.dither(1, x, y, z, list(c)) == exp
    # mode 0: clamp, round half away from zero
    assert O.dither(0, 0, 0, 0, [0.5, 1.5, -1.0, 0.998]) == [128, 255, 0, 254]


def test_dither_mode1_mask_value_64_never_rounds_up():
    # mask value 64 at index 61 -> threshold 1.0; fract is < 1 so never rounds up
    x, y, z = 61 % 4, (61 // 4) % 4, 61 // 16
    assert O.dither(1, x, y, z, [0.999] * 4) == [254] * 4


def test_halton():
    assert O.halton(1, 2) == 0.5
    assert O.halton(3, 2) == 0.75
    assert O.halton(1, 3) == pytest.approx(1 / 3)
    assert O.halton(0, 3) == 0.0
    assert O.halton(5, 3) == pytest.approx(2 / 3 + 1 / 9, rel=1e-6)


def test_hsva():
    assert O.hsva(0.0, 1, 1, 1) == [1.0, 0.0, 0.0, 1.0]
    r = O.hsva(math.pi / 2, 1, 1, 0.5)  # hi = 1, f = 0.5 -> (q, v, p) = (0.5, 1, 0)
    assert r == pytest.approx([0.5, 1.0, 0.0, 0.5])
    r = O.hsva(float(np.float32(math.pi)), 1, 1, 1)  # hi = 3 -> (p, q, v)
    assert r[0] == 0.0 and r[2] == 1.0 and r[1] == pytest.approx(1.0, abs=1e-6)


def _tiny(n=4, fdims=(1,), nvol=1, fb=(8, 8)):
    return O.Oracle(fb, (n, n, n), (n, n, n), (2, 2, 2), (0, 0, 0), (1, 1, 1), list(fdims), [1] * len(fdims), nvol)


def test_default_transfer_tables():
    o = _tiny(fdims=(1, 1), nvol=2)
    lut0 = o.lut(0)
    # source 0 of 2: hue 0 -> (1,0,0); alpha ramps 0 -> 1 over keys 0..1024 (lib/isaac.hpp:759-793)
    assert lut0[0] == pytest.approx([1, 0, 0, 0])
    assert lut0[512] == pytest.approx([1, 0, 0, 0.5])
    assert lut0[1023] == pytest.approx([1, 0, 0, 1023 / 1024])
    lut1 = o.lut(1)
    assert lut1[0][0] == 0.0 and lut1[0][2] == 1.0


def test_transfer_interpolation_and_duplicates():
    o = _tiny()
    o.set_transfer(0, {0: (0, 0, 0, 0), 512: (1, 1, 1, 1), 1024: (0, 0, 0, 1)})
    lut = o.lut(0)
    assert lut[256] == pytest.approx([0.5, 0.5, 0.5, 0.5])
    assert lut[768] == pytest.approx([0.5, 0.5, 0.5, 1.0])
    # a repeated key keeps its first value (std::map::insert)
    keys = np.array([0, 1024, 1024], dtype=np.uint32)
    o2 = _tiny()
    o2.lib.or_set_transfer(
        o2.ctx,
        0,
        3,
        keys.ctypes.data_as(O._u32p),
        np.array([0, 0, 0, 0, 1, 1, 1, 1, 0, 0, 0, 0], dtype=np.float32).ctypes.data_as(O._fp),
    )
    assert o2.lut(0)[512] == pytest.approx([0.5, 0.5, 0.5, 0.5])


def test_merge_constant_field_known_answer():
    # one source, value 0.5 everywhere, chain idem, default weight 2, transfer (1,0,0,j/1024)
    n = 4
    o = _tiny(n=n)
    data = np.full((n, n, n), 0.5, dtype=np.float32)
    o.set_source(0, data)
    o.set_dither_mode(0)
    o.update()
    vol, iso = o.combined()
    # lut[512] = (1,0,0,0.5); a = 0.5*2 = 1; color = (1*1, 0, 0, 1)/2 = (0.5, 0, 0, 0.5) -> round(127.5) = 128
    assert (vol == np.array([128, 0, 0, 128], dtype=np.uint8)).all()
    assert (iso == 0).all()


def test_minmax_closed_form():
    n = 6
    o = _tiny(n=n)
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    data = ((x - 2.0) * 0.25 + y * 0.5 - z * 0.125).astype(np.float32)
    o.set_source(0, data)
    o.set_functions(0, "mul(2)|add(1)")
    mn, mx = o.minmax()
    vals = data * np.float32(2) + np.float32(1)
    assert mn[0] == vals.min() and mx[0] == vals.max()


def test_minmax_signed_zero_follows_scan_order():
    # column (x,y) order first, then z: the first zero in that order decides the sign
    n = 2
    o = _tiny(n=n)
    data = np.ones((n, n, n), dtype=np.float32)
    data[1, 0, 0] = -0.0  # column (0,0), z = 1
    data[0, 1, 0] = 0.0  # column (0,1), z = 0
    o.set_source(0, data)
    mn, _ = o.minmax()
    assert mn[0] == 0.0 and np.signbit(mn[0])  # column (0,0) scanned first


def test_minmax_ignores_nan():
    n = 3
    o = _tiny(n=n)
    data = np.linspace(-1, 1, n ** 3, dtype=np.float32).reshape(n, n, n)
    data[0, 0, 0] = np.nan
    o.set_source(0, data)
    mn, mx = o.minmax()
    assert mn[0] == np.nanmin(data) and mx[0] == np.nanmax(data)


def test_bf16_fp16_rounding():
    lib = O.load()
    for v in [1.0, 1.00390625, 1.0 + 2 ** -9, 3.14159, 65519.0, 65520.0, 1e-8, -2.5e-5]:
        f16 = float(np.float32(np.float16(np.float32(v))))
        assert lib.or_round_fp16(v) == pytest.approx(f16, rel=0, abs=0) or (math.isinf(f16) and math.isinf(lib.or_round_fp16(v)))
    assert lib.or_round_bf16(1.0 + 2 ** -8) == 1.0  # tie to even
    assert lib.or_round_bf16(1.0 + 3 * 2 ** -8) == 1.0 + 2 ** -6


def test_fp64_oracle_close_to_fp32():
    from harness import build_oracle, gaussian_pair, image_diff

    s = gaussian_pair(n=24, fb=(40, 32))
    a = build_oracle(s).frame()
    b = build_oracle(s, f64=True).frame()
    st = image_diff(a, b)
    assert st["max"] <= 3 and st["frac_le1"] > 0.99


def test_dither_blue_noise_modes():
    # mode 3: 8^3 mask (isaac_dither_kernel.hpp:42-74), value/512; first entries 140, 428
    assert O.dither(3, 0, 0, 0, [0.5] * 4) == [128] * 4  # .5 > 140/512
    assert O.dither(3, 1, 0, 0, [0.5] * 4) == [127] * 4  # .5 < 428/512
    assert O.dither(3, 8, 8, 8, [0.5] * 4) == [128] * 4  # wraps every 8
    # modes >= 4: 16^3 mask (:76-310), value/4096; entries 0 and 4 are 1940 and 2568
    assert O.dither(4, 0, 0, 0, [0.5] * 4) == [128] * 4  # .5 > 1940/4096
    assert O.dither(4, 4, 0, 0, [0.5] * 4) == [127] * 4  # .5 < 2568/4096
    assert O.dither(7, 4, 16, 32, [0.5] * 4) == [127] * 4  # any larger mode, wraps every 16
