"""Tensor-core (tcgen05) convolutions against the float64 CPU oracle.

Inputs are bf16-representable; the kernels accumulate in FP32, so outputs
stored as bf16 agree with the oracle to bf16 rounding (relative 2^-8) plus
FP32 summation noise: |gpu - ref| <= 1e-2 * |ref| + 2e-3 * scale, where
scale is the RMS of the reference.  FP32 outputs (y_f32, dw) use 2e-3."""

import ctypes as C

import numpy as np
import pytest
import torch

from isaac_b200 import _lib
from oracle import recon_oracle as R

pytestmark = pytest.mark.gpu


def _bf16(a):
    return torch.from_numpy(np.ascontiguousarray(R.round_bf16(a))).to(torch.bfloat16).cuda()


def _close(got, ref, rel, name):
    ref = np.asarray(ref, np.float64)
    got = np.asarray(got, np.float64)
    scale = float(np.sqrt(np.mean(ref**2))) + 1e-12
    err = np.abs(got - ref)
    bound = rel * np.abs(ref) + 2e-3 * scale
    bad = err > bound
    assert not bad.any(), (name, float(err.max()), scale, int(bad.sum()), bad.size)


def _run(fn, **kw):
    a = _lib.ConvArgs()
    for k, v in kw.items():
        setattr(a, k, v)
    lib = _lib.load()
    _lib.check(getattr(lib, fn)(C.byref(a), C.c_void_p(torch.cuda.current_stream().cuda_stream)))


CASES = [
    # B, H, W, Ci, Co, ks, s, pad
    (2, 13, 11, 8, 16, 3, 1, 1),
    (2, 13, 11, 32, 32, 3, 1, 1),
    (1, 17, 15, 32, 64, 3, 2, 1),
    (2, 9, 10, 64, 96, 3, 2, 1),
    (1, 12, 9, 96, 128, 2, 2, 0),
    (2, 14, 13, 224, 96, 1, 1, 0),
    (1, 16, 16, 32, 16, 1, 1, 0),
    (2, 120, 90, 32, 32, 3, 1, 1),  # more tiles than SMs: several tiles per CTA
    (1, 40, 300, 16, 32, 3, 1, 1),  # rows of 2 full and 1 ragged 128-pixel tiles
    (1, 33, 290, 32, 64, 3, 2, 1),  # stride 2 on row tiles, ragged
    (2, 31, 260, 64, 64, 3, 1, 1),
]


@pytest.mark.parametrize("case", CASES, ids=[str(c) for c in CASES])
def test_conv_forward_dgrad_wgrad(case):
    B, H, W, Ci, Co, ks, s, pad = case
    rng = np.random.default_rng(hash(case) % (1 << 32))
    Ho, Wo = R.out_size(H, ks, s, pad), R.out_size(W, ks, s, pad)
    x = R.round_bf16(rng.standard_normal((B, H, W, Ci)).astype(np.float32))
    w = R.round_bf16((rng.standard_normal((Co, ks, ks, Ci)) / np.sqrt(ks * ks * Ci)).astype(np.float32))
    bias = rng.standard_normal(Co).astype(np.float32) * 0.1
    dy = R.round_bf16(rng.standard_normal((B, Ho, Wo, Co)).astype(np.float32))
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    dims = dict(batch=B, ksize=ks, stride=s, pad=pad, error_flag=flag.data_ptr())

    # forward, bias + ReLU, bf16 out
    xd, wd = _bf16(x), _bf16(R.pack_weights(w))
    bd = torch.from_numpy(bias).cuda()
    y = torch.zeros((B, Ho, Wo, Co), dtype=torch.bfloat16, device="cuda")
    _run("isaacb_conv_forward", x=xd.data_ptr(), w=wd.data_ptr(), bias=bd.data_ptr(), y=y.data_ptr(), in_h=H, in_w=W,
         c_in=Ci, out_h=Ho, out_w=Wo, c_out=Co, relu=1, **dims)
    ref = np.maximum(R.conv_forward(x, w, s, pad) + bias, 0.0)
    _close(y.float().cpu().numpy(), ref, 1e-2, "forward")

    # forward, FP32 out, no epilogue
    yf = torch.zeros((B, Ho, Wo, Co), dtype=torch.float32, device="cuda")
    _run("isaacb_conv_forward", x=xd.data_ptr(), w=wd.data_ptr(), y_f32=yf.data_ptr(), in_h=H, in_w=W, c_in=Ci,
         out_h=Ho, out_w=Wo, c_out=Co, **dims)
    _close(yf.cpu().numpy(), R.conv_forward(x, w, s, pad), 2e-3, "forward fp32")

    # input gradient (transposed gather) with the ReLU mask of y and accumulation
    dyd = _bf16(dy)
    wt = _bf16(R.pack_weights_transposed(w))
    prev = R.round_bf16(rng.standard_normal((B, H, W, Ci)).astype(np.float32))
    mask = R.round_bf16(rng.standard_normal((B, H, W, Ci)).astype(np.float32))
    dx = _bf16(prev)
    md = _bf16(mask)
    _run("isaacb_conv_forward", x=dyd.data_ptr(), w=wt.data_ptr(), y=dx.data_ptr(), mask=md.data_ptr(), in_h=Ho,
         in_w=Wo, c_in=Co, out_h=H, out_w=W, c_out=Ci, transposed=1, accumulate=1, **dims)
    ref = np.where(mask > 0, R.conv_dgrad(dy, w, (H, W), s, pad), 0.0) + prev
    _close(dx.float().cpu().numpy(), ref, 1e-2, "dgrad")

    # weight gradient, accumulated into FP32
    dw0 = rng.standard_normal((ks * ks * Ci, (Co + 15) // 16 * 16)).astype(np.float32)
    dw = torch.from_numpy(dw0.copy()).cuda()
    _run("isaacb_conv_wgrad", x=xd.data_ptr(), dy=dyd.data_ptr(), dw=dw.data_ptr(), in_h=H, in_w=W, c_in=Ci,
         out_h=Ho, out_w=Wo, c_out=Co, **dims)
    ref = R.conv_wgrad(x, dy, ks, s, pad)  # [co][ky][kx][ci]
    ref_mat = np.transpose(ref, (1, 2, 3, 0)).reshape(ks * ks * Ci, Co)
    got = dw.cpu().numpy()[:, :Co] - dw0[:, :Co]
    _close(got, ref_mat, 2e-3, "wgrad")
    torch.cuda.synchronize()
    assert int(flag.item()) == 0


@pytest.mark.parametrize("case", CASES, ids=[str(c) for c in CASES])
def test_tma_and_cp_async_producers_agree(case):
    """The row-tile kernel loads its halo with tiled TMA copies where the input allows
    (stride 1; stride 2 with an even width) and with cp.async gathers otherwise; both
    fill the same shared-memory runs, so the outputs are bit-identical."""
    B, H, W, Ci, Co, ks, s, pad = case
    rng = np.random.default_rng(7)
    Ho, Wo = R.out_size(H, ks, s, pad), R.out_size(W, ks, s, pad)
    x = _bf16(rng.standard_normal((B, H, W, Ci)).astype(np.float32))
    w = R.round_bf16((rng.standard_normal((Co, ks, ks, Ci)) / np.sqrt(ks * ks * Ci)).astype(np.float32))
    wd, wt = _bf16(R.pack_weights(w)), _bf16(R.pack_weights_transposed(w))
    dy = _bf16(rng.standard_normal((B, Ho, Wo, Co)).astype(np.float32))
    lib = _lib.load()
    outs = []
    try:
        for tma in (1, 0):
            _lib.check(lib.isaacb_conv_set_producer(tma))
            yf = torch.zeros((B, Ho, Wo, Co), dtype=torch.float32, device="cuda")
            _run("isaacb_conv_forward", x=x.data_ptr(), w=wd.data_ptr(), y_f32=yf.data_ptr(), batch=B, in_h=H, in_w=W,
                 c_in=Ci, out_h=Ho, out_w=Wo, c_out=Co, ksize=ks, stride=s, pad=pad)
            dx = torch.zeros((B, H, W, Ci), dtype=torch.float32, device="cuda")
            if s == 1:
                _run("isaacb_conv_forward", x=dy.data_ptr(), w=wt.data_ptr(), y_f32=dx.data_ptr(), batch=B, in_h=Ho,
                     in_w=Wo, c_in=Co, out_h=H, out_w=W, c_out=Ci, ksize=ks, stride=s, pad=pad, transposed=1)
            torch.cuda.synchronize()
            outs.append((yf.cpu(), dx.cpu()))
    finally:
        _lib.check(lib.isaacb_conv_set_producer(1))
    assert torch.equal(outs[0][0], outs[1][0])
    assert torch.equal(outs[0][1], outs[1][1])
