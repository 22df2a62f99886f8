"""Failure detection in the tensor-core kernels, without a fault.

Every wait of the tcgen05 convolutions on an mbarrier is bounded: when it gives
up, the kernel raises the caller's error flag, lets nothing it issued stay in
flight, releases its TMEM and returns, so the context stays usable.  These tests
make such a wait run out on purpose -- the `wait_check_us` budget makes the
kernel wait, before any copy or MMA, on an mbarrier that nothing arrives at --
and check the status, that no output was written, and that the next launches
(which allocate TMEM again) run normally and give the oracle's result."""

import ctypes as C

import numpy as np
import pytest
import torch

from isaac_b200 import _lib
from oracle import recon_oracle as R

pytestmark = pytest.mark.gpu

BUDGET_US = 2000


def _conv(x, w, y, flag, B, H, W, Ci, Co, ks, s, pad, check_us):
    a = _lib.ConvArgs(x=x.data_ptr(), w=w.data_ptr(), y_f32=y.data_ptr(), error_flag=flag.data_ptr(), batch=B, in_h=H,
                      in_w=W, c_in=Ci, out_h=(H + 2 * pad - ks) // s + 1, out_w=(W + 2 * pad - ks) // s + 1, c_out=Co,
                      ksize=ks, stride=s, pad=pad, wait_check_us=check_us)
    lib = _lib.load()
    _lib.check(lib.isaacb_conv_forward(C.byref(a), C.c_void_p(torch.cuda.current_stream().cuda_stream)))


# (B, H, W, Ci, Co, ks, stride, pad): 32 input channels take the row-tile kernel
# (k_conv_row), 8 the general implicit GEMM (k_conv_gemm)
CASES = [(1, 40, 300, 32, 32, 3, 1, 1), (2, 13, 11, 8, 16, 3, 1, 1)]


@pytest.mark.parametrize("case", CASES, ids=["row_tiles", "implicit_gemm"])
def test_conv_wait_expiry_raises_flag_and_releases_tmem(case):
    B, H, W, Ci, Co, ks, s, pad = case
    Ho, Wo = (H + 2 * pad - ks) // s + 1, (W + 2 * pad - ks) // s + 1
    rng = np.random.default_rng(3)
    xh = R.round_bf16(rng.standard_normal((B, H, W, Ci)).astype(np.float32))
    wh = R.round_bf16((rng.standard_normal((Co, ks, ks, Ci)) / np.sqrt(ks * ks * Ci)).astype(np.float32))
    x = torch.from_numpy(xh).to(torch.bfloat16).cuda()
    w = torch.from_numpy(R.pack_weights(wh)).to(torch.bfloat16).cuda()
    ref = R.conv_forward(xh, wh, s, pad)
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    for _ in range(2):  # twice: a leaked TMEM allocation would stall the launches after it
        y = torch.full((B, Ho, Wo, Co), float("nan"), dtype=torch.float32, device="cuda")
        flag.zero_()
        _conv(x, w, y, flag, B, H, W, Ci, Co, ks, s, pad, BUDGET_US)
        torch.cuda.synchronize()
        assert int(flag.item()) == 1
        assert torch.isnan(y).all()  # the kernel gave up before writing anything
        flag.zero_()
        _conv(x, w, y, flag, B, H, W, Ci, Co, ks, s, pad, 0)
        torch.cuda.synchronize()
        assert int(flag.item()) == 0
        got = y.cpu().numpy().astype(np.float64)
        scale = float(np.sqrt(np.mean(ref**2)))
        assert (np.abs(got - ref) <= 2e-3 * np.abs(ref) + 2e-3 * scale).all()


def test_reconstructor_reports_wait_expiry_and_recovers():
    from isaac_b200.recon import Reconstructor

    h, w = 48, 80
    rng = np.random.default_rng(5)
    low = torch.from_numpy(rng.integers(0, 256, (h, w, 4), dtype=np.uint8)).cuda()
    net = Reconstructor(1, h, w, seed=1)
    ref = torch.empty((2 * h, 2 * w, 4), dtype=torch.uint8, device="cuda")
    net.infer(low, ref)
    torch.cuda.synchronize()
    assert net.error_flag() == 0
    out = torch.empty_like(ref)
    net.arm_wait_check(BUDGET_US)
    net.infer(low, out)
    torch.cuda.synchronize()
    assert net.error_flag() == 1  # read and cleared
    net.infer(low, out)
    torch.cuda.synchronize()
    assert net.error_flag() == 0
    assert torch.equal(out, ref)
    net.close()
