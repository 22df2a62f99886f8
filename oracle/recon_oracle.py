"""CPU oracle of the learned frame reconstructor (test infrastructure only).

The reference has no learned component; the reconstructor is an extension, so
this file restates the mathematics the CUDA kernels implement -- NHWC
convolutions, their input and weight gradients, the U-Net built from them, the
loss and the optimiser -- in float64 numpy.  It is the checker the GPU tests
compare against; nothing in the product imports it.

Layouts follow the kernels: activations NHWC, weights [c_out][ky][kx][c_in].
"""

from __future__ import annotations

import numpy as np


def round_bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest bf16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = ((u + 0x7FFF + lsb) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32)


def out_size(n: int, k: int, s: int, p: int) -> int:
    return (n + 2 * p - k) // s + 1


def _taps(n_out: int, n_in: int, k: int, s: int, p: int, t: int):
    """Output positions whose tap t lands inside the input, and those input positions."""
    o = np.arange(n_out)
    i = o * s - p + t
    ok = (i >= 0) & (i < n_in)
    return o[ok], i[ok]


def conv_forward(x, w, stride=1, pad=1, out_hw=None):
    """y[b,oy,ox,co] = sum_{ky,kx,ci} x[b, oy*s-p+ky, ox*s-p+kx, ci] * w[co,ky,kx,ci] (zero outside)."""
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    B, H, W, Ci = x.shape
    Co, ks, _, _ = w.shape
    Ho, Wo = out_hw if out_hw else (out_size(H, ks, stride, pad), out_size(W, ks, stride, pad))
    y = np.zeros((B, Ho, Wo, Co))
    for ky in range(ks):
        oy, iy = _taps(Ho, H, ks, stride, pad, ky)
        for kx in range(ks):
            ox, ix = _taps(Wo, W, ks, stride, pad, kx)
            if len(oy) == 0 or len(ox) == 0:
                continue
            y[:, oy[:, None], ox[None, :], :] += x[:, iy[:, None], ix[None, :], :] @ w[:, ky, kx, :].T
    return y


def conv_dgrad(dy, w, in_hw, stride=1, pad=1):
    """Gradient of conv_forward with respect to x (the adjoint scatter)."""
    dy = np.asarray(dy, np.float64)
    w = np.asarray(w, np.float64)
    B, Ho, Wo, Co = dy.shape
    _, ks, _, Ci = w.shape
    H, W = in_hw
    dx = np.zeros((B, H, W, Ci))
    for ky in range(ks):
        oy, iy = _taps(Ho, H, ks, stride, pad, ky)
        for kx in range(ks):
            ox, ix = _taps(Wo, W, ks, stride, pad, kx)
            if len(oy) == 0 or len(ox) == 0:
                continue
            dx[:, iy[:, None], ix[None, :], :] += dy[:, oy[:, None], ox[None, :], :] @ w[:, ky, kx, :]
    return dx


def conv_wgrad(x, dy, ks, stride=1, pad=1):
    """Gradient of conv_forward with respect to w: dw[co,ky,kx,ci]."""
    x = np.asarray(x, np.float64)
    dy = np.asarray(dy, np.float64)
    B, H, W, Ci = x.shape
    _, Ho, Wo, Co = dy.shape
    dw = np.zeros((Co, ks, ks, Ci))
    for ky in range(ks):
        oy, iy = _taps(Ho, H, ks, stride, pad, ky)
        for kx in range(ks):
            ox, ix = _taps(Wo, W, ks, stride, pad, kx)
            if len(oy) == 0 or len(ox) == 0:
                continue
            xs = x[:, iy[:, None], ix[None, :], :].reshape(-1, Ci)
            ds = dy[:, oy[:, None], ox[None, :], :].reshape(-1, Co)
            dw[:, ky, kx, :] = ds.T @ xs
    return dw


def pack_weights(w: np.ndarray) -> np.ndarray:
    """[co][ky][kx][ci] -> the kernels' bf16 GEMM matrix [roundup(co,16)][roundup(ks*ks*ci,64)] (float32 values)."""
    Co, ks, _, Ci = w.shape
    K = ks * ks * Ci
    out = np.zeros(((Co + 15) // 16 * 16, (K + 63) // 64 * 64), np.float32)
    out[:Co, :K] = w.reshape(Co, K)
    return out


def pack_weights_transposed(w: np.ndarray) -> np.ndarray:
    """The input-gradient GEMM matrix: per tap the transpose, [ci][ky][kx][co], packed like pack_weights."""
    return pack_weights(np.ascontiguousarray(np.transpose(w, (3, 1, 2, 0))))


# ---------------------------------------------------------------------------- the U-Net
# (name, ksize, stride, pad, c_in, c_out, relu, input)
#   input: "x" (the 8-channel input), a layer name, or ("cat", coarse, fine): channel
#   concatenation of the nearest-neighbour x2 upsampled coarse map (indices clamped
#   to the coarse grid) and the fine map.
LAYERS = [
    ("E1", 3, 1, 1, 8, 32, True, "x"),
    ("E1b", 3, 1, 1, 32, 32, True, "E1"),
    ("D12", 3, 2, 1, 32, 64, True, "E1b"),
    ("E2", 3, 1, 1, 64, 64, True, "D12"),
    ("D23", 3, 2, 1, 64, 96, True, "E2"),
    ("D34", 2, 2, 0, 96, 128, True, "D23"),
    ("U43", 1, 1, 0, 224, 96, True, ("cat", "D34", "D23")),
    ("U32", 1, 1, 0, 160, 64, True, ("cat", "U43", "E2")),
    ("U21", 1, 1, 0, 96, 32, True, ("cat", "U32", "E1b")),
    ("U21b", 3, 1, 1, 32, 32, True, "U21"),
    ("OUT", 1, 1, 0, 32, 16, False, "U21b"),
]


def param_count() -> int:
    return sum(co * k * k * ci + co for _, k, _, _, ci, co, _, _ in LAYERS)


def unflatten(params: np.ndarray) -> dict:
    """Flat parameter vector (per layer: weights [co][ky][kx][ci], then bias [co]) -> dict."""
    out, o = {}, 0
    for name, k, _, _, ci, co, _, _ in LAYERS:
        n = co * k * k * ci
        out[name] = (params[o : o + n].reshape(co, k, k, ci), params[o + n : o + n + co])
        o += n + co
    return out


def flatten(d: dict) -> np.ndarray:
    return np.concatenate([np.concatenate([d[n][0].ravel(), d[n][1].ravel()]) for n, *_ in LAYERS])


def up_index(n_fine: int, n_coarse: int) -> np.ndarray:
    return np.minimum(np.arange(n_fine) // 2, n_coarse - 1)


def cat_up(coarse, fine):
    iy = up_index(fine.shape[1], coarse.shape[1])
    ix = up_index(fine.shape[2], coarse.shape[2])
    return np.concatenate([coarse[:, iy[:, None], ix[None, :], :], fine], axis=-1)


def cat_up_backward(d, coarse_shape, c1):
    """Split the gradient of cat_up into (coarse, fine) gradients (children summed)."""
    B, h, w, _ = d.shape
    dc = np.zeros(coarse_shape)
    iy = up_index(h, coarse_shape[1])
    ix = up_index(w, coarse_shape[2])
    np.add.at(dc, (slice(None), iy[:, None], ix[None, :]), d[..., :c1])
    return dc, d[..., c1:]


def upsample_bilinear2(low):
    """x2 upsampling aligned with the renderer's pixel centres (pixel X of the full
    frame sits at X/2 of the half-size frame): even pixels copy, odd ones average
    their two neighbours (the last one clamps)."""
    B, h, w, C = low.shape

    def axis_weights(n):
        X = np.arange(2 * n)
        a = X // 2
        b = np.minimum((X + 1) // 2, n - 1)
        wb = np.where(X % 2 == 1, 0.5, 0.0)
        return a, b, wb

    ay, by, wy = axis_weights(h)
    ax, bx, wx = axis_weights(w)
    rows = low[:, ay] * (1 - wy)[None, :, None, None] + low[:, by] * wy[None, :, None, None]
    return rows[:, :, ax] * (1 - wx)[None, None, :, None] + rows[:, :, bx] * wx[None, None, :, None]


def shuffle(r):
    """[B][h][w][16] residual -> [B][2h][2w][4]: channel (dy*2+dx)*4+c goes to (2y+dy, 2x+dx, c)."""
    B, h, w, _ = r.shape
    return r.reshape(B, h, w, 2, 2, 4).transpose(0, 1, 3, 2, 4, 5).reshape(B, 2 * h, 2 * w, 4)


def unshuffle(g):
    B, H, W, _ = g.shape
    return g.reshape(B, H // 2, 2, W // 2, 2, 4).transpose(0, 1, 3, 2, 4, 5).reshape(B, H // 2, W // 2, 16)


def net_input(low_u8):
    """RGBA8 half-size frames -> the network input: RGBA / 255 and 4 zero channels."""
    x = np.zeros(low_u8.shape[:3] + (8,))
    x[..., :4] = low_u8 / 255.0
    return x


class UNet:
    """Forward, loss and backward in float64.  With ``bf16`` the values the GPU
    stores in bf16 (activations, gradients, the network input) are rounded at
    the same points."""

    def __init__(self, params: np.ndarray, bf16: bool = True):
        self.p = unflatten(np.asarray(params, np.float64))
        self.bf16 = bf16

    def _r(self, a):
        return R_bf16(a) if self.bf16 else a

    def forward(self, low_u8):
        x = self._r(net_input(low_u8))
        act = {"x": x}
        ins = {}
        for name, k, s, p, ci, co, relu, src in LAYERS:
            if isinstance(src, tuple):
                inp = cat_up(act[src[1]], act[src[2]])
            else:
                inp = act[src]
            ins[name] = inp
            w, b = self.p[name]
            y = conv_forward(inp, self._r(w), s, p) + b
            if relu:
                y = np.maximum(y, 0.0)
            if name != "OUT":
                act[name] = self._r(y)
            else:  # the residual is stored in FP32
                act[name] = y.astype(np.float32).astype(np.float64) if self.bf16 else y
        self.act, self.ins = act, ins
        self.low = low_u8
        return act["OUT"]

    def predict(self, low_u8):
        r = self.forward(low_u8)
        return upsample_bilinear2(low_u8 / 255.0) + shuffle(r)

    def loss_and_backward(self, low_u8, high_u8):
        r = self.forward(low_u8)
        pred = upsample_bilinear2(low_u8 / 255.0) + shuffle(r)
        diff = pred - high_u8 / 255.0
        n = diff.size
        loss = float(np.sum(diff**2) / n)
        dr = self._r(unshuffle(2.0 * diff / n))
        grads = {}
        dact = {"OUT": dr}
        for name, k, s, p, ci, co, relu, src in reversed(LAYERS):
            g = dact[name]
            if relu:
                g = np.where(self.act[name] > 0, g, 0.0)
            w, _ = self.p[name]
            inp = self.ins[name]
            grads[name] = (conv_wgrad(inp, g, k, s, p), g.sum(axis=(0, 1, 2)))
            if src == "x":
                continue
            dx = conv_dgrad(g, self._r(w), inp.shape[1:3], s, p)
            if isinstance(src, tuple):
                c1 = self.act[src[1]].shape[-1]
                dc, df = cat_up_backward(dx, self.act[src[1]].shape, c1)
                for nm, d in ((src[1], dc), (src[2], df)):
                    dact[nm] = dact.get(nm, 0.0) + d
            else:
                dact[src] = dact.get(src, 0.0) + dx
        self.grads = grads
        return loss, flatten(grads)


def R_bf16(a):
    return round_bf16(np.asarray(a, np.float32)).astype(np.float64)


def adam_step(params, grads, m, v, t, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam update (bias-corrected), in place on float64 arrays; t counts from 1."""
    m[:] = beta1 * m + (1 - beta1) * grads
    v[:] = beta2 * v + (1 - beta2) * grads * grads
    mh = m / (1 - beta1**t)
    vh = v / (1 - beta2**t)
    params[:] = params - lr * mh / (np.sqrt(vh) + eps)
    return params
