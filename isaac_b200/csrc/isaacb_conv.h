// Launch interface of the tensor-core convolution kernels (recon_gemm.cu),
// shared with the frame reconstructor (recon.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace isaacb
{
    // forward / input-gradient implicit GEMM (see recon_gemm.cu)
    struct ConvGemmParams
    {
        const __nv_bfloat16* x; // gather source, NHWC [B][H][W][Cg]
        const __nv_bfloat16* w; // packed weights [Npad][Kpad]
        const float* bias; // [Cout] or null
        __nv_bfloat16* y; // NHWC [B][Ho][Wo][Cout] (unless yf)
        float* yf; // FP32 output instead of y
        const __nv_bfloat16* mask; // output *= (mask > 0), NHWC like y, or null
        int B, H, W, Cg;
        int Ho, Wo, Cout, Npad, Kpad;
        int ks, stride, pad, transposed;
        int relu, accumulate;
        int* errorFlag;
        // failure-detection check: non-zero = before any copy or MMA, wait this many ns on
        // an mbarrier that nothing arrives at, raise errorFlag, release TMEM and return
        unsigned long long waitCheckNs;
        // row-tile kernel only (k_conv_row):
        // implicit concatenation (cp.async producer, 1x1): the first upC input channels
        // come from xUp, [B][upInH][upInW][upC], read at the nearest coarse pixel
        // (min(y/2, upInH-1), min(x/2, upInW-1)); the other Cg - upC from x, whose pixels
        // then hold Cg - upC channels; null = off
        const __nv_bfloat16* xUp;
        int upC, upInH, upInW;
        // host launch hint (row-tile kernel): launch as a programmatic dependent of the
        // stream's previous kernel, so that its CTAs load their weights while that kernel
        // drains; the kernel reads its input only after griddepcontrol.wait
        int pdl;
    };

    // bilinear x2 of a half-size RGBA8 frame at full-size pixel (X, Y), aligned with the
    // renderer's pixel positions (integer coordinates): even pixels copy, odd ones
    // average two neighbours; values in [0, 1]
    __device__ __forceinline__ float4 bilinear2_rgba(const uchar4* __restrict__ low, int h, int w, int X, int Y)
    {
        const int ya = Y >> 1, yb = min((Y + 1) >> 1, h - 1);
        const int xa = X >> 1, xb = min((X + 1) >> 1, w - 1);
        const float wy = (Y & 1) ? 0.5f : 0.0f, wx = (X & 1) ? 0.5f : 0.0f;
        const uchar4 a = __ldg(low + size_t(ya) * w + xa), b = __ldg(low + size_t(ya) * w + xb);
        const uchar4 c = __ldg(low + size_t(yb) * w + xa), d = __ldg(low + size_t(yb) * w + xb);
        auto mix = [&](float va, float vb, float vc, float vd) {
            const float r0 = va * (1.0f - wx) + vb * wx;
            const float r1 = vc * (1.0f - wx) + vd * wx;
            return (r0 * (1.0f - wy) + r1 * wy) / 255.0f;
        };
        return make_float4(mix(a.x, b.x, c.x, d.x), mix(a.y, b.y, c.y, d.y), mix(a.z, b.z, c.z, d.z), mix(a.w, b.w, c.w, d.w));
    }

    // a value in [0, 1] as a byte: round to nearest, clamped
    __device__ __forceinline__ uint8_t unit_byte(float v)
    {
        return uint8_t(__float2int_rn(fminf(fmaxf(v * 255.0f, 0.0f), 255.0f)));
    }

    // weight gradient (see recon_gemm.cu)
    struct WgradParams
    {
        const __nv_bfloat16* x; // layer input [B][H][W][Cin]
        const __nv_bfloat16* dy; // output gradient [B][Ho][Wo][Cout]
        float* dw; // [Mtot][Npad], accumulated
        int B, H, W, Cin, Ho, Wo, Cout, Npad;
        int ks, stride, pad;
        int Mtot; // ks*ks*Cin
        int chunksPerSplit; // set by the launcher
        int* errorFlag;
    };

    size_t conv_gemm_smem(int Npad, int Kpad);
    // the row-tile kernel takes this convolution (and then honours xUp)
    bool row_tiles_apply(const ConvGemmParams& p);
    size_t conv_wgrad_smem(int Npad);
    bool launch_conv_gemm(const ConvGemmParams& p, cudaStream_t s);
    bool launch_conv_wgrad(WgradParams p, cudaStream_t s);
} // namespace isaacb
