// Launch interface of the tensor-core convolution kernels (recon_gemm.cu),
// shared with the frame reconstructor (recon.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstddef>

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
    };

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
    size_t conv_wgrad_smem(int Npad);
    bool launch_conv_gemm(const ConvGemmParams& p, cudaStream_t s);
    bool launch_conv_wgrad(WgradParams p, cudaStream_t s);
} // namespace isaacb
