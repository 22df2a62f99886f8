// Learned frame reconstructor: a 4-level convolutional U-Net that rebuilds
// the full-size frame from a half-size render taken at twice the step.  No
// counterpart in the reference; it sits beside the plain renderer, which
// produces its training pairs and stays its judge and fallback.
//
// Network (NHWC bf16 activations, FP32 accumulation on the tensor cores):
//   x    half-size RGBA / 255 and 4 zero channels (8)
//   E1   3x3     8 -> 32  ReLU        E1b  3x3   32 -> 32 ReLU
//   D12  3x3/2  32 -> 64  ReLU        E2   3x3   64 -> 64 ReLU
//   D23  3x3/2  64 -> 96  ReLU        D34  2x2/2 96 -> 128 ReLU
//   U43  1x1 on [up(D34), D23] 224 -> 96 ReLU
//   U32  1x1 on [up(U43), E2]  160 -> 64 ReLU
//   U21  1x1 on [up(U32), E1b]  96 -> 32 ReLU
//   U21b 3x3    32 -> 32 ReLU         OUT  1x1   32 -> 16 (FP32)
//   frame = bilinear x2 of the half-size frame + pixel-shuffle(OUT)
// up() is nearest-neighbour x2 with indices clamped to the coarse grid.
// 216,464 parameters; FP32 master weights, Adam, bf16 copies packed for the
// forward and input-gradient GEMMs.  Loss: mean squared error over the
// full-size RGBA in [0,1].
#include "../../include/isaac_b200.h"
#include "isaacb_conv.h"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

namespace isaacb
{
    void set_global_error(const std::string& msg);
}

using namespace isaacb;
using bf16 = __nv_bfloat16;

namespace
{
    constexpr int kLayers = 11;
    enum Src
    {
        SRC_X = -1
    };
    struct LayerDef
    {
        const char* name;
        int ks, stride, pad, cin, cout, relu;
        int src; // producing layer, or SRC_X
        int coarse, fine; // for concatenation inputs (src == -2)
    };
    // src == -2: the input is [up(coarse), fine]
    const LayerDef kDefs[kLayers] = {
        {"E1", 3, 1, 1, 8, 32, 1, SRC_X, 0, 0},
        {"E1b", 3, 1, 1, 32, 32, 1, 0, 0, 0},
        {"D12", 3, 2, 1, 32, 64, 1, 1, 0, 0},
        {"E2", 3, 1, 1, 64, 64, 1, 2, 0, 0},
        {"D23", 3, 2, 1, 64, 96, 1, 3, 0, 0},
        {"D34", 2, 2, 0, 96, 128, 1, 4, 0, 0},
        {"U43", 1, 1, 0, 224, 96, 1, -2, 5, 4},
        {"U32", 1, 1, 0, 160, 64, 1, -2, 6, 3},
        {"U21", 1, 1, 0, 96, 32, 1, -2, 7, 1},
        {"U21b", 3, 1, 1, 32, 32, 1, 8, 0, 0},
        {"OUT", 1, 1, 0, 32, 16, 0, 9, 0, 0},
    };

    int round_up(int v, int m)
    {
        return (v + m - 1) / m * m;
    }
    int out_size(int n, int k, int s, int p)
    {
        return (n + 2 * p - k) / s + 1;
    }

    // ------------------------------------------------------------------ elementwise kernels
    __device__ __forceinline__ uint4 pack8(const float (&v)[8])
    {
        uint4 o;
        __nv_bfloat162 h;
        h = __floats2bfloat162_rn(v[0], v[1]);
        o.x = *reinterpret_cast<uint32_t*>(&h);
        h = __floats2bfloat162_rn(v[2], v[3]);
        o.y = *reinterpret_cast<uint32_t*>(&h);
        h = __floats2bfloat162_rn(v[4], v[5]);
        o.z = *reinterpret_cast<uint32_t*>(&h);
        h = __floats2bfloat162_rn(v[6], v[7]);
        o.w = *reinterpret_cast<uint32_t*>(&h);
        return o;
    }
    __device__ __forceinline__ void unpack8(uint4 u, float (&v)[8])
    {
        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for(int i = 0; i < 4; ++i)
        {
            v[2 * i] = __uint_as_float(w[i] << 16);
            v[2 * i + 1] = __uint_as_float(w[i] & 0xFFFF0000u);
        }
    }

    // half-size RGBA8 frames (batch entry b is frame index[b]) -> network input: RGBA / 255
    // and zeros, 16 channels (the parameters see the first 8; the GEMM wants multiples of 16)
    __global__ void k_input(const uint8_t* __restrict__ low, const int32_t* __restrict__ index, int B, int h, int w, bf16* __restrict__ x)
    {
        // the first convolution may start loading its weights (it waits for this grid
        // before reading x)
        asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
        // a batch holds at most 2^26 pixels (isaacb_recon_create), so 32-bit indices suffice
        const uint32_t n = uint32_t(B) * uint32_t(h) * uint32_t(w), hw = uint32_t(h) * uint32_t(w);
        for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        {
            const uint32_t b = i / hw, pp = i - b * hw;
            const int f = index ? __ldg(index + b) : int(b);
            const uchar4 c = __ldg(reinterpret_cast<const uchar4*>(low) + size_t(f) * hw + pp);
            float v[8] = {float(c.x) / 255.0f, float(c.y) / 255.0f, float(c.z) / 255.0f, float(c.w) / 255.0f, 0, 0, 0, 0};
            reinterpret_cast<uint4*>(x)[2 * i] = pack8(v);
            reinterpret_cast<uint4*>(x)[2 * i + 1] = make_uint4(0, 0, 0, 0);
        }
    }

    // [up(coarse), fine] along channels, 8 channels per thread step
    __global__ void k_cat_up(const bf16* __restrict__ coarse, const bf16* __restrict__ fine, bf16* __restrict__ out, int B, int h, int w, int hc, int wc, int c1, int c2)
    {
        const int cc = (c1 + c2) / 8;
        const size_t n = size_t(B) * h * w * cc;
        for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        {
            const int j = int(i % cc);
            const size_t p = i / cc;
            uint4 v;
            if(j * 8 < c1)
            {
                const int x = int(p % w);
                const size_t t = p / w;
                const int y = int(t % h), b = int(t / h);
                const int yc = min(y / 2, hc - 1), xc = min(x / 2, wc - 1);
                v = __ldg(reinterpret_cast<const uint4*>(coarse + ((size_t(b) * hc + yc) * wc + xc) * c1 + j * 8));
            }
            else
                v = __ldg(reinterpret_cast<const uint4*>(fine + p * c2 + (j * 8 - c1)));
            reinterpret_cast<uint4*>(out)[i] = v;
        }
    }

    // gradient of k_cat_up: fine part copied, coarse part summed over its children; both
    // multiplied by (activation > 0), the derivative of the producing layer's ReLU
    __global__ void k_cat_up_backward(
        const bf16* __restrict__ dcat,
        const bf16* __restrict__ coarseAct,
        const bf16* __restrict__ fineAct,
        bf16* __restrict__ dcoarse,
        bf16* __restrict__ dfine,
        int B,
        int h,
        int w,
        int hc,
        int wc,
        int c1,
        int c2)
    {
        const int ctot = c1 + c2;
        const size_t nf = size_t(B) * h * w * (c2 / 8);
        const size_t nc = size_t(B) * hc * wc * (c1 / 8);
        for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < nf + nc; i += size_t(gridDim.x) * blockDim.x)
        {
            if(i < nf)
            {
                const int j = int(i % (c2 / 8));
                const size_t p = i / (c2 / 8);
                float d[8], a[8];
                unpack8(__ldg(reinterpret_cast<const uint4*>(dcat + p * ctot + c1 + j * 8)), d);
                unpack8(__ldg(reinterpret_cast<const uint4*>(fineAct + p * c2 + j * 8)), a);
#pragma unroll
                for(int k = 0; k < 8; ++k)
                    d[k] = a[k] > 0.0f ? d[k] : 0.0f;
                reinterpret_cast<uint4*>(dfine + p * c2 + j * 8)[0] = pack8(d);
            }
            else
            {
                const size_t ii = i - nf;
                const int j = int(ii % (c1 / 8));
                const size_t q = ii / (c1 / 8);
                const int xc = int(q % wc);
                const size_t t = q / wc;
                const int yc = int(t % hc), b = int(t / hc);
                const int y0 = 2 * yc, y1 = yc == hc - 1 ? h - 1 : min(2 * yc + 1, h - 1);
                const int x0 = 2 * xc, x1 = xc == wc - 1 ? w - 1 : min(2 * xc + 1, w - 1);
                float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                for(int y = y0; y <= y1; ++y)
                    for(int x = x0; x <= x1; ++x)
                    {
                        float d[8];
                        unpack8(__ldg(reinterpret_cast<const uint4*>(dcat + ((size_t(b) * h + y) * w + x) * ctot + j * 8)), d);
#pragma unroll
                        for(int k = 0; k < 8; ++k)
                            s[k] += d[k];
                    }
                float a[8];
                unpack8(__ldg(reinterpret_cast<const uint4*>(coarseAct + q * c1 + j * 8)), a);
#pragma unroll
                for(int k = 0; k < 8; ++k)
                    s[k] = a[k] > 0.0f ? s[k] : 0.0f;
                reinterpret_cast<uint4*>(dcoarse + q * c1 + j * 8)[0] = pack8(s);
            }
        }
    }

    __device__ __forceinline__ float4 bilinear2(const uchar4* __restrict__ low, int h, int w, int X, int Y)
    {
        return bilinear2_rgba(low, h, w, X, Y);
    }

    // per half-size pixel: the 4 full-size predictions, their squared error against the
    // target and the loss gradient with respect to the 16 residual channels
    __global__ void k_loss(
        const uint8_t* __restrict__ low,
        const uint8_t* __restrict__ high,
        const int32_t* __restrict__ index,
        const float* __restrict__ r,
        bf16* __restrict__ dr,
        float* __restrict__ lossSum,
        int B,
        int h,
        int w,
        float gradScale,
        float invCount)
    {
        float acc = 0.0f;
        const size_t n = size_t(B) * h * w;
        for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        {
            const int x = int(i % w);
            const size_t t = i / w;
            const int y = int(t % h), b = int(t / h);
            const int f = index ? __ldg(index + b) : b;
            const uchar4* lo = reinterpret_cast<const uchar4*>(low) + size_t(f) * h * w;
            const uchar4* hi = reinterpret_cast<const uchar4*>(high) + size_t(f) * 4 * h * w;
            float rv[16], g[16];
            const float4* rp = reinterpret_cast<const float4*>(r + i * 16);
#pragma unroll
            for(int k = 0; k < 4; ++k)
            {
                const float4 q = rp[k];
                rv[4 * k] = q.x, rv[4 * k + 1] = q.y, rv[4 * k + 2] = q.z, rv[4 * k + 3] = q.w;
            }
#pragma unroll
            for(int s = 0; s < 4; ++s)
            {
                const int X = 2 * x + (s & 1), Y = 2 * y + (s >> 1);
                const float4 bl = bilinear2(lo, h, w, X, Y);
                const uchar4 tg = __ldg(hi + size_t(Y) * (2 * w) + X);
                const float d0 = bl.x + rv[4 * s] - float(tg.x) / 255.0f;
                const float d1 = bl.y + rv[4 * s + 1] - float(tg.y) / 255.0f;
                const float d2 = bl.z + rv[4 * s + 2] - float(tg.z) / 255.0f;
                const float d3 = bl.w + rv[4 * s + 3] - float(tg.w) / 255.0f;
                acc += d0 * d0 + d1 * d1 + d2 * d2 + d3 * d3;
                g[4 * s] = gradScale * d0, g[4 * s + 1] = gradScale * d1, g[4 * s + 2] = gradScale * d2, g[4 * s + 3] = gradScale * d3;
            }
            float a[8], c[8];
#pragma unroll
            for(int k = 0; k < 8; ++k)
            {
                a[k] = g[k];
                c[k] = g[8 + k];
            }
            uint4* dp = reinterpret_cast<uint4*>(dr + i * 16);
            dp[0] = pack8(a);
            dp[1] = pack8(c);
        }
        // block reduction of the squared error
        __shared__ float red[32];
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if((threadIdx.x & 31) == 0)
            red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if(threadIdx.x == 0)
        {
            float s = 0.0f;
            for(int k = 0; k < int(blockDim.x >> 5); ++k)
                s += red[k];
            atomicAdd(lossSum, s * invCount);
        }
    }

    // the reconstructed full-size frame, RGBA8 (round to nearest, clamped): bilinear x2 of
    // the half-size frame plus the pixel-shuffled residual (4 channels per full-size pixel)
    __global__ void k_frame(const uint8_t* __restrict__ low, const float* __restrict__ r, uint8_t* __restrict__ out, int h, int w)
    {
        // r comes from the output layer, which this kernel follows as a programmatic dependent
        asm volatile("griddepcontrol.wait;" ::: "memory");
        // one thread per half-size pixel (x, y): blockIdx.y is the row
        const int x = int(blockIdx.x * blockDim.x + threadIdx.x), y = int(blockIdx.y);
        if(x < w && y < h)
        {
            const size_t i = size_t(y) * w + x;
            const uchar4* lo = reinterpret_cast<const uchar4*>(low);
            const float4* rp = reinterpret_cast<const float4*>(r + i * 16);
#pragma unroll
            for(int s = 0; s < 4; ++s)
            {
                const int X = 2 * x + (s & 1), Y = 2 * y + (s >> 1);
                const float4 bl = bilinear2(lo, h, w, X, Y);
                const float4 q = rp[s];
                reinterpret_cast<uchar4*>(out)[size_t(Y) * (2 * w) + X]
                    = make_uchar4(unit_byte(bl.x + q.x), unit_byte(bl.y + q.y), unit_byte(bl.z + q.z), unit_byte(bl.w + q.w));
            }
        }
    }

    // the method without the network: bilinear x2 alone, RGBA8
    __global__ void k_bilinear_frame(const uint8_t* __restrict__ low, uint8_t* __restrict__ out, int h, int w)
    {
        const size_t n = size_t(4) * h * w;
        for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        {
            const int X = int(i % (2 * w)), Y = int(i / (2 * w));
            const float4 bl = bilinear2(reinterpret_cast<const uchar4*>(low), h, w, X, Y);
            reinterpret_cast<uchar4*>(out)[i] = make_uchar4(unit_byte(bl.x), unit_byte(bl.y), unit_byte(bl.z), unit_byte(bl.w));
        }
    }

    // per-channel sums of a gradient (the bias gradient), added to db
    __global__ void k_bias_grad(const bf16* __restrict__ g, size_t pixels, int C, float* __restrict__ db)
    {
        __shared__ float part[256];
        const int t = threadIdx.x;
        const int lanesPerPix = C; // one thread per channel, 256 / C pixels side by side
        const int pixPerIter = blockDim.x / lanesPerPix;
        const int c = t % lanesPerPix, pofs = t / lanesPerPix;
        float s = 0.0f;
        if(pofs < pixPerIter)
            for(size_t p = blockIdx.x * size_t(pixPerIter) + pofs; p < pixels; p += size_t(gridDim.x) * pixPerIter)
                s += __bfloat162float(g[p * C + c]);
        part[t] = (pofs < pixPerIter) ? s : 0.0f;
        __syncthreads();
        if(t < C)
        {
            float a = 0.0f;
            for(int k = t; k < pixPerIter * C; k += C)
                a += part[k];
            atomicAdd(db + t, a);
        }
    }

    // sum of squared byte differences of two RGBA8 images (for PSNR)
    __global__ void k_sq_error(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b, size_t n, unsigned long long* __restrict__ out)
    {
        unsigned long long acc = 0;
        for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n / 4; i += size_t(gridDim.x) * blockDim.x)
        {
            const uchar4 x = __ldg(reinterpret_cast<const uchar4*>(a) + i), y = __ldg(reinterpret_cast<const uchar4*>(b) + i);
            const int d0 = int(x.x) - y.x, d1 = int(x.y) - y.y, d2 = int(x.z) - y.z, d3 = int(x.w) - y.w;
            acc += unsigned(d0 * d0 + d1 * d1 + d2 * d2 + d3 * d3);
        }
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if((threadIdx.x & 31) == 0 && acc)
            atomicAdd(out, acc);
    }

    // ------------------------------------------------------------------ parameters and Adam
    struct LayerTable
    {
        int off[kLayers + 1]; // flat offsets of each layer's weights (then its bias)
        int ks[kLayers], cin[kLayers], cout[kLayers];
        int cg[kLayers]; // input channels of the GEMM layout (cin rounded up to 16)
        int Npad[kLayers], Kpad[kLayers], NpadT[kLayers], KpadT[kLayers];
        bf16* wf[kLayers];
        bf16* wt[kLayers];
        const float* dw[kLayers];
        const float* db[kLayers];
    };

    // one thread per parameter: optional Adam step on the FP32 master, then the bf16
    // copies in the forward ([co][tap*cin+ci]) and input-gradient ([ci][tap*cout+co]) layouts
    __global__ void k_params(
        const __grid_constant__ LayerTable T,
        float* __restrict__ master,
        float* __restrict__ m,
        float* __restrict__ v,
        int total,
        int step,
        float lr,
        float* __restrict__ gradOut)
    {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if(i >= total)
            return;
        int L = 0;
        while(L + 1 < kLayers && i >= T.off[L + 1])
            ++L;
        const int ks = T.ks[L], cin = T.cin[L], cout = T.cout[L], cg = T.cg[L];
        const int taps = ks * ks;
        const int o = i - T.off[L];
        const int nw = cout * taps * cin;
        int co, t = 0, ci = 0;
        float g = 0.0f;
        if(o < nw)
        {
            co = o / (taps * cin);
            const int r = o - co * taps * cin;
            t = r / cin;
            ci = r - t * cin;
            if(T.dw[L])
                g = T.dw[L][size_t(t * cg + ci) * T.Npad[L] + co];
        }
        else
        {
            co = o - nw;
            if(T.db[L])
                g = T.db[L][co];
        }
        if(gradOut)
            gradOut[i] = g;
        float p = master[i];
        if(step > 0)
        {
            const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
            const float mi = b1 * m[i] + (1.0f - b1) * g;
            const float vi = b2 * v[i] + (1.0f - b2) * g * g;
            m[i] = mi;
            v[i] = vi;
            const float mh = mi / (1.0f - powf(b1, float(step)));
            const float vh = vi / (1.0f - powf(b2, float(step)));
            p -= lr * mh / (sqrtf(vh) + eps);
            master[i] = p;
        }
        if(o < nw)
        {
            const bf16 pb = __float2bfloat16_rn(p);
            T.wf[L][size_t(co) * T.Kpad[L] + t * cg + ci] = pb;
            if(T.wt[L])
                T.wt[L][size_t(ci) * T.KpadT[L] + t * cout + co] = pb;
        }
    }

    int grid_for(size_t n, int threads = 256)
    {
        size_t b = (n + threads - 1) / threads;
        if(b > 148 * 16)
            b = 148 * 16;
        return int(b < 1 ? 1 : b);
    }
} // namespace

struct isaacb_recon
{
    int maxBatch = 0, maxH = 0, maxW = 0;
    int total = 0; // parameters
    LayerTable T{};
    float* master = nullptr;
    float* adamM = nullptr;
    float* adamV = nullptr;
    float* bias[kLayers] = {};
    float* dw[kLayers] = {};
    float* db[kLayers] = {};
    bf16* wf[kLayers] = {};
    bf16* wt[kLayers] = {};
    bf16* act[kLayers] = {}; // outputs (OUT: unused, see r)
    bf16* dpre[kLayers] = {}; // gradient with respect to each layer's pre-activation output
    bf16* cat[kLayers] = {}; // concatenated inputs
    bf16* dcat = nullptr; // gradient of a concatenated input (largest one)
    bf16* x = nullptr;
    float* r = nullptr; // OUT, FP32
    float* lossSum = nullptr;
    float* gradHost = nullptr; // device staging for the flat gradient
    unsigned long long* sqErr = nullptr;
    int32_t* errorFlag = nullptr;
    unsigned long long waitCheckNs = 0; // armed failure-path check for the next convolution
    int step = 0;
    // per-level sizes for the current call
    int lh[4], lw[4];
    std::vector<void*> allocs;
};

namespace
{
    isaacb_status fail_r(isaacb_status st, const std::string& m)
    {
        set_global_error(m);
        return st;
    }

    template<class T>
    bool dalloc(isaacb_recon* R, T*& p, size_t count)
    {
        void* q = nullptr;
        if(cudaMalloc(&q, count * sizeof(T) + 16) != cudaSuccess)
            return false;
        cudaMemset(q, 0, count * sizeof(T) + 16);
        R->allocs.push_back(q);
        p = static_cast<T*>(q);
        return true;
    }

    // output level of each layer (0 = half-size frame, 3 = coarsest)
    const int kLevel[kLayers] = {0, 0, 1, 1, 2, 3, 2, 1, 0, 0, 0};

    void level_sizes(int h, int w, int (&lh)[4], int (&lw)[4])
    {
        lh[0] = h;
        lw[0] = w;
        lh[1] = out_size(h, 3, 2, 1);
        lw[1] = out_size(w, 3, 2, 1);
        lh[2] = out_size(lh[1], 3, 2, 1);
        lw[2] = out_size(lw[1], 3, 2, 1);
        lh[3] = out_size(lh[2], 2, 2, 0);
        lw[3] = out_size(lw[2], 2, 2, 0);
    }

    int in_level(int L)
    {
        const LayerDef& d = kDefs[L];
        if(d.src == SRC_X)
            return 0;
        if(d.src == -2)
            return kLevel[d.fine];
        return kLevel[d.src];
    }

    const bf16* layer_input(const isaacb_recon* R, int L)
    {
        const LayerDef& d = kDefs[L];
        if(d.src == SRC_X)
            return R->x;
        if(d.src == -2)
            return R->cat[L];
        return R->act[d.src];
    }

    bool conv_layer(isaacb_recon* R, int L, int B, cudaStream_t s, bool pdl = false)
    {
        const LayerDef& d = kDefs[L];
        const int li = in_level(L), lo = kLevel[L];
        ConvGemmParams p{};
        p.x = layer_input(R, L);
        p.w = R->wf[L];
        p.bias = R->bias[L];
        p.y = L == kLayers - 1 ? nullptr : R->act[L];
        p.yf = L == kLayers - 1 ? R->r : nullptr;
        p.B = B;
        p.H = R->lh[li];
        p.W = R->lw[li];
        p.Cg = R->T.cg[L];
        p.Ho = R->lh[lo];
        p.Wo = R->lw[lo];
        p.Cout = d.cout;
        p.Npad = R->T.Npad[L];
        p.Kpad = R->T.Kpad[L];
        p.ks = d.ks;
        p.stride = d.stride;
        p.pad = d.pad;
        p.relu = d.relu;
        p.errorFlag = R->errorFlag;
        p.waitCheckNs = R->waitCheckNs;
        R->waitCheckNs = 0;
        p.pdl = pdl ? 1 : 0;
        return launch_conv_gemm(p, s);
    }

    bool forward(isaacb_recon* R, int B, cudaStream_t s)
    {
        for(int L = 0; L < kLayers; ++L)
        {
            const LayerDef& d = kDefs[L];
            if(d.src == -2)
            {
                const int lf = kLevel[d.fine], lc = kLevel[d.coarse];
                const size_t n = size_t(B) * R->lh[lf] * R->lw[lf] * (d.cin / 8);
                k_cat_up<<<grid_for(n), 256, 0, s>>>(
                    R->act[d.coarse],
                    R->act[d.fine],
                    R->cat[L],
                    B,
                    R->lh[lf],
                    R->lw[lf],
                    R->lh[lc],
                    R->lw[lc],
                    kDefs[d.coarse].cout,
                    kDefs[d.fine].cout);
            }
            if(!conv_layer(R, L, B, s))
                return false;
        }
        return true;
    }

    // One image, inference only.  A concatenating 1x1 layer reads its two inputs in place:
    // the row-tile producer gathers the coarse tensor's channels at the nearest coarse
    // pixel and the fine tensor's after them, which is [up(coarse), fine] without the
    // concatenated tensor ever being formed.  The sums are the training forward's.
    bool forward_infer(isaacb_recon* R, const uint8_t* low, uint8_t* out, cudaStream_t s)
    {
        for(int L = 0; L < kLayers; ++L)
        {
            const LayerDef& d = kDefs[L];
            if(d.src == -2)
            {
                // [up(coarse), fine] read in place by the producer (implicit concatenation)
                const int lf = kLevel[d.fine], lc = kLevel[d.coarse];
                ConvGemmParams p{};
                p.x = R->act[d.fine];
                p.xUp = R->act[d.coarse];
                p.upC = kDefs[d.coarse].cout;
                p.upInH = R->lh[lc];
                p.upInW = R->lw[lc];
                p.w = R->wf[L];
                p.bias = R->bias[L];
                p.y = R->act[L];
                p.B = 1;
                p.H = p.Ho = R->lh[lf];
                p.W = p.Wo = R->lw[lf];
                p.Cg = R->T.cg[L];
                p.Cout = d.cout;
                p.Npad = R->T.Npad[L];
                p.Kpad = R->T.Kpad[L];
                p.ks = 1;
                p.stride = 1;
                p.relu = d.relu;
                p.errorFlag = R->errorFlag;
                p.pdl = 1;
                if(p.Cg != d.cin || !row_tiles_apply(p) || !launch_conv_gemm(p, s))
                    return false;
                continue;
            }
            if(L == kLayers - 1)
            {
                ConvGemmParams p{};
                p.x = R->act[d.src];
                p.w = R->wf[L];
                p.bias = R->bias[L];
                p.B = 1;
                p.H = p.Ho = R->lh[0];
                p.W = p.Wo = R->lw[0];
                p.Cg = R->T.cg[L];
                p.Cout = d.cout;
                p.Npad = R->T.Npad[L];
                p.Kpad = R->T.Kpad[L];
                p.ks = 1;
                p.stride = 1;
                p.errorFlag = R->errorFlag;
                p.yf = R->r;
                p.pdl = 1;
                if(!launch_conv_gemm(p, s))
                    return false;
                cudaLaunchConfig_t cfg{};
                cfg.gridDim = dim3(unsigned((R->lw[0] + 255) / 256), unsigned(R->lh[0]));
                cfg.blockDim = dim3(256);
                cfg.stream = s;
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                attr[0].val.programmaticStreamSerializationAllowed = 1;
                cfg.attrs = attr;
                cfg.numAttrs = 1;
                const uint8_t* lowc = low;
                const float* rc = R->r;
                cudaLaunchKernelEx(&cfg, k_frame, lowc, rc, out, R->lh[0], R->lw[0]);
                continue;
            }
            // the first layer follows k_input, a plain launch; the others each follow a
            // row-tile convolution, launched as its programmatic dependent
            if(!conv_layer(R, L, 1, s, true))
                return false;
        }
        return true;
    }

    bool backward(isaacb_recon* R, int B, cudaStream_t s)
    {
        bool has[kLayers] = {};
        for(int L = 0; L < kLayers; ++L)
        {
            cudaMemsetAsync(R->dw[L], 0, size_t(kDefs[L].ks * kDefs[L].ks * R->T.cg[L]) * R->T.Npad[L] * sizeof(float), s);
            cudaMemsetAsync(R->db[L], 0, size_t(kDefs[L].cout) * sizeof(float), s);
        }
        for(int L = kLayers - 1; L >= 0; --L)
        {
            const LayerDef& d = kDefs[L];
            const int li = in_level(L), lo = kLevel[L];
            const bf16* g = R->dpre[L];
            // weight and bias gradients
            WgradParams wp{};
            wp.x = layer_input(R, L);
            wp.dy = g;
            wp.dw = R->dw[L];
            wp.B = B;
            wp.H = R->lh[li];
            wp.W = R->lw[li];
            wp.Cin = R->T.cg[L];
            wp.Ho = R->lh[lo];
            wp.Wo = R->lw[lo];
            wp.Cout = d.cout;
            wp.Npad = R->T.Npad[L];
            wp.ks = d.ks;
            wp.stride = d.stride;
            wp.pad = d.pad;
            wp.Mtot = d.ks * d.ks * R->T.cg[L];
            wp.errorFlag = R->errorFlag;
            if(!launch_conv_wgrad(wp, s))
                return false;
            const size_t pix = size_t(B) * R->lh[lo] * R->lw[lo];
            k_bias_grad<<<grid_for(pix / 8 + 1), 256, 0, s>>>(g, pix, d.cout, R->db[L]);
            if(d.src == SRC_X)
                continue;
            // input gradient
            ConvGemmParams p{};
            p.x = g;
            p.w = R->wt[L];
            p.B = B;
            p.H = R->lh[lo];
            p.W = R->lw[lo];
            p.Cg = d.cout;
            p.Ho = R->lh[li];
            p.Wo = R->lw[li];
            p.Cout = d.cin;
            p.Npad = R->T.NpadT[L];
            p.Kpad = R->T.KpadT[L];
            p.ks = d.ks;
            p.stride = d.stride;
            p.pad = d.pad;
            p.transposed = 1;
            p.errorFlag = R->errorFlag;
            if(d.src == -2)
            {
                p.y = R->dcat;
                if(!launch_conv_gemm(p, s))
                    return false;
                const int lf = kLevel[d.fine], lc = kLevel[d.coarse];
                const int c1 = kDefs[d.coarse].cout, c2 = kDefs[d.fine].cout;
                const size_t n = size_t(B) * (size_t(R->lh[lf]) * R->lw[lf] * (c2 / 8) + size_t(R->lh[lc]) * R->lw[lc] * (c1 / 8));
                k_cat_up_backward<<<grid_for(n), 256, 0, s>>>(
                    R->dcat,
                    R->act[d.coarse],
                    R->act[d.fine],
                    R->dpre[d.coarse],
                    R->dpre[d.fine],
                    B,
                    R->lh[lf],
                    R->lw[lf],
                    R->lh[lc],
                    R->lw[lc],
                    c1,
                    c2);
                has[d.coarse] = has[d.fine] = true;
            }
            else
            {
                p.y = R->dpre[d.src];
                p.mask = R->act[d.src];
                p.accumulate = has[d.src] ? 1 : 0;
                if(!launch_conv_gemm(p, s))
                    return false;
                has[d.src] = true;
            }
        }
        return true;
    }

    isaacb_status check_dims(const isaacb_recon* R, uint32_t batch, uint32_t h, uint32_t w)
    {
        if(!R || batch == 0 || h < 8 || w < 8 || h > 16384 || w > 16384)
            return ISAACB_INVALID_ARG;
        // every level must fit the buffers sized for the creation-time maximum
        int lh[4], lw[4], mh[4], mw[4];
        level_sizes(int(h), int(w), lh, lw);
        level_sizes(R->maxH, R->maxW, mh, mw);
        for(int l = 0; l < 4; ++l)
            if(size_t(batch) * lh[l] * lw[l] > size_t(R->maxBatch) * mh[l] * mw[l])
                return ISAACB_INVALID_ARG;
        return ISAACB_OK;
    }

    void table_pointers(isaacb_recon* R, bool withGrads)
    {
        for(int L = 0; L < kLayers; ++L)
        {
            R->T.wf[L] = R->wf[L];
            R->T.wt[L] = R->wt[L];
            R->T.dw[L] = withGrads ? R->dw[L] : nullptr;
            R->T.db[L] = withGrads ? R->db[L] : nullptr;
        }
    }

    // the master weights -> bias buffers and the packed bf16 copies
    void sync_params(isaacb_recon* R, cudaStream_t s)
    {
        table_pointers(R, false);
        k_params<<<(R->total + 255) / 256, 256, 0, s>>>(R->T, R->master, R->adamM, R->adamV, R->total, 0, 0.0f, nullptr);
        for(int L = 0; L < kLayers; ++L)
        {
            const int nw = kDefs[L].cout * kDefs[L].ks * kDefs[L].ks * kDefs[L].cin;
            cudaMemcpyAsync(R->bias[L], R->master + R->T.off[L] + nw, kDefs[L].cout * sizeof(float), cudaMemcpyDeviceToDevice, s);
        }
    }
} // namespace

extern "C"
{
    uint32_t isaacb_recon_param_count(void)
    {
        uint32_t n = 0;
        for(int L = 0; L < kLayers; ++L)
            n += uint32_t(kDefs[L].cout * kDefs[L].ks * kDefs[L].ks * kDefs[L].cin + kDefs[L].cout);
        return n;
    }

    isaacb_status isaacb_recon_create(uint32_t max_batch, uint32_t max_h, uint32_t max_w, uint64_t seed, isaacb_recon** out)
    {
        if(!out || max_batch == 0 || max_h < 8 || max_w < 8 || uint64_t(max_batch) * max_h * max_w > (1ull << 26))
            return fail_r(ISAACB_INVALID_ARG, "isaacb_recon_create: bad sizes");
        *out = nullptr;
        isaacb_recon* R = new isaacb_recon;
        R->maxBatch = int(max_batch);
        R->maxH = int(max_h);
        R->maxW = int(max_w);
        int mh[4], mw[4];
        level_sizes(R->maxH, R->maxW, mh, mw);
        bool ok = true;
        int off = 0;
        size_t maxCat = 0;
        for(int L = 0; L < kLayers && ok; ++L)
        {
            const LayerDef& d = kDefs[L];
            const int cg = round_up(d.cin, 16);
            const int K = d.ks * d.ks * cg, KT = d.ks * d.ks * d.cout;
            R->T.off[L] = off;
            R->T.ks[L] = d.ks;
            R->T.cin[L] = d.cin;
            R->T.cg[L] = cg;
            R->T.cout[L] = d.cout;
            R->T.Npad[L] = round_up(d.cout, 16);
            R->T.Kpad[L] = round_up(K, 64);
            R->T.NpadT[L] = round_up(d.cin, 16);
            R->T.KpadT[L] = round_up(KT, 64);
            off += d.cout * d.ks * d.ks * d.cin + d.cout;
            const size_t pix = size_t(R->maxBatch) * mh[kLevel[L]] * mw[kLevel[L]];
            ok = ok && dalloc(R, R->wf[L], size_t(R->T.Npad[L]) * R->T.Kpad[L]);
            ok = ok && (d.src == SRC_X || dalloc(R, R->wt[L], size_t(R->T.NpadT[L]) * R->T.KpadT[L]));
            ok = ok && dalloc(R, R->bias[L], d.cout);
            ok = ok && dalloc(R, R->dw[L], size_t(K) * R->T.Npad[L]);
            ok = ok && dalloc(R, R->db[L], d.cout);
            ok = ok && dalloc(R, R->dpre[L], pix * d.cout);
            if(L != kLayers - 1)
                ok = ok && dalloc(R, R->act[L], pix * d.cout);
            if(d.src == -2)
            {
                ok = ok && dalloc(R, R->cat[L], pix * d.cin);
                maxCat = std::max(maxCat, pix * d.cin);
            }
            if(ok && conv_gemm_smem(R->T.Npad[L], R->T.Kpad[L]) > 227 * 1024)
                ok = false;
        }
        R->T.off[kLayers] = off;
        R->total = off;
        const size_t pix0 = size_t(R->maxBatch) * mh[0] * mw[0];
        ok = ok && dalloc(R, R->dcat, maxCat) && dalloc(R, R->x, pix0 * 16) && dalloc(R, R->r, pix0 * 16);
        ok = ok && dalloc(R, R->master, size_t(off)) && dalloc(R, R->adamM, size_t(off)) && dalloc(R, R->adamV, size_t(off));
        ok = ok && dalloc(R, R->lossSum, 1) && dalloc(R, R->gradHost, size_t(off)) && dalloc(R, R->sqErr, 1) && dalloc(R, R->errorFlag, 1);
        if(!ok)
        {
            isaacb_recon_destroy(R);
            return fail_r(ISAACB_OOM, "isaacb_recon_create: allocation failed");
        }
        // He-normal weights from the seed, zero biases; the output layer starts small so
        // the first frames are close to the bilinear upsampling
        std::vector<float> host(size_t(off), 0.0f);
        std::mt19937_64 rng(seed);
        std::normal_distribution<float> nd(0.0f, 1.0f);
        for(int L = 0; L < kLayers; ++L)
        {
            const LayerDef& d = kDefs[L];
            const int fan = d.ks * d.ks * d.cin;
            const float sc = std::sqrt(2.0f / float(fan)) * (L == kLayers - 1 ? 0.1f : 1.0f);
            for(int i = 0; i < d.cout * fan; ++i)
                host[size_t(R->T.off[L] + i)] = nd(rng) * sc;
        }
        cudaMemcpy(R->master, host.data(), host.size() * sizeof(float), cudaMemcpyHostToDevice);
        sync_params(R, 0);
        if(cudaDeviceSynchronize() != cudaSuccess)
        {
            isaacb_recon_destroy(R);
            return fail_r(ISAACB_CUDA_ERROR, "isaacb_recon_create: initialisation failed");
        }
        *out = R;
        return ISAACB_OK;
    }

    isaacb_status isaacb_recon_destroy(isaacb_recon* R)
    {
        if(!R)
            return ISAACB_OK;
        for(void* p : R->allocs)
            cudaFree(p);
        delete R;
        return ISAACB_OK;
    }

    isaacb_status isaacb_recon_get_params(isaacb_recon* R, float* host)
    {
        if(!R || !host)
            return ISAACB_INVALID_ARG;
        if(cudaMemcpy(host, R->master, size_t(R->total) * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
            return fail_r(ISAACB_CUDA_ERROR, "isaacb_recon_get_params");
        return ISAACB_OK;
    }

    isaacb_status isaacb_recon_set_params(isaacb_recon* R, const float* host)
    {
        if(!R || !host)
            return ISAACB_INVALID_ARG;
        if(cudaMemcpy(R->master, host, size_t(R->total) * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
            return fail_r(ISAACB_CUDA_ERROR, "isaacb_recon_set_params");
        cudaMemset(R->adamM, 0, size_t(R->total) * sizeof(float));
        cudaMemset(R->adamV, 0, size_t(R->total) * sizeof(float));
        R->step = 0;
        sync_params(R, 0);
        return cudaDeviceSynchronize() == cudaSuccess ? ISAACB_OK : fail_r(ISAACB_CUDA_ERROR, "isaacb_recon_set_params");
    }

    isaacb_status isaacb_recon_train_step(
        isaacb_recon* R,
        const uint8_t* low,
        const uint8_t* high,
        const int32_t* index,
        uint32_t batch,
        uint32_t h,
        uint32_t w,
        float lr,
        float* loss_dev,
        float* grads_host,
        void* stream)
    {
        if(check_dims(R, batch, h, w) != ISAACB_OK || !low || !high)
            return fail_r(ISAACB_INVALID_ARG, "isaacb_recon_train_step: bad arguments");
        cudaStream_t s = (cudaStream_t) stream;
        const int B = int(batch);
        level_sizes(int(h), int(w), R->lh, R->lw);
        const size_t pix0 = size_t(B) * h * w;
        k_input<<<grid_for(pix0), 256, 0, s>>>(low, index, B, int(h), int(w), R->x);
        if(!forward(R, B, s))
            return fail_r(ISAACB_INVALID_ARG, "isaacb_recon_train_step: layer does not fit");
        cudaMemsetAsync(R->lossSum, 0, sizeof(float), s);
        const float n = float(pix0) * 16.0f;
        k_loss<<<grid_for(pix0), 256, 0, s>>>(low, high, index, R->r, R->dpre[kLayers - 1], R->lossSum, B, int(h), int(w), 2.0f / n, 1.0f / n);
        if(!backward(R, B, s))
            return fail_r(ISAACB_INVALID_ARG, "isaacb_recon_train_step: layer does not fit");
        table_pointers(R, true);
        const bool update = grads_host == nullptr;
        if(update)
            R->step++;
        k_params<<<(R->total + 255) / 256, 256, 0, s>>>(
            R->T, R->master, R->adamM, R->adamV, R->total, update ? R->step : 0, lr, update ? nullptr : R->gradHost);
        if(update)
        {
            for(int L = 0; L < kLayers; ++L)
            {
                const int nw = kDefs[L].cout * kDefs[L].ks * kDefs[L].ks * kDefs[L].cin;
                cudaMemcpyAsync(R->bias[L], R->master + R->T.off[L] + nw, kDefs[L].cout * sizeof(float), cudaMemcpyDeviceToDevice, s);
            }
        }
        if(loss_dev)
            cudaMemcpyAsync(loss_dev, R->lossSum, sizeof(float), cudaMemcpyDeviceToDevice, s);
        if(grads_host)
        {
            if(cudaMemcpyAsync(grads_host, R->gradHost, size_t(R->total) * sizeof(float), cudaMemcpyDeviceToHost, s) != cudaSuccess
               || cudaStreamSynchronize(s) != cudaSuccess)
                return fail_r(ISAACB_CUDA_ERROR, "isaacb_recon_train_step: gradient readback");
        }
        const cudaError_t e = cudaGetLastError();
        if(e != cudaSuccess)
            return fail_r(ISAACB_CUDA_ERROR, std::string("isaacb_recon_train_step: ") + cudaGetErrorString(e));
        return ISAACB_OK;
    }

    isaacb_status isaacb_recon_infer(isaacb_recon* R, const uint8_t* low, uint32_t h, uint32_t w, uint8_t* out, void* stream)
    {
        if(check_dims(R, 1, h, w) != ISAACB_OK || !low || !out)
            return fail_r(ISAACB_INVALID_ARG, "isaacb_recon_infer: bad arguments");
        cudaStream_t s = (cudaStream_t) stream;
        level_sizes(int(h), int(w), R->lh, R->lw);
        const size_t pix0 = size_t(h) * w;
        k_input<<<grid_for(pix0), 256, 0, s>>>(low, nullptr, 1, int(h), int(w), R->x);
        if(!forward_infer(R, low, out, s))
            return fail_r(ISAACB_INVALID_ARG, "isaacb_recon_infer: layer does not fit");
        const cudaError_t e = cudaGetLastError();
        if(e != cudaSuccess)
            return fail_r(ISAACB_CUDA_ERROR, std::string("isaacb_recon_infer: ") + cudaGetErrorString(e));
        return ISAACB_OK;
    }

    isaacb_status isaacb_recon_error(isaacb_recon* R, int32_t* flag)
    {
        if(!R || !flag)
            return ISAACB_INVALID_ARG;
        if(cudaMemcpy(flag, R->errorFlag, sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
            return ISAACB_CUDA_ERROR;
        cudaMemset(R->errorFlag, 0, sizeof(int32_t));
        return ISAACB_OK;
    }

    isaacb_status isaacb_recon_arm_wait_check(isaacb_recon* R, uint32_t budget_us)
    {
        if(!R || budget_us == 0)
            return fail_r(ISAACB_INVALID_ARG, "isaacb_recon_arm_wait_check: bad arguments");
        R->waitCheckNs = 1000ull * budget_us;
        return ISAACB_OK;
    }

    isaacb_status isaacb_upsample_bilinear2(const uint8_t* low, uint32_t h, uint32_t w, uint8_t* out, void* stream)
    {
        if(!low || !out || h == 0 || w == 0)
            return fail_r(ISAACB_INVALID_ARG, "isaacb_upsample_bilinear2: bad arguments");
        k_bilinear_frame<<<grid_for(size_t(4) * h * w), 256, 0, (cudaStream_t) stream>>>(low, out, int(h), int(w));
        return cudaGetLastError() == cudaSuccess ? ISAACB_OK : fail_r(ISAACB_CUDA_ERROR, "isaacb_upsample_bilinear2");
    }

    isaacb_status isaacb_image_sq_error(const uint8_t* a, const uint8_t* b, uint64_t bytes, unsigned long long* sum_dev, void* stream)
    {
        if(!a || !b || !sum_dev || bytes % 4 != 0)
            return fail_r(ISAACB_INVALID_ARG, "isaacb_image_sq_error: bad arguments");
        k_sq_error<<<grid_for(bytes / 4), 256, 0, (cudaStream_t) stream>>>(a, b, size_t(bytes), sum_dev);
        return cudaGetLastError() == cudaSuccess ? ISAACB_OK : fail_r(ISAACB_CUDA_ERROR, "isaacb_image_sq_error");
    }
}
