// Stereo compositing of two rendered passes on the GPU (the reference does it on
// the host after IceT, lib/isaac/isaac_compositors.hpp:37-116):
//   mode 0  the first image (DefaultCompositor)
//   mode 1  left and right side by side, 2W x H (StereoCompositorSideBySide)
//   mode 2  per pixel (left & leftFilter) | (right & rightFilter) on the 32-bit RGBA8
//           word (StereoCompositorAnaglyph)
// Rows, pixels and bytes keep the frame layout (row 0 = bottom).
#include "../../include/isaac_b200.h"

#include <cuda_runtime.h>
#include <string>

namespace isaacb
{
    void set_global_error(const std::string& msg);

    namespace
    {
        __global__ void k_composite(int mode, const uint32_t* __restrict__ left, const uint32_t* __restrict__ right, int w, int h, uint32_t lf, uint32_t rf, uint32_t* __restrict__ out)
        {
            const int outW = mode == 1 ? 2 * w : w;
            const size_t n = size_t(outW) * h;
            for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
            {
                const int x = int(i % outW);
                const size_t y = i / outW;
                uint32_t v;
                if(mode == 1)
                    v = x < w ? __ldg(left + y * w + x) : __ldg(right + y * w + (x - w));
                else if(mode == 2)
                    v = (__ldg(left + i) & lf) | (__ldg(right + i) & rf);
                else
                    v = __ldg(left + i);
                out[i] = v;
            }
        }

        // ---------------------------------------------------------------- sort-last blend
        // IceT's ordered BLEND composite of the ranks' RGBA8 images
        // (lib/isaac.hpp:820-826, 2015-2055): premultiplied colours folded front to back
        // with the "under" operator in 8-bit integers, each channel
        //   acc += src * (255 - acc.alpha) / 255   (integer division, result kept mod 256),
        // with acc.alpha taken before the step.  The images arrive already sorted front to
        // back; an optional background goes under the result.
        constexpr int kMaxBlendImages = 64;
        struct BlendArgs
        {
            const uint32_t* img[kMaxBlendImages];
            int32_t count;
            int32_t hasBg;
            uint32_t bg;
        };

        // Two channels per 32-bit word, one in each 16-bit lane: b * f <= 255 * 255 fits a
        // lane, and for 0 <= x <= 65025, floor(x / 255) == (x + 1 + (x >> 8)) >> 8 with
        // the sum <= 65280, so no lane carries into the next.  Byte permutes pick the
        // lanes' bytes; the final permute keeps the low byte of each channel sum, which is
        // the mod-256 result.
        __device__ __forceinline__ uint32_t div255_lanes(uint32_t x)
        {
            const uint32_t t = x + 0x00010001u + __byte_perm(x, 0u, 0x4341);
            return __byte_perm(t, 0u, 0x4341);
        }

        __device__ __forceinline__ uint32_t under(uint32_t acc, uint32_t src)
        {
            const uint32_t f = 255u - (acc >> 24);
            const uint32_t lo = __byte_perm(acc, 0u, 0x4240) + div255_lanes(__byte_perm(src, 0u, 0x4240) * f);
            const uint32_t hi = __byte_perm(acc, 0u, 0x4341) + div255_lanes(__byte_perm(src, 0u, 0x4341) * f);
            return __byte_perm(lo, hi, 0x6240);
        }

        // four pixels per thread: one 16-byte load per image, all issued before the fold
        __global__ void __launch_bounds__(256) k_blend_under4(const __grid_constant__ BlendArgs a, size_t quads, uint4* __restrict__ out)
        {
            for(size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < quads; q += size_t(gridDim.x) * blockDim.x)
            {
                // the first image under an empty accumulator is itself (f = 255)
                uint4 acc = __ldg(reinterpret_cast<const uint4*>(a.img[0]) + q);
                for(int k0 = 1; k0 < a.count; k0 += 8)
                {
                    uint4 v[8];
                    const int m = min(8, a.count - k0);
#pragma unroll
                    for(int k = 0; k < 8; ++k)
                        if(k < m)
                            v[k] = __ldg(reinterpret_cast<const uint4*>(a.img[k0 + k]) + q);
#pragma unroll
                    for(int k = 0; k < 8; ++k)
                        if(k < m)
                        {
                            acc.x = under(acc.x, v[k].x);
                            acc.y = under(acc.y, v[k].y);
                            acc.z = under(acc.z, v[k].z);
                            acc.w = under(acc.w, v[k].w);
                        }
                }
                if(a.hasBg)
                    acc = make_uint4(under(acc.x, a.bg), under(acc.y, a.bg), under(acc.z, a.bg), under(acc.w, a.bg));
                out[q] = acc;
            }
        }

        __global__ void __launch_bounds__(256) k_blend_under(const __grid_constant__ BlendArgs a, size_t n, uint32_t* __restrict__ out)
        {
            for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
            {
                uint32_t acc = 0;
                for(int k = 0; k < a.count; ++k)
                    acc = under(acc, __ldg(a.img[k] + i));
                out[i] = a.hasBg ? under(acc, a.bg) : acc;
            }
        }
    } // namespace
} // namespace isaacb

extern "C" isaacb_status isaacb_blend_ordered(
    const uint8_t* const* images,
    uint32_t count,
    const int32_t* order,
    uint32_t pixels,
    const uint8_t* background,
    uint8_t* out,
    void* stream)
{
    using namespace isaacb;
    if(!images || !order || !out || count == 0 || count > uint32_t(kMaxBlendImages))
    {
        set_global_error("isaacb_blend_ordered: bad arguments (1 to 64 images, order and output required)");
        return ISAACB_INVALID_ARG;
    }
    BlendArgs a{};
    bool aligned = (reinterpret_cast<uintptr_t>(out) & 15u) == 0 && pixels % 4 == 0;
    uint64_t seen = 0;
    for(uint32_t k = 0; k < count; ++k)
    {
        const int32_t r = order[k];
        if(r < 0 || uint32_t(r) >= count || (seen >> r) & 1u || !images[r])
        {
            set_global_error("isaacb_blend_ordered: order must be a permutation of the images");
            return ISAACB_INVALID_ARG;
        }
        seen |= uint64_t(1) << r;
        a.img[k] = reinterpret_cast<const uint32_t*>(images[r]);
        aligned = aligned && (reinterpret_cast<uintptr_t>(images[r]) & 15u) == 0;
    }
    a.count = int32_t(count);
    a.hasBg = background ? 1 : 0;
    if(background)
        a.bg = uint32_t(background[0]) | (uint32_t(background[1]) << 8) | (uint32_t(background[2]) << 16)
            | (uint32_t(background[3]) << 24);
    if(pixels == 0)
        return ISAACB_OK;
    const size_t work = aligned ? pixels / 4 : pixels;
    size_t blocks = (work + 255) / 256;
    if(blocks > 148 * 16)
        blocks = 148 * 16;
    if(aligned)
        k_blend_under4<<<unsigned(blocks), 256, 0, (cudaStream_t) stream>>>(a, work, reinterpret_cast<uint4*>(out));
    else
        k_blend_under<<<unsigned(blocks), 256, 0, (cudaStream_t) stream>>>(a, work, reinterpret_cast<uint32_t*>(out));
    const cudaError_t e = cudaGetLastError();
    if(e != cudaSuccess)
    {
        set_global_error(std::string("isaacb_blend_ordered: ") + cudaGetErrorString(e));
        return ISAACB_CUDA_ERROR;
    }
    return ISAACB_OK;
}

extern "C" isaacb_status isaacb_composite(
    int32_t mode,
    const uint8_t* left,
    const uint8_t* right,
    uint32_t width,
    uint32_t height,
    uint32_t left_filter,
    uint32_t right_filter,
    uint8_t* out,
    void* stream)
{
    if(!left || !out || width == 0 || height == 0 || width > 32768 || height > 32768 || mode < 0 || mode > 2
       || (mode != 0 && !right))
    {
        isaacb::set_global_error("isaacb_composite: bad arguments");
        return ISAACB_INVALID_ARG;
    }
    const size_t n = size_t(mode == 1 ? 2 * width : width) * height;
    size_t blocks = (n + 255) / 256;
    if(blocks > 148 * 8)
        blocks = 148 * 8;
    isaacb::k_composite<<<unsigned(blocks), 256, 0, (cudaStream_t) stream>>>(
        mode,
        reinterpret_cast<const uint32_t*>(left),
        reinterpret_cast<const uint32_t*>(right),
        int(width),
        int(height),
        left_filter,
        right_filter,
        reinterpret_cast<uint32_t*>(out));
    const cudaError_t e = cudaGetLastError();
    if(e != cudaSuccess)
    {
        isaacb::set_global_error(std::string("isaacb_composite: ") + cudaGetErrorString(e));
        return ISAACB_CUDA_ERROR;
    }
    return ISAACB_OK;
}
