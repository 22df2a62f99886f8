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
    } // namespace
} // namespace isaacb

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
