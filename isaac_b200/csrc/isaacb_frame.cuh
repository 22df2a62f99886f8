// Per-pixel helpers shared by the combined and the per-source frame kernels.
#pragma once

#include "isaacb_internal.h"

namespace isaacb
{
    __device__ __forceinline__ size_t pix(const FrameParams& p, int x, int y)
    {
        return size_t(y) * p.v.W + x;
    }

    __device__ __forceinline__ void count_samples(unsigned long long* ctr, unsigned long long n)
    {
        // one atomic per warp
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            n += __shfl_xor_sync(0xffffffffu, n, o);
        if((threadIdx.x & 31) == 0 && n)
            atomicAdd(ctr, n);
    }

    // ------------------------------------------------------------------ shading + volume
    // ShadingKernel (lib/isaac/isaac_common_kernel.hpp:220-320) for rank 0
    __device__ __forceinline__ float4 hsva_rank0(float a)
    {
        // getHSVA(halton(0,3)*2pi, 1, 1, a) = (1, 0, 0, a)
        return make_float4(1.0f, 0.0f, 0.0f, a);
    }

    // the settings ShadingKernel reads
    struct ShadeParams
    {
        int32_t renderMode;
        float aoWeight;
        float4 bg;
    };

    // ShadingKernel on one pixel's G-buffer values: colour and depth are updated in place
    __device__ __forceinline__ void shade_values(
        const ShadeParams& sp,
        const View& v,
        const Geom& g,
        int px,
        int py,
        uchar4& gcolor,
        float3 normal,
        float aoRaw,
        float& depth)
    {
        float4 color = from_byte4(gcolor);
        const float aoStrength = 1.0f - aoRaw;
        const int mode = sp.renderMode;
        if(mode == 7)
            color = hsva_rank0(color.w);
        if(mode < 3 || mode == 7)
        {
            const Ray ray = pixel_to_ray(v, g, px, py);
            const float3 lightDir = neg3(ray.dir);
            float lightFactor = fabsf(dot3(normal, lightDir));
            const float3 halfVector = normalize3(add3(neg3(ray.dir), lightDir));
            float specular = dot3(normal, halfVector);
            const double s2 = double(specular) * double(specular);
            specular = float(s2 * s2);
            specular *= 0.5f;
            if(mode == 1)
                specular = 0.0f;
            const float w = sp.aoWeight;
            const float aoFactor = ((1.0f - w) + w * aoStrength);
            lightFactor += aoFactor;
            lightFactor *= 0.5f;
            float4 sh;
            sh.x = gmin(color.x * lightFactor + specular, 1.0f);
            sh.y = gmin(color.y * lightFactor + specular, 1.0f);
            sh.z = gmin(color.z * lightFactor + specular, 1.0f);
            sh.w = color.w;
            gcolor = to_byte4(sh);
            if(mode == 2 || mode == 7)
                depth = 0.0f;
        }
        else if(mode == 3)
        {
            gcolor = to_byte4(make_float4(sp.bg.w, sp.bg.z, sp.bg.y, color.w));
        }
        else if(mode == 4)
        {
            gcolor = to_byte4(make_float4(normal.x * 0.5f + 0.5f, normal.y * 0.5f + 0.5f, normal.z * 0.5f + 0.5f, color.w));
            depth = 0.0f;
        }
        else if(mode == 5)
        {
            const float d = depth / float(g.maxGss);
            gcolor = to_byte4(make_float4(d, d, d, color.w));
            depth = 0.0f;
        }
        else if(mode == 6)
        {
            const float w = sp.aoWeight;
            const float aoFactor = ((1.0f - w) + w * aoStrength);
            gcolor = to_byte4(make_float4(aoFactor, aoFactor, aoFactor, color.w));
            depth = 0.0f;
        }
        else if(mode == 8)
        {
            gcolor = to_byte4(hsva_rank0(1.0f));
            depth = 0.0f;
        }
    }

    __device__ __forceinline__ void shade_pixel(const FrameParams& p, int px, int py, size_t o)
    {
        const ShadeParams sp{p.renderMode, p.aoWeight, p.bg};
        uchar4 c = p.color[o];
        float d = p.depth[o];
        shade_values(sp, p.v, p.g, px, py, c, f3(p.normal[3 * o], p.normal[3 * o + 1], p.normal[3 * o + 2]), p.ao[o], d);
        p.color[o] = c;
        p.depth[o] = d;
    }
} // namespace isaacb
