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

    __device__ __forceinline__ void shade_pixel(const FrameParams& p, int px, int py, size_t o)
    {
        float4 color = from_byte4(p.color[o]);
        const float3 normal = f3(p.normal[3 * o], p.normal[3 * o + 1], p.normal[3 * o + 2]);
        const float aoStrength = 1.0f - p.ao[o];
        const int mode = p.renderMode;
        if(mode == 7)
            color = hsva_rank0(color.w);
        if(mode < 3 || mode == 7)
        {
            const Ray ray = pixel_to_ray(p.v, p.g, px, py);
            const float3 lightDir = neg3(ray.dir);
            float lightFactor = fabsf(dot3(normal, lightDir));
            const float3 halfVector = normalize3(add3(neg3(ray.dir), lightDir));
            float specular = dot3(normal, halfVector);
            const double s2 = double(specular) * double(specular);
            specular = float(s2 * s2);
            specular *= 0.5f;
            if(mode == 1)
                specular = 0.0f;
            const float w = p.aoWeight;
            const float aoFactor = ((1.0f - w) + w * aoStrength);
            lightFactor += aoFactor;
            lightFactor *= 0.5f;
            float4 sh;
            sh.x = gmin(color.x * lightFactor + specular, 1.0f);
            sh.y = gmin(color.y * lightFactor + specular, 1.0f);
            sh.z = gmin(color.z * lightFactor + specular, 1.0f);
            sh.w = color.w;
            p.color[o] = to_byte4(sh);
            if(mode == 2 || mode == 7)
                p.depth[o] = 0.0f;
        }
        else if(mode == 3)
        {
            p.color[o] = to_byte4(make_float4(p.bg.w, p.bg.z, p.bg.y, color.w));
        }
        else if(mode == 4)
        {
            p.color[o] = to_byte4(make_float4(normal.x * 0.5f + 0.5f, normal.y * 0.5f + 0.5f, normal.z * 0.5f + 0.5f, color.w));
            p.depth[o] = 0.0f;
        }
        else if(mode == 5)
        {
            const float d = p.depth[o] / float(p.g.maxGss);
            p.color[o] = to_byte4(make_float4(d, d, d, color.w));
            p.depth[o] = 0.0f;
        }
        else if(mode == 6)
        {
            const float w = p.aoWeight;
            const float aoFactor = ((1.0f - w) + w * aoStrength);
            p.color[o] = to_byte4(make_float4(aoFactor, aoFactor, aoFactor, color.w));
            p.depth[o] = 0.0f;
        }
        else if(mode == 8)
        {
            p.color[o] = to_byte4(hsva_rank0(1.0f));
            p.depth[o] = 0.0f;
        }
    }

} // namespace isaacb
