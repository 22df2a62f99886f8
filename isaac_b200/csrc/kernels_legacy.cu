// Frame kernels of the per-source renderer (the reference's legacy path,
// ISAAC_RENDERER_LEGACY): every sample interpolates each source's own bricks,
// applies its functor chain and transfer function and accumulates.
//   getColorValue        lib/isaac/isaac_volume_kernel.hpp:101-168
//   VolumeRenderKernel   lib/isaac/isaac_volume_kernel.hpp:302-432
//   IsoStepRenderKernel  lib/isaac/isaac_iso_kernel.hpp:463-778
//
// Bricks hold FP32, BF16 or FP16 values; interpolation, chain, lookup and
// compositing stay FP32.
#include "isaacb_frame.cuh"

#include <cfloat>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace isaacb
{
    __device__ __forceinline__ float load_elem(const void* base, int dtype, size_t i)
    {
        if(dtype == 1)
            return __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(base)[i]);
        if(dtype == 2)
            return __half2float(reinterpret_cast<const __half*>(base)[i]);
        return __ldg(reinterpret_cast<const float*>(base) + i);
    }

    // one source's colour at pos (getColorValue)
    __device__ float4 per_source_color(const FrameParams& p, int s, float3 pos, bool linear)
    {
        const PerSourceSrc& S = p.ps[s];
        const Geom& g = p.g;
        const int per = 4 * S.ncomp;
        float v[4] = {0, 0, 0, 0};
        float result;
        if(linear)
        {
            const float cx = pos.x - 0.5f, cy = pos.y - 0.5f, cz = pos.z - 0.5f;
            const float flx = floorf(cx), fly = floorf(cy), flz = floorf(cz);
            const float fx = cx - flx, fy = cy - fly, fz = cz - flz;
            int ix, iy, iz;
            if(S.persistent)
            {
                // isaac_int(offsetPos) truncates; the mirror at the upper border equals a clamp
                ix = f2i(cx);
                iy = f2i(cy);
                iz = f2i(cz);
            }
            else
            {
                ix = f2i(flx);
                iy = f2i(fly);
                iz = f2i(flz);
            }
            ix = iclamp(ix, -1, g.ls[0] - 1);
            iy = iclamp(iy, -1, g.ls[1] - 1);
            iz = iclamp(iz, -1, g.ls[2] - 1);
            size_t above;
            const size_t s0 = source_slot(g, ix, iy, iz, above) * per;
            const size_t s1 = above * per;
#pragma unroll
            for(int c = 0; c < 4; ++c)
            {
                if(c < S.ncomp)
                {
                    v[c] = tri_q(
                        fx,
                        fy,
                        fz,
                        load_elem(S.bricks, S.dtype, s0 + 4 * c),
                        load_elem(S.bricks, S.dtype, s0 + 4 * c + 1),
                        load_elem(S.bricks, S.dtype, s0 + 4 * c + 2),
                        load_elem(S.bricks, S.dtype, s0 + 4 * c + 3),
                        load_elem(S.bricks, S.dtype, s1 + 4 * c),
                        load_elem(S.bricks, S.dtype, s1 + 4 * c + 1),
                        load_elem(S.bricks, S.dtype, s1 + 4 * c + 2),
                        load_elem(S.bricks, S.dtype, s1 + 4 * c + 3));
                }
            }
        }
        else
        {
            const int ix = iclamp(f2i(pos.x), 0, g.ls[0] - 1);
            const int iy = iclamp(f2i(pos.y), 0, g.ls[1] - 1);
            const int iz = iclamp(f2i(pos.z), 0, g.ls[2] - 1);
            size_t above;
            const size_t s0 = source_slot(g, ix, iy, iz, above) * per;
#pragma unroll
            for(int c = 0; c < 4; ++c)
                if(c < S.ncomp)
                    v[c] = load_elem(S.bricks, S.dtype, s0 + 4 * c);
        }
        if(S.persistent)
            result = apply_chain(v, S.fdim, S.chain);
        else
            result = v[0];
        return __ldg(p.lut + size_t(s) * p.ts + lut_index(result, p.ts));
    }

    // checkCoord (lib/isaac/isaac_volume_kernel.hpp:206-214) for guard 0
    __device__ __forceinline__ float3 check_coord(const Geom& g, float3 c)
    {
        return f3(
            gclamp(c.x, 0.0f, float(g.ls[0] - 1) - FLT_MIN),
            gclamp(c.y, 0.0f, float(g.ls[1] - 1) - FLT_MIN),
            gclamp(c.z, 0.0f, float(g.ls[2] - 1) - FLT_MIN));
    }
    __device__ __forceinline__ float4 accessor_value(const FrameParams& p, int s, float3 pos, bool linear)
    {
        if(p.ps[s].persistent)
            pos = check_coord(p.g, pos);
        return per_source_color(p, s, pos, linear);
    }

    // start/end step adjustment of the legacy kernels (lib/isaac/isaac_volume_kernel.hpp:362-376)
    __device__ __forceinline__ bool inside_local(const Geom& g, float3 pos)
    {
        return !(pos.x < 0.0f || pos.y < 0.0f || pos.z < 0.0f || pos.x >= float(g.ls[0]) || pos.y >= float(g.ls[1])
                 || pos.z >= float(g.ls[2]));
    }
    __device__ __forceinline__ void legacy_bounds(const Geom& g, March& m)
    {
        float3 pos = march_pos(m, m.startSteps);
        while(!inside_local(g, pos) && m.startSteps <= m.endSteps)
        {
            m.startSteps++;
            pos = march_pos(m, m.startSteps);
        }
        pos = march_pos(m, m.endSteps);
        while(!inside_local(g, pos) && m.startSteps <= m.endSteps)
        {
            m.endSteps--;
            pos = march_pos(m, m.endSteps);
        }
    }

    __device__ __forceinline__ void count_warp(unsigned long long* ctr, unsigned long long n)
    {
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            n += __shfl_xor_sync(0xffffffffu, n, o);
        if((threadIdx.x & 31) == 0 && n)
            atomicAdd(ctr, n);
    }

    __global__ void __launch_bounds__(256) k_iso_per_source(const __grid_constant__ FrameParams p)
    {
        int px, py;
        thread_pixel(px, py);
        unsigned long long n = 0;
        const bool linear = p.interpolation != 0;
        bool any = false;
        for(int s = 0; s < p.nVol; ++s)
            any |= p.ps[s].iso != 0.0f;
        if(any && px < p.v.W && py < p.v.H)
        {
            const size_t o = size_t(py) * p.v.W + px;
            Ray ray = pixel_to_ray(p.v, p.g, px, py);
            if(clip_ray(ray, p.v, p.g))
            {
                ray.endDepth = gmin(ray.endDepth, p.depth[o]);
                if(!(ray.endDepth <= ray.startDepth))
                {
                    March m = march_setup(ray, p.g, p.v.scale, p.step);
                    legacy_bounds(p.g, m);
                    bool hit = false;
                    float hitDepth = ray.endDepth;
                    float4 hitColor = make_float4(0, 0, 0, 0);
                    float3 hitNormal = f3(0, 0, 0);
                    float oldValues[kMaxSources];
                    for(int s = 0; s < kMaxSources; ++s)
                        oldValues[s] = 0.0f;
                    for(int i = m.startSteps; i <= m.endSteps && !hit; i++)
                    {
                        ++n;
                        const float3 pos = march_pos(m, i);
                        const bool first = ray.isClipped && i == m.startSteps;
                        const float t = float(i) * m.stepU;
                        for(int s = 0; s < p.nVol; ++s)
                        {
                            const float thr = p.ps[s].iso;
                            if(thr == 0.0f)
                                continue;
                            const float value = accessor_value(p, s, pos, linear).w;
                            const float prev = oldValues[s];
                            oldValues[s] = value;
                            if(value < thr)
                                continue;
                            float testDepth;
                            if(first)
                                testDepth = ray.startDepth;
                            else
                                testDepth = t + m.stepU * (thr - prev) / (value - prev);
                            if(testDepth > hitDepth)
                                continue;
                            hitDepth = testDepth;
                            hit = true;
                            const float3 np = add3(ray.start, muls3(ray.dir, hitDepth));
                            const float3 pu = div3(np, p.v.scale);
                            hitColor = accessor_value(p, s, pu, linear);
                            hitColor.w = 1.0f;
                            float3 gr;
                            gr.x = accessor_value(p, s, add3(pu, f3(1, 0, 0)), linear).w
                                - accessor_value(p, s, sub3(pu, f3(1, 0, 0)), linear).w;
                            gr.y = accessor_value(p, s, add3(pu, f3(0, 1, 0)), linear).w
                                - accessor_value(p, s, sub3(pu, f3(0, 1, 0)), linear).w;
                            gr.z = accessor_value(p, s, add3(pu, f3(0, 0, 1)), linear).w
                                - accessor_value(p, s, sub3(pu, f3(0, 0, 1)), linear).w;
                            float gl = length3(gr);
                            if(first)
                            {
                                gr = ray.clippingNormal;
                                gl = 1.0f;
                            }
                            hitNormal = divs3(neg3(gr), gl);
                        }
                    }
                    if(hit)
                    {
                        p.color[o] = to_byte4(hitColor);
                        p.normal[3 * o] = hitNormal.x;
                        p.normal[3 * o + 1] = hitNormal.y;
                        p.normal[3 * o + 2] = hitNormal.z;
                        p.depth[o] = hitDepth;
                    }
                }
            }
        }
        if(p.counters)
            count_warp(p.counters + 1, n);
    }

    void launch_iso_per_source(const FrameParams& p, cudaStream_t s)
    {
        dim3 grid((p.v.W + 31) / 32, (p.v.H + 7) / 8);
        k_iso_per_source<<<grid, 256, 0, s>>>(p);
    }

    __global__ void __launch_bounds__(256) k_shade_volume_per_source(const __grid_constant__ FrameParams p)
    {
        int px, py;
        thread_pixel(px, py);
        unsigned long long n = 0;
        const bool linear = p.interpolation != 0;
        if(px < p.v.W && py < p.v.H)
        {
            const size_t o = size_t(py) * p.v.W + px;
            shade_pixel(p, px, py, o);
            bool any = false;
            for(int s = 0; s < p.nVol; ++s)
                any |= p.ps[s].weight != 0.0f;
            Ray ray = pixel_to_ray(p.v, p.g, px, py);
            if(any && clip_ray(ray, p.v, p.g))
            {
                ray.endDepth = gmin(ray.endDepth, p.depth[o]);
                if(!(ray.endDepth <= ray.startDepth))
                {
                    March m = march_setup(ray, p.g, p.v.scale, p.step);
                    legacy_bounds(p.g, m);
                    float4 value = make_float4(0, 0, 0, 0);
                    float4 color = make_float4(0, 0, 0, 0);
                    for(int i = m.startSteps; i <= m.endSteps; i++)
                    {
                        ++n;
                        const float3 pos = march_pos(m, i);
                        for(int s = 0; s < p.nVol; ++s)
                        {
                            const float w = p.ps[s].weight;
                            if(w == 0.0f)
                                continue;
                            float4 c = per_source_color(p, s, pos, linear);
                            c.w *= w;
                            value.x += c.x * c.w;
                            value.y += c.y * c.w;
                            value.z += c.z * c.w;
                            value.w += c.w;
                        }
                        const float oma = 1.0f - color.w;
                        value = make_float4(value.x * m.factor, value.y * m.factor, value.z * m.factor, value.w * m.factor);
                        color.x += oma * value.x;
                        color.y += oma * value.y;
                        color.z += oma * value.z;
                        color.w += oma * value.w;
                        if(color.w > 0.99f)
                            break;
                    }
                    const float4 solid = from_byte4(p.color[o]);
                    const float r = 1.0f - color.w;
                    color = make_float4(color.x + r * solid.x, color.y + r * solid.y, color.z + r * solid.z, color.w + r * solid.w);
                    p.color[o] = to_byte4(color);
                }
            }
        }
        if(p.counters)
            count_warp(p.counters, n);
    }

    // 4 consecutive stored values (one x-quad of a slot) as floats
    template<int DT>
    __device__ __forceinline__ void load_quad(const void* base, size_t slot, float (&v)[4])
    {
        if constexpr(DT == 0)
        {
            const float4 q = __ldg(reinterpret_cast<const float4*>(base) + slot);
            v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
        }
        else
        {
            const uint2 q = __ldg(reinterpret_cast<const uint2*>(base) + slot);
            if constexpr(DT == 1)
            {
                v[0] = __uint_as_float(q.x << 16);
                v[1] = __uint_as_float(q.x & 0xFFFF0000u);
                v[2] = __uint_as_float(q.y << 16);
                v[3] = __uint_as_float(q.y & 0xFFFF0000u);
            }
            else
            {
                const __half2 a = *reinterpret_cast<const __half2*>(&q.x), b = *reinterpret_cast<const __half2*>(&q.y);
                const float2 fa = __half22float2(a), fb = __half22float2(b);
                v[0] = fa.x, v[1] = fa.y, v[2] = fb.x, v[3] = fb.y;
            }
        }
    }

    // The same march as k_shade_volume_per_source for the common case of scalar,
    // persistent sources that share one storage type: the trilinear footprint (slot
    // and fractions) is found once per sample for all sources, and each source's
    // two x-quads come in two vector loads.  Arithmetic and order are unchanged,
    // so the frame is bit-identical to the general kernel's.
    template<int DT, bool LINEAR>
    __global__ void __launch_bounds__(256) k_shade_volume_per_source_scalar(const __grid_constant__ FrameParams p)
    {
        int px, py;
        thread_pixel(px, py);
        unsigned long long n = 0;
        if(px < p.v.W && py < p.v.H)
        {
            const size_t o = size_t(py) * p.v.W + px;
            shade_pixel(p, px, py, o);
            bool any = false;
            for(int s = 0; s < p.nVol; ++s)
                any |= p.ps[s].weight != 0.0f;
            Ray ray = pixel_to_ray(p.v, p.g, px, py);
            if(any && clip_ray(ray, p.v, p.g))
            {
                ray.endDepth = gmin(ray.endDepth, p.depth[o]);
                if(!(ray.endDepth <= ray.startDepth))
                {
                    March m = march_setup(ray, p.g, p.v.scale, p.step);
                    legacy_bounds(p.g, m);
                    const Geom& g = p.g;
                    float4 value = make_float4(0, 0, 0, 0);
                    float4 color = make_float4(0, 0, 0, 0);
                    for(int i = m.startSteps; i <= m.endSteps; i++)
                    {
                        ++n;
                        const float3 pos = march_pos(m, i);
                        size_t q0, q1;
                        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
                        if(LINEAR)
                        {
                            const float cx = pos.x - 0.5f, cy = pos.y - 0.5f, cz = pos.z - 0.5f;
                            fx = cx - floorf(cx);
                            fy = cy - floorf(cy);
                            fz = cz - floorf(cz);
                            // persistent sources: isaac_int(offsetPos) truncates
                            const int ix = iclamp(f2i(cx), -1, g.ls[0] - 1);
                            const int iy = iclamp(f2i(cy), -1, g.ls[1] - 1);
                            const int iz = iclamp(f2i(cz), -1, g.ls[2] - 1);
                            q0 = source_slot(g, ix, iy, iz, q1);
                        }
                        else
                        {
                            const int ix = iclamp(f2i(pos.x), 0, g.ls[0] - 1);
                            const int iy = iclamp(f2i(pos.y), 0, g.ls[1] - 1);
                            const int iz = iclamp(f2i(pos.z), 0, g.ls[2] - 1);
                            q0 = source_slot(g, ix, iy, iz, q1);
                        }
                        for(int s = 0; s < p.nVol; ++s)
                        {
                            const PerSourceSrc& S = p.ps[s];
                            const float w = S.weight;
                            if(w == 0.0f)
                                continue;
                            float a[4], b[4];
                            load_quad<DT>(S.bricks, q0, a);
                            float v[4] = {0, 0, 0, 0};
                            if(LINEAR)
                            {
                                load_quad<DT>(S.bricks, q1, b);
                                v[0] = tri_q(fx, fy, fz, a[0], a[1], a[2], a[3], b[0], b[1], b[2], b[3]);
                            }
                            else
                                v[0] = a[0];
                            const float result = apply_chain(v, S.fdim, S.chain);
                            float4 c = __ldg(p.lut + size_t(s) * p.ts + lut_index(result, p.ts));
                            c.w *= w;
                            value.x += c.x * c.w;
                            value.y += c.y * c.w;
                            value.z += c.z * c.w;
                            value.w += c.w;
                        }
                        const float oma = 1.0f - color.w;
                        value = make_float4(value.x * m.factor, value.y * m.factor, value.z * m.factor, value.w * m.factor);
                        color.x += oma * value.x;
                        color.y += oma * value.y;
                        color.z += oma * value.z;
                        color.w += oma * value.w;
                        if(color.w > 0.99f)
                            break;
                    }
                    const float4 solid = from_byte4(p.color[o]);
                    const float r = 1.0f - color.w;
                    color = make_float4(color.x + r * solid.x, color.y + r * solid.y, color.z + r * solid.z, color.w + r * solid.w);
                    p.color[o] = to_byte4(color);
                }
            }
        }
        if(p.counters)
            count_warp(p.counters, n);
    }

    // Weighted sources of a frame, in source order (zero weights dropped): the
    // specialised kernel below keeps their pointers and weights in registers.
    struct ActiveSources
    {
        int n;
        int idx[kMaxSources];
        const void* bricks[kMaxSources];
        float weight[kMaxSources];
        // active source k's premultiplied table, biased so that the float bits of
        // 1.5 * 2^23 + index address entry index (see transfer_entry)
        const char* pre[kMaxSources];
    };

    // The volume term of every table entry of the active sources, once per frame instead
    // of once per sample: a = c.w * weight, (c.x * a, c.y * a, c.z * a, a).  These are the
    // products the per-sample loop of PerSourceVolumeRenderKernel forms
    // (lib/isaac/isaac_volume_kernel.hpp:365-377: color.w *= weight; value += color * color.w),
    // so the sums that use them round the same way.
    __global__ void __launch_bounds__(256) k_ps_premultiply(const float4* __restrict__ lut, ActiveSources act, float4* __restrict__ out, int ts)
    {
        const int k = blockIdx.y;
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if(i >= ts)
            return;
        const float4 c = __ldg(lut + size_t(act.idx[k]) * ts + i);
        const float a = c.w * act.weight[k];
        out[size_t(k) * ts + i] = make_float4(c.x * a, c.y * a, c.z * a, a);
    }

    // the premultiplied entry of lut_index_fast(v, ts) as two FP32 pairs (r, g) and (b, a):
    // round(clamp(v * ts, 0, ts - 1)) is floor(x + 0.5) with the add rounded down (it never
    // crosses the next integer), and the floor comes as float bits from a magic-number add
    // also rounded down; both give lut_index_fast's index for every v, NaN included
    __device__ __forceinline__ void transfer_entry(const char* biased, float v, float tsf, float tsMax, f2p& rg, f2p& ba)
    {
        const float xi = fminf(fmaxf(v * tsf, 0.0f), tsMax);
        const float t = __fadd_rd(__fadd_rd(xi, 0.5f), 12582912.0f);
        const ulonglong2 e = __ldg(reinterpret_cast<const ulonglong2*>(biased + size_t(uint32_t(__float_as_int(t))) * sizeof(float4)));
        rg.v = e.x;
        ba.v = e.y;
    }

    // a*(1-o) + b*o on two lanes (two sources), each lane rounded exactly like lin():
    // both products round before the add (f2p_mul_exact)
    __device__ __forceinline__ f2p lin2(f2p omo, f2p o, f2p a, f2p b, f2p nz)
    {
        return f2p_add(f2p_mul_exact(a, omo, nz), f2p_mul_exact(b, o, nz));
    }

    // k_shade_volume_per_source_scalar for 1..4 weighted sources known at compile time:
    // the sources' quads are all loaded before any is used, pairs of sources share packed
    // FP32 trilinear arithmetic (two lanes, the scalar roundings), and with IDEM the
    // functor chain is skipped.  The weighted premultiplied table entries come from
    // k_ps_premultiply, found with a 6-instruction index, and value and colour run as
    // FP32 pairs.  Same operations in the same order per source, so the frame is
    // bit-identical to the general kernels'.
    // (4 CTAs per SM: 58 registers without spills, twice the warps of the unbounded 88)
    template<int DT, bool LINEAR, int NS, bool IDEM>
    __global__ void __launch_bounds__(256, 4) k_shade_volume_per_source_n(
        const __grid_constant__ FrameParams p,
        const __grid_constant__ ActiveSources act)
    {
        int px, py;
        thread_pixel(px, py);
        unsigned long long n = 0;
        if(px < p.v.W && py < p.v.H)
        {
            const size_t o = size_t(py) * p.v.W + px;
            shade_pixel(p, px, py, o);
            Ray ray = pixel_to_ray(p.v, p.g, px, py);
            if(clip_ray(ray, p.v, p.g))
            {
                ray.endDepth = gmin(ray.endDepth, p.depth[o]);
                if(!(ray.endDepth <= ray.startDepth))
                {
                    March m = march_setup(ray, p.g, p.v.scale, p.step);
                    legacy_bounds(p.g, m);
                    const Geom& g = p.g;
                    const void* br[NS];
#pragma unroll
                    for(int k = 0; k < NS; ++k)
                        br[k] = act.bricks[k];
                    const float tsf = float(p.ts), tsMax = float(p.ts - 1);
                    const f2p fac = f2p_make(m.factor, m.factor);
                    const f2p nz = f2p_make(p.negZero, p.negZero);
                    // value and colour as FP32 pairs (r, g), (b, a); every lane rounds like
                    // the scalar op
                    f2p vrg = f2p_make(0.0f, 0.0f), vba = f2p_make(0.0f, 0.0f);
                    f2p crg = f2p_make(0.0f, 0.0f), cba = f2p_make(0.0f, 0.0f);
                    float cw = 0.0f;
                    // The warp walks absolute step indices together from its earliest first
                    // step, each lane sampling only inside its own range: lanes then sample
                    // the same depth shell at once, which keeps their taps close where the
                    // entry face is oblique to the view.  Each ray's samples and their
                    // order are unchanged.
                    const int wStart = __reduce_min_sync(__activemask(), m.startSteps);
                    for(int i = wStart; i <= m.endSteps; i++)
                    {
                        if(i < m.startSteps)
                            continue;
                        ++n;
                        const float3 pos = march_pos(m, i);
                        uint32_t q0, q1 = 0;
                        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
                        size_t above;
                        if(LINEAR)
                        {
                            const float cx = pos.x - 0.5f, cy = pos.y - 0.5f, cz = pos.z - 0.5f;
                            fx = cx - floorf(cx);
                            fy = cy - floorf(cy);
                            fz = cz - floorf(cz);
                            const int ix = iclamp(f2i(cx), -1, g.ls[0] - 1);
                            const int iy = iclamp(f2i(cy), -1, g.ls[1] - 1);
                            const int iz = iclamp(f2i(cz), -1, g.ls[2] - 1);
                            q0 = uint32_t(source_slot(g, ix, iy, iz, above));
                            q1 = uint32_t(above);
                        }
                        else
                        {
                            const int ix = iclamp(f2i(pos.x), 0, g.ls[0] - 1);
                            const int iy = iclamp(f2i(pos.y), 0, g.ls[1] - 1);
                            const int iz = iclamp(f2i(pos.z), 0, g.ls[2] - 1);
                            q0 = uint32_t(source_slot(g, ix, iy, iz, above));
                        }
                        float a[NS][4], b[NS][4], val[NS];
#pragma unroll
                        for(int k = 0; k < NS; ++k)
                        {
                            load_quad<DT>(br[k], q0, a[k]);
                            if(LINEAR)
                                load_quad<DT>(br[k], q1, b[k]);
                        }
                        if(LINEAR)
                        {
                            const f2p omz = f2p_make(1.0f - fz, 1.0f - fz), vz = f2p_make(fz, fz);
                            const f2p omy = f2p_make(1.0f - fy, 1.0f - fy), vy = f2p_make(fy, fy);
                            const f2p omx = f2p_make(1.0f - fx, 1.0f - fx), vx = f2p_make(fx, fx);
#pragma unroll
                            for(int k = 0; k + 1 < NS; k += 2)
                            {
                                // quad order (x0,y0),(x0+1,y0),(x0,y0+1),(x0+1,y0+1); tri_q's lerp tree
                                const f2p z00 = lin2(omz, vz, f2p_make(a[k][0], a[k + 1][0]), f2p_make(b[k][0], b[k + 1][0]), nz);
                                const f2p z01 = lin2(omz, vz, f2p_make(a[k][2], a[k + 1][2]), f2p_make(b[k][2], b[k + 1][2]), nz);
                                const f2p z10 = lin2(omz, vz, f2p_make(a[k][1], a[k + 1][1]), f2p_make(b[k][1], b[k + 1][1]), nz);
                                const f2p z11 = lin2(omz, vz, f2p_make(a[k][3], a[k + 1][3]), f2p_make(b[k][3], b[k + 1][3]), nz);
                                const f2p A = lin2(omy, vy, z00, z01, nz);
                                const f2p B = lin2(omy, vy, z10, z11, nz);
                                f2p_split(lin2(omx, vx, A, B, nz), val[k], val[k + 1]);
                            }
                            if(NS & 1)
                            {
                                const int k = NS - 1;
                                val[k] = tri_q(fx, fy, fz, a[k][0], a[k][1], a[k][2], a[k][3], b[k][0], b[k][1], b[k][2], b[k][3]);
                            }
                        }
                        else
                        {
#pragma unroll
                            for(int k = 0; k < NS; ++k)
                                val[k] = a[k][0];
                        }
                        // value gains the weighted premultiplied entries (it carries over
                        // from the previous sample, scaled by the factor, as in the reference)
#pragma unroll
                        for(int k = 0; k < NS; ++k)
                        {
                            float result = val[k];
                            if(!IDEM)
                            {
                                float v[4] = {val[k], 0.0f, 0.0f, 0.0f};
                                result = apply_chain(v, 1, p.ps[act.idx[k]].chain);
                            }
                            f2p erg, eba;
                            transfer_entry(act.pre[k], result, tsf, tsMax, erg, eba);
                            vrg = f2p_add(vrg, erg);
                            vba = f2p_add(vba, eba);
                        }
                        const float oma = 1.0f - cw;
                        const f2p om = f2p_make(oma, oma);
                        vrg = f2p_mul_exact(vrg, fac, nz);
                        vba = f2p_mul_exact(vba, fac, nz);
                        crg = f2p_add(crg, f2p_mul_exact(om, vrg, nz));
                        cba = f2p_add(cba, f2p_mul_exact(om, vba, nz));
                        float cb;
                        f2p_split(cba, cb, cw);
                        if(cw > 0.99f)
                            break;
                    }
                    float4 color;
                    f2p_split(crg, color.x, color.y);
                    f2p_split(cba, color.z, color.w);
                    const float4 solid = from_byte4(p.color[o]);
                    const float r = 1.0f - color.w;
                    color = make_float4(color.x + r * solid.x, color.y + r * solid.y, color.z + r * solid.z, color.w + r * solid.w);
                    p.color[o] = to_byte4(color);
                }
            }
        }
        if(p.counters)
            count_warp(p.counters, n);
    }

    template<int DT, bool LINEAR, bool IDEM>
    void launch_ps_n(const FrameParams& p, const ActiveSources& act, dim3 grid, cudaStream_t s)
    {
        k_ps_premultiply<<<dim3((p.ts + 255) / 256, act.n), 256, 0, s>>>(p.lut, act, p.psPre, p.ts);
        switch(act.n)
        {
        case 1: k_shade_volume_per_source_n<DT, LINEAR, 1, IDEM><<<grid, 256, 0, s>>>(p, act); break;
        case 2: k_shade_volume_per_source_n<DT, LINEAR, 2, IDEM><<<grid, 256, 0, s>>>(p, act); break;
        case 3: k_shade_volume_per_source_n<DT, LINEAR, 3, IDEM><<<grid, 256, 0, s>>>(p, act); break;
        default: k_shade_volume_per_source_n<DT, LINEAR, 4, IDEM><<<grid, 256, 0, s>>>(p, act); break;
        }
    }
    template<int DT>
    void launch_ps_dt(const FrameParams& p, const ActiveSources& act, bool lin, bool idem, dim3 grid, cudaStream_t s)
    {
        if(lin)
            idem ? launch_ps_n<DT, true, true>(p, act, grid, s) : launch_ps_n<DT, true, false>(p, act, grid, s);
        else
            idem ? launch_ps_n<DT, false, true>(p, act, grid, s) : launch_ps_n<DT, false, false>(p, act, grid, s);
    }

    int launch_shade_volume_per_source(const FrameParams& p, cudaStream_t s)
    {
        dim3 grid((p.v.W + 31) / 32, (p.v.H + 7) / 8);
        // the scalar kernel serves frames whose weighted sources are all scalar, persistent and of one type
        int dt = -1;
        bool scalar = true;
        for(int k = 0; k < p.nVol && scalar; ++k)
        {
            const PerSourceSrc& S = p.ps[k];
            if(S.weight == 0.0f)
                continue;
            scalar = S.fdim == 1 && S.ncomp == 1 && S.persistent && (dt < 0 || dt == S.dtype);
            dt = S.dtype;
        }
        if(scalar && dt >= 0)
        {
            const bool lin = p.interpolation != 0;
            ActiveSources act{};
            bool idem = true;
            for(int k = 0; k < p.nVol; ++k)
            {
                const PerSourceSrc& S = p.ps[k];
                if(S.weight == 0.0f)
                    continue;
                act.idx[act.n] = k;
                act.bricks[act.n] = S.bricks;
                act.weight[act.n] = S.weight;
                act.pre[act.n] = reinterpret_cast<const char*>(p.psPre + size_t(act.n) * p.ts)
                    - size_t(0x4B400000u) * sizeof(float4);
                act.n++;
                idem = idem && S.chain.op[0] == OP_IDEM && S.chain.op[1] == OP_IDEM && S.chain.op[2] == OP_IDEM;
            }
            // slot indices of the specialised kernel are 32-bit
            const bool fits = size_t(p.g.nb[0]) * p.g.nb[1] * p.g.nb[2] * kSlotsPerBrick < (1ull << 31);
            if(act.n >= 1 && act.n <= 4 && fits)
            {
                if(dt == 0)
                    launch_ps_dt<0>(p, act, lin, idem, grid, s);
                else if(dt == 1)
                    launch_ps_dt<1>(p, act, lin, idem, grid, s);
                else
                    launch_ps_dt<2>(p, act, lin, idem, grid, s);
                return 2;
            }
            if(dt == 0)
                lin ? k_shade_volume_per_source_scalar<0, true><<<grid, 256, 0, s>>>(p)
                    : k_shade_volume_per_source_scalar<0, false><<<grid, 256, 0, s>>>(p);
            else if(dt == 1)
                lin ? k_shade_volume_per_source_scalar<1, true><<<grid, 256, 0, s>>>(p)
                    : k_shade_volume_per_source_scalar<1, false><<<grid, 256, 0, s>>>(p);
            else
                lin ? k_shade_volume_per_source_scalar<2, true><<<grid, 256, 0, s>>>(p)
                    : k_shade_volume_per_source_scalar<2, false><<<grid, 256, 0, s>>>(p);
            return 1;
        }
        k_shade_volume_per_source<<<grid, 256, 0, s>>>(p);
        return 1;
    }
} // namespace isaacb
