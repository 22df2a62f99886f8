// Frame kernels of the combined (pre-classified) renderer: drawCallBack
// (lib/isaac.hpp:2140-2543).
//
//   k_clear_particles  ClearBufferKernel + ParticleRenderKernel
//                      (lib/isaac/isaac_common_kernel.hpp:195-217,
//                       lib/isaac/isaac_particle_kernel.hpp:32-260)
//   k_iso              CombinedIsoRenderKernel (lib/isaac/isaac_iso_kernel.hpp:25-128)
//   k_ssao             SSAOKernel (+ optional SSAOFilterKernel)
//                      (lib/isaac/isaac_ssao_kernel.hpp:38-230)
//   k_shade_volume     ShadingKernel + CombinedVolumeRenderKernel
//                      (lib/isaac/isaac_common_kernel.hpp:220-320,
//                       lib/isaac/isaac_volume_kernel.hpp:23-88)
//
// The reference launches these six passes with a blocking wait after each;
// here the per-pixel passes that need no neighbour are fused, so a frame is
// two launches (four with iso surfaces and SSAO).
#include "isaacb_frame.cuh"
#include "isaacb_march.cuh"

#include <algorithm>
#include <cfloat>

namespace isaacb
{
    // ------------------------------------------------------------------ particles
    __device__ void particle_pixel(const FrameParams& p, int px, int py)
    {
        bool any = false;
        for(int s = 0; s < p.nPart; ++s)
            any |= p.part[s].weight != 0.0f;
        if(!any)
            return;
        Ray ray = pixel_to_ray(p.v, p.g, px, py);
        if(!clip_ray(ray, p.v, p.g))
            return;
        const size_t o = pix(p, px, py);
        ray.endDepth = gmin(ray.endDepth, p.depth[o]);
        const float3 ps = p.pscale;
        float4 pColor = make_float4(0, 0, 0, 0);
        float depth = FLT_MAX;
        bool hit = false;
        int ds[3];
        ds[0] = int(gsign(ray.dir.x));
        ds[1] = int(gsign(ray.dir.y));
        ds[2] = int(gsign(ray.dir.z));
        const float3 cur = add3(ray.start, muls3(ray.dir, ray.startDepth));
        uint32_t cell[3];
        cell[0] = uint32_t(iclamp(f2i(cur.x / ps.x), 0, p.g.lps[0] - 1));
        cell[1] = uint32_t(iclamp(f2i(cur.y / ps.y), 0, p.g.lps[1] - 1));
        cell[2] = uint32_t(iclamp(f2i(cur.z / ps.z), 0, p.g.lps[2] - 1));
        const float rayLength = ray.endDepth - ray.startDepth;
        float tested = 0.0f;
        float t[3], dT[3];
        const float dr[3] = {ray.dir.x, ray.dir.y, ray.dir.z};
        const float pc[3] = {ps.x, ps.y, ps.z};
        const float cu[3] = {cur.x, cur.y, cur.z};
#pragma unroll
        for(int i = 0; i < 3; ++i)
        {
            t[i] = ((float(cell[i]) + float(max(ds[i], 0))) * pc[i] - cu[i]) / dr[i];
            dT[i] = pc[i] / dr[i] * float(ds[i]);
            if(dr[i] == 0.0f)
                t[i] = FLT_MAX;
        }
        float3 pNormal = f3(0, 0, 0);
        while(cell[0] < uint32_t(p.g.lps[0]) && cell[1] < uint32_t(p.g.lps[1]) && cell[2] < uint32_t(p.g.lps[2])
              && !hit && tested <= rayLength)
        {
            const size_t ci = (size_t(cell[2]) * p.g.lps[1] + cell[1]) * p.g.lps[0] + cell[0];
            const float3 cellf = f3(float(cell[0]), float(cell[1]), float(cell[2]));
            for(int s = 0; s < p.nPart; ++s)
            {
                const ParticleSrc& P = p.part[s];
                if(P.weight == 0.0f)
                    continue;
                const uint32_t k1 = __ldg(P.offsets + ci + 1);
                for(uint32_t k = __ldg(P.offsets + ci); k < k1; ++k)
                {
                    const float3 pp
                        = f3(__ldg(P.pos + 3 * size_t(k)), __ldg(P.pos + 3 * size_t(k) + 1), __ldg(P.pos + 3 * size_t(k) + 2));
                    const float3 ppos = mul3(add3(pp, cellf), ps);
                    const float3 L = sub3(ppos, cur);
                    const float radius = (P.radius ? __ldg(P.radius + k) : P.constRadius) * P.weight;
                    const float r2 = radius * radius;
                    const float tca = dot3(L, ray.dir);
                    const float d2 = dot3(L, L) - tca * tca;
                    if(d2 <= r2)
                    {
                        const float thc = sqrtf(r2 - d2);
                        const float t0 = tca - thc;
                        const float t1 = tca + thc;
                        if(t1 >= 0.0f && t0 < depth)
                        {
                            float a[4];
                            const float* ap = P.attr + size_t(k) * P.fdim;
                            a[0] = __ldg(ap);
                            a[1] = P.fdim > 1 ? __ldg(ap + 1) : 0.0f;
                            a[2] = P.fdim > 2 ? __ldg(ap + 2) : 0.0f;
                            a[3] = P.fdim > 3 ? __ldg(ap + 3) : 0.0f;
                            const float res = apply_chain(a, P.fdim, P.chain);
                            const float4 value = __ldg(p.lut + P.lutBase + lut_index(res, p.ts));
                            if(value.w >= 0.5f)
                            {
                                pColor = value;
                                depth = t0;
                                hit = true;
                                pNormal = sub3(add3(cur, smul3(t0, ray.dir)), ppos);
                                if(t0 < 0.0f && ray.isClipped)
                                    pNormal = neg3(ray.clippingNormal);
                            }
                        }
                    }
                }
            }
            if(t[0] < t[1] && t[0] < t[2])
            {
                cell[0] += uint32_t(ds[0]);
                tested = t[0];
                t[0] += dT[0];
            }
            else if(t[1] < t[0] && t[1] < t[2])
            {
                cell[1] += uint32_t(ds[1]);
                tested = t[1];
                t[1] += dT[1];
            }
            else
            {
                cell[2] += uint32_t(ds[2]);
                tested = t[2];
                t[2] += dT[2];
            }
        }
        if(!hit)
            return;
        pNormal = normalize3(pNormal);
        pColor.w = 1.0f;
        p.color[o] = to_byte4(pColor);
        p.normal[3 * o] = pNormal.x;
        p.normal[3 * o + 1] = pNormal.y;
        p.normal[3 * o + 2] = pNormal.z;
        p.depth[o] = depth + ray.startDepth;
    }

    __global__ void __launch_bounds__(256) k_clear_particles(const __grid_constant__ FrameParams p)
    {
        int px, py;
        thread_pixel(px, py);
        if(px >= p.v.W || py >= p.v.H)
            return;
        const size_t o = pix(p, px, py);
        p.color[o] = to_byte4(p.bgSwizzled);
        p.normal[3 * o] = 0.0f;
        p.normal[3 * o + 1] = 0.0f;
        p.normal[3 * o + 2] = 0.0f;
        p.depth[o] = FLT_MAX;
        p.ao[o] = 0.0f;
        if(p.nPart > 0)
            particle_pixel(p, px, py);
    }

    void launch_clear_particles(const FrameParams& p, cudaStream_t s)
    {
        dim3 grid((p.v.W + 31) / 32, (p.v.H + 7) / 8);
        k_clear_particles<<<grid, 256, 0, s>>>(p);
    }

    // ------------------------------------------------------------------ iso
    // interpolated alpha byte (0..255 scale) of the iso alpha quads at c = pos - 0.5,
    // FMA/ALU pipes only; brick index and emptiness (max alpha <= 127) returned
    // slot of apron-shifted coordinates inside their brick for a known slot order
    template<bool YFAST>
    __device__ __forceinline__ uint32_t slot_in_brick_as(int ax, int ay, int az)
    {
        return uint32_t(az & 7) * 64u + (YFAST ? uint32_t((ax & 7) * 8 + (ay & 7)) : uint32_t((ay & 7) * 8 + (ax & 7)));
    }

    template<bool LINEAR, bool YFAST>
    __device__ __forceinline__ float iso_alpha_fast(const FrameParams& p, float cx, float cy, float cz, int& brick)
    {
        const Geom& g = p.g;
        const float lo = LINEAR ? -1.0f : 0.0f;
        cx = fminf(fmaxf(cx, lo), float(g.ls[0] - 1));
        cy = fminf(fmaxf(cy, lo), float(g.ls[1] - 1));
        cz = fminf(fmaxf(cz, lo), float(g.ls[2] - 1));
        const int magic = 0x4B400000 - 1;
        const float tx = __fadd_rd(cx, 12582912.0f), ty = __fadd_rd(cy, 12582912.0f), tz = __fadd_rd(cz, 12582912.0f);
        const int ax = __float_as_int(tx) - magic, ay = __float_as_int(ty) - magic, az = __float_as_int(tz) - magic;
        brick = ((az >> 3) * g.nb[1] + (ay >> 3)) * g.nb[0] + (ax >> 3);
        const uint32_t slot = uint32_t(brick) * uint32_t(kSlotsPerBrick) + slot_in_brick_as<YFAST>(ax, ay, az);
        if(!LINEAR)
            return ubyte_f(__ldg(p.isoAQ + slot), 0);
        const uint32_t A = __ldg(p.isoAQ + slot), B = __ldg(p.isoAQ + slot + 64);
        const float fx = cx - (tx - 12582912.0f), fy = cy - (ty - 12582912.0f), fz = cz - (tz - 12582912.0f);
        // bytes as b 2^-133 and z weights times 2^64 (ubyte_pair_tiny): each product and
        // sum is the unscaled one times 2^-69, and the last multiply undoes it exactly
        const float fz64 = fz * 0x1p64f;
        const float gx = 1.0f - fx, gy = 1.0f - fy, gz64 = 0x1p64f - fz64;
        const float w00 = gx * gy, w10 = fx * gy, w01 = gx * fy, w11 = fx * fy;
        float v = ubyte_tiny(A, 0) * (w00 * gz64);
        v = fmaf(ubyte_tiny(A, 1), w10 * gz64, v);
        v = fmaf(ubyte_tiny(A, 2), w01 * gz64, v);
        v = fmaf(ubyte_tiny(A, 3), w11 * gz64, v);
        v = fmaf(ubyte_tiny(B, 0), w00 * fz64, v);
        v = fmaf(ubyte_tiny(B, 1), w10 * fz64, v);
        v = fmaf(ubyte_tiny(B, 2), w01 * fz64, v);
        v = fmaf(ubyte_tiny(B, 3), w11 * fz64, v);
        return v * 0x1p69f;
    }

    // Interpolated alpha byte (0..255 scale) of the iso alpha quads at the reference's
    // sample position pos = startU + stepVec * i, with the reference's arithmetic: the
    // position and c = pos - 0.5 rounded as separate operations, floor/fraction of the
    // unclamped c, CLAMP on the texel indices and the z -> y -> x lerp order of
    // Sampler/trilinear (lib/isaac/isaac_texture.hpp:140-305, isaac_helper.hpp:124-144).
    template<bool LINEAR, bool YFAST>
    __device__ __forceinline__ float iso_alpha_exact(const FrameParams& p, const March& m, int i)
    {
        const Geom& g = p.g;
        const float3 pos = march_pos(m, i);
        if(!LINEAR)
        {
            const int ax = iclamp(f2i(pos.x), 0, g.ls[0] - 1) + 1, ay = iclamp(f2i(pos.y), 0, g.ls[1] - 1) + 1,
                      az = iclamp(f2i(pos.z), 0, g.ls[2] - 1) + 1;
            const int brick = ((az >> 3) * g.nb[1] + (ay >> 3)) * g.nb[0] + (ax >> 3);
            const uint32_t slot
                = uint32_t(brick) * uint32_t(kSlotsPerBrick) + slot_in_brick_as<YFAST>(ax, ay, az);
            return byte_f(__ldg(p.isoAQ + slot), 0);
        }
        const float cx = pos.x - 0.5f, cy = pos.y - 0.5f, cz = pos.z - 0.5f;
        const float flx = floorf(cx), fly = floorf(cy), flz = floorf(cz);
        const float fx = cx - flx, fy = cy - fly, fz = cz - flz;
        // a footprint whose base lies below -1 or above L-1 reads clamped texels only; the
        // quad at base -1 (L-1) holds exactly those values
        const int ax = iclamp(f2i(flx), -1, g.ls[0] - 1) + 1, ay = iclamp(f2i(fly), -1, g.ls[1] - 1) + 1,
                  az = iclamp(f2i(flz), -1, g.ls[2] - 1) + 1;
        const int brick = ((az >> 3) * g.nb[1] + (ay >> 3)) * g.nb[0] + (ax >> 3);
        const uint32_t slot
            = uint32_t(brick) * uint32_t(kSlotsPerBrick) + slot_in_brick_as<YFAST>(ax, ay, az);
        const uint32_t A = __ldg(p.isoAQ + slot), B = __ldg(p.isoAQ + slot + 64);
        return tri_q(fx, fy, fz, byte_f(A, 0), byte_f(A, 1), byte_f(A, 2), byte_f(A, 3), byte_f(B, 0), byte_f(B, 1),
                     byte_f(B, 2), byte_f(B, 3));
    }

    // CombinedIsoRenderKernel (lib/isaac/isaac_iso_kernel.hpp:25-128).  The march reads
    // alpha with the fast sampler and skips bricks whose alpha bytes are all <= 127 (a
    // trilinear value there is below the 0.5 threshold).  The fast sampler (fused
    // position, 8-weight trilinear) differs from the reference's arithmetic by far less
    // than kIsoMargin bytes, so a sample further than that below the threshold is a
    // miss for both; any other sample is evaluated again with the reference's arithmetic
    // (iso_alpha_exact), which decides the hit.  At the hit, the previous sample's value
    // for the depth interpolation is the exact one too, and value / 255 is a division as
    // in the reference.  So hit, depth, colour and normal follow the reference's float
    // operations exactly.
    constexpr float kIsoMargin = 0.125f; // alpha bytes
    template<bool LINEAR, bool YFAST>
    __global__ void __launch_bounds__(256) k_iso(const __grid_constant__ FrameParams p)
    {
        int px, py;
        thread_pixel(px, py);
        unsigned long long n = 0;
        if(px < p.v.W && py < p.v.H)
        {
            Ray ray = pixel_to_ray(p.v, p.g, px, py);
            const size_t o = pix(p, px, py);
            if(clip_ray(ray, p.v, p.g))
            {
                ray.endDepth = gmin(ray.endDepth, p.depth[o]);
                if(!(ray.endDepth <= ray.startDepth))
                {
                    const March m = march_setup(ray, p.g, p.v.scale, p.step);
                    const float off = LINEAR ? 0.5f : 0.0f;
                    const float c0x = m.startU.x - off, c0y = m.startU.y - off, c0z = m.startU.z - off;
                    bool hit = false;
                    float depth = ray.endDepth;
                    float4 hitColor = make_float4(0, 0, 0, 0);
                    float3 hitNormal = f3(0, 0, 0);
                    int curBrick = -1;
                    bool skip = false;
                    int i = m.startSteps;
                    for(; i <= m.endSteps; ++i)
                    {
                        const float fi = float(i);
                        const float cx = fmaf(m.stepVec.x, fi, c0x), cy = fmaf(m.stepVec.y, fi, c0y),
                                    cz = fmaf(m.stepVec.z, fi, c0z);
                        int brick;
                        const float a = iso_alpha_fast<LINEAR, YFAST>(p, cx, cy, cz, brick);
                        if(brick != curBrick)
                        {
                            curBrick = brick;
                            skip = __ldg(p.isoFlag + brick) <= 127;
                        }
                        if(skip || a < 127.5f - kIsoMargin)
                            continue;
                        const float value = iso_alpha_exact<LINEAR, YFAST>(p, m, i) / 255.0f;
                        if(value < 0.5f)
                            continue;
                        // the reference's previous value: 0 before the first sample
                        const float tmp = i == m.startSteps ? 0.0f : iso_alpha_exact<LINEAR, YFAST>(p, m, i - 1) / 255.0f;
                        const bool first = ray.isClipped && i == m.startSteps;
                        const float t = fi * m.stepU;
                        if(first)
                            depth = ray.startDepth;
                        else
                            depth = t + m.stepU * (0.5f - tmp) / (value - tmp);
                        hit = true;
                        const float3 np = add3(ray.start, muls3(ray.dir, depth));
                        const float3 pu = div3(np, p.v.scale);
                        hitColor = sample_linear_rgba8(p.isoLin, p.g, pu, LINEAR);
                        hitColor.w = 1.0f;
                        float3 gr;
                        gr.x = sample_linear_rgba8(p.isoLin, p.g, add3(pu, f3(1, 0, 0)), LINEAR).w
                            - sample_linear_rgba8(p.isoLin, p.g, sub3(pu, f3(1, 0, 0)), LINEAR).w;
                        gr.y = sample_linear_rgba8(p.isoLin, p.g, add3(pu, f3(0, 1, 0)), LINEAR).w
                            - sample_linear_rgba8(p.isoLin, p.g, sub3(pu, f3(0, 1, 0)), LINEAR).w;
                        gr.z = sample_linear_rgba8(p.isoLin, p.g, add3(pu, f3(0, 0, 1)), LINEAR).w
                            - sample_linear_rgba8(p.isoLin, p.g, sub3(pu, f3(0, 0, 1)), LINEAR).w;
                        float gl = length3(gr);
                        if(first || gl == 0.0f)
                        {
                            gr = ray.clippingNormal;
                            gl = 1.0f;
                        }
                        hitNormal = divs3(neg3(gr), gl);
                        ++i;
                        break;
                    }
                    n += (unsigned long long) (i - m.startSteps);
                    if(hit)
                    {
                        p.color[o] = to_byte4(hitColor);
                        p.normal[3 * o] = hitNormal.x;
                        p.normal[3 * o + 1] = hitNormal.y;
                        p.normal[3 * o + 2] = hitNormal.z;
                        p.depth[o] = depth;
                    }
                }
            }
        }
        if(p.counters)
            count_samples(p.counters + 1, n);
    }

    void launch_iso(const FrameParams& p, cudaStream_t s)
    {
        dim3 grid((p.v.W + 31) / 32, (p.v.H + 7) / 8);
        if(p.interpolation)
            p.g.yfast ? k_iso<true, true><<<grid, 256, 0, s>>>(p) : k_iso<true, false><<<grid, 256, 0, s>>>(p);
        else
            p.g.yfast ? k_iso<false, true><<<grid, 256, 0, s>>>(p) : k_iso<false, false><<<grid, 256, 0, s>>>(p);
    }

    // ------------------------------------------------------------------ SSAO
    __global__ void __launch_bounds__(256) k_ssao(const __grid_constant__ FrameParams p)
    {
        int px, py;
        thread_pixel(px, py);
        if(px >= p.v.W || py >= p.v.H)
            return;
        const size_t o = pix(p, px, py);
        const float ref = p.depth[o];
        float occ = 0.0f;
        float ao;
        if(p.aoSamples == 0)
        {
            for(int i = -3; i <= 3; ++i)
            {
                const int x = iclamp(px + i * 10, 0, p.v.W - 1);
                for(int j = -3; j <= 3; ++j)
                {
                    const int y = iclamp(py + j * 10, 0, p.v.H - 1);
                    if(__ldg(p.depth + pix(p, x, y)) < ref)
                        occ += 1.0f;
                }
            }
            ao = gclamp(occ / 42.0f, 0.0f, 1.0f);
        }
        else
        {
            // the configurable pattern (no reference counterpart): the same occlusion
            // test over aoSamples taps, CLAMP at the frame border
            for(int k = 0; k < p.aoSamples; ++k)
            {
                const int x = iclamp(px + p.aoOffsets[2 * k], 0, p.v.W - 1);
                const int y = iclamp(py + p.aoOffsets[2 * k + 1], 0, p.v.H - 1);
                if(__ldg(p.depth + pix(p, x, y)) < ref)
                    occ += 1.0f;
            }
            ao = gclamp(occ / (float(p.aoSamples) * (42.0f / 48.0f)), 0.0f, 1.0f);
        }
        p.ao[o] = ao;
        if(p.aoFilter)
        {
            const float4 c = from_byte4(p.color[o]);
            const float w = p.aoWeight;
            const float f = (1.0f - w) + w * (1.0f - ao);
            p.color[o] = to_byte4(make_float4(f * c.x, f * c.y, f * c.z, c.w));
        }
    }

    void launch_ssao(const FrameParams& p, cudaStream_t s)
    {
        dim3 grid((p.v.W + 31) / 32, (p.v.H + 7) / 8);
        k_ssao<<<grid, 256, 0, s>>>(p);
    }

    // A k_shade_volume block is 128 threads, 4 warps of 8 x 4 pixels, covering a tile of
    // tile_w(FULL) x tile_h(FULL) pixels.
    constexpr int kShadeThreads = 128;
    // tile width of the FULL form (the short launches): 16 x 8 pixels keep a block's rays
    // closer together than 32 x 4 (the 960x540 half-size render: 0.953 -> 0.931 ms)
    constexpr int kShortTileW = 16;
    // tile width and minimum blocks per SM of the uncapped form (the long launches)
    constexpr int kLongTileW = 32;
    constexpr int kLongMinBlocks = 1;
    __host__ __device__ constexpr int shade_tile_w(bool full)
    {
        return full ? kShortTileW : kLongTileW;
    }
    __host__ __device__ constexpr int shade_tile_h(bool full)
    {
        return kShadeThreads / shade_tile_w(full);
    }

    // FULL: registers capped so that a whole SM's threads are resident (16 blocks, 32
    // registers, a few bytes spilled).  Launches of only a few waves take it: more
    // resident rays shorten their tail.  Longer launches keep the uncapped form (46
    // registers, 10 blocks per SM), whose loop runs faster.
    // tile of a y-fastest texture's blocks (4 warps of 4 x 8 pixels)
    constexpr int kYTileW = 16;
    __host__ __device__ constexpr int shade_tile_w(bool full, bool yfast)
    {
        return yfast ? kYTileW : shade_tile_w(full);
    }
    __host__ __device__ constexpr int shade_tile_h(bool full, bool yfast)
    {
        return kShadeThreads / shade_tile_w(full, yfast);
    }

    // YFAST: the texture's slots are y fastest; each warp then covers 4 x 8 pixels, so that
    // the image's columns, which views about the y axis keep along y, walk the fastest axis
    template<bool VOLUME, bool LINEAR, bool FULL, bool YFAST>
    __global__ void __launch_bounds__(kShadeThreads, FULL ? 2048 / kShadeThreads : kLongMinBlocks) k_shade_volume(const __grid_constant__ FrameParams p)
    {
        // empty-space skipping only pays when the texture has empty bricks; the merge that
        // wrote it counted them (either choice renders the same image)
        const bool skip = VOLUME && __ldg(p.emptyCount) != 0u;
        constexpr int TW = shade_tile_w(FULL, YFAST), TH = shade_tile_h(FULL, YFAST);
        constexpr int WW = YFAST ? 4 : 8, WH = 32 / WW, WX = TW / WW; // warp tile and warps per row
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        const int px = int(blockIdx.x) * TW + (w % WX) * WW + (l % WW);
        const int py = int(blockIdx.y) * TH + (w / WX) * WH + (l / WW);
        unsigned long long n = 0;
        if(px < p.v.W && py < p.v.H)
        {
            const size_t o = pix(p, px, py);
            shade_pixel(p, px, py, o);
            if(VOLUME)
            {
                Ray ray = pixel_to_ray(p.v, p.g, px, py);
                if(clip_ray(ray, p.v, p.g))
                {
                    ray.endDepth = gmin(ray.endDepth, p.depth[o]);
                    if(!(ray.endDepth <= ray.startDepth))
                    {
                        const March m = march_setup(ray, p.g, p.v.scale, p.step);
                        const float factor = m.factor * p.totalWeightAll;
                        float4 color;
                        const VolTexRef tex{p.g, p.volQ, p.volFlag};
                        if(LINEAR && march_in_range(p.g, m))
                            color = skip ? march_combined<LINEAR, false, true, YFAST>(tex, m, factor, n)
                                         : march_combined<LINEAR, false, false, YFAST>(tex, m, factor, n);
                        else
                            color = skip ? march_combined<LINEAR, true, true, YFAST>(tex, m, factor, n)
                                         : march_combined<LINEAR, true, false, YFAST>(tex, m, factor, n);
                        const float4 solid = from_byte4(p.color[o]);
                        const float r = 1.0f - color.w;
                        color = make_float4(color.x + r * solid.x, color.y + r * solid.y, color.z + r * solid.z, color.w + r * solid.w);
                        p.color[o] = to_byte4(color);
                    }
                }
            }
        }
        if(VOLUME && p.counters)
            count_samples(p.counters, n);
    }

    template<bool FULL, bool YFAST>
    void launch_shade_volume_as(const FrameParams& p, bool volume, cudaStream_t s)
    {
        constexpr int TW = shade_tile_w(FULL, YFAST), TH = shade_tile_h(FULL, YFAST);
        const dim3 grid((p.v.W + TW - 1) / TW, (p.v.H + TH - 1) / TH);
        if(!volume)
            k_shade_volume<false, false, FULL, YFAST><<<grid, kShadeThreads, 0, s>>>(p);
        else if(p.interpolation)
            k_shade_volume<true, true, FULL, YFAST><<<grid, kShadeThreads, 0, s>>>(p);
        else
            k_shade_volume<true, false, FULL, YFAST><<<grid, kShadeThreads, 0, s>>>(p);
    }

    // launches of fewer than this many waves of the uncapped form take the FULL form
    constexpr int kShadeShortWaves = 4;

    void launch_shade_volume(const FrameParams& p, bool volume, cudaStream_t s)
    {
        const long long blocks = (long long) ((p.v.W + shade_tile_w(false) - 1) / shade_tile_w(false))
            * ((p.v.H + shade_tile_h(false) - 1) / shade_tile_h(false));
        // resident blocks of the uncapped form on the whole device, once per device (a
        // property of the kernel and the device, valid in any context on it)
        static int resident[64] = {0};
        int dev = 0;
        cudaGetDevice(&dev);
        if(dev >= 0 && dev < 64 && resident[dev] == 0)
        {
            int sms = 0, perSm = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_shade_volume<true, true, false, false>, kShadeThreads, 0);
            resident[dev] = std::max(1, sms * perSm);
        }
        const long long waves = blocks / std::max(1, dev >= 0 && dev < 64 ? resident[dev] : 1);
        const bool full = volume && waves < kShadeShortWaves;
        if(p.g.yfast)
            full ? launch_shade_volume_as<true, true>(p, volume, s) : launch_shade_volume_as<false, true>(p, volume, s);
        else
            full ? launch_shade_volume_as<true, false>(p, volume, s) : launch_shade_volume_as<false, false>(p, volume, s);
    }
} // namespace isaacb
