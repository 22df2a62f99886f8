// The combined-texture ray-march shared by the single-view and the batched
// kernels.  Included by the kernel translation units only.
#pragma once

#include "isaacb_internal.h"

namespace isaacb
{
    // the texture a march reads: geometry, quad bricks and per-brick emptiness
    struct VolTexRef
    {
        Geom g;
        const uint4* volQ;
        const uint8_t* volFlag;
    };

    // the trilinear sample of channel-major slots A (plane z0) and B (plane z0 + 1) at the
    // fractional position (fx, fy, fz), in units of 1/65535 byte: an exact integer sum of
    // 16-bit fixed-point weights times bytes
    __device__ __forceinline__ float4 trilinear_dp2a(uint4 A, uint4 B, float fx, float fy, float fz)
    {
        constexpr float kUnit = 65535.0f;
        const float gx = 1.0f - fx, gy = 1.0f - fy;
        const float fzU = fz * kUnit, gzU = kUnit - fzU;
        // the xy weights of a texel row as packed pairs (texel x0, texel x0 + 1):
        // (w00, w10) = (gx, fx) * gy and (w01, w11) = (gx, fx) * fy
        const f2p X = f2p_make(gx, fx);
        const f2p R0 = f2p_mul(X, f2p_make(gy, gy)), R1 = f2p_mul(X, f2p_make(fy, fy));
        // round(w * 65535) lands in the low bits of 2^23 + w * 65535 (one rounding per lane,
        // to nearest, as the scalar fmaf); <= 65535, so the low 16 bits are the weight
        const f2p M = f2p_make(8388608.0f, 8388608.0f), GZ = f2p_make(gzU, gzU), FZ = f2p_make(fzU, fzU);
        auto pack = [](f2p q) {
            float lo, hi;
            f2p_split(q, lo, hi);
            return __byte_perm(__float_as_uint(lo), __float_as_uint(hi), 0x5410u);
        };
        // weight pairs (texel (x0,y) | texel (x0+1,y) << 16) for rows y0 and y0+1 of each plane
        const uint32_t W0a = pack(f2p_fma(R0, GZ, M));
        const uint32_t W1a = pack(f2p_fma(R1, GZ, M));
        const uint32_t W0b = pack(f2p_fma(R0, FZ, M));
        const uint32_t W1b = pack(f2p_fma(R1, FZ, M));
        // Σ weights <= 65535 + 4, so every channel sum is an exact integer below 2^24
        auto tri = [&](uint32_t a, uint32_t b) {
            return __uint2float_rn(dp2a_hi(W1b, b, dp2a_lo(W0b, b, dp2a_hi(W1a, a, dp2a_lo(W0a, a, 0u)))));
        };
        return make_float4(tri(A.x, B.x), tri(A.y, B.y), tri(A.z, B.z), tri(A.w, B.w));
    }

    // Front-to-back march of CombinedVolumeRenderKernel (lib/isaac/isaac_volume_kernel.hpp:61-87)
    // at the reference's sample positions.  Differences from the exact form, all far
    // below one output LSB and covered by the parity tests:
    //  * pos - 0.5 is one fmaf per axis and the /255 normalisation is folded into the
    //    per-ray factor;
    //  * the trilinear is an integer dot product: the 8 FP32 weights are rounded to
    //    16-bit fixed point (w * 65535), and each channel-major slot word (channel c of
    //    the 2x2 texels of one plane) is weighed whole by dp2a.lo + dp2a.hi.  The sums
    //    are exact integers below 2^24, so the only error is the weights' rounding,
    //    at most 8 * 0.5 / 65535 * 255 = 0.016 byte units per sample;
    //  * empty-space skipping: a brick whose texels (apron included) are all zero
    //    yields exactly zero samples, so the samples inside it are counted but not
    //    evaluated -- adding zero leaves the colour unchanged.
    // CLAMP keeps every coordinate inside the volume; a LINEAR ray whose first and
    // last sample lie strictly inside needs no per-sample clamp (positions are affine
    // in the step index, rounding is far below the 1e-3 margin).
    // YFAST: the texture's slots are y fastest (Geom::yfast), else x fastest.
    template<bool LINEAR, bool CLAMP, bool SKIP, bool YFAST = false>
    __device__ __forceinline__ float4 march_combined(
        const VolTexRef& p,
        const March& m,
        float factor,
        unsigned long long& count)
    {
        const Geom& g = p.g;
        const float k = factor / 255.0f;
        // trilinear samples come out scaled by the weights' fixed-point unit 65535
        constexpr float kUnit = 65535.0f;
        const float kS = LINEAR ? k / kUnit : k;
        const float off = LINEAR ? 0.5f : 0.0f;
        const float c0x = m.startU.x - off, c0y = m.startU.y - off, c0z = m.startU.z - off;
        const float svx = m.stepVec.x, svy = m.stepVec.y, svz = m.stepVec.z;
        const float lo = LINEAR ? -1.0f : 0.0f;
        const float hx = float(g.ls[0] - 1), hy = float(g.ls[1] - 1), hz = float(g.ls[2] - 1);
        const int nb0 = g.nb[0], nb1 = g.nb[1];
        // the slot of apron-shifted coordinates as a sum over the axes: with b = a >> 3 and
        // l = a & 7 per axis, b * stride + l * step == a * step + b * (stride - 8 * step);
        // the in-brick steps of x and y are (1, 8), or (8, 1) for y-fastest slots
        constexpr uint32_t stepX = YFAST ? 8u : 1u, stepY = YFAST ? 1u : 8u;
        const uint32_t sy = uint32_t(nb0) * uint32_t(kSlotsPerBrick) - 8u * stepY;
        const uint32_t sz = uint32_t(nb1) * uint32_t(nb0) * uint32_t(kSlotsPerBrick) - 512u;
        // floor(c) + 1 (the apron-shifted coordinate) straight from the magic-number add
        const int magic = 0x4B400000 - 1;
        float4 color = make_float4(0, 0, 0, 0);
        int curBrick = -1;
        bool empty = false;
        const float fs = float(m.startSteps), fe = float(m.endSteps);
        float fi = fs;
        while(fi <= fe)
        {
            float cx = fmaf(svx, fi, c0x), cy = fmaf(svy, fi, c0y), cz = fmaf(svz, fi, c0z);
            if(CLAMP)
            {
                cx = fminf(fmaxf(cx, lo), hx);
                cy = fminf(fmaxf(cy, lo), hy);
                cz = fminf(fmaxf(cz, lo), hz);
            }
            const float tx = __fadd_rd(cx, 12582912.0f), ty = __fadd_rd(cy, 12582912.0f),
                        tz = __fadd_rd(cz, 12582912.0f);
            const int ax = __float_as_int(tx) - magic, ay = __float_as_int(ty) - magic, az = __float_as_int(tz) - magic;
            const int brick = SKIP ? ((az >> 3) * nb1 + (ay >> 3)) * nb0 + (ax >> 3) : 0;
            if(SKIP && brick != curBrick)
            {
                curBrick = brick;
                empty = __ldg(p.volFlag + brick) == 0;
            }
            if(SKIP && empty)
            {
                // last step index whose position stays inside this brick's sample region
                // [8b-1, 8b+7) per axis, with a 1e-3-step margin against rounding
                float tEnd = 3.0e38f;
                const float bl[3] = {float(ax & ~7) - 1.0f, float(ay & ~7) - 1.0f, float(az & ~7) - 1.0f};
                const float sv[3] = {svx, svy, svz};
                const float c0[3] = {c0x, c0y, c0z};
#pragma unroll
                for(int a = 0; a < 3; ++a)
                {
                    if(sv[a] > 0.0f)
                        tEnd = fminf(tEnd, (bl[a] + 8.0f - c0[a]) / sv[a]);
                    else if(sv[a] < 0.0f)
                        tEnd = fminf(tEnd, (bl[a] - c0[a]) / sv[a]);
                }
                // margin: 1e-3 steps plus the float rounding of tEnd itself
                const float last = fminf(fmaxf(floorf(tEnd - (1.0e-3f + 1.0e-6f * fabsf(tEnd))), fi), fe);
                fi = last + 1.0f;
                continue;
            }
            const uint32_t slot = stepX * uint32_t(ax) + (576u - 8u * stepX) * uint32_t(ax >> 3) + stepY * uint32_t(ay)
                + sy * uint32_t(ay >> 3) + 64u * uint32_t(az) + sz * uint32_t(az >> 3);
            float r0, r1, r2, r3;
            if(LINEAR)
            {
                // channel-major slots: A.c / B.c = channel c of the 2x2 texels of planes z0 / z0+1
                const uint4 A = __ldg(p.volQ + slot);
                const uint4 B = __ldg(p.volQ + slot + 64);
                const float4 r = trilinear_dp2a(A, B, cx - (tx - 12582912.0f), cy - (ty - 12582912.0f), cz - (tz - 12582912.0f));
                r0 = r.x, r1 = r.y, r2 = r.z, r3 = r.w;
            }
            else
            {
                // texel (x0, y0) of the slot: byte 0 of each channel word
                const uint4 Q = __ldg(p.volQ + slot);
                r0 = ubyte_f(Q.x, 0), r1 = ubyte_f(Q.y, 0), r2 = ubyte_f(Q.z, 0), r3 = ubyte_f(Q.w, 0);
            }
            const float s = (1.0f - color.w) * kS;
            color.x = fmaf(s, r0, color.x);
            color.y = fmaf(s, r1, color.y);
            color.z = fmaf(s, r2, color.z);
            color.w = fmaf(s, r3, color.w);
            fi += 1.0f;
            if(color.w > 0.99f)
                break;
        }
        count += (unsigned long long) (fminf(fi, fe + 1.0f) - fs);
        return color;
    }

    // a LINEAR ray needs no clamp if both end samples are inside [-1, L) by a margin
    __device__ __forceinline__ bool march_in_range(const Geom& g, const March& m)
    {
        const float fs = float(m.startSteps), fe = float(m.endSteps);
        const float c0[3] = {m.startU.x - 0.5f, m.startU.y - 0.5f, m.startU.z - 0.5f};
        const float sv[3] = {m.stepVec.x, m.stepVec.y, m.stepVec.z};
        bool ok = true;
#pragma unroll
        for(int a = 0; a < 3; ++a)
        {
            const float a0 = fmaf(sv[a], fs, c0[a]), a1 = fmaf(sv[a], fe, c0[a]);
            ok = ok && fminf(a0, a1) >= -0.999f && fmaxf(a0, a1) <= float(g.ls[a]) - 0.001f;
        }
        return ok;
    }

} // namespace isaacb
