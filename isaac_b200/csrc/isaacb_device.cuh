// Device-side building blocks of the B200 ISAAC hot path: parameter structs,
// glm-semantics float helpers, the functor-chain interpreter, ray setup and
// the brick samplers.
//
// Exactness: every translation unit that includes this header is compiled with
// --fmad=false, so plain float expressions round exactly like the reference's
// CPU backend (no fused multiply-add).  Where a kernel trades that exactness
// for speed it calls fmaf() explicitly and says so.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace isaacb
{
    constexpr int kMaxSources = 16;
    constexpr int kMaxFunctors = 3;
    constexpr int kMaxClip = 16;
    constexpr int kMaxAoSamples = 32; // taps of the configurable SSAO pattern
    // Quad-packed apron brick: 8x8 (x,y) slots x 9 z-planes.  Slot (lx,ly,lz) of
    // brick (bx,by,bz) holds the four texels (x0,y0),(x0+1,y0),(x0,y0+1),(x0+1,y0+1)
    // of plane z, with x0 = 8bx-1+lx, y0 = 8by-1+ly, z = 8bz-1+lz, each clamped to
    // the volume.  A trilinear footprint whose base texel is (x0,y0,z0) is the two
    // slots (lx,ly,lz) and (lx,ly,lz+1) of one brick.  The combined RGBA8 texture
    // stores a slot channel-major (quad_channel_major), the iso alpha texture one
    // byte per texel in the same order.  Inside a brick the slots are stored x fastest
    // or y fastest, as the merge chose for its camera (Geom::yfast, slot_in_brick).
    constexpr int kSlotsPerBrick = 576;
    constexpr int kApron = 9;

    enum Op : int32_t
    {
        OP_IDEM = 0,
        OP_ADD = 1,
        OP_MUL = 2,
        OP_LENGTH = 3,
        OP_POW = 4,
        OP_SUM = 5
    };

    struct Chain
    {
        int32_t op[kMaxFunctors];
        float p[4 * kMaxFunctors];
    };

    // SimulationSizeStruct (lib/isaac/isaac_types.hpp:119-131) with the integer
    // values the reference stores in size_t / int vectors.
    struct Geom
    {
        int32_t gs[3], ls[3], lps[3], pos[3], gss[3], lss[3], posS[3];
        int32_t maxGss;
        int32_t nb[3]; // bricks per axis = (ls >> 3) + 1
        // slot order of the combined textures' bricks, set by the merge that wrote them:
        // 0 x fastest (slot lz * 64 + ly * 8 + lx), 1 y fastest (lz * 64 + lx * 8 + ly)
        int32_t yfast;
    };

    __host__ __device__ inline int32_t bricks_per_axis(int32_t l)
    {
        return (l >> 3) + 1;
    }

    // ------------------------------------------------------------- glm semantics
    __device__ __forceinline__ float gmin(float a, float b)
    {
        return (b < a) ? b : a;
    }
    __device__ __forceinline__ float gmax(float a, float b)
    {
        return (a < b) ? b : a;
    }
    __device__ __forceinline__ float gclamp(float x, float lo, float hi)
    {
        return gmin(gmax(x, lo), hi);
    }
    __device__ __forceinline__ float gsign(float x)
    {
        return float((0.0f < x) ? 1 : 0) - float((x < 0.0f) ? 1 : 0);
    }
    __device__ __forceinline__ float gfract(float x)
    {
        return x - floorf(x);
    }
    __device__ __forceinline__ int iclamp(int x, int lo, int hi)
    {
        return min(max(x, lo), hi);
    }
    // float -> int conversion of the GPU (saturating, NaN -> 0)
    __device__ __forceinline__ int f2i(float x)
    {
        return __float2int_rz(x);
    }

    __device__ __forceinline__ float3 f3(float x, float y, float z)
    {
        return make_float3(x, y, z);
    }
    __device__ __forceinline__ float3 add3(float3 a, float3 b)
    {
        return f3(a.x + b.x, a.y + b.y, a.z + b.z);
    }
    __device__ __forceinline__ float3 sub3(float3 a, float3 b)
    {
        return f3(a.x - b.x, a.y - b.y, a.z - b.z);
    }
    __device__ __forceinline__ float3 mul3(float3 a, float3 b)
    {
        return f3(a.x * b.x, a.y * b.y, a.z * b.z);
    }
    __device__ __forceinline__ float3 muls3(float3 a, float s)
    {
        return f3(a.x * s, a.y * s, a.z * s);
    }
    __device__ __forceinline__ float3 smul3(float s, float3 a)
    {
        return f3(s * a.x, s * a.y, s * a.z);
    }
    __device__ __forceinline__ float3 div3(float3 a, float3 b)
    {
        return f3(a.x / b.x, a.y / b.y, a.z / b.z);
    }
    __device__ __forceinline__ float3 divs3(float3 a, float s)
    {
        return f3(a.x / s, a.y / s, a.z / s);
    }
    __device__ __forceinline__ float3 neg3(float3 a)
    {
        return f3(-a.x, -a.y, -a.z);
    }
    __device__ __forceinline__ float dot3(float3 a, float3 b)
    {
        float tx = a.x * b.x, ty = a.y * b.y, tz = a.z * b.z;
        return (tx + ty) + tz;
    }
    __device__ __forceinline__ float length3(float3 a)
    {
        return sqrtf(dot3(a, a));
    }
    __device__ __forceinline__ float3 normalize3(float3 a)
    {
        float inv = 1.0f / sqrtf(dot3(a, a));
        return muls3(a, inv);
    }
    __device__ __forceinline__ float comp(float3 v, int i)
    {
        return i == 0 ? v.x : (i == 1 ? v.y : v.z);
    }

    // transformColor (lib/isaac/isaac_helper.hpp:71-79)
    __device__ __forceinline__ uint32_t byte_of(float v)
    {
        return (uint32_t) min(max(f2i(gclamp(v, 0.0f, 1.0f) * 255.0f), 0), 255);
    }
    __device__ __forceinline__ uchar4 to_byte4(float4 c)
    {
        return make_uchar4(byte_of(c.x), byte_of(c.y), byte_of(c.z), byte_of(c.w));
    }
    __device__ __forceinline__ float4 from_byte4(uchar4 b)
    {
        return make_float4(float(b.x) / 255.0f, float(b.y) / 255.0f, float(b.z) / 255.0f, float(b.w) / 255.0f);
    }

    // ------------------------------------------------------------- functor chain
    // generateFunctorChain (lib/isaac/isaac_functor_chain.hpp:95-108) as a
    // register interpreter over the bytecode the host parser produced; the
    // reference dispatches the same chain through a device function-pointer table.
    __device__ __forceinline__ float dotN(const float (&v)[4], int n)
    {
        if(n == 1)
            return v[0] * v[0];
        if(n == 2)
        {
            float a = v[0] * v[0], b = v[1] * v[1];
            return a + b;
        }
        if(n == 3)
        {
            float a = v[0] * v[0], b = v[1] * v[1], c = v[2] * v[2];
            return (a + b) + c;
        }
        float a = v[0] * v[0], b = v[1] * v[1], c = v[2] * v[2], d = v[3] * v[3];
        return (a + b) + (c + d);
    }

    __device__ __forceinline__ float apply_chain(float (&v)[4], int dim, const Chain& ch)
    {
        int n = dim;
#pragma unroll
        for(int k = 0; k < kMaxFunctors; ++k)
        {
            const int op = ch.op[k];
            if(op == OP_ADD)
            {
#pragma unroll
                for(int i = 0; i < 4; ++i)
                    if(i < n)
                        v[i] = v[i] + ch.p[4 * k + i];
            }
            else if(op == OP_MUL)
            {
#pragma unroll
                for(int i = 0; i < 4; ++i)
                    if(i < n)
                        v[i] = v[i] * ch.p[4 * k + i];
            }
            else if(op == OP_LENGTH)
            {
                v[0] = sqrtf(dotN(v, n));
                n = 1;
            }
            else if(op == OP_POW)
            {
#pragma unroll
                for(int i = 0; i < 4; ++i)
                    if(i < n)
                        v[i] = powf(v[i], ch.p[4 * k + i]);
            }
            else if(op == OP_SUM)
            {
                float r = 0.0f;
#pragma unroll
                for(int i = 0; i < 4; ++i)
                    if(i < n)
                        r += v[i];
                v[0] = r;
                n = 1;
            }
        }
        return v[0];
    }

    // transfer-function index round(v*TS) clamped to [0,TS-1], NaN -> 0
    // (lib/isaac/isaac_common_kernel.hpp:589-591)
    __device__ __forceinline__ int lut_index(float v, int ts)
    {
        float c = gclamp(roundf(v * float(ts)), 0.0f, float(ts - 1));
        return f2i(c);
    }

    // ------------------------------------------------------------- ray setup
    struct Ray
    {
        float3 dir, start;
        float startDepth, endDepth;
        bool isClipped;
        float3 clippingNormal;
    };

    struct View
    {
        float inv[16]; // inverse(P*MV), column major
        int32_t W, H;
        float3 scale;
        int32_t clipCount;
        float clipPos[kMaxClip][3];
        float clipNrm[kMaxClip][3];
    };

    // pixelToRay (lib/isaac/isaac_common_kernel.hpp:51-92)
    __device__ __forceinline__ Ray pixel_to_ray(const View& v, const Geom& g, int px, int py)
    {
        float vx = float(px) / float(v.W) * 2.0f - 1.0f;
        float vy = float(py) / float(v.H) * 2.0f - 1.0f;
        float s4[4], e4[4];
#pragma unroll
        for(int i = 0; i < 4; ++i)
        {
            float m0 = v.inv[0 * 4 + i] * vx;
            float m1 = v.inv[1 * 4 + i] * vy;
            float a0 = m0 + m1;
            float ms = v.inv[2 * 4 + i] * -1.0f;
            float me = v.inv[2 * 4 + i] * 1.0f;
            float m3 = v.inv[3 * 4 + i] * 1.0f;
            s4[i] = a0 + (ms + m3);
            e4[i] = a0 + (me + m3);
        }
        Ray r;
        float3 start = f3(s4[0] / s4[3], s4[1] / s4[3], s4[2] / s4[3]);
        float3 end = f3(e4[0] / e4[3], e4[1] / e4[3], e4[2] / e4[3]);
        float maxSize = float(g.maxGss) * 0.5f;
        start = muls3(start, maxSize);
        end = muls3(end, maxSize);
        r.start = start;
        r.dir = normalize3(sub3(end, start));
        r.isClipped = false;
        r.clippingNormal = f3(0, 0, 0);
        r.startDepth = r.endDepth = 0.0f;
        return r;
    }

    // clipRay (lib/isaac/isaac_common_kernel.hpp:94-193)
    __device__ __forceinline__ bool clip_ray(Ray& ray, const View& v, const Geom& g)
    {
        float off[3];
#pragma unroll
        for(int i = 0; i < 3; ++i)
            off[i] = float(g.gss[i] / 2 - g.posS[i]);
        ray.start = add3(ray.start, f3(off[0], off[1], off[2]));
        float bbMin[3], bbMax[3];
        float st[3] = {ray.start.x, ray.start.y, ray.start.z};
        float dr[3] = {ray.dir.x, ray.dir.y, ray.dir.z};
#pragma unroll
        for(int i = 0; i < 3; ++i)
        {
            int mnl = max(0, -g.posS[i]);
            int mxl = min(g.lss[i], g.gss[i] - g.posS[i]);
            float a = (float(mnl) - st[i]) / dr[i];
            float b = (float(mxl) - st[i]) / dr[i];
            if(b < a)
            {
                float t = a;
                a = b;
                b = t;
            }
            bbMin[i] = a;
            bbMax[i] = b;
        }
        ray.startDepth = gmax(bbMin[0], gmax(bbMin[1], bbMin[2]));
        ray.endDepth = gmin(bbMax[0], gmin(bbMax[1], bbMax[2]));
        float cn[3] = {0, 0, 0};
#pragma unroll
        for(int i = 0; i < 3; ++i)
        {
            float sign = gsign(dr[i]);
            bool outerLow = g.pos[i] == 0 && (sign + 1.0f) != 0.0f;
            bool outerHigh = g.pos[i] + g.ls[i] == g.gs[i] && (sign - 1.0f) != 0.0f;
            if(bbMin[i] == ray.startDepth && (outerLow || outerHigh))
            {
                ray.isClipped = true;
                cn[i] = sign;
            }
        }
        ray.clippingNormal = f3(cn[0], cn[1], cn[2]);
        for(int i = 0; i < v.clipCount; ++i)
        {
            float3 n = f3(v.clipNrm[i][0], v.clipNrm[i][1], v.clipNrm[i][2]);
            float3 p = f3(
                v.clipPos[i][0] * float(g.gss[0]) * 0.5f + off[0],
                v.clipPos[i][1] * float(g.gss[1]) * 0.5f + off[1],
                v.clipPos[i][2] * float(g.gss[2]) * 0.5f + off[2]);
            float d = dot3(ray.dir, n);
            float depth = (dot3(p, n) - dot3(ray.start, n)) / d;
            if(d > 0.0f)
            {
                if(ray.endDepth < depth)
                    return false;
                if(ray.startDepth <= depth)
                {
                    ray.clippingNormal = n;
                    ray.isClipped = true;
                    ray.startDepth = depth;
                }
            }
            else
            {
                if(ray.startDepth > depth)
                    return false;
                if(ray.endDepth > depth)
                    ray.endDepth = depth;
            }
        }
        ray.startDepth = gmax(ray.startDepth, 0.002f);
        if(ray.startDepth > ray.endDepth || isinf(ray.startDepth) || isinf(ray.endDepth))
            return false;
        return true;
    }

    // ray-march preamble shared by the volume and iso kernels
    // (lib/isaac/isaac_volume_kernel.hpp:56-65)
    struct March
    {
        float stepU, factor;
        int startSteps, endSteps;
        float3 stepVec, startU;
    };
    __device__ __forceinline__ March march_setup(const Ray& ray, const Geom& g, float3 scale, float step)
    {
        March m;
        float minSize = float(min(g.gs[0], min(g.gs[1], g.gs[2])));
        m.stepU = step * (length3(ray.dir) / length3(div3(ray.dir, scale)));
        m.factor = m.stepU / minSize * 2.0f;
        m.startSteps = f2i(ceilf(ray.startDepth / m.stepU));
        m.endSteps = f2i(floorf(ray.endDepth / m.stepU));
        m.stepVec = div3(smul3(m.stepU, ray.dir), scale);
        m.startU = div3(ray.start, scale);
        return m;
    }
    __device__ __forceinline__ float3 march_pos(const March& m, int i)
    {
        return add3(m.startU, muls3(m.stepVec, float(i)));
    }

    // ------------------------------------------------------------- brick addressing
    // slot of apron-shifted coordinates (ax, ay, az) inside their brick, in the texture's order
    __device__ __forceinline__ uint32_t slot_in_brick(const Geom& g, int ax, int ay, int az)
    {
        const uint32_t xy = g.yfast ? uint32_t((ax & 7) * 8 + (ay & 7)) : uint32_t((ay & 7) * 8 + (ax & 7));
        return uint32_t(az & 7) * 64u + xy;
    }
    __device__ __forceinline__ size_t brick_slot(const Geom& g, int x0, int y0, int z0)
    {
        // x0 in [-1, L-1]: base texel of a trilinear footprint
        int ax = x0 + 1, ay = y0 + 1, az = z0 + 1;
        size_t brick = (size_t(az >> 3) * g.nb[1] + size_t(ay >> 3)) * g.nb[0] + size_t(ax >> 3);
        return brick * kSlotsPerBrick + size_t(slot_in_brick(g, ax, ay, az));
    }

    // Per-source bricks order their slots along a Morton curve: slot (lx, ly, lz) of a
    // brick is the bit interleave of lx, ly, lz (bits x0 y0 z0 x1 y1 z1 x2 y2 z2) for the
    // 8 layers of its own voxels, and 512 + ly * 8 + lx in the apron layer lz = 8.  The
    // rays of a warp sample a small patch of voxels that faces the camera; in x-fastest
    // order a patch facing the x axis spans 64- and 512-byte strides, in Morton order
    // every 2x2x2 block is contiguous whatever the view direction.
    __device__ __forceinline__ uint32_t spread3(int v)
    {
        // 3-bit v -> bits 0, 3, 6: byte v of the table 0x49 48 41 40 09 08 01 00
        return __byte_perm(0x09080100u, 0x49484140u, uint32_t(v));
    }
    __device__ __forceinline__ uint32_t morton_slot(int lx, int ly, int lz)
    {
        return lz < 8 ? (spread3(lx) | (spread3(ly) << 1) | (spread3(lz) << 2)) : uint32_t(512 + ly * 8 + lx);
    }
    // the slot of the trilinear footprint based at (x0, y0, z0) in [-1, L-1] in the
    // per-source bricks, and in `above` the slot of the layer z0 + 1
    __device__ __forceinline__ size_t source_slot(const Geom& g, int x0, int y0, int z0, size_t& above)
    {
        const int ax = x0 + 1, ay = y0 + 1, az = z0 + 1;
        const size_t base = ((size_t(az >> 3) * g.nb[1] + size_t(ay >> 3)) * g.nb[0] + size_t(ax >> 3)) * kSlotsPerBrick;
        const int lx = ax & 7, ly = ay & 7, lz = az & 7;
        const uint32_t xy = spread3(lx) | (spread3(ly) << 1);
        above = base + (lz < 7 ? (xy | (spread3(lz + 1) << 2)) : uint32_t(512 + ly * 8 + lx));
        return base + (xy | (spread3(lz) << 2));
    }

    __device__ __forceinline__ float byte_f(uint32_t w, int c)
    {
        return float((w >> (8 * c)) & 0xffu);
    }

    // linear(o, a, b) = a*(1-o) + b*o (lib/isaac/isaac_helper.hpp:124-128)
    __device__ __forceinline__ float lin(float o, float a, float b)
    {
        return a * (1.0f - o) + b * o;
    }

    // trilinear over the 8 texels of a footprint, z first then y then x
    // (lib/isaac/isaac_helper.hpp:138-144).  q0 = plane z0, q1 = plane z0+1;
    // each .x/.y/.z/.w = (x0,y0),(x0+1,y0),(x0,y0+1),(x0+1,y0+1).
    __device__ __forceinline__ float tri_q(float fx, float fy, float fz, float d000, float d100, float d010, float d110,
                                           float d001, float d101, float d011, float d111)
    {
        float A = lin(fy, lin(fz, d000, d001), lin(fz, d010, d011));
        float B = lin(fy, lin(fz, d100, d101), lin(fz, d110, d111));
        return lin(fx, A, B);
    }

    // alpha channel of the combined iso texture (alpha quads, 4 bytes per slot)
    __device__ __forceinline__ float sample_alpha(const uint32_t* __restrict__ q, const Geom& g, float3 pos, bool linear)
    {
        if(linear)
        {
            float cx = pos.x - 0.5f, cy = pos.y - 0.5f, cz = pos.z - 0.5f;
            float flx = floorf(cx), fly = floorf(cy), flz = floorf(cz);
            float fx = cx - flx, fy = cy - fly, fz = cz - flz;
            int ix = iclamp(f2i(flx), -1, g.ls[0] - 1);
            int iy = iclamp(f2i(fly), -1, g.ls[1] - 1);
            int iz = iclamp(f2i(flz), -1, g.ls[2] - 1);
            size_t s = brick_slot(g, ix, iy, iz);
            uint32_t a = __ldg(q + s);
            uint32_t b = __ldg(q + s + 64);
            float r = tri_q(
                fx,
                fy,
                fz,
                byte_f(a, 0),
                byte_f(a, 1),
                byte_f(a, 2),
                byte_f(a, 3),
                byte_f(b, 0),
                byte_f(b, 1),
                byte_f(b, 2),
                byte_f(b, 3));
            return r / 255.0f;
        }
        int ix = iclamp(f2i(pos.x), 0, g.ls[0] - 1);
        int iy = iclamp(f2i(pos.y), 0, g.ls[1] - 1);
        int iz = iclamp(f2i(pos.z), 0, g.ls[2] - 1);
        uint32_t w = __ldg(q + brick_slot(g, ix, iy, iz));
        return byte_f(w, 0) / 255.0f;
    }

    // full RGBA8 sample of a linear (x fastest) texture, exact arithmetic
    __device__ __forceinline__ float4 sample_linear_rgba8(
        const uint32_t* __restrict__ t,
        const Geom& g,
        float3 pos,
        bool linear)
    {
        const int LX = g.ls[0], LY = g.ls[1], LZ = g.ls[2];
        auto tex = [&](int x, int y, int z) -> uint32_t {
            x = iclamp(x, 0, LX - 1);
            y = iclamp(y, 0, LY - 1);
            z = iclamp(z, 0, LZ - 1);
            return __ldg(t + (size_t(z) * LY + y) * LX + x);
        };
        if(linear)
        {
            float cx = pos.x - 0.5f, cy = pos.y - 0.5f, cz = pos.z - 0.5f;
            float flx = floorf(cx), fly = floorf(cy), flz = floorf(cz);
            float fx = cx - flx, fy = cy - fly, fz = cz - flz;
            int ix = f2i(flx), iy = f2i(fly), iz = f2i(flz);
            uint32_t d000 = tex(ix, iy, iz), d100 = tex(ix + 1, iy, iz), d010 = tex(ix, iy + 1, iz),
                     d110 = tex(ix + 1, iy + 1, iz);
            uint32_t d001 = tex(ix, iy, iz + 1), d101 = tex(ix + 1, iy, iz + 1), d011 = tex(ix, iy + 1, iz + 1),
                     d111 = tex(ix + 1, iy + 1, iz + 1);
            float r[4];
#pragma unroll
            for(int c = 0; c < 4; ++c)
                r[c] = tri_q(
                    fx,
                    fy,
                    fz,
                    byte_f(d000, c),
                    byte_f(d100, c),
                    byte_f(d010, c),
                    byte_f(d110, c),
                    byte_f(d001, c),
                    byte_f(d101, c),
                    byte_f(d011, c),
                    byte_f(d111, c));
            return make_float4(r[0] / 255.0f, r[1] / 255.0f, r[2] / 255.0f, r[3] / 255.0f);
        }
        uint32_t w = tex(f2i(pos.x), f2i(pos.y), f2i(pos.z));
        return make_float4(byte_f(w, 0) / 255.0f, byte_f(w, 1) / 255.0f, byte_f(w, 2) / 255.0f, byte_f(w, 3) / 255.0f);
    }

    // ------------------------------------------------------------- fast paths (FMA / ALU pipes only)
    // The ray-march is issue-bound; these helpers keep its per-sample work off the
    // XU pipe (conversions, rounding, reciprocal), which the exact forms above use.

    // byte c of w as a float, exactly: the bit pattern 0x4B0000bb is 2^23 + b
    __device__ __forceinline__ float ubyte_f(uint32_t w, int c)
    {
        return __int_as_float(int(__byte_perm(w, 0x4B000000u, 0x7440u + unsigned(c)))) - 8388608.0f;
    }

    // floor(x) as float and int for |x| < 2^22: adding 1.5*2^23 rounded toward -inf leaves
    // floor(x) in the low mantissa bits (exact)
    __device__ __forceinline__ void floor_split(float x, float& fl, int& ix)
    {
        const float t = __fadd_rd(x, 12582912.0f);
        fl = t - 12582912.0f;
        ix = __float_as_int(t) - 0x4B400000;
    }

    // trunc(x) as int for 0 <= x < 2^22 (exact): adding 2^23 rounded toward zero
    __device__ __forceinline__ int trunc_nonneg(float x, float& tr)
    {
        const float t = __fadd_rz(x, 8388608.0f);
        tr = t - 8388608.0f;
        return __float_as_int(t) - 0x4B000000;
    }

    // round half away from zero of x in [0, 2^22) (roundf for non-negative x), exact
    __device__ __forceinline__ int round_nonneg(float x)
    {
        float tr;
        const int t = trunc_nonneg(x, tr);
        return t + ((x - tr) >= 0.5f ? 1 : 0);
    }

    // lut_index with the same result for every input, NaN included, without the
    // conversion pipe: clamp first (NaN -> 0), then round half away from zero
    __device__ __forceinline__ int lut_index_fast(float v, int ts)
    {
        const float x = v * float(ts);
        const float xc = fminf(fmaxf(x, 0.0f), float(ts));
        return min(round_nonneg(xc), ts - 1);
    }

    // ------------------------------------------------------------- packed FP32 pairs (sm_100a f32x2)
    // Two FP32 lanes per instruction; each lane rounds exactly like the scalar op.
    struct f2p
    {
        unsigned long long v;
    };
    __device__ __forceinline__ f2p f2p_make(float lo, float hi)
    {
        f2p r;
        asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
        return r;
    }
    __device__ __forceinline__ void f2p_split(f2p a, float& lo, float& hi)
    {
        asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
    }
    __device__ __forceinline__ f2p f2p_fma(f2p a, f2p b, f2p c)
    {
        f2p r;
        asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
        return r;
    }
    // a * b rounded once per lane; only for a product that does not feed an add (the
    // assembler may contract mul.rn.f32x2 + add.rn.f32x2 into one fma, see f2p_mul_exact)
    __device__ __forceinline__ f2p f2p_mul(f2p a, f2p b)
    {
        f2p r;
        asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
        return r;
    }
    __device__ __forceinline__ f2p f2p_add(f2p a, f2p b)
    {
        f2p r;
        asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
        return r;
    }
    // a * b rounded once, for a product that feeds an add.  The assembler contracts
    // mul.rn.f32x2 followed by add.rn.f32x2 into one fma.rn.f32x2 (the explicit rounding
    // does not stop it for the packed forms, as it does for mul.rn.f32), which rounds
    // once instead of twice.  An fma whose addend is -0 is the rounded product for every
    // a and b (x + -0 = x, +0 included), and with the -0 taken from a kernel parameter the
    // assembler cannot turn it back into a multiply.
    __device__ __forceinline__ f2p f2p_mul_exact(f2p a, f2p b, f2p negZero)
    {
        return f2p_fma(a, b, negZero);
    }
    // byte c of w as the exact float b_c 2^-133: the byte in bits 16-23 and zeros
    // elsewhere, one byte permute and no add.  Below 128 the value is subnormal, from 128
    // on bit 23 is the exponent's lowest bit and the value is normal, and in both ranges
    // it equals b 2^-133; zero stays zero.  fma (no .ftz) takes subnormal operands as they
    // are; with weights scaled by 2^64 every product and sum is a normal number, each the
    // unscaled one times 2^-69.
    __device__ __forceinline__ float ubyte_tiny(uint32_t w, int c)
    {
        return __int_as_float(int(__byte_perm(w, 0u, 0x4044u + 256u * unsigned(c))));
    }

    // ------------------------------------------------------------- channel-major quad slots
    // A slot of the combined volume texture holds the 2x2 texels (x0,y0), (x0+1,y0),
    // (x0,y0+1), (x0+1,y0+1) of one z-plane channel by channel: word c of the slot
    // carries channel c of the four texels in bytes 0-3, in that order.  The march then
    // weighs a whole word with two integer dot products (dp2a.lo on bytes 0-1, dp2a.hi
    // on bytes 2-3) and never extracts a byte.

    // the slot of four RGBA8 texels t0..t3 (texel order above): a 4x4 byte transpose
    __device__ __forceinline__ uint4 quad_channel_major(uint32_t t0, uint32_t t1, uint32_t t2, uint32_t t3)
    {
        const uint32_t rg01 = __byte_perm(t0, t1, 0x5140u), ba01 = __byte_perm(t0, t1, 0x7362u);
        const uint32_t rg23 = __byte_perm(t2, t3, 0x5140u), ba23 = __byte_perm(t2, t3, 0x7362u);
        return make_uint4(__byte_perm(rg01, rg23, 0x5410u), __byte_perm(rg01, rg23, 0x7632u),
                          __byte_perm(ba01, ba23, 0x5410u), __byte_perm(ba01, ba23, 0x7632u));
    }
    // texel k (0..3) of a channel-major slot as an RGBA8 word
    __device__ __forceinline__ uint32_t quad_texel(uint4 q, int k)
    {
        const uint32_t sel = uint32_t(k) | (uint32_t(k) << 4);
        return __byte_perm(__byte_perm(q.x, q.y, 0x0040u + sel), __byte_perm(q.z, q.w, 0x0040u + sel), 0x5410u);
    }

    // d = c + a.lo16 * b.byte0 + a.hi16 * b.byte1 (unsigned, exact)
    __device__ __forceinline__ uint32_t dp2a_lo(uint32_t a, uint32_t b, uint32_t c)
    {
        uint32_t d;
        asm("dp2a.lo.u32.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
        return d;
    }
    // d = c + a.lo16 * b.byte2 + a.hi16 * b.byte3 (unsigned, exact)
    __device__ __forceinline__ uint32_t dp2a_hi(uint32_t a, uint32_t b, uint32_t c)
    {
        uint32_t d;
        asm("dp2a.hi.u32.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
        return d;
    }

    // pixel of a thread: a block of 256 threads covers 32x8 pixels and each warp an 8x4 tile
    __device__ __forceinline__ void thread_pixel(int& px, int& py)
    {
        int t = threadIdx.x;
        int w = t >> 5, l = t & 31;
        px = blockIdx.x * 32 + (w & 3) * 8 + (l & 7);
        py = blockIdx.y * 8 + (w >> 2) * 4 + (l >> 3);
    }
} // namespace isaacb
