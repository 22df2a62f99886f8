// Buffer update kernels: the merge of all volume sources into the combined
// RGBA8 volume / iso textures (MergeToCombinedTextureKernel,
// lib/isaac/isaac_common_kernel.hpp:553-759) and the per-source bricks of the
// per-source renderer (UpdatePersistendTextureKernel,
// lib/isaac/isaac_common_kernel.hpp:432-451).
//
// The merge runs in two passes: every voxel is evaluated once, in x-rows, into
// linear RGBA8 textures; then one CTA per row of quad-packed apron bricks gathers
// their texels (each brick's 8^3 voxels plus the apron on the low side, clamped at
// the volume border) and writes the bricks' slots as coalesced 16-byte stores.  The per-brick
// flags feed empty-space skipping.
#include "isaacb_blue_noise.h"
#include "isaacb_internal.h"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>

namespace isaacb
{
    // 4x4x4 ordered dither masks (lib/isaac/isaac_dither_kernel.hpp:22-40)
    __constant__ uint8_t c_dither1[64]
        = {17, 46, 55, 1,  57, 7,  38, 31, 9,  52, 2,  54, 36, 26, 19, 44, 53, 20, 47, 22, 29, 60,
           62, 12, 45, 14, 26, 33, 8,  39, 11, 63, 13, 56, 6,  50, 40, 32, 23, 48, 21, 42, 51, 5,
           61, 3,  34, 27, 41, 10, 30, 37, 4,  35, 15, 59, 49, 24, 43, 18, 25, 64, 58, 16};
    __constant__ uint8_t c_dither2[64]
        = {13, 61, 45, 51, 59, 39, 16, 40, 10, 49, 2,  46, 36, 43, 15, 60, 26, 52, 23, 9,  32, 6,
           31, 0,  54, 21, 58, 24, 17, 5,  28, 38, 56, 41, 11, 63, 14, 47, 37, 48, 42, 62, 12, 18,
           3,  35, 50, 44, 19, 1,  20, 34, 29, 25, 57, 4,  22, 8,  33, 53, 30, 55, 27, 7};

    // 8^3 and 16^3 blue-noise masks of dither modes 3 and >= 4 (lib/isaac/isaac_dither_kernel.hpp:42-310)
    __device__ const uint16_t g_blue8[512] = {ISAACB_BLUE_NOISE8_VALUES};
    __device__ const uint16_t g_blue16[4096] = {ISAACB_BLUE_NOISE16_VALUES};

    // the mode's threshold for voxel (x, y, z >= 0); mask: the 64-entry table of modes 1 and 2
    __device__ __forceinline__ float dither_threshold(int mode, const uint8_t* mask, int x, int y, int z)
    {
        if(mode == 1 || mode == 2)
            return float(mask[(x & 3) + (y & 3) * 4 + (z & 3) * 16]) / 64.0f;
        if(mode == 3)
            return float(__ldg(&g_blue8[(x & 7) + (y & 7) * 8 + (z & 7) * 64])) / 512.0f;
        return float(__ldg(&g_blue16[(x & 15) + (y & 15) * 16 + (z & 15) * 256])) / 4096.0f;
    }

    // applyDither3D (lib/isaac/isaac_dither_kernel.hpp:7-329), every mode, bit-exact,
    // with truncation, floor and rounding done by exact magic-number adds on the FMA pipe
    __device__ __forceinline__ uint32_t round_byte(float v)
    {
        // round(clamp(v,0,1)*255); clamp maps NaN to 0 as the GPU conversion does
        return uint32_t(round_nonneg(fminf(fmaxf(v, 0.0f), 1.0f) * 255.0f));
    }

    // dither for colours known to be finite and >= 0 (every table entry and weight >= 0,
    // total weight > 0): int(s) = floor(s), so one magic-number floor serves both terms
    __device__ __forceinline__ uint32_t dither_rgba_nonneg(int mode, const uint8_t* mask, int x, int y, int z, float4 c)
    {
        const float v[4] = {c.x, c.y, c.z, c.w};
        uint32_t out = 0;
        if(mode == 0)
        {
#pragma unroll
            for(int i = 0; i < 4; ++i)
                out |= uint32_t(min(round_nonneg(fminf(v[i], 1.0f) * 255.0f), 255)) << (8 * i);
            return out;
        }
        const float d = dither_threshold(mode, mask, x, y, z);
#pragma unroll
        for(int i = 0; i < 4; ++i)
        {
            const float s = fminf(v[i] * 255.0f, 257.0f);
            float fl;
            int fi;
            floor_split(s, fl, fi);
            out |= uint32_t(min(fi + ((s - fl) > d ? 1 : 0), 255)) << (8 * i);
        }
        return out;
    }

    // mask: the mode's 64-entry table (shared memory copy), unused for mode 0
    __device__ __forceinline__ uint32_t dither_rgba(int mode, const uint8_t* mask, int x, int y, int z, float4 c)
    {
        float v[4] = {c.x, c.y, c.z, c.w};
        uint32_t out = 0;
        if(mode == 0)
        {
#pragma unroll
            for(int i = 0; i < 4; ++i)
            {
                // gclamp keeps the reference's NaN path (NaN -> byte 0)
                const float cl = gclamp(v[i], 0.0f, 1.0f);
                out |= (cl == cl ? uint32_t(round_nonneg(cl * 255.0f)) : 0u) << (8 * i);
            }
            return out;
        }
        const float d = dither_threshold(mode, mask, x, y, z); // x, y, z >= 0
#pragma unroll
        for(int i = 0; i < 4; ++i)
        {
            // int(s) + (fract(s) > d), clamped to [0,255]; s is clamped to [-2,257] first,
            // which changes no clamped result (NaN -> -2 -> 0, like the conversion's 0)
            const float s = fminf(fmaxf(v[i] * 255.0f, -2.0f), 257.0f);
            float tr;
            int ti = trunc_nonneg(fabsf(s), tr);
            if(s < 0.0f)
                ti = -ti;
            float fl;
            int fi;
            floor_split(s, fl, fi);
            int ci = ti + ((s - fl) > d ? 1 : 0);
            out |= uint32_t(min(max(ci, 0), 255)) << (8 * i);
        }
        return out;
    }

    __device__ __forceinline__ void read_voxel(const float* __restrict__ src, int fdim, size_t idx, float (&v)[4])
    {
        const float* p = src + idx * fdim;
        v[0] = __ldg(p);
        v[1] = fdim > 1 ? __ldg(p + 1) : 0.0f;
        v[2] = fdim > 2 ? __ldg(p + 2) : 0.0f;
        v[3] = fdim > 3 ? __ldg(p + 3) : 0.0f;
    }

    // ---------------------------------------------------------------- merge, pass 1: per voxel
    // One thread per voxel (rows of x, so every source read and texture write is
    // coalesced): the functor chain, the transfer lookup, the field alpha of advected
    // sources, the weighted sum and the dither, in the reference's source order.  The
    // results go to two linear RGBA8 textures, the volume (a scratch buffer) and the iso
    // texture (the iso output).

    // the weighted or iso sources of a merge, in source order
    struct MergeActive
    {
        int n;
        const float* src[kMaxSources];
        const float4* lut[kMaxSources];
        float weight[kMaxSources];
        float iso[kMaxSources];
        const float4* pre[kMaxSources]; // weighted premultiplied tables (k_merge_premultiply)
    };

    // the volume term of every table entry of the active sources, computed once per merge
    // instead of once per voxel: a = c.w * weight, (c.x * a, c.y * a, c.z * a, a) -- the
    // same float products merge_accumulate forms, so the sums that use them are unchanged
    __global__ void __launch_bounds__(256) k_merge_premultiply(const __grid_constant__ MergeActive act, float4* __restrict__ out, int ts)
    {
        const int k = blockIdx.y;
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if(i >= ts)
            return;
        const float4 c = __ldg(act.lut[k] + i);
        const float a = c.w * act.weight[k];
        out[size_t(k) * ts + i] = make_float4(c.x * a, c.y * a, c.z * a, a);
    }

    // the voxel's volume texel (weighted sum / total weight, dithered) and iso texel
    __device__ __forceinline__ uint32_t merge_volume_texel(const MergeParams& p, const uint8_t* mask, int x, int y, int z, float4 vc)
    {
        if(p.invTotalWeight != 0.0f)
        {
            // totalWeight is a power of two: x * 2^-k is the correctly rounded x / 2^k
            vc = make_float4(vc.x * p.invTotalWeight, vc.y * p.invTotalWeight, vc.z * p.invTotalWeight, vc.w * p.invTotalWeight);
        }
        else
            vc = make_float4(vc.x / p.totalWeight, vc.y / p.totalWeight, vc.z / p.totalWeight, vc.w / p.totalWeight);
        return p.nonNegative ? dither_rgba_nonneg(p.ditherMode, mask, x, y, z, vc) : dither_rgba(p.ditherMode, mask, x, y, z, vc);
    }
    __device__ __forceinline__ uint32_t merge_iso_texel(float4 ic)
    {
        return round_byte(ic.x) | (round_byte(ic.y) << 8) | (round_byte(ic.z) << 16) | (round_byte(ic.w) << 24);
    }

    template<bool ISO>
    __device__ __forceinline__ void merge_store(const MergeParams& p, const uint8_t* mask, size_t i, int x, int y, int z, float4 vc, float4 ic)
    {
        p.volLin[i] = merge_volume_texel(p, mask, x, y, z, vc);
        if(ISO)
            p.isoLin[i] = merge_iso_texel(ic);
    }

    __device__ __forceinline__ void merge_accumulate(float4 c, float vw, float it, bool iso, float4& vc, float4& ic)
    {
        if(vw > 0.0f)
        {
            const float a = c.w * vw;
            vc.x += c.x * a;
            vc.y += c.y * a;
            vc.z += c.z * a;
            vc.w += a;
        }
        if(iso && it > 0.0f)
        {
            const float a = c.w / it * 0.5f;
            if(ic.w < a)
                ic = make_float4(c.x, c.y, c.z, a);
        }
    }

    // NS (1..4) scalar sources whose chains are all idem, none advected: the sources'
    // pointers, tables and weights live in registers and all values load up front
    template<bool ISO, int NS>
    __global__ void __launch_bounds__(256) k_merge_voxels_n(const __grid_constant__ MergeParams p, const __grid_constant__ MergeActive act)
    {
        __shared__ uint8_t sMask[64];
        if(threadIdx.x < 64)
            sMask[threadIdx.x] = p.ditherMode == 2 ? c_dither2[threadIdx.x] : c_dither1[threadIdx.x];
        __syncthreads();
        const Geom& g = p.g;
        const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
        if(x >= g.ls[0])
            return;
        const size_t i = (size_t(z) * g.ls[1] + y) * g.ls[0] + x;
        float val[NS];
#pragma unroll
        for(int k = 0; k < NS; ++k)
            val[k] = __ldg(act.src[k] + i);
        float4 vc = make_float4(0, 0, 0, 0), ic = make_float4(0, 0, 0, 0);
#pragma unroll
        for(int k = 0; k < NS; ++k)
            merge_accumulate(__ldg(act.lut[k] + lut_index_fast(val[k], p.ts)), act.weight[k], act.iso[k], ISO, vc, ic);
        merge_store<ISO>(p, sMask, i, x, y, z, vc, ic);
    }

    // the largest float below 1: a threshold of exactly 1 behaves as this one below
    constexpr float kDitherMax = 0x1.fffffep-1f;

    // the non-negative dither with threshold d (already capped at kDitherMax):
    // floor(s) + (fract(s) > d) == ceil(s - d) for 0 <= d < 1 and s >= 0, and the
    // round-up subtraction keeps the ceiling exact; ceil by an exact magic-number add
    __device__ __forceinline__ uint32_t dither_rgba_ceil(float4 c, float d)
    {
        const float v[4] = {c.x, c.y, c.z, c.w};
        uint32_t out = 0;
#pragma unroll
        for(int i = 0; i < 4; ++i)
        {
            const float s = fminf(v[i] * 255.0f, 257.0f);
            const float t = __fadd_ru(__fsub_ru(s, d), 12582912.0f);
            out |= uint32_t(min(__float_as_int(t) - 0x4B400000, 255)) << (8 * i);
        }
        return out;
    }

    // Four x-adjacent voxels (the quad q of rows of rowQuads) of the scalar merge: one
    // 16-byte load per source and one 16-byte store per texture.  The transfer index is
    // round(clamp(v * ts, 0, ts - 1)) (the same as clamping the rounded value), with the
    // rounding as a round-down add of 0.5 and an exact magic-number floor; `entry(k, bits)`
    // returns source k's table entry for the floor's float bits (0x4B400000 + index).
    // Without iso output the tables are the premultiplied ones (k_merge_premultiply).
    template<bool ISO, int NS, class Entry>
    __device__ __forceinline__ void merge_quad(const MergeParams& p, const MergeActive& act, const uint8_t* sMask, uint32_t q, uint32_t rowQuads, Entry entry)
    {
        const Geom& g = p.g;
        const uint32_t row = q / rowQuads;
        const int x = int(q - row * rowQuads) * 4;
        const int y = int(row % uint32_t(g.ls[1])), z = int(row / uint32_t(g.ls[1]));
        float4 val[NS];
#pragma unroll
        for(int k = 0; k < NS; ++k)
            val[k] = __ldg(reinterpret_cast<const float4*>(act.src[k]) + q);
        const float tsf = float(p.ts), tsMax = float(p.ts - 1);
        // the four thresholds of modes 1 and 2: x is a multiple of 4, so they are the mask
        // bytes (y&3)*4 + (z&3)*16 + 0..3, one aligned word
        const bool fast = p.nonNegative && p.ditherMode != 0;
        const uint32_t maskWord = *reinterpret_cast<const uint32_t*>(sMask + (y & 3) * 4 + (z & 3) * 16);
        uint32_t vo[4], io[4];
#pragma unroll
        for(int j = 0; j < 4; ++j)
        {
            float4 vc = make_float4(0, 0, 0, 0), ic = make_float4(0, 0, 0, 0);
#pragma unroll
            for(int k = 0; k < NS; ++k)
            {
                const float v = j == 0 ? val[k].x : j == 1 ? val[k].y : j == 2 ? val[k].z : val[k].w;
                const float xi = fminf(fmaxf(v * tsf, 0.0f), tsMax);
                const float t = __fadd_rd(__fadd_rd(xi, 0.5f), 12582912.0f);
                const float4 c = entry(k, __float_as_uint(t));
                if(ISO)
                    merge_accumulate(c, act.weight[k], act.iso[k], true, vc, ic);
                else if(act.weight[k] > 0.0f)
                {
                    vc.x += c.x;
                    vc.y += c.y;
                    vc.z += c.z;
                    vc.w += c.w;
                }
            }
            if(fast)
            {
                if(p.invTotalWeight != 0.0f)
                    vc = make_float4(vc.x * p.invTotalWeight, vc.y * p.invTotalWeight, vc.z * p.invTotalWeight, vc.w * p.invTotalWeight);
                else
                    vc = make_float4(vc.x / p.totalWeight, vc.y / p.totalWeight, vc.z / p.totalWeight, vc.w / p.totalWeight);
                const float d = (p.ditherMode == 1 || p.ditherMode == 2)
                    ? float((maskWord >> (8 * j)) & 0xFFu) / 64.0f
                    : dither_threshold(p.ditherMode, sMask, x + j, y, z);
                vo[j] = dither_rgba_ceil(vc, fminf(d, kDitherMax));
            }
            else
                vo[j] = merge_volume_texel(p, sMask, x + j, y, z, vc);
            io[j] = ISO ? merge_iso_texel(ic) : 0u;
        }
        reinterpret_cast<uint4*>(p.volLin)[q] = make_uint4(vo[0], vo[1], vo[2], vo[3]);
        if(ISO)
            reinterpret_cast<uint4*>(p.isoLin)[q] = make_uint4(io[0], io[1], io[2], io[3]);
    }

    // As k_merge_voxels_n, four x-adjacent voxels per thread (rows a multiple of 4 voxels,
    // 16-byte aligned sources, fewer than 2^32 groups of four); table entries from global
    // memory through a pointer biased so that the floor's bits address them
    template<bool ISO, int NS>
    __global__ void __launch_bounds__(256) k_merge_voxels_x4(const __grid_constant__ MergeParams p, const __grid_constant__ MergeActive act)
    {
        __shared__ __align__(4) uint8_t sMask[64];
        if(threadIdx.x < 64)
            sMask[threadIdx.x] = p.ditherMode == 2 ? c_dither2[threadIdx.x] : c_dither1[threadIdx.x];
        __syncthreads();
        const uint32_t rowQuads = uint32_t(p.g.ls[0]) >> 2;
        const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
        if(q >= rowQuads * uint32_t(p.g.ls[1]) * uint32_t(p.g.ls[2]))
            return;
        merge_quad<ISO, NS>(p, act, sMask, q, rowQuads, [&](int k, uint32_t bits) {
            const float4* table = ISO ? act.lut[k] : act.pre[k];
            const char* biased = reinterpret_cast<const char*>(table) - size_t(0x4B400000u) * sizeof(float4);
            return __ldg(reinterpret_cast<const float4*>(biased + size_t(bits) * sizeof(float4)));
        });
    }

    // The same without iso output, with the NS premultiplied tables (NS * ts entries) in
    // shared memory: persistent CTAs load them once and walk the quads, so each of the
    // four gathers per voxel reads shared memory instead of scattering over L1 sectors.
    template<int NS>
    __global__ void __launch_bounds__(512) k_merge_voxels_x4_smem(const __grid_constant__ MergeParams p, const __grid_constant__ MergeActive act)
    {
        extern __shared__ float4 sLut[];
        __shared__ __align__(4) uint8_t sMask[64];
        if(threadIdx.x < 64)
            sMask[threadIdx.x] = p.ditherMode == 2 ? c_dither2[threadIdx.x] : c_dither1[threadIdx.x];
        const int ts = p.ts;
        for(int i = threadIdx.x; i < NS * ts; i += blockDim.x)
            sLut[i] = __ldg(p.lutPre + i);
        __syncthreads();
        const uint32_t rowQuads = uint32_t(p.g.ls[0]) >> 2;
        const uint32_t quads = rowQuads * uint32_t(p.g.ls[1]) * uint32_t(p.g.ls[2]);
        for(uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < quads; q += gridDim.x * blockDim.x)
            merge_quad<false, NS>(p, act, sMask, q, rowQuads, [&](int k, uint32_t bits) {
                return sLut[k * ts + int(bits - 0x4B400000u)];
            });
    }

    template<bool ISO>
    __global__ void __launch_bounds__(256) k_merge_voxels(const __grid_constant__ MergeParams p)
    {
        __shared__ uint8_t sMask[64];
        if(threadIdx.x < 64)
            sMask[threadIdx.x] = p.ditherMode == 2 ? c_dither2[threadIdx.x] : c_dither1[threadIdx.x];
        __syncthreads();
        const Geom& g = p.g;
        const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
        if(x >= g.ls[0])
            return;
        const size_t i = (size_t(z) * g.ls[1] + y) * g.ls[0] + x;
        float4 vc = make_float4(0, 0, 0, 0), ic = make_float4(0, 0, 0, 0);
        for(int s = 0; s < p.nVol; ++s)
        {
            const float vw = p.weight[s];
            const float it = p.iso[s];
            if(!(vw + it > 0.0f))
                continue;
            float val;
            if(p.chainIdem[s] != 0)
                val = __ldg(p.src[s] + i * p.fdim[s]); // every functor idem: the x component
            else
            {
                float v[4];
                read_voxel(p.src[s], p.fdim[s], i, v);
                val = apply_chain(v, p.fdim[s], p.chain[s]);
            }
            float4 c = __ldg(p.lut + size_t(s) * p.ts + lut_index_fast(val, p.ts));
            if(p.adv[s])
            {
                // field source: alpha blended with the advection texture
                // (MergeAdvectionToCombinedTextureIterator, isaac_common_kernel.hpp:664-665)
                const size_t ai = (size_t(z + p.advG[2]) * (g.ls[1] + 2 * p.advG[1]) + (y + p.advG[1])) * (g.ls[0] + 2 * p.advG[0])
                    + (x + p.advG[0]);
                c.w *= float(__ldg(p.adv[s] + ai)) / 255.0f;
            }
            merge_accumulate(c, vw, it, ISO, vc, ic);
        }
        merge_store<ISO>(p, sMask, i, x, y, z, vc, ic);
    }

    // ---------------------------------------------------------------- merge, pass 2: bricks
    // One CTA per row of kPackRow = 4 bricks along x.  The row's 33 x 9 x 9 texels (the
    // bricks' voxels plus the apron on the low side, clamped at the volume border) come
    // from the linear textures into shared memory (staged row r = lz * 9 + ly at pitch
    // kPackPitch), texel rows per warp with the lanes along x.  A lane's texels all have the same x, so they belong to the same one or two
    // bricks: the lane keeps one "any non-zero" bit and one maximum alpha byte, and a warp
    // reduction per brick gives the flags that drive empty-space skipping.  Then the 4
    // bricks' 576-slot quad blocks, contiguous in memory, go out as 16-byte stores: thread
    // (lx, ly) walks the slot layers lz of all 4 bricks, and slot index = layer * 64 + lxy.
    // A slot is stored channel-major (quad_channel_major: word c = channel c of its four
    // texels), the form the march's integer dot products read.
    // Every texel is a copy of a voxel pass 1 computed once.
    constexpr int kPackRow = 4;
    constexpr int kPackPitch = 40; // row pitch in words: 40 = 8 mod 32 keeps the quad reads conflict-free
    constexpr int kPackRows = kApron * kApron; // (ly, lz) rows
    constexpr int kPackWords = kPackRows * kPackPitch;
    // k_merge_pack's pitch for y-fastest slots: its quad reads then walk y across a warp's
    // lanes, and 36 = 4 mod 32 puts the 8 rows x 4 columns of a warp on 32 different banks
    constexpr int kPackPitchY = 36;

    template<bool ISO, bool YFAST>
    __global__ void __launch_bounds__(256) k_merge_pack(const __grid_constant__ MergeParams p)
    {
        // staging pitch: conflict-free quad reads for the slot order
        constexpr int kPitch = YFAST ? kPackPitchY : kPackPitch;
        __shared__ uint32_t volS[kPackWords];
        __shared__ uint32_t isoS[ISO ? kPackWords : 1];
        __shared__ int anyS[kPackRow], isoMaxS[kPackRow];
        const Geom& g = p.g;
        const int bx0 = blockIdx.x * kPackRow, by = blockIdx.y, bz = blockIdx.z;
        const int nRow = min(kPackRow, g.nb[0] - bx0);
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if(threadIdx.x < kPackRow)
        {
            anyS[threadIdx.x] = 0;
            isoMaxS[threadIdx.x] = 0;
        }
        // staged texel lx belongs to the bricks j with 8j <= lx <= 8j + 8
        const int x0 = iclamp(bx0 * 8 - 1 + lane, 0, g.ls[0] - 1);
        const int x32 = iclamp(bx0 * 8 + 31, 0, g.ls[0] - 1); // lx = 32, brick 3, read by lane 0
        const int jlo = lane >= 1 ? (lane - 1) >> 3 : 0, jhi = min(lane >> 3, kPackRow - 1);
        int laneAny = 0, laneIso = 0, any32 = 0, iso32 = 0;
        // all of the warp's row loads are issued before any is used, so that enough
        // bytes are in flight to cover the memory latency (lane 0 also reads the row's
        // 33rd texel, lx = 32).  Warp w stages the rows ly = w of all 9 planes lz and the
        // row ly = 8 of plane w (warp 0 also of plane 8): one y offset per warp and one
        // multiply per plane, as the kernel is bound by instruction issue.
        const size_t plane = size_t(g.ls[0]) * size_t(g.ls[1]);
        const size_t yA = size_t(iclamp(by * 8 - 1 + warp, 0, g.ls[1] - 1)) * size_t(g.ls[0]);
        const size_t yB = size_t(iclamp(by * 8 + 7, 0, g.ls[1] - 1)) * size_t(g.ls[0]);
        constexpr int kRows = kApron + 2; // 9 planes of row ly = w, then row ly = 8 of planes w and 8
        uint32_t v[kRows], w[kRows], v2[kRows], w2[kRows];
        int rr[kRows];
#pragma unroll
        for(int i = 0; i < kRows; ++i)
        {
            const int lz = i < kApron ? i : (i == kApron ? warp : 8);
            const int ly = i < kApron ? warp : 8;
            rr[i] = lz * kApron + ly;
            if(i == kApron + 1 && warp != 0)
            {
                rr[i] = -1;
                continue;
            }
            const size_t row = size_t(iclamp(bz * 8 - 1 + lz, 0, g.ls[2] - 1)) * plane + (i < kApron ? yA : yB);
            v[i] = __ldg(p.volLin + row + x0);
            if(ISO)
                w[i] = __ldg(p.isoLin + row + x0);
            if(lane == 0)
            {
                v2[i] = __ldg(p.volLin + row + x32);
                if(ISO)
                    w2[i] = __ldg(p.isoLin + row + x32);
            }
        }
#pragma unroll
        for(int i = 0; i < kRows; ++i)
        {
            const int r = rr[i];
            if(r >= 0)
            {
                volS[r * kPitch + lane] = v[i];
                laneAny |= v[i] != 0u;
                if(ISO)
                {
                    isoS[r * kPitch + lane] = w[i];
                    laneIso = max(laneIso, int(w[i] >> 24));
                }
                if(lane == 0)
                {
                    volS[r * kPitch + 32] = v2[i];
                    any32 |= v2[i] != 0u;
                    if(ISO)
                    {
                        isoS[r * kPitch + 32] = w2[i];
                        iso32 = max(iso32, int(w2[i] >> 24));
                    }
                }
            }
        }
        __syncthreads(); // the flag slots are initialised
#pragma unroll
        for(int j = 0; j < kPackRow; ++j)
        {
            const bool mine = jlo <= j && j <= jhi;
            const bool extra = j == kPackRow - 1 && lane == 0; // the lx = 32 texel
            const int a = __any_sync(0xFFFFFFFFu, (mine && laneAny) || (extra && any32));
            int m = 0;
            if(ISO)
                m = int(__reduce_max_sync(0xFFFFFFFFu, unsigned(max(mine ? laneIso : 0, extra ? iso32 : 0))));
            if(lane == 0)
            {
                if(a)
                    atomicOr(&anyS[j], 1);
                if(ISO && m)
                    atomicMax(&isoMaxS[j], m);
            }
        }
        __syncthreads();
        const size_t brick0 = (size_t(bz) * g.nb[1] + by) * g.nb[0] + bx0;
        if(threadIdx.x < nRow)
        {
            const int j = threadIdx.x;
            p.volFlag[brick0 + j] = anyS[j] ? 1 : 0;
            if(!anyS[j])
                atomicAdd(p.emptyBricks, 1u);
            if(ISO)
                p.isoFlag[brick0 + j] = uint8_t(isoMaxS[j]);
        }
        // thread lxy writes slot lxy of each layer: (lx, ly) = (lxy & 7, lxy >> 3) for x-fastest
        // slots, (lxy >> 3, lxy & 7) for y-fastest ones
        const int lxy = threadIdx.x & 63;
        const int base = YFAST ? (lxy & 7) * kPitch + (lxy >> 3) : (lxy >> 3) * kPitch + (lxy & 7);
        for(int layer = threadIdx.x >> 6; layer < nRow * kApron; layer += 4)
        {
            const int j = layer / kApron, lz = layer - j * kApron;
            const int t = lz * (kApron * kPitch) + base + 8 * j;
            const size_t slot = brick0 * kSlotsPerBrick + size_t(layer) * 64 + lxy;
            p.volQ[slot] = quad_channel_major(volS[t], volS[t + 1], volS[t + kPitch], volS[t + kPitch + 1]);
            if(ISO)
                p.isoAQ[slot] = (isoS[t] >> 24) | ((isoS[t + 1] >> 24) << 8) | ((isoS[t + kPitch] >> 24) << 16)
                    | ((isoS[t + kPitch + 1] >> 24) << 24);
        }
    }

    // largest set of premultiplied tables the persistent merge keeps in shared memory
    // (4 sources x 1024 entries = 64 KiB leaves room for two 512-thread CTAs per SM)
    constexpr size_t kMergeSmemTables = 96 * 1024;

    template<int NS>
    void launch_x4_smem(const MergeParams& p, const MergeActive& act, size_t quads, size_t tableBytes, cudaStream_t s)
    {
        // the opt-in to more than 48 KiB of dynamic shared memory, once per device
        static uint64_t configured = 0;
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        if(dev < 64 && !((configured >> dev) & 1u)
           && cudaFuncSetAttribute(k_merge_voxels_x4_smem<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kMergeSmemTables))
               == cudaSuccess)
            configured |= uint64_t(1) << dev;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const size_t resident = size_t(sms) * ctas_per_sm(k_merge_voxels_x4_smem<NS>, 512, tableBytes);
        const size_t grid = std::max<size_t>(1, std::min(resident, (quads + 511) / 512));
        k_merge_voxels_x4_smem<NS><<<unsigned(grid), 512, tableBytes, s>>>(p, act);
    }

    // returns the number of kernels launched
    template<bool ISO>
    int launch_merge_iso(const MergeParams& p, cudaStream_t s)
    {
        const dim3 vgrid((p.g.ls[0] + 255) / 256, p.g.ls[1], p.g.ls[2]);
        MergeActive act{};
        bool scalar = true;
        for(int k = 0; k < p.nVol; ++k)
        {
            if(!(p.weight[k] + p.iso[k] > 0.0f))
                continue;
            scalar = scalar && p.chainIdem[k] && p.fdim[k] == 1 && !p.adv[k];
            act.src[act.n] = p.src[k];
            act.lut[act.n] = p.lut + size_t(k) * p.ts;
            act.weight[act.n] = p.weight[k];
            act.iso[act.n] = p.iso[k];
            act.n++;
        }
        bool x4 = (p.g.ls[0] & 3) == 0 && size_t(p.g.ls[0] / 4) * p.g.ls[1] * p.g.ls[2] < (size_t(1) << 32);
        for(int k = 0; k < act.n; ++k)
            x4 = x4 && (reinterpret_cast<uintptr_t>(act.src[k]) & 15u) == 0;
        int launches = 2;
        if(scalar && x4 && act.n >= 1 && act.n <= 4)
        {
            const size_t quads = size_t(p.g.ls[0] / 4) * p.g.ls[1] * p.g.ls[2];
            const unsigned blocks = unsigned((quads + 255) / 256);
            if(!ISO)
            {
                for(int k = 0; k < act.n; ++k)
                    act.pre[k] = p.lutPre + size_t(k) * p.ts;
                k_merge_premultiply<<<dim3((p.ts + 255) / 256, act.n), 256, 0, s>>>(act, p.lutPre, p.ts);
                launches++;
            }
            const size_t tableBytes = size_t(act.n) * p.ts * sizeof(float4);
            if(!ISO && tableBytes <= kMergeSmemTables)
            {
                switch(act.n)
                {
                case 1: launch_x4_smem<1>(p, act, quads, tableBytes, s); break;
                case 2: launch_x4_smem<2>(p, act, quads, tableBytes, s); break;
                case 3: launch_x4_smem<3>(p, act, quads, tableBytes, s); break;
                default: launch_x4_smem<4>(p, act, quads, tableBytes, s); break;
                }
            }
            else
            {
                switch(act.n)
                {
                case 1: k_merge_voxels_x4<ISO, 1><<<blocks, 256, 0, s>>>(p, act); break;
                case 2: k_merge_voxels_x4<ISO, 2><<<blocks, 256, 0, s>>>(p, act); break;
                case 3: k_merge_voxels_x4<ISO, 3><<<blocks, 256, 0, s>>>(p, act); break;
                default: k_merge_voxels_x4<ISO, 4><<<blocks, 256, 0, s>>>(p, act); break;
                }
            }
        }
        else if(scalar && act.n >= 1 && act.n <= 4)
        {
            switch(act.n)
            {
            case 1: k_merge_voxels_n<ISO, 1><<<vgrid, 256, 0, s>>>(p, act); break;
            case 2: k_merge_voxels_n<ISO, 2><<<vgrid, 256, 0, s>>>(p, act); break;
            case 3: k_merge_voxels_n<ISO, 3><<<vgrid, 256, 0, s>>>(p, act); break;
            default: k_merge_voxels_n<ISO, 4><<<vgrid, 256, 0, s>>>(p, act); break;
            }
        }
        else
            k_merge_voxels<ISO><<<vgrid, 256, 0, s>>>(p);
        const dim3 pgrid((p.g.nb[0] + kPackRow - 1) / kPackRow, p.g.nb[1], p.g.nb[2]);
        if(p.g.yfast)
            k_merge_pack<ISO, true><<<pgrid, 256, 0, s>>>(p);
        else
            k_merge_pack<ISO, false><<<pgrid, 256, 0, s>>>(p);
        return launches;
    }

    int launch_merge(const MergeParams& p, cudaStream_t s)
    {
        return p.writeIso ? launch_merge_iso<true>(p, s) : launch_merge_iso<false>(p, s);
    }

    // ---------------------------------------------------------------- field-source advection
    // updateNoiseTexture (lib/isaac.hpp:499-562) with HaltonSeedingKernel, GaussBlur7Kernel
    // and MultiplyClampKernel (lib/isaac/isaac_common_kernel.hpp:334-430), and
    // GenerateAdvectionTextureKernel (:500-550).  The reference leaves the advection
    // textures (and their guard cells) uninitialised; here they start at zero, so a
    // sample outside the local volume reads 0 like its VALUE border.

    // trilinear sample of a scalar texture through Sampler<LINEAR, ...>::interpolate
    // (isaac_texture.hpp:237-257): fetch(ix, iy, iz) returns the bordered texel
    template<class F>
    __device__ __forceinline__ float sample_linear(float cx, float cy, float cz, F fetch)
    {
        cx -= 0.5f;
        cy -= 0.5f;
        cz -= 0.5f;
        const float flx = floorf(cx), fly = floorf(cy), flz = floorf(cz);
        const int ix = int(flx), iy = int(fly), iz = int(flz);
        const float ox = cx - flx, oy = cy - fly, oz = cz - flz;
        return tri_q(
            ox,
            oy,
            oz,
            fetch(ix, iy, iz),
            fetch(ix + 1, iy, iz),
            fetch(ix, iy + 1, iz),
            fetch(ix + 1, iy + 1, iz),
            fetch(ix, iy, iz + 1),
            fetch(ix + 1, iy, iz + 1),
            fetch(ix, iy + 1, iz + 1),
            fetch(ix + 1, iy + 1, iz + 1));
    }

    __device__ __forceinline__ float halton_f(uint32_t index, uint32_t base)
    {
        // isaac_helper.hpp:57-69
        float result = 0.0f, f = 1.0f;
        while(index > 0)
        {
            f /= float(base);
            result += f * float(index % base);
            index /= base;
        }
        return result;
    }

    __global__ void k_noise_seed(NoiseParams p, float* __restrict__ noise)
    {
        // every seed writes 1, so the serial reference loop and this one agree in any order
        const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
        if(i > p.seedPoints)
            return;
        const int x = int(float(p.LX) * halton_f(uint32_t(i), 3));
        const int y = int(float(p.LY) * halton_f(uint32_t(i), 5));
        const int z = int(float(p.LZ) * halton_f(uint32_t(i), 7));
        noise[(size_t(z) * p.LY + y) * p.LX + x] = 1.0f;
    }

    __global__ void k_noise_blur(NoiseParams p, const float* __restrict__ src, float* __restrict__ dst, int axis)
    {
        const size_t n = size_t(p.LX) * p.LY * p.LZ;
        const float g7[4] = {64.0f, 40.5f, 10.0f, 1.0f};
        const float mx = axis == 0 ? 1.0f : 0.0f, my = axis == 1 ? 1.0f : 0.0f, mz = axis == 2 ? 1.0f : 0.0f;
        auto fetch = [&](int x, int y, int z) {
            // REPEAT border, no guard
            x = (p.LX + (x % p.LX)) % p.LX;
            y = (p.LY + (y % p.LY)) % p.LY;
            z = (p.LZ + (z % p.LZ)) % p.LZ;
            return __ldg(src + (size_t(z) * p.LY + y) * p.LX + x);
        };
        for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        {
            const int x = int(i % p.LX);
            const size_t t = i / p.LX;
            const int y = int(t % p.LY), z = int(t / p.LY);
            float r = 0.0f;
            for(int k = -3; k < 4; ++k)
            {
                const float cx = float(x) + mx * float(k) / p.scale[0];
                const float cy = float(y) + my * float(k) / p.scale[1];
                const float cz = float(z) + mz * float(k) / p.scale[2];
                r += sample_linear(cx, cy, cz, fetch) * g7[k < 0 ? -k : k];
            }
            dst[i] = r / 167.0f;
        }
    }

    __global__ void k_noise_clamp(size_t n, const float* __restrict__ src, float* __restrict__ dst)
    {
        for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
            dst[i] = gclamp(src[i] * 30.0f, 0.0f, 1.0f);
    }

    // one thread per float of the compact copy: consecutive threads read consecutive
    // floats of one guarded row
    __global__ void __launch_bounds__(256)
        k_compact_guarded(const float* __restrict__ src, float* __restrict__ dst, int X, int Y, int Z, int g, int fd)
    {
        const size_t rowF = size_t(X) * fd;
        const size_t n = rowF * Y * Z;
        const size_t gx = size_t(X + 2 * g), gy = size_t(Y + 2 * g);
        for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        {
            const size_t row = i / rowF, k = i - row * rowF;
            const size_t y = row % Y, z = row / Y;
            dst[i] = __ldg(src + (((z + g) * gy + (y + g)) * gx + g) * fd + k);
        }
    }

    void launch_compact_guarded(const float* src, float* dst, int X, int Y, int Z, int guard, int fdim, cudaStream_t s)
    {
        const size_t n = size_t(X) * Y * Z * fdim;
        const size_t blocks = std::min<size_t>((n + 255) / 256, size_t(148) * 32);
        k_compact_guarded<<<unsigned(blocks), 256, 0, s>>>(src, dst, X, Y, Z, guard, fdim);
    }

    void launch_noise(const NoiseParams& p, float* noise, float* tmp, cudaStream_t s)
    {
        const size_t n = size_t(p.LX) * p.LY * p.LZ;
        cudaMemsetAsync(noise, 0, n * sizeof(float), s);
        if(p.seedPoints > 0)
            k_noise_seed<<<(p.seedPoints + 255) / 256, 256, 0, s>>>(p, noise);
        const int blocks = int(std::min<size_t>((n + 255) / 256, 148 * 16));
        k_noise_blur<<<blocks, 256, 0, s>>>(p, noise, tmp, 0);
        k_noise_blur<<<blocks, 256, 0, s>>>(p, tmp, noise, 1);
        k_noise_blur<<<blocks, 256, 0, s>>>(p, noise, tmp, 2);
        k_noise_clamp<<<blocks, 256, 0, s>>>(n, tmp, noise);
    }

    __global__ void k_advect(const __grid_constant__ AdvectParams p)
    {
        const size_t n = size_t(p.LX) * p.LY * p.LZ;
        const int SX = p.LX + 2 * p.G[0], SY = p.LY + 2 * p.G[1];
        auto at = [&](int x, int y, int z) {
            return (size_t(z + p.G[2]) * SY + (y + p.G[1])) * SX + (x + p.G[0]);
        };
        auto fetch = [&](int x, int y, int z) {
            // VALUE border 0 outside the guard band (Sampler::safeMemoryAccess,
            // isaac_texture.hpp:201-206); the band holds zeros or a neighbour's slabs
            if(x < -p.G[0] || y < -p.G[1] || z < -p.G[2] || x >= p.LX + p.G[0] || y >= p.LY + p.G[1] || z >= p.LZ + p.G[2])
                return 0.0f;
            return float(__ldg(p.back + at(x, y, z)));
        };
        for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        {
            const int x = int(i % p.LX);
            const size_t t = i / p.LX;
            const int y = int(t % p.LY), z = int(t / p.LY);
            float vx = __ldg(p.field + 3 * i), vy = __ldg(p.field + 3 * i + 1), vz = __ldg(p.field + 3 * i + 2);
            // glm::length: sqrt((x*x + y*y) + z*z); at least FLT_MIN
            const float len = gmax(sqrtf((vx * vx + vy * vy) + vz * vz), 1.17549435e-38f);
            vx = vx / len;
            vy = vy / len;
            vz = vz / len;
            const float cx = (float(x) + 0.5f) - vx * p.stepSize / p.scale[0];
            const float cy = (float(y) + 0.5f) - vy * p.stepSize / p.scale[1];
            const float cz = (float(z) + 0.5f) - vz * p.stepSize / p.scale[2];
            const float history = sample_linear(cx, cy, cz, fetch) / 255.0f;
            const float nv = p.seedNoise ? __ldg(p.noise + i) : 0.0f;
            const float v = nv + history * p.historyWeight * (1.0f - nv);
            // applyDither3D(5, coord, v): the 16^3 blue-noise mask, int(s) + (fract(s) > d), clamped
            const float d = dither_threshold(5, nullptr, x, y, z);
            const float sv = fminf(fmaxf(v * 255.0f, -2.0f), 257.0f);
            float tr;
            int ti = trunc_nonneg(fabsf(sv), tr);
            if(sv < 0.0f)
                ti = -ti;
            float fl;
            int fi;
            floor_split(sv, fl, fi);
            p.out[at(x, y, z)] = uint8_t(min(max(ti + ((sv - fl) > d ? 1 : 0), 0), 255));
        }
    }

    void launch_advect(const AdvectParams& p, cudaStream_t s)
    {
        const size_t n = size_t(p.LX) * p.LY * p.LZ;
        k_advect<<<int(std::min<size_t>((n + 255) / 256, 148 * 16)), 256, 0, s>>>(p);
    }

    // guard slab voxel c <-> texture voxel, per axis (the reference's index arithmetic,
    // including where it places the positive-side slabs):
    //   pack (SyncToOwnGuard, isaac_common_kernel.hpp:454-474):
    //     source = max(d, 0) * (L - e - 1) + c
    //   unpack (SyncFromNeighbourGuard, :477-498):
    //     target = max(d, 0) * (L - 1) + min(d, 0) * e + c
    template<bool PACK>
    __global__ void k_guard(const __grid_constant__ GuardParams p)
    {
        const size_t n = size_t(p.e[0]) * p.e[1] * p.e[2];
        const int SX = p.L[0] + 2 * p.G[0], SY = p.L[1] + 2 * p.G[1];
        for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        {
            const int c[3] = {int(i % p.e[0]), int((i / p.e[0]) % p.e[1]), int(i / (size_t(p.e[0]) * p.e[1]))};
            int t[3];
#pragma unroll
            for(int a = 0; a < 3; ++a)
                t[a] = PACK ? (p.d[a] > 0 ? p.L[a] - p.e[a] - 1 : 0) + c[a]
                            : (p.d[a] > 0 ? p.L[a] - 1 : 0) + (p.d[a] < 0 ? -p.e[a] : 0) + c[a];
            const size_t ti = (size_t(t[2] + p.G[2]) * SY + (t[1] + p.G[1])) * SX + (t[0] + p.G[0]);
            if(PACK)
                p.slab[i] = p.tex[ti];
            else
                p.tex[ti] = p.slab[i];
        }
    }

    void launch_pack_guard(const GuardParams& p, cudaStream_t s)
    {
        const size_t n = size_t(p.e[0]) * p.e[1] * p.e[2];
        k_guard<true><<<int(std::min<size_t>((n + 255) / 256, 148 * 8)), 256, 0, s>>>(p);
    }
    void launch_unpack_guard(const GuardParams& p, cudaStream_t s)
    {
        const size_t n = size_t(p.e[0]) * p.e[1] * p.e[2];
        k_guard<false><<<int(std::min<size_t>((n + 255) / 256, 148 * 8)), 256, 0, s>>>(p);
    }

    // ---------------------------------------------------------------- per-source bricks
    template<int DT>
    __device__ __forceinline__ void store_elem(void* base, size_t i, float v)
    {
        if(DT == 0)
            reinterpret_cast<float*>(base)[i] = v;
        else if(DT == 1)
            reinterpret_cast<__nv_bfloat16*>(base)[i] = __float2bfloat16_rn(v);
        else
            reinterpret_cast<__half*>(base)[i] = __float2half_rn(v);
    }

    template<int DT>
    __global__ void __launch_bounds__(256) k_source_bricks(const __grid_constant__ SourceBrickParams p)
    {
        __shared__ float valS[4][kApron * kApron * kApron];
        const Geom& g = p.g;
        const int bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z;
        for(int t = threadIdx.x; t < kApron * kApron * kApron; t += blockDim.x)
        {
            const int lx = t % kApron, ly = (t / kApron) % kApron, lz = t / (kApron * kApron);
            const int x = iclamp(bx * 8 - 1 + lx, 0, g.ls[0] - 1);
            const int y = iclamp(by * 8 - 1 + ly, 0, g.ls[1] - 1);
            const int z = iclamp(bz * 8 - 1 + lz, 0, g.ls[2] - 1);
            const size_t idx = (size_t(z) * g.ls[1] + y) * g.ls[0] + x;
            float v[4];
            const float* sp = p.src + idx * p.fdim;
            v[0] = __ldg(sp);
            v[1] = p.fdim > 1 ? __ldg(sp + 1) : 0.0f;
            v[2] = p.fdim > 2 ? __ldg(sp + 2) : 0.0f;
            v[3] = p.fdim > 3 ? __ldg(sp + 3) : 0.0f;
            if(p.applyChain)
            {
                valS[0][t] = apply_chain(v, p.fdim, p.chain);
            }
            else
            {
#pragma unroll
                for(int c = 0; c < 4; ++c)
                    if(c < p.ncomp)
                        valS[c][t] = v[c];
            }
        }
        __syncthreads();
        const size_t brick = (size_t(bz) * g.nb[1] + by) * g.nb[0] + bx;
        const int per = 4 * p.ncomp;
        for(int s = threadIdx.x; s < kSlotsPerBrick; s += blockDim.x)
        {
            const int lx = s & 7, ly = (s >> 3) & 7, lz = s >> 6;
            const int t = (lz * kApron + ly) * kApron + lx;
            const size_t base = (brick * kSlotsPerBrick + morton_slot(lx, ly, lz)) * per;
            for(int c = 0; c < p.ncomp; ++c)
            {
                store_elem<DT>(p.out, base + 4 * c + 0, valS[c][t]);
                store_elem<DT>(p.out, base + 4 * c + 1, valS[c][t + 1]);
                store_elem<DT>(p.out, base + 4 * c + 2, valS[c][t + kApron]);
                store_elem<DT>(p.out, base + 4 * c + 3, valS[c][t + kApron + 1]);
            }
        }
    }

    // the stored value of voxel idx of a one-component brick set: the functor chain's
    // result (non-persistent sources) or the first component
    __device__ __forceinline__ float source_value(const SourceBrickParams& p, size_t idx)
    {
        const float* sp = p.src + idx * p.fdim;
        if(!p.applyChain)
            return __ldg(sp);
        float v[4];
        v[0] = __ldg(sp);
        v[1] = p.fdim > 1 ? __ldg(sp + 1) : 0.0f;
        v[2] = p.fdim > 2 ? __ldg(sp + 2) : 0.0f;
        v[3] = p.fdim > 3 ? __ldg(sp + 3) : 0.0f;
        return apply_chain(v, p.fdim, p.chain);
    }

    // two values as one 32-bit word of BF16 (DT 1) or FP16 (DT 2), the first in the low
    // half, each rounded to nearest even as __float2bfloat16_rn / __float2half_rn do
    template<int DT>
    __device__ __forceinline__ void pack_pair(float a, float b, uint32_t& out)
    {
        if(DT == 1)
        {
            const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
            out = *reinterpret_cast<const uint32_t*>(&h);
        }
        else
        {
            const __half2 h = __floats2half2_rn(a, b);
            out = *reinterpret_cast<const uint32_t*>(&h);
        }
    }

    // one quad slot of 4 elements as one store: 16 bytes (FP32) or 8 bytes (BF16 / FP16,
    // rounded to nearest even as __float2bfloat16_rn / __float2half_rn do)
    template<int DT>
    __device__ __forceinline__ void store_quad(void* out, size_t slot, float a, float b, float c, float d)
    {
        if(DT == 0)
            reinterpret_cast<float4*>(out)[slot] = make_float4(a, b, c, d);
        else if(DT == 1)
        {
            const __nv_bfloat162 lo = __floats2bfloat162_rn(a, b), hi = __floats2bfloat162_rn(c, d);
            reinterpret_cast<uint2*>(out)[slot]
                = make_uint2(*reinterpret_cast<const uint32_t*>(&lo), *reinterpret_cast<const uint32_t*>(&hi));
        }
        else
        {
            const __half2 lo = __floats2half2_rn(a, b), hi = __floats2half2_rn(c, d);
            reinterpret_cast<uint2*>(out)[slot]
                = make_uint2(*reinterpret_cast<const uint32_t*>(&lo), *reinterpret_cast<const uint32_t*>(&hi));
        }
    }

    // the stored value of voxel idx: with SIMPLE the source has one component and no
    // functor chain, and the value is the voxel itself
    template<bool SIMPLE>
    __device__ __forceinline__ float source_value_t(const SourceBrickParams& p, size_t idx)
    {
        if constexpr(SIMPLE)
            return __ldg(p.src + idx);
        else
            return source_value(p, idx);
    }

    // One-component bricks as k_merge_pack builds the combined ones: one CTA per row of 4
    // bricks along x, texel rows staged with the lanes along x, then every slot of the 4
    // bricks as one vector store, contiguous in memory.  The kernel is bound by
    // instruction issue, so the staging is arranged for little index arithmetic: warp w
    // stages the rows ly = w of all 9 planes lz (one y offset per warp, one multiply per
    // plane) and the row ly = 8 of plane w (warp 0 also of plane 8).
    template<int DT, bool SIMPLE>
    __global__ void __launch_bounds__(256) k_source_bricks_row(const __grid_constant__ SourceBrickParams p)
    {
        __shared__ float valS[kPackWords];
        const Geom& g = p.g;
        const int bx0 = blockIdx.x * kPackRow, by = blockIdx.y, bz = blockIdx.z;
        const int nRow = min(kPackRow, g.nb[0] - bx0);
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int x0 = iclamp(bx0 * 8 - 1 + lane, 0, g.ls[0] - 1);
        const int x32 = iclamp(bx0 * 8 + 31, 0, g.ls[0] - 1);
        const size_t plane = size_t(g.ls[0]) * size_t(g.ls[1]);
        const size_t yA = size_t(iclamp(by * 8 - 1 + warp, 0, g.ls[1] - 1)) * size_t(g.ls[0]);
        const size_t yB = size_t(iclamp(by * 8 + 7, 0, g.ls[1] - 1)) * size_t(g.ls[0]);
        // all of the warp's row loads are issued before any is used (lane 0 also reads
        // the row's 33rd texel, lx = 32)
        float v[kApron], v2[kApron], u[2], u2[2];
#pragma unroll
        for(int lz = 0; lz < kApron; ++lz)
        {
            const size_t row = size_t(iclamp(bz * 8 - 1 + lz, 0, g.ls[2] - 1)) * plane + yA;
            v[lz] = source_value_t<SIMPLE>(p, row + x0);
            if(lane == 0)
                v2[lz] = source_value_t<SIMPLE>(p, row + x32);
        }
        {
            const size_t row = size_t(iclamp(bz * 8 - 1 + warp, 0, g.ls[2] - 1)) * plane + yB;
            u[0] = source_value_t<SIMPLE>(p, row + x0);
            if(lane == 0)
                u2[0] = source_value_t<SIMPLE>(p, row + x32);
        }
        if(warp == 0)
        {
            const size_t row = size_t(iclamp(bz * 8 + 7, 0, g.ls[2] - 1)) * plane + yB;
            u[1] = source_value_t<SIMPLE>(p, row + x0);
            if(lane == 0)
                u2[1] = source_value_t<SIMPLE>(p, row + x32);
        }
        // staged row r = lz * 9 + ly
#pragma unroll
        for(int lz = 0; lz < kApron; ++lz)
        {
            const int r = lz * kApron + warp;
            valS[r * kPackPitch + lane] = v[lz];
            if(lane == 0)
                valS[r * kPackPitch + 32] = v2[lz];
        }
        {
            const int r = warp * kApron + 8;
            valS[r * kPackPitch + lane] = u[0];
            if(lane == 0)
                valS[r * kPackPitch + 32] = u2[0];
        }
        if(warp == 0)
        {
            const int r = 8 * kApron + 8;
            valS[r * kPackPitch + lane] = u[1];
            if(lane == 0)
                valS[r * kPackPitch + 32] = u2[1];
        }
        __syncthreads();
        const size_t brick0 = (size_t(bz) * g.nb[1] + by) * g.nb[0] + bx0;
        if(DT == 0)
        {
            // one 16-byte slot per thread
            const int lxy = threadIdx.x & 63;
            const int base = (lxy >> 3) * kPackPitch + (lxy & 7);
            for(int layer = threadIdx.x >> 6; layer < nRow * kApron; layer += 4)
            {
                const int j = layer / kApron, lz = layer - j * kApron;
                const int t = lz * (kApron * kPackPitch) + base + 8 * j;
                store_quad<0>(p.out, (brick0 + j) * kSlotsPerBrick + morton_slot(lxy & 7, lxy >> 3, lz), valS[t],
                              valS[t + 1], valS[t + kPackPitch], valS[t + kPackPitch + 1]);
            }
        }
        else
        {
            // 8-byte slots: two x-adjacent slots per thread, one 16-byte store
            const int pair = threadIdx.x & 31; // lx = 2 * (pair & 3), ly = pair >> 2
            const int lxy = (pair >> 2) * 8 + 2 * (pair & 3);
            const int base = (pair >> 2) * kPackPitch + 2 * (pair & 3);
            for(int layer = threadIdx.x >> 5; layer < nRow * kApron; layer += 8)
            {
                const int j = layer / kApron, lz = layer - j * kApron;
                const int t = lz * (kApron * kPackPitch) + base + 8 * j;
                const float a0 = valS[t], a1 = valS[t + 1], a2 = valS[t + 2];
                const float b0 = valS[t + kPackPitch], b1 = valS[t + kPackPitch + 1], b2 = valS[t + kPackPitch + 2];
                uint32_t w[4];
                pack_pair<DT>(a0, a1, w[0]);
                pack_pair<DT>(b0, b1, w[1]);
                pack_pair<DT>(a1, a2, w[2]);
                pack_pair<DT>(b1, b2, w[3]);
                // x-adjacent slots (lx even, lx + 1) are adjacent in Morton order too
                const size_t slot = (brick0 + j) * kSlotsPerBrick + morton_slot(lxy & 7, lxy >> 3, lz); // even
                reinterpret_cast<uint4*>(p.out)[slot >> 1] = make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
    }

    void launch_source_bricks(const SourceBrickParams& p, cudaStream_t s)
    {
        if(p.ncomp == 1)
        {
            const dim3 grid((p.g.nb[0] + kPackRow - 1) / kPackRow, p.g.nb[1], p.g.nb[2]);
            const bool simple = p.fdim == 1 && !p.applyChain;
            if(p.dtype == 1)
                simple ? k_source_bricks_row<1, true><<<grid, 256, 0, s>>>(p) : k_source_bricks_row<1, false><<<grid, 256, 0, s>>>(p);
            else if(p.dtype == 2)
                simple ? k_source_bricks_row<2, true><<<grid, 256, 0, s>>>(p) : k_source_bricks_row<2, false><<<grid, 256, 0, s>>>(p);
            else
                simple ? k_source_bricks_row<0, true><<<grid, 256, 0, s>>>(p) : k_source_bricks_row<0, false><<<grid, 256, 0, s>>>(p);
            return;
        }
        dim3 grid(p.g.nb[0], p.g.nb[1], p.g.nb[2]);
        if(p.dtype == 1)
            k_source_bricks<1><<<grid, 256, 0, s>>>(p);
        else if(p.dtype == 2)
            k_source_bricks<2><<<grid, 256, 0, s>>>(p);
        else
            k_source_bricks<0><<<grid, 256, 0, s>>>(p);
    }

    // ---------------------------------------------------------------- diagnostics
    __global__ void k_unbrick(Geom g, const uint4* __restrict__ q, uint32_t* __restrict__ out)
    {
        const size_t n = size_t(g.ls[0]) * g.ls[1] * g.ls[2];
        for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        {
            const int x = int(i % g.ls[0]);
            const int y = int((i / g.ls[0]) % g.ls[1]);
            const int z = int(i / (size_t(g.ls[0]) * g.ls[1]));
            out[i] = quad_texel(__ldg(q + brick_slot(g, x, y, z)), 0);
        }
    }

    void launch_unbrick(const Geom& g, const uint4* volQ, uint32_t* out, cudaStream_t s)
    {
        k_unbrick<<<148 * 8, 256, 0, s>>>(g, volQ, out);
    }
} // namespace isaacb
