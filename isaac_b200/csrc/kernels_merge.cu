// Buffer update kernels: the merge of all volume sources into the combined
// RGBA8 volume / iso textures (MergeToCombinedTextureKernel,
// lib/isaac/isaac_common_kernel.hpp:553-759) and the per-source bricks of the
// per-source renderer (UpdatePersistendTextureKernel,
// lib/isaac/isaac_common_kernel.hpp:432-451).
//
// One CTA builds one quad-packed apron brick.  It evaluates the 9^3 texels of
// the brick (its 8^3 voxels plus the apron on the low side, clamped at the
// volume border) once into shared memory, then writes the 576 slots as
// coalesced 16-byte stores.  The per-brick flags feed empty-space skipping.
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

    // ---------------------------------------------------------------- TMA / mbarrier helpers
    __device__ __forceinline__ uint32_t smem_u32(const void* p)
    {
        return static_cast<uint32_t>(__cvta_generic_to_shared(p));
    }
    __device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t phase)
    {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred P;\n mbarrier.test_wait.parity.shared::cta.b64 P, [%1], %2;\n selp.u32 %0, 1, 0, P;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        return done != 0;
    }
    // bounded wait: about 0.5 s at most, then false
    __device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t phase)
    {
        for(int it = 0; it < (1 << 22); ++it)
        {
            if(mbar_test(bar, phase))
                return true;
            __nanosleep(100);
        }
        return false;
    }

    // The 9^3 texels of one brick.  Each thread owns up to three texels (t, t+256,
    // t+512) and keeps their colour sums in registers while the sources are visited
    // in the outer loop, so per-source state (chain, table, weights) is uniform and
    // loaded once.  fetch(s, x, y, z, v) reads a clamped voxel.
    template<bool ISO, class Fetch>
    __device__ __forceinline__ void merge_brick(
        const MergeParams& p,
        int bx,
        int by,
        int bz,
        uint32_t* volS,
        uint32_t* isoS,
        int& anyVol,
        int& myIsoMax,
        const uint8_t* mask,
        Fetch fetch)
    {
        constexpr int kPer = 3;
        constexpr int kTex = kApron * kApron * kApron;
        const Geom& g = p.g;
        int xs[kPer], ys[kPer], zs[kPer];
        float4 vc[kPer], ic[kPer];
#pragma unroll
        for(int j = 0; j < kPer; ++j)
        {
            const int t = min(int(threadIdx.x) + 256 * j, kTex - 1);
            const int lx = t % kApron, ly = (t / kApron) % kApron, lz = t / (kApron * kApron);
            xs[j] = iclamp(bx * 8 - 1 + lx, 0, g.ls[0] - 1);
            ys[j] = iclamp(by * 8 - 1 + ly, 0, g.ls[1] - 1);
            zs[j] = iclamp(bz * 8 - 1 + lz, 0, g.ls[2] - 1);
            vc[j] = make_float4(0, 0, 0, 0);
            ic[j] = make_float4(0, 0, 0, 0);
        }
        const int nMine = int(threadIdx.x) + 512 < kTex ? 3 : 2; // 729 texels over 256 threads
        for(int s = 0; s < p.nVol; ++s)
        {
            const float vw = p.weight[s];
            const float it = p.iso[s];
            if(!(vw + it > 0.0f))
                continue;
            const float4* lut = p.lut + size_t(s) * p.ts;
            const uint8_t* adv = p.adv[s];
            auto accumulate = [&](int j, float val) {
                float4 c = __ldg(lut + lut_index_fast(val, p.ts));
                if(adv)
                {
                    // field source: alpha blended with the advection texture
                    // (MergeAdvectionToCombinedTextureIterator, isaac_common_kernel.hpp:664-665)
                    const size_t vox = (size_t(zs[j]) * g.ls[1] + ys[j]) * g.ls[0] + xs[j];
                    c.w *= float(__ldg(adv + vox)) / 255.0f;
                }
                if(vw > 0.0f)
                {
                    const float a = c.w * vw;
                    vc[j].x += c.x * a;
                    vc[j].y += c.y * a;
                    vc[j].z += c.z * a;
                    vc[j].w += a;
                }
                if(ISO && it > 0.0f)
                {
                    const float a = c.w / it * 0.5f;
                    if(ic[j].w < a)
                        ic[j] = make_float4(c.x, c.y, c.z, a);
                }
            };
            if(p.chainIdem[s] != 0)
            {
                // all functors idem: the value is the first component
#pragma unroll
                for(int j = 0; j < kPer; ++j)
                {
                    if(j < nMine)
                        accumulate(j, fetch.first(s, xs[j], ys[j], zs[j]));
                }
            }
            else
            {
#pragma unroll
                for(int j = 0; j < kPer; ++j)
                {
                    if(j < nMine)
                    {
                        float v[4];
                        fetch(s, xs[j], ys[j], zs[j], v);
                        accumulate(j, apply_chain(v, p.fdim[s], p.chain[s]));
                    }
                }
            }
        }
#pragma unroll
        for(int j = 0; j < kPer; ++j)
        {
            if(j >= nMine)
                break;
            const int t = int(threadIdx.x) + 256 * j;
            float4 c = vc[j];
            if(p.invTotalWeight != 0.0f)
            {
                // totalWeight is a power of two: x * 2^-k is the correctly rounded x / 2^k
                c = make_float4(c.x * p.invTotalWeight, c.y * p.invTotalWeight, c.z * p.invTotalWeight, c.w * p.invTotalWeight);
            }
            else
            {
                c = make_float4(c.x / p.totalWeight, c.y / p.totalWeight, c.z / p.totalWeight, c.w / p.totalWeight);
            }
            const uint32_t vb = p.nonNegative ? dither_rgba_nonneg(p.ditherMode, mask, xs[j], ys[j], zs[j], c)
                                              : dither_rgba(p.ditherMode, mask, xs[j], ys[j], zs[j], c);
            volS[t] = vb;
            anyVol |= vb != 0u;
            if(ISO)
            {
                const float4 q = ic[j];
                const uint32_t ib = round_byte(q.x) | (round_byte(q.y) << 8) | (round_byte(q.z) << 16) | (round_byte(q.w) << 24);
                isoS[t] = ib;
                myIsoMax = max(myIsoMax, int(ib >> 24));
            }
        }
    }

    // merge_brick for the common case of scalar sources with all-idem chains staged by
    // TMA: one tile offset per texel serves every source, the value is one shared-memory
    // load, and the source loop has no per-source layout arithmetic.  Same operations in
    // the same order as merge_brick, so the bytes are identical.
    template<bool ISO>
    __device__ __forceinline__ void merge_brick_scalar(
        const MergeParams& p,
        int bx,
        int by,
        int bz,
        uint32_t* volS,
        uint32_t* isoS,
        int& anyVol,
        int& myIsoMax,
        const uint8_t* mask,
        const unsigned char* tiles,
        int x0,
        int y0,
        int z0)
    {
        constexpr int kPer = 3;
        constexpr int kTex = kApron * kApron * kApron;
        const Geom& g = p.g;
        int xs[kPer], ys[kPer], zs[kPer], off[kPer];
        float4 vc[kPer], ic[kPer];
#pragma unroll
        for(int j = 0; j < kPer; ++j)
        {
            const int t = min(int(threadIdx.x) + 256 * j, kTex - 1);
            const int lz = t / (kApron * kApron);
            const int r = t - lz * (kApron * kApron);
            const int ly = r / kApron, lx = r - ly * kApron;
            xs[j] = iclamp(bx * 8 - 1 + lx, 0, g.ls[0] - 1);
            ys[j] = iclamp(by * 8 - 1 + ly, 0, g.ls[1] - 1);
            zs[j] = iclamp(bz * 8 - 1 + lz, 0, g.ls[2] - 1);
            off[j] = ((zs[j] - z0) * kApron + (ys[j] - y0)) * 16 + (xs[j] - x0);
            vc[j] = make_float4(0, 0, 0, 0);
            ic[j] = make_float4(0, 0, 0, 0);
        }
        const int nMine = int(threadIdx.x) + 512 < kTex ? 3 : 2;
        const int ts = p.ts;
        for(int s = 0; s < p.nVol; ++s)
        {
            const float vw = p.weight[s];
            const float it = p.iso[s];
            if(!(vw + it > 0.0f))
                continue;
            const float* tile = reinterpret_cast<const float*>(tiles + p.tileOffset[s]);
            const float4* lut = p.lut + size_t(s) * ts;
#pragma unroll
            for(int j = 0; j < kPer; ++j)
            {
                if(j >= nMine)
                    break;
                const float4 c = __ldg(lut + lut_index_fast(tile[off[j]], ts));
                if(vw > 0.0f)
                {
                    const float a = c.w * vw;
                    vc[j].x += c.x * a;
                    vc[j].y += c.y * a;
                    vc[j].z += c.z * a;
                    vc[j].w += a;
                }
                if(ISO && it > 0.0f)
                {
                    const float a = c.w / it * 0.5f;
                    if(ic[j].w < a)
                        ic[j] = make_float4(c.x, c.y, c.z, a);
                }
            }
        }
#pragma unroll
        for(int j = 0; j < kPer; ++j)
        {
            if(j >= nMine)
                break;
            const int t = int(threadIdx.x) + 256 * j;
            float4 c = vc[j];
            if(p.invTotalWeight != 0.0f)
                c = make_float4(c.x * p.invTotalWeight, c.y * p.invTotalWeight, c.z * p.invTotalWeight, c.w * p.invTotalWeight);
            else
                c = make_float4(c.x / p.totalWeight, c.y / p.totalWeight, c.z / p.totalWeight, c.w / p.totalWeight);
            const uint32_t vb = p.nonNegative ? dither_rgba_nonneg(p.ditherMode, mask, xs[j], ys[j], zs[j], c)
                                              : dither_rgba(p.ditherMode, mask, xs[j], ys[j], zs[j], c);
            volS[t] = vb;
            anyVol |= vb != 0u;
            if(ISO)
            {
                const float4 q = ic[j];
                const uint32_t ib = round_byte(q.x) | (round_byte(q.y) << 8) | (round_byte(q.z) << 16) | (round_byte(q.w) << 24);
                isoS[t] = ib;
                myIsoMax = max(myIsoMax, int(ib >> 24));
            }
        }
    }

    // voxel readers of merge_brick: the TMA-staged tile in shared memory, or global memory
    struct TileFetch
    {
        const MergeParams& p;
        const unsigned char* tiles;
        int x0, y0, z0;
        __device__ __forceinline__ const float* at(int s, int x, int y, int z) const
        {
            const int fd = p.fdim[s];
            const float* tile = reinterpret_cast<const float*>(tiles + p.tileOffset[s]);
            return tile + ((z - z0) * kApron + (y - y0)) * (16 * fd) + (x - x0) * fd;
        }
        __device__ __forceinline__ float first(int s, int x, int y, int z) const
        {
            return *at(s, x, y, z);
        }
        __device__ __forceinline__ void operator()(int s, int x, int y, int z, float (&v)[4]) const
        {
            const int fd = p.fdim[s];
            const float* q = at(s, x, y, z);
            v[0] = q[0];
            v[1] = fd > 1 ? q[1] : 0.0f;
            v[2] = fd > 2 ? q[2] : 0.0f;
            v[3] = fd > 3 ? q[3] : 0.0f;
        }
    };
    struct GlobalFetch
    {
        const MergeParams& p;
        __device__ __forceinline__ size_t idx(int x, int y, int z) const
        {
            return (size_t(z) * p.g.ls[1] + y) * p.g.ls[0] + x;
        }
        __device__ __forceinline__ float first(int s, int x, int y, int z) const
        {
            return __ldg(p.src[s] + idx(x, y, z) * p.fdim[s]);
        }
        __device__ __forceinline__ void operator()(int s, int x, int y, int z, float (&v)[4]) const
        {
            read_voxel(p.src[s], p.fdim[s], idx(x, y, z), v);
        }
    };

    // One CTA per brick.  With TMA, thread 0 stages each active source's region
    // [8b-4, 8b+12) x [8b-1, 8b+8) x [8b-1, 8b+8) (the x start rounded down to a
    // 16-byte boundary; out-of-volume elements are never read) into shared memory
    // with one cp.async.bulk.tensor per source, completing on an mbarrier.
    template<bool TMA, bool ISO>
    __global__ void __launch_bounds__(256, 5) k_merge(const __grid_constant__ MergeParams p)
    {
        extern __shared__ __align__(128) unsigned char dsm[];
        __shared__ uint32_t volS[kApron * kApron * kApron];
        __shared__ uint32_t isoS[kApron * kApron * kApron];
        __shared__ int isoMax;
        __shared__ __align__(8) unsigned long long mbar;
        __shared__ uint8_t sMask[64];
        if(threadIdx.x < 64)
            sMask[threadIdx.x] = p.ditherMode == 2 ? c_dither2[threadIdx.x] : c_dither1[threadIdx.x];
        const Geom& g = p.g;
        const int bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z;
        const int x0 = bx * 8 - 4, y0 = by * 8 - 1, z0 = bz * 8 - 1;
        const uint32_t bar = smem_u32(&mbar);
        // tiles start on a 128-byte boundary of the dynamic shared memory (128 spare bytes requested)
        unsigned char* tiles = dsm + ((128u - (smem_u32(dsm) & 127u)) & 127u);
        if(threadIdx.x == 0)
        {
            isoMax = 0;
            if(TMA)
            {
                asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1) : "memory");
                asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            }
        }
        __syncthreads();
        if(TMA)
        {
            if(threadIdx.x == 0)
            {
                asm volatile(
                    "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(p.txBytes) : "memory");
                for(int s = 0; s < p.nVol; ++s)
                {
                    if(p.tileOffset[s] < 0)
                        continue;
                    const uint32_t dst = smem_u32(tiles + p.tileOffset[s]);
                    const uint64_t map = reinterpret_cast<uint64_t>(&p.tmap[s]);
                    asm volatile(
                        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                        :
                        : "r"(dst), "l"(map), "r"(x0 * p.fdim[s]), "r"(y0), "r"(z0), "r"(bar)
                        : "memory");
                }
            }
            if(!mbar_wait_bounded(bar, 0))
            {
                atomicOr(p.errorFlag, 1);
                // let the copies land before the block's shared memory is released
                mbar_wait_bounded(bar, 0);
                return;
            }
        }
        int anyVol = 0;
        int myIsoMax = 0;
        if(TMA)
        {
            if(p.scalarIdem)
                merge_brick_scalar<ISO>(p, bx, by, bz, volS, isoS, anyVol, myIsoMax, sMask, tiles, x0, y0, z0);
            else
                merge_brick<ISO>(p, bx, by, bz, volS, isoS, anyVol, myIsoMax, sMask, TileFetch{p, tiles, x0, y0, z0});
        }
        else
        {
            merge_brick<ISO>(p, bx, by, bz, volS, isoS, anyVol, myIsoMax, sMask, GlobalFetch{p});
        }
        if(ISO)
            atomicMax(&isoMax, myIsoMax);
        anyVol = __syncthreads_or(anyVol);
        const size_t brick = (size_t(bz) * g.nb[1] + by) * g.nb[0] + bx;
        if(threadIdx.x == 0)
        {
            p.volFlag[brick] = anyVol ? 1 : 0;
            if(!anyVol)
                atomicAdd(p.emptyBricks, 1u);
            if(ISO)
                p.isoFlag[brick] = uint8_t(isoMax);
        }
        for(int s = threadIdx.x; s < kSlotsPerBrick; s += blockDim.x)
        {
            const int lx = s & 7, ly = (s >> 3) & 7, lz = s >> 6;
            const int t = (lz * kApron + ly) * kApron + lx;
            uint4 q = make_uint4(volS[t], volS[t + 1], volS[t + kApron], volS[t + kApron + 1]);
            p.volQ[brick * kSlotsPerBrick + s] = q;
            if(ISO)
            {
                uint32_t a = (isoS[t] >> 24) | ((isoS[t + 1] >> 24) << 8) | ((isoS[t + kApron] >> 24) << 16)
                    | ((isoS[t + kApron + 1] >> 24) << 24);
                p.isoAQ[brick * kSlotsPerBrick + s] = a;
            }
        }
        if(ISO)
        {
            // interior voxels 8b..8b+7 of this brick in the linear iso texture
            for(int t = threadIdx.x; t < 512; t += blockDim.x)
            {
                const int lx = t & 7, ly = (t >> 3) & 7, lz = t >> 6;
                const int x = bx * 8 + lx, y = by * 8 + ly, z = bz * 8 + lz;
                if(x < g.ls[0] && y < g.ls[1] && z < g.ls[2])
                    p.isoLin[(size_t(z) * g.ls[1] + y) * g.ls[0] + x]
                        = isoS[((lz + 1) * kApron + (ly + 1)) * kApron + (lx + 1)];
            }
        }
    }

    void launch_merge(const MergeParams& p, cudaStream_t s)
    {
        dim3 grid(p.g.nb[0], p.g.nb[1], p.g.nb[2]);
        if(p.useTma)
        {
            if(p.writeIso)
            {
                cudaFuncSetAttribute(k_merge<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, p.tileBytes + 128);
                k_merge<true, true><<<grid, 256, p.tileBytes + 128, s>>>(p);
            }
            else
            {
                cudaFuncSetAttribute(k_merge<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, p.tileBytes + 128);
                k_merge<true, false><<<grid, 256, p.tileBytes + 128, s>>>(p);
            }
        }
        else if(p.writeIso)
            k_merge<false, true><<<grid, 256, 0, s>>>(p);
        else
            k_merge<false, false><<<grid, 256, 0, s>>>(p);
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
        auto fetch = [&](int x, int y, int z) {
            // VALUE border 0 (the guard cells are zero too)
            if(x < 0 || y < 0 || z < 0 || x >= p.LX || y >= p.LY || z >= p.LZ)
                return 0.0f;
            return float(__ldg(p.back + (size_t(z) * p.LY + y) * p.LX + x));
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
            p.out[i] = uint8_t(min(max(ti + ((sv - fl) > d ? 1 : 0), 0), 255));
        }
    }

    void launch_advect(const AdvectParams& p, cudaStream_t s)
    {
        const size_t n = size_t(p.LX) * p.LY * p.LZ;
        k_advect<<<int(std::min<size_t>((n + 255) / 256, 148 * 16)), 256, 0, s>>>(p);
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
            const size_t base = (brick * kSlotsPerBrick + s) * per;
            for(int c = 0; c < p.ncomp; ++c)
            {
                store_elem<DT>(p.out, base + 4 * c + 0, valS[c][t]);
                store_elem<DT>(p.out, base + 4 * c + 1, valS[c][t + 1]);
                store_elem<DT>(p.out, base + 4 * c + 2, valS[c][t + kApron]);
                store_elem<DT>(p.out, base + 4 * c + 3, valS[c][t + kApron + 1]);
            }
        }
    }

    void launch_source_bricks(const SourceBrickParams& p, cudaStream_t s)
    {
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
            out[i] = reinterpret_cast<const uint32_t*>(q)[brick_slot(g, x, y, z) * 4];
        }
    }

    void launch_unbrick(const Geom& g, const uint4* volQ, uint32_t* out, cudaStream_t s)
    {
        k_unbrick<<<148 * 8, 256, 0, s>>>(g, volQ, out);
    }
} // namespace isaacb
