// Internal launch interface between the C-ABI host code (api.cu) and the
// kernel translation units.  Not installed; not part of the C ABI.
#pragma once

#include <algorithm>

#include "isaacb_device.cuh"

#include <cstdint>
#include <cuda_runtime.h>

namespace isaacb
{
    // -------------------------------------------------------------- merge / update
    struct MergeParams
    {
        Geom g;
        int32_t nVol;
        int32_t ts;
        int32_t ditherMode;
        int32_t writeIso;
        const float* src[kMaxSources];
        int32_t fdim[kMaxSources];
        Chain chain[kMaxSources];
        int32_t chainIdem[kMaxSources]; // 1: every functor is idem, the value is the x component
        const float4* lut; // nTotal * ts, source s at s*ts
        float4* lutPre; // scratch of nTotal * ts: weighted premultiplied entries of the scalar merge
        float weight[kMaxSources];
        float iso[kMaxSources];
        float totalWeight;
        float invTotalWeight; // 2^-k when totalWeight == 2^k exactly, else 0
        int32_t nonNegative; // every colour sum is finite and >= 0 (tables and weights >= 0, total > 0)
        const uint8_t* adv[kMaxSources]; // field sources: advection texture (guarded, x fastest), else null
        int32_t advG[3]; // the advection textures' guard band per axis
        uint32_t* volLin; // combined volume RGBA8, linear (merge scratch between the two passes)
        uint4* volQ; // combined volume, quad bricks
        uint32_t* isoAQ; // combined iso alpha, quad bricks
        uint32_t* isoLin; // combined iso RGBA8, linear
        uint8_t* volFlag; // per brick: 1 if any texel (apron included) is non-zero
        uint8_t* isoFlag; // per brick: max alpha byte (apron included)
        unsigned int* emptyBricks; // count of all-zero bricks (zeroed by the host before the merge)
    };
    // CTAs of `kernel` that fit on one SM with `threads` threads and `dynSmem` bytes of
    // dynamic shared memory (registers, threads, shared memory; at most 4)
    template<class K>
    inline int ctas_per_sm(K kernel, int threads, size_t dynSmem)
    {
        cudaFuncAttributes fa{};
        int dev = 0, smemSm = 0, reserved = 0, regsSm = 0, thrSm = 0;
        if(cudaFuncGetAttributes(&fa, kernel) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess)
            return 1;
        cudaDeviceGetAttribute(&smemSm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
        cudaDeviceGetAttribute(&regsSm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&thrSm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
        const size_t perCta = dynSmem + fa.sharedSizeBytes + size_t(reserved);
        int n = perCta ? int(size_t(smemSm) / perCta) : 4;
        const int warps = (threads + 31) / 32;
        const int regsPerWarp = ((fa.numRegs * 32 + 255) / 256) * 256;
        if(regsPerWarp > 0)
            n = std::min(n, regsSm / (regsPerWarp * warps));
        n = std::min(n, thrSm / (warps * 32));
        return std::max(1, std::min(n, 4));
    }

    // returns the number of kernels it launched
    int launch_merge(const MergeParams& p, cudaStream_t s);

    // field-source advection (kernels_merge.cu)
    struct NoiseParams
    {
        int LX, LY, LZ;
        float scale[3];
        int seedPoints;
    };
    // noise texture: Halton seeds, three 7-tap blur passes, x30 clamped (tmp: scratch of the same size)
    void launch_noise(const NoiseParams& p, float* noise, float* tmp, cudaStream_t s);
    struct AdvectParams
    {
        const float* field; // float3 per voxel, x fastest
        const uint8_t* back; // last frame's advection texture
        uint8_t* out;
        const float* noise;
        int LX, LY, LZ;
        int G[3]; // guard band of the advection textures, (L + 2G) per axis, x fastest
        float scale[3];
        float stepSize; // step factor * ISAAC_MAX_ADVECTION_STEP_SIZE
        float historyWeight;
        int seedNoise; // 1: this step adds the noise (timeStep % period < seeding time)
    };
    void launch_advect(const AdvectParams& p, cudaStream_t s);

    // one guard slab of an advection texture (the reference's SyncToOwnGuard /
    // SyncFromNeighbourGuard): direction d, slab extent e (G across d, L along it)
    struct GuardParams
    {
        uint8_t* tex; // guarded advection texture
        uint8_t* slab; // e[0] * e[1] * e[2] bytes, x fastest
        int L[3], G[3];
        int d[3], e[3];
    };
    void launch_pack_guard(const GuardParams& p, cudaStream_t s);
    void launch_unpack_guard(const GuardParams& p, cudaStream_t s);

    // per-source renderer bricks: persistent sources keep their raw components,
    // non-persistent sources their functor-chain value (UpdatePersistendTextureKernel)
    struct SourceBrickParams
    {
        Geom g;
        const float* src;
        int32_t fdim; // components of the source
        int32_t ncomp; // components stored (fdim or 1)
        int32_t applyChain;
        int32_t dtype; // 0 f32, 1 bf16, 2 f16
        Chain chain;
        void* out; // slots of ncomp*4 elements, component major
    };
    void launch_source_bricks(const SourceBrickParams& p, cudaStream_t s);
    // interior of a source with `guard` cells per side ((X+2g)(Y+2g)(Z+2g) voxels, x fastest)
    // into a compact X*Y*Z copy, fdim floats per voxel
    void launch_compact_guarded(const float* src, float* dst, int X, int Y, int Z, int guard, int fdim, cudaStream_t s);

    // quad bricks -> linear RGBA8 (diagnostics)
    void launch_unbrick(const Geom& g, const uint4* volQ, uint32_t* out, cudaStream_t s);

    // -------------------------------------------------------------- min / max
    struct MinMaxParams
    {
        Geom g;
        const float* src;
        int32_t fdim;
        Chain chain;
        // particles
        const uint32_t* offsets;
        const float* attr;
        int32_t particle;
        float* partial; // 2 floats per block
        unsigned long long* keys; // 4 keys: first +0 / -0 for min and max
    };
    int minmax_blocks(const MinMaxParams& p);
    void launch_minmax(const MinMaxParams& p, int blocks, float* result, cudaStream_t s);
    void launch_minmax_zero_keys(const MinMaxParams& p, cudaStream_t s);

    // -------------------------------------------------------------- frame
    struct ParticleSrc
    {
        const uint32_t* offsets;
        const float* pos;
        const float* attr;
        const float* radius;
        float constRadius;
        int32_t fdim;
        float weight;
        int32_t lutBase;
        Chain chain;
    };

    struct PerSourceSrc
    {
        const void* bricks;
        int32_t dtype;
        int32_t ncomp;
        int32_t persistent;
        int32_t fdim;
        float weight;
        float iso;
        Chain chain;
    };

    struct FrameParams
    {
        View v;
        Geom g;
        int32_t ts;
        int32_t interpolation;
        float step;
        float4 bgSwizzled; // (bg[3], bg[2], bg[1], 0)
        float4 bg;
        int32_t renderMode;
        float aoWeight;
        int32_t aoFilter;
        // SSAO taps: 0 = the reference's 7x7 grid at 10 px; else aoSamples pixel offsets
        // (x, y pairs in aoOffsets), normalised by aoSamples * 42/48 like the grid's 42
        int32_t aoSamples;
        int8_t aoOffsets[2 * kMaxAoSamples];
        float totalWeightAll;
        // all-zero bricks counted by the last merge of the combined texture (device memory,
        // written earlier on the same stream): the volume march skips empty bricks when it
        // is nonzero, a choice made on the GPU so that it always matches the texture
        const unsigned int* emptyCount;
        const float4* lut;
        // combined textures
        const uint4* volQ;
        const uint32_t* isoAQ;
        const uint32_t* isoLin;
        const uint8_t* volFlag;
        const uint8_t* isoFlag;
        // particles
        int32_t nVol;
        int32_t nPart;
        float3 pscale;
        ParticleSrc part[kMaxSources];
        // per-source renderer
        PerSourceSrc ps[kMaxSources];
        float4* psPre; // scratch: the weighted premultiplied tables of the active sources
        float negZero; // -0.0f, the addend of packed products that must round on their own (f2p_mul_exact)
        // G-buffer
        uchar4* color;
        float* depth;
        float* normal; // 3 floats per pixel
        float* ao;
        unsigned long long* counters; // [0] volume samples, [1] iso samples; null = off
    };

    // -------------------------------------------------------------- batched views
    // one context (e.g. one timestep) of a batch: its texture and frame settings
    struct BatchCtx
    {
        Geom g;
        const uint4* volQ;
        const uint8_t* volFlag;
        float step;
        float totalWeightAll;
        int32_t interpolation;
        int32_t skipEmpty; // 0 or 1, or -1: skip when *emptyCount (the last merge's all-zero bricks) is nonzero
        const unsigned int* emptyCount;
        int32_t volume; // totalWeightAll > 0
        int32_t renderMode;
        float aoWeight;
        float4 bg;
        float4 bgSwizzled;
        float3 scale;
        int32_t clipCount;
        float clipPos[kMaxClip][3];
        float clipNrm[kMaxClip][3];
    };
    // one view of a batch: camera inverse, size, context and output
    struct BatchView
    {
        float inv[16];
        int32_t W, H;
        int32_t ctx;
        int32_t tilesX;
        int32_t tileBase;
        int32_t tiles;
        uchar4* out;
    };
    struct BatchParams
    {
        const BatchCtx* ctxs;
        const BatchView* views;
        int32_t nViews;
        int32_t totalTiles;
        int32_t tileW, tileH; // tileW * tileH == 256, tileW % 8 == 0, tileH % 4 == 0
        int32_t* counter; // work queue head, zero before the launch
        unsigned long long* samples; // optional sample counter
    };
    void launch_batch(const BatchParams& p, int blocks, cudaStream_t s);
    int batch_max_blocks_per_sm();

    void launch_clear_particles(const FrameParams& p, cudaStream_t s);
    void launch_iso(const FrameParams& p, cudaStream_t s);
    void launch_iso_per_source(const FrameParams& p, cudaStream_t s);
    void launch_ssao(const FrameParams& p, cudaStream_t s);
    void launch_shade_volume(const FrameParams& p, bool volume, cudaStream_t s);
    // returns the number of kernels it launched
    int launch_shade_volume_per_source(const FrameParams& p, cudaStream_t s);
} // namespace isaacb
