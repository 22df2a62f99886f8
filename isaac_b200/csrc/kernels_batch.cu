// Many views of one or more contexts (e.g. the timesteps of a simulation) in
// one persistent launch.  No counterpart in the reference, which renders one
// view per doVisualization (lib/isaac.hpp:2008-2061).
//
// Every CTA pulls 32x8-pixel-sized tiles (any 256-pixel shape) from an atomic
// work queue over all views, stages the tile's view and context in shared
// memory, and renders each pixel exactly as the single-view pipeline does for a
// volume-only context: clear (ClearBufferKernel), shading of the empty G-buffer
// (ShadingKernel) and the combined volume march.  The frames are therefore
// bit-identical to isaacb_render's.
#include "isaacb_frame.cuh"
#include "isaacb_march.cuh"

#include <cfloat>

namespace isaacb
{
    template<bool LINEAR, bool SKIP>
    __device__ __forceinline__ uchar4 batch_pixel(const BatchCtx& c, const View& v, int px, int py, unsigned long long& n)
    {
        uchar4 col = to_byte4(c.bgSwizzled);
        float depth = FLT_MAX;
        const ShadeParams sp{c.renderMode, c.aoWeight, c.bg};
        shade_values(sp, v, c.g, px, py, col, f3(0, 0, 0), 0.0f, depth);
        if(!c.volume)
            return col;
        Ray ray = pixel_to_ray(v, c.g, px, py);
        if(!clip_ray(ray, v, c.g))
            return col;
        ray.endDepth = gmin(ray.endDepth, depth);
        if(ray.endDepth <= ray.startDepth)
            return col;
        const March m = march_setup(ray, c.g, v.scale, c.step);
        const float factor = m.factor * c.totalWeightAll;
        const VolTexRef tex{c.g, c.volQ, c.volFlag};
        float4 color;
        if(LINEAR && march_in_range(c.g, m))
            color = march_combined<LINEAR, false, SKIP>(tex, m, factor, n);
        else
            color = march_combined<LINEAR, true, SKIP>(tex, m, factor, n);
        const float4 solid = from_byte4(col);
        const float r = 1.0f - color.w;
        color = make_float4(color.x + r * solid.x, color.y + r * solid.y, color.z + r * solid.z, color.w + r * solid.w);
        return to_byte4(color);
    }

    __global__ void __launch_bounds__(256) k_batch(const __grid_constant__ BatchParams bp)
    {
        __shared__ View sv;
        __shared__ BatchCtx sc;
        __shared__ int sTile, sView;
        unsigned long long n = 0;
        const int t = threadIdx.x;
        // pixel of this thread inside a tile: warps cover 8x4 blocks
        const int warpsX = bp.tileW / 8;
        const int w = t >> 5, l = t & 31;
        const int ox = (w % warpsX) * 8 + (l & 7), oy = (w / warpsX) * 4 + (l >> 3);
        for(;;)
        {
            if(t == 0)
            {
                const int tile = atomicAdd(bp.counter, 1);
                int v = -1;
                if(tile < bp.totalTiles)
                    for(int i = 0; i < bp.nViews; ++i)
                        if(tile >= bp.views[i].tileBase && tile < bp.views[i].tileBase + bp.views[i].tiles)
                        {
                            v = i;
                            break;
                        }
                sTile = tile;
                sView = v;
            }
            __syncthreads();
            const int tile = sTile, vi = sView;
            if(tile >= bp.totalTiles || vi < 0)
                break;
            const BatchView& bv = bp.views[vi];
            // stage the view and its context in shared memory
            {
                const int* src = reinterpret_cast<const int*>(&bp.ctxs[bv.ctx]);
                int* dst = reinterpret_cast<int*>(&sc);
                for(int i = t; i < int(sizeof(BatchCtx) / 4); i += blockDim.x)
                    dst[i] = src[i];
                if(t < 16)
                    sv.inv[t] = bv.inv[t];
                if(t == 0)
                {
                    sv.W = bv.W;
                    sv.H = bv.H;
                }
            }
            __syncthreads();
            if(t == 0)
            {
                sv.scale = sc.scale;
                sv.clipCount = sc.clipCount;
            }
            for(int i = t; i < kMaxClip * 3; i += blockDim.x)
            {
                sv.clipPos[i / 3][i % 3] = sc.clipPos[i / 3][i % 3];
                sv.clipNrm[i / 3][i % 3] = sc.clipNrm[i / 3][i % 3];
            }
            __syncthreads();
            const int local = tile - bv.tileBase;
            const int px = (local % bv.tilesX) * bp.tileW + ox;
            const int py = (local / bv.tilesX) * bp.tileH + oy;
            if(px < sv.W && py < sv.H)
            {
                uchar4 c;
                // auto (-1): skip when the context's last merge found empty bricks
                const bool skip = sc.skipEmpty >= 0 ? sc.skipEmpty != 0 : __ldg(sc.emptyCount) != 0u;
                if(sc.interpolation)
                    c = skip ? batch_pixel<true, true>(sc, sv, px, py, n) : batch_pixel<true, false>(sc, sv, px, py, n);
                else
                    c = skip ? batch_pixel<false, true>(sc, sv, px, py, n) : batch_pixel<false, false>(sc, sv, px, py, n);
                bv.out[size_t(py) * sv.W + px] = c;
            }
            __syncthreads();
        }
        if(bp.samples)
            count_samples(bp.samples, n);
    }

    void launch_batch(const BatchParams& p, int blocks, cudaStream_t s)
    {
        k_batch<<<blocks, 256, 0, s>>>(p);
    }

    int batch_max_blocks_per_sm()
    {
        int n = 0;
        if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch, 256, 0) != cudaSuccess)
            return 1;
        return n > 0 ? n : 1;
    }
} // namespace isaacb
