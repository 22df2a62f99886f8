// Convolutions as implicit GEMMs on the sm_100a tensor cores (tcgen05).
//
// Forward and input-gradient ("dgrad") passes share k_conv_gemm:
//   Y[p][n] = sum_k A[p][k] * Wp[n][k],  k = tap * Cg + c,
// where A is the im2col gather of the NHWC bf16 source (never materialised:
// each CTA gathers its 128-row x 64-column K-slices straight into shared
// memory with zero-filling cp.async), Wp is the packed bf16 weight matrix
// held whole in shared memory, and the FP32 accumulator lives in TMEM.  One
// thread issues the MMAs (M=128, N=Npad, K=16 per instruction) and commits
// them to per-stage mbarriers that recycle the shared-memory stages; the
// epilogue reads TMEM with tcgen05.ld and fuses bias, ReLU, the ReLU mask of
// the backward pass, accumulation into an existing gradient and the bf16 or
// FP32 store.  The gather has two forms:
//   forward     input pixel = out * stride - pad + tap
//   transposed  input pixel = (out + pad - tap) / stride when divisible
// The transposed form with the per-tap transposed weights is the gradient
// of the forward form with respect to its input.
//
// The weight gradient ("wgrad") is k_conv_wgrad:
//   dW[(tap, ci)][co] = sum_p X[in(p, tap)][ci] * dY[p][co]
// with both operands MN-major (channels contiguous in NHWC), the pixel axis
// as the reduction split over CTAs, and FP32 partial sums added atomically.
//
// Every mbarrier wait is bounded; on a timeout the kernel raises the error
// flag, stops issuing work, waits (bounded) for its MMAs and frees its TMEM.
#include "../../include/isaac_b200.h"
#include "isaacb_internal.h"
#include "isaacb_conv.h"
#include "isaacb_tc.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <algorithm>
#include <string>

namespace isaacb
{
    void set_global_error(const std::string& msg);

    namespace
    {
        using bf16 = __nv_bfloat16;
        constexpr int kThreads = 256;
        constexpr int kStages = 4;
        constexpr int kTileM = 128;
        constexpr int kChunkK = 64; // K elements per pipeline stage
        constexpr int kStageBytesA = kTileM * kChunkK * 2; // 16 KiB

        __host__ __device__ inline uint32_t tmem_columns(int n)
        {
            uint32_t c = 32;
            while(c < uint32_t(n))
                c <<= 1;
            return c;
        }

        __device__ __forceinline__ void raise_error(int* flag, bool& abortLocal)
        {
            abortLocal = true;
            if(flag)
                atomicExch(flag, 1);
        }

        __device__ __forceinline__ uint4 pack_bf16x8(const float (&v)[8])
        {
            uint4 o;
            __nv_bfloat162 h;
            h = __floats2bfloat162_rn(v[0], v[1]);
            o.x = *reinterpret_cast<uint32_t*>(&h);
            h = __floats2bfloat162_rn(v[2], v[3]);
            o.y = *reinterpret_cast<uint32_t*>(&h);
            h = __floats2bfloat162_rn(v[4], v[5]);
            o.z = *reinterpret_cast<uint32_t*>(&h);
            h = __floats2bfloat162_rn(v[6], v[7]);
            o.w = *reinterpret_cast<uint32_t*>(&h);
            return o;
        }
        __device__ __forceinline__ void unpack_bf16x8(uint4 u, float (&v)[8])
        {
            const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
            for(int i = 0; i < 4; ++i)
            {
                v[2 * i] = __uint_as_float(w[i] << 16);
                v[2 * i + 1] = __uint_as_float(w[i] & 0xFFFF0000u);
            }
        }

        // ------------------------------------------------------------------ forward / dgrad
        __global__ void __launch_bounds__(kThreads, 1) k_conv_gemm(const __grid_constant__ ConvGemmParams p)
        {
            extern __shared__ unsigned char dsm[];
            __shared__ uint32_t sTmem;
            __shared__ __align__(8) uint64_t sEmpty[kStages];
            __shared__ __align__(8) uint64_t sDone;
            unsigned char* base = dsm + ((128u - (tc::smem_addr(dsm) & 127u)) & 127u);
            const uint32_t sB = tc::smem_addr(base);
            const uint32_t sA = sB + uint32_t(p.Npad) * uint32_t(p.Kpad) * 2u;
            const int tid = threadIdx.x;
            const uint32_t cols = tmem_columns(p.Npad);
            if(tid < 32)
            {
                tc::tmem_alloc(&sTmem, cols);
                tc::tmem_relinquish();
            }
            if(tid == 0)
            {
                for(int s = 0; s < kStages; ++s)
                    tc::mbar_init(&sEmpty[s], 1);
                tc::mbar_init(&sDone, 1);
                tc::mbar_init_fence();
            }
            bool abortLocal = false, aborted = false;
            // the whole packed weight matrix, canonical K-major: core (n/8, k/8) at (n/8)*Kpad*16 + (k/8)*128
            {
                const int kb = p.Kpad / 8;
                const int pieces = p.Npad * kb;
                for(int i = tid; i < pieces; i += kThreads)
                {
                    const int n = i / kb, k8 = i - n * kb;
                    const uint32_t dst = sB + uint32_t(n >> 3) * uint32_t(p.Kpad) * 16u + uint32_t(k8) * 128u + uint32_t(n & 7) * 16u;
                    tc::cp_async16(dst, p.w + size_t(n) * p.Kpad + size_t(k8) * 8, 16);
                }
                tc::cp_async_commit();
                tc::cp_async_wait<0>();
                tc::fence_async_smem();
            }
            tc::fence_before_sync();
            __syncthreads();
            tc::fence_after_sync();
            const uint32_t tmem = sTmem;
            if(p.waitCheckNs != 0)
            {
                // failure-detection check: sDone has had no arrival, so this bounded wait
                // runs out; no copy or MMA is in flight when the TMEM is released
                if(tid == 0 && !tc::mbar_wait(&sDone, 0, p.waitCheckNs) && p.errorFlag)
                    atomicExch(p.errorFlag, 1);
                tc::fence_before_sync();
                __syncthreads();
                if(tid < 32)
                    tc::tmem_dealloc(tmem, cols);
                return;
            }

            const int P = p.B * p.Ho * p.Wo;
            const int nTiles = (P + kTileM - 1) / kTileM;
            const int nk = p.Kpad / kChunkK;
            const int taps = p.ks * p.ks;
            const int m = tid & (kTileM - 1);
            const int jBase = tid >> 7;
            const uint32_t idesc = tc::idesc_bf16(kTileM, p.Npad, false, false);
            const uint32_t sboB = uint32_t(p.Kpad) * 16u;
            uint32_t G0 = 0;
            uint32_t donePhase = 0;

            for(int tile = blockIdx.x; tile < nTiles; tile += gridDim.x)
            {
                const int pix = tile * kTileM + m;
                const bool valid = pix < P;
                int b = 0, oy = 0, ox = 0;
                if(valid)
                {
                    ox = pix % p.Wo;
                    const int t = pix / p.Wo;
                    oy = t % p.Ho;
                    b = t / p.Ho;
                }
                auto load_chunk = [&](int kc, uint32_t G) {
                    const uint32_t stage = sA + (G % kStages) * uint32_t(kStageBytesA);
#pragma unroll
                    for(int q = 0; q < 4; ++q)
                    {
                        const int j = jBase + 2 * q;
                        const int k = kc * kChunkK + j * 8;
                        const int t = k / p.Cg;
                        const int c = k - t * p.Cg;
                        const bf16* src = p.x;
                        uint32_t bytes = 0;
                        if(valid && t < taps)
                        {
                            const int ty = t / p.ks, tx = t - ty * p.ks;
                            int iy, ix;
                            bool ok;
                            if(!p.transposed)
                            {
                                iy = oy * p.stride - p.pad + ty;
                                ix = ox * p.stride - p.pad + tx;
                                ok = iy >= 0 && ix >= 0 && iy < p.H && ix < p.W;
                            }
                            else
                            {
                                const int ny = oy + p.pad - ty, nx = ox + p.pad - tx;
                                ok = ny >= 0 && nx >= 0 && (ny % p.stride) == 0 && (nx % p.stride) == 0;
                                iy = ny / p.stride;
                                ix = nx / p.stride;
                                ok = ok && iy < p.H && ix < p.W;
                            }
                            if(ok)
                            {
                                src = p.x + ((size_t(b) * p.H + iy) * p.W + ix) * p.Cg + c;
                                bytes = 16;
                            }
                        }
                        const uint32_t dst = stage + uint32_t(m >> 3) * 1024u + uint32_t(j) * 128u + uint32_t(m & 7) * 16u;
                        tc::cp_async16(dst, src, bytes);
                    }
                };

                for(int c = 0; c < kStages - 1; ++c)
                {
                    if(c < nk)
                    {
                        const uint32_t G = G0 + c;
                        if(G >= kStages && !tc::mbar_wait(&sEmpty[G % kStages], ((G / kStages) - 1) & 1))
                            raise_error(p.errorFlag, abortLocal);
                        load_chunk(c, G);
                    }
                    tc::cp_async_commit();
                }
                for(int kc = 0; kc < nk; ++kc)
                {
                    const int kn = kc + kStages - 1;
                    if(kn < nk)
                    {
                        const uint32_t G = G0 + kn;
                        if(G >= kStages && !tc::mbar_wait(&sEmpty[G % kStages], ((G / kStages) - 1) & 1))
                            raise_error(p.errorFlag, abortLocal);
                        load_chunk(kn, G);
                    }
                    tc::cp_async_commit();
                    tc::cp_async_wait<kStages - 1>();
                    tc::fence_async_smem();
                    if(__syncthreads_or(abortLocal))
                    {
                        aborted = true;
                        break;
                    }
                    if(tid == 0)
                    {
                        tc::fence_after_sync();
                        const uint32_t G = G0 + kc;
                        const uint32_t stage = sA + (G % kStages) * uint32_t(kStageBytesA);
#pragma unroll
                        for(int j = 0; j < kChunkK / 16; ++j)
                        {
                            const uint64_t ad = tc::smem_desc(stage + uint32_t(j) * 256u, 128u, 1024u);
                            const uint64_t bd = tc::smem_desc(sB + uint32_t(kc * 8 + 2 * j) * 128u, 128u, sboB);
                            tc::mma_bf16(tmem, ad, bd, idesc, (kc | j) != 0 ? 1u : 0u);
                        }
                        tc::mma_commit(&sEmpty[G % kStages]);
                    }
                }
                tc::cp_async_wait<0>();
                if(tid == 0)
                    tc::mma_commit(&sDone);
                if(!tc::mbar_wait(&sDone, donePhase))
                    raise_error(p.errorFlag, abortLocal);
                donePhase ^= 1u;
                G0 += uint32_t(nk);
                if(__syncthreads_or(abortLocal))
                {
                    aborted = true;
                    break;
                }
                tc::fence_after_sync();

                // epilogue: thread = TMEM lane = tile row; the two warpgroups split the columns
                {
                    const int warp = tid >> 5;
                    const uint32_t lane0 = uint32_t(warp & 3) * 32u;
                    const int half = warp >> 2;
                    const int cpw = p.Npad / 2;
                    for(int c0 = half * cpw; c0 < (half + 1) * cpw; c0 += 8)
                    {
                        float v[8];
                        tc::tmem_ld8(tmem + (lane0 << 16) + uint32_t(c0), v);
                        tc::tmem_wait_ld();
                        if(!valid || c0 >= p.Cout)
                            continue;
                        const size_t o = size_t(pix) * p.Cout + c0;
                        if(p.bias)
                        {
#pragma unroll
                            for(int i = 0; i < 8; ++i)
                                v[i] += __ldg(p.bias + c0 + i);
                        }
                        if(p.relu)
                        {
#pragma unroll
                            for(int i = 0; i < 8; ++i)
                                v[i] = fmaxf(v[i], 0.0f);
                        }
                        if(p.mask)
                        {
                            float mk[8];
                            unpack_bf16x8(__ldg(reinterpret_cast<const uint4*>(p.mask + o)), mk);
#pragma unroll
                            for(int i = 0; i < 8; ++i)
                                v[i] = mk[i] > 0.0f ? v[i] : 0.0f;
                        }
                        if(p.yf)
                        {
                            float4* dst = reinterpret_cast<float4*>(p.yf + o);
                            if(p.accumulate)
                            {
                                const float4 a = dst[0], bq = dst[1];
                                v[0] += a.x, v[1] += a.y, v[2] += a.z, v[3] += a.w;
                                v[4] += bq.x, v[5] += bq.y, v[6] += bq.z, v[7] += bq.w;
                            }
                            dst[0] = make_float4(v[0], v[1], v[2], v[3]);
                            dst[1] = make_float4(v[4], v[5], v[6], v[7]);
                        }
                        else
                        {
                            uint4* dst = reinterpret_cast<uint4*>(p.y + o);
                            if(p.accumulate)
                            {
                                float a[8];
                                unpack_bf16x8(*dst, a);
#pragma unroll
                                for(int i = 0; i < 8; ++i)
                                    v[i] += a[i];
                            }
                            *dst = pack_bf16x8(v);
                        }
                    }
                }
                tc::fence_before_sync();
                __syncthreads();
            }
            // drain: every MMA this CTA issued has completed before TMEM is released
            if(aborted)
            {
                if(tid == 0)
                    tc::mma_commit(&sDone);
                tc::mbar_wait(&sDone, donePhase);
            }
            tc::fence_before_sync();
            __syncthreads();
            if(tid < 32)
                tc::tmem_dealloc(tmem, cols);
        }

        // ------------------------------------------------------------------ row tiles
        // Convolutions of stride 1 (forward, or the input gradient with `transposed`) or
        // stride 2 (forward) whose gathered channel count is a multiple of 16.  A tile is
        // 128 consecutive output pixels of one image row.  Its input rows (ks of them)
        // are loaded into shared memory once, channel chunks of 8 stored as separate
        // runs of 16-byte pixels; for stride 2 each run is split into its even and odd
        // input columns.  Every tap then reads the same halo through a descriptor whose
        // start is shifted by the tap's column offset: the no-swizzle core matrix is 8
        // consecutive 16-byte rows, and consecutive output pixels are consecutive
        // entries of a run (of a parity plane for stride 2).  Warp roles:
        //   warps 0-3  epilogue (TMEM lane = pixel), double-buffered accumulators
        //   warps 4-7  producers: cp.async of the halo, arrival on the stage's mbarrier
        //   warp 8     one thread issues the MMAs and commits them
        // With TMA the halo comes in one tiled bulk-tensor load per run (a box of 8 channels
        // x the run's pixels) issued by one thread of warp 9, and warps 4-7 join the
        // epilogue: warps 0-3 take the first half of the accumulator columns, warps 4-7 the
        // second (a warp reads TMEM lanes 32*(w%4)..+31, so both groups see every pixel).
        constexpr int kRowThreads = 288;
        template<bool TMA>
        __host__ __device__ constexpr int row_threads()
        {
            return TMA ? 320 : kRowThreads;
        }

        struct RowGeom
        {
            int S; // stride: 1 or 2
            int HWp; // entries between runs (per parity plane for stride 2)
            int HWn; // entries a run needs (<= HWp; HWp is padded to 8 for TMA destinations)
            int stages; // halo buffers: 1 or 2
            int rowB; // swizzled staging: bytes per staged pixel (Cg * 2 = 32, 64 or 128); 0 = chunked runs
            // implicit concatenation by TMA (1x1, xUp): channel chunks of cwc (coarse) and cwf
            // (fine) channels, each staged as 128 swizzled rows; 0 = off
            int cwc, cwf;
        };

        __host__ __device__ inline RowGeom row_geom(int stride, int ks, int pad, int stages, bool tma = false)
        {
            RowGeom g;
            g.S = stride;
            g.HWn = stride == 1 ? kTileM + 2 * pad : kTileM + (ks - 1) / 2 + 1;
            // a TMA destination starts on a 128-byte boundary: runs of a multiple of 8 entries
            g.HWp = tma ? (g.HWn + 7) / 8 * 8 : g.HWn;
            g.stages = stages;
            g.rowB = 0;
            g.cwc = g.cwf = 0;
            return g;
        }

        // Epilogue of one 128-pixel output tile (row y of image b, column tile xt): this
        // thread's pixel px, accumulator columns [cBeg, cBeg + colsPer) of the TMEM tile at
        // tAcc (this warp's lanes); bias, ReLU, mask, then the bf16 / FP32 store.
        __device__ __forceinline__ void row_epilogue(
            const ConvGemmParams& p,
            uint32_t tAcc,
            int xt,
            int b,
            int y,
            int px,
            int cBeg,
            int colsPer,
            const float* sBias)
        {
            const int x = xt * kTileM + px;
            const bool valid = x < p.Wo;
            const size_t pix = (size_t(b) * p.Ho + y) * p.Wo + x;
            // 16 accumulator columns per TMEM wait (8 where a column group ends)
            for(int c16 = cBeg; c16 < cBeg + colsPer; c16 += 16)
            {
                const bool two = c16 + 16 <= cBeg + colsPer;
                float v[2][8];
                const uint32_t ta = tAcc + uint32_t(c16);
                tc::tmem_ld8(ta, v[0]);
                if(two)
                    tc::tmem_ld8(ta + 8u, v[1]);
                tc::tmem_wait_ld();
                if(!valid)
                    continue;
#pragma unroll
                for(int hh = 0; hh < 2; ++hh)
                {
                    const int c0 = c16 + 8 * hh;
                    if(c0 >= p.Cout || (hh == 1 && !two))
                        break;
                    float(&w)[8] = v[hh];
                    const size_t o = pix * p.Cout + c0;
                    if(p.bias)
                    {
#pragma unroll
                        for(int k = 0; k < 8; ++k)
                            w[k] += sBias[c0 + k];
                    }
                    if(p.relu)
                    {
#pragma unroll
                        for(int k = 0; k < 8; ++k)
                            w[k] = fmaxf(w[k], 0.0f);
                    }
                    if(p.mask)
                    {
                        float mk[8];
                        unpack_bf16x8(__ldg(reinterpret_cast<const uint4*>(p.mask + o)), mk);
#pragma unroll
                        for(int k = 0; k < 8; ++k)
                            w[k] = mk[k] > 0.0f ? w[k] : 0.0f;
                    }
                    if(p.yf)
                    {
                        float4* dst = reinterpret_cast<float4*>(p.yf + o);
                        if(p.accumulate)
                        {
                            const float4 u = dst[0], t2 = dst[1];
                            w[0] += u.x, w[1] += u.y, w[2] += u.z, w[3] += u.w;
                            w[4] += t2.x, w[5] += t2.y, w[6] += t2.z, w[7] += t2.w;
                        }
                        dst[0] = make_float4(w[0], w[1], w[2], w[3]);
                        dst[1] = make_float4(w[4], w[5], w[6], w[7]);
                    }
                    else
                    {
                        uint4* dst = reinterpret_cast<uint4*>(p.y + o);
                        if(p.accumulate)
                        {
                            float u[8];
                            unpack_bf16x8(*dst, u);
#pragma unroll
                            for(int k = 0; k < 8; ++k)
                                w[k] += u[k];
                        }
                        *dst = pack_bf16x8(w);
                    }
                }
            }
        }

        template<bool TMA>
        __global__ void __launch_bounds__(row_threads<TMA>(), 1)
            k_conv_row(const __grid_constant__ ConvGemmParams p, const RowGeom rg, const __grid_constant__ CUtensorMap tmap,
                       const __grid_constant__ CUtensorMap tmapUp)
        {
            extern __shared__ unsigned char dsm[];
            __shared__ uint32_t sTmem;
            __shared__ float sBias[256];
            __shared__ __align__(8) uint64_t sFull[2];
            __shared__ __align__(8) uint64_t sEmpty[2];
            __shared__ __align__(8) uint64_t sAccFull[2];
            __shared__ __align__(8) uint64_t sAccEmpty[2];
            __shared__ __align__(8) uint64_t sDrain;
            unsigned char* base = dsm + ((128u - (tc::smem_addr(dsm) & 127u)) & 127u);
            const uint32_t sB = tc::smem_addr(base);
            const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
            const int pad = p.pad, ks = p.ks, S = rg.S, HWp = rg.HWp, NS = rg.stages;
            const int nC = p.Cg / 8;
            const uint32_t runBytes = uint32_t(HWp) * 16u;
            // swizzled staging: each input row is HWp pixels of rowB bytes, the row buffers
            // and the halo start on multiples of the swizzle pattern's period (8 rows)
            const int rowB = rg.rowB;
            const bool cat = TMA && rg.cwc != 0;
            const uint32_t swSpan = cat ? 1024u : 8u * uint32_t(rowB);
            const uint32_t rowPitch = rowB ? (uint32_t(HWp * rowB) + swSpan - 1u) / swSpan * swSpan : 0u;
            const uint32_t haloBytes = rowB ? uint32_t(ks * S) * rowPitch : uint32_t(ks * nC * S) * runBytes;
            const uint32_t wEnd = sB + uint32_t(p.Npad) * uint32_t(p.Kpad) * 2u;
            const uint32_t sH = (rowB || cat) ? (wEnd + swSpan - 1u) / swSpan * swSpan : wEnd;
            const uint32_t half = tmem_columns(p.Npad);
            const uint32_t cols = 2 * half;
            if(warp == 0)
            {
                tc::tmem_alloc(&sTmem, cols);
                tc::tmem_relinquish();
            }
            if(tid == 0)
            {
                for(int s = 0; s < 2; ++s)
                {
                    tc::mbar_init(&sFull[s], TMA ? 1 : 128);
                    tc::mbar_init(&sEmpty[s], 1);
                    tc::mbar_init(&sAccFull[s], 1);
                    tc::mbar_init(&sAccEmpty[s], TMA ? 256 : 128);
                }
                tc::mbar_init(&sDrain, 1);
                tc::mbar_init_fence();
            }
            {
                const int kb = p.Kpad / 8;
                const int pieces = p.Npad * kb;
                for(int i = tid; i < pieces; i += row_threads<TMA>())
                {
                    const int n = i / kb, k8 = i - n * kb;
                    const uint32_t dst = sB + uint32_t(n >> 3) * uint32_t(p.Kpad) * 16u + uint32_t(k8) * 128u + uint32_t(n & 7) * 16u;
                    tc::cp_async16(dst, p.w + size_t(n) * p.Kpad + size_t(k8) * 8, 16);
                }
                tc::cp_async_commit();
                // the per-channel bias, read by every epilogue thread for every pixel
                for(int c = tid; c < p.Npad && c < 256; c += row_threads<TMA>())
                    sBias[c] = (p.bias && c < p.Cout) ? __ldg(p.bias + c) : 0.0f;
                tc::cp_async_wait<0>();
                tc::fence_async_smem();
            }
            tc::fence_before_sync();
            __syncthreads();
            tc::fence_after_sync();
            // everything above (weights, bias, barriers, TMEM) is independent of the
            // previous layer; its output is read only from here on
            tc::grid_dependency_wait();
            tc::grid_launch_dependents();
            const uint32_t tmem = sTmem;
            if(p.waitCheckNs != 0)
            {
                // failure-detection check: sDrain has had no arrival, so this bounded wait
                // runs out; no copy or MMA is in flight when the TMEM is released
                if(tid == 0 && !tc::mbar_wait(&sDrain, 0, p.waitCheckNs) && p.errorFlag)
                    atomicExch(p.errorFlag, 1);
                tc::fence_before_sync();
                __syncthreads();
                if(warp == 0)
                    tc::tmem_dealloc(tmem, cols);
                return;
            }
            const int tilesPerRow = (p.Wo + kTileM - 1) / kTileM;
            const int nTiles = p.B * p.Ho * tilesPerRow;

            if(TMA && warp == 9)
            {
                // entry (ty, chunk j, parity q, idx) holds input column S*x0 - pad + S*idx + q:
                // one box per run.  Stride 1: map (C, W, H, B), box (8, HWn, 1, 1) at
                // (8j, x0 - pad, row, b).  Stride 2: map (C, 2, W/2, H, B), the column split
                // into its parity and half, box (8, 1, HWn, 1, 1) at (8j, c & 1, c >> 1, row,
                // b) with c = 2*x0 - pad + q.  Swizzled staging (16-64 channels): one box of
                // all channels per run, (C, HWp, 1, 1) at (0, x0 - pad, row, b) or
                // (C, 1, HWp, 1, 1) at (0, c & 1, c >> 1, row, b), written with the map's
                // 32/64/128-byte swizzle.  Rows and columns outside the image read zeros.
                if(lane == 0)
                {
                    const uint32_t txBytes = cat ? uint32_t(kTileM * p.Cg * 2)
                        : rowB                   ? uint32_t(ks * S * HWp * rowB)
                                                 : uint32_t(ks * nC * S * rg.HWn) * 16u;
                    int i = 0;
                    for(int tile = blockIdx.x; tile < nTiles; tile += gridDim.x, ++i)
                    {
                        const int s = i % NS, n = i / NS;
                        if(n >= 1 && !tc::mbar_wait(&sEmpty[s], uint32_t(n - 1) & 1u))
                        {
                            if(p.errorFlag)
                                atomicExch(p.errorFlag, 1);
                            break;
                        }
                        const int xt = tile % tilesPerRow;
                        const int row = tile / tilesPerRow;
                        const int y = row % p.Ho, b = row / p.Ho;
                        const int x0 = xt * kTileM;
                        const uint32_t st = sH + uint32_t(s) * haloBytes;
                        tc::mbar_arrive_expect_tx(&sFull[s], txBytes);
                        if(cat)
                        {
                            // tile rows in parity order: row m < 64 is pixel x0 + 2m, row 64 + m
                            // is pixel x0 + 2m + 1; both halves read coarse pixel x0/2 + m, so
                            // the coarse chunk is copied to both, the fine chunk by parity
                            uint32_t dst = st;
                            const int yc = min(y >> 1, p.upInH - 1); // the nearest coarse row, clamped
                            for(int c = 0; c < p.upC; c += rg.cwc)
                            {
                                for(int h = 0; h < 2; ++h)
                                    tc::tma_load_4d(dst + uint32_t(h * 64 * rg.cwc * 2), &tmapUp, c, x0 >> 1, yc, b, &sFull[s]);
                                dst += uint32_t(kTileM * rg.cwc * 2);
                            }
                            for(int c = 0; c < p.Cg - p.upC; c += rg.cwf)
                            {
                                for(int q = 0; q < 2; ++q)
                                    tc::tma_load_5d(dst + uint32_t(q * 64 * rg.cwf * 2), &tmap, c, q, x0 >> 1, y, b, &sFull[s]);
                                dst += uint32_t(kTileM * rg.cwf * 2);
                            }
                            continue;
                        }
                        for(int ty = 0; ty < ks; ++ty)
                        {
                            const int iy = p.transposed ? y + pad - ty : S * y - pad + ty;
                            if(rowB)
                            {
                                if(S == 1)
                                    tc::tma_load_4d(st + uint32_t(ty) * rowPitch, &tmap, 0, x0 - pad, iy, b, &sFull[s]);
                                else
                                    for(int q = 0; q < 2; ++q)
                                    {
                                        const int c = 2 * x0 - pad + q;
                                        tc::tma_load_5d(st + uint32_t(ty * 2 + q) * rowPitch, &tmap, 0, c & 1, c >> 1, iy, b,
                                                        &sFull[s]);
                                    }
                                continue;
                            }
                            for(int j = 0; j < nC; ++j)
                                for(int q = 0; q < S; ++q)
                                {
                                    const uint32_t dst = st + uint32_t((ty * nC + j) * S + q) * runBytes;
                                    if(S == 1)
                                        tc::tma_load_4d(dst, &tmap, 8 * j, x0 - pad, iy, b, &sFull[s]);
                                    else
                                    {
                                        const int c = 2 * x0 - pad + q;
                                        tc::tma_load_5d(dst, &tmap, 8 * j, c & 1, c >> 1, iy, b, &sFull[s]);
                                    }
                                }
                        }
                    }
                }
            }
            else if(!TMA && warp >= 4 && warp < 8)
            {
                // producers: entry (ty, chunk j, parity q, idx) holds input column S*x0 - pad + S*idx + q
                const int pt = tid - 128;
                const int dj = 128 % nC, dc = 128 / nC;
                int i = 0;
                for(int tile = blockIdx.x; tile < nTiles; tile += gridDim.x, ++i)
                {
                    const int s = i % NS, n = i / NS;
                    if(n >= 1 && !tc::mbar_wait(&sEmpty[s], uint32_t(n - 1) & 1u))
                    {
                        if(p.errorFlag)
                            atomicExch(p.errorFlag, 1);
                        break;
                    }
                    const int xt = tile % tilesPerRow;
                    const int row = tile / tilesPerRow;
                    const int y = row % p.Ho, b = row / p.Ho;
                    const int x0 = xt * kTileM;
                    const uint32_t st = sH + uint32_t(s) * haloBytes;
                    // flat index g = (c * nC + j) within one halo row, c = S*idx + q the input column
                    // offset; consecutive threads take consecutive 16-byte pieces of global memory and
                    // step by 128 pieces, so j and c advance by fixed amounts
                    const int perRow = nC * S * HWp;
                    for(int ty = 0; ty < ks; ++ty)
                    {
                        const int iy = p.transposed ? y + pad - ty : S * y - pad + ty;
                        const bool rowOk = iy >= 0 && iy < p.H;
                        // implicit concatenation: chunks below nUp come from the coarse tensor at
                        // the nearest coarse pixel, the rest from x, whose pixels hold cX channels
                        const int nUp = p.xUp ? p.upC / 8 : 0;
                        const int cX = p.Cg - 8 * nUp;
                        const bf16* rowPtr = p.x + (size_t(b) * p.H + (rowOk ? iy : 0)) * p.W * cX;
                        const bf16* upRow = p.xUp
                            ? p.xUp + (size_t(b) * p.upInH + min((rowOk ? iy : 0) >> 1, p.upInH - 1)) * p.upInW * p.upC
                            : nullptr;
                        const uint32_t rowBase = st + uint32_t(ty * nC * S) * runBytes;
                        int j = pt % nC, c = pt / nC;
                        for(int g = pt; g < perRow; g += 128)
                        {
                            const int ix = S * x0 - pad + c;
                            const int q = c & (S - 1), idx = S == 1 ? c : (c >> 1);
                            const bool ok = rowOk && ix >= 0 && ix < p.W;
                            const bf16* src = !ok ? p.x
                                : j < nUp ? upRow + size_t(min(ix >> 1, p.upInW - 1)) * p.upC + j * 8
                                          : rowPtr + size_t(ix) * cX + (j - nUp) * 8;
                            tc::cp_async16(rowBase + uint32_t(j * S + q) * runBytes + uint32_t(idx) * 16u, src, ok ? 16u : 0u);
                            j += dj;
                            c += dc;
                            if(j >= nC)
                            {
                                j -= nC;
                                ++c;
                            }
                        }
                    }
                    tc::cp_async_arrive(&sFull[s]);
                }
                tc::cp_async_wait<0>();
            }
            else if(warp == 8)
            {
                if(lane == 0)
                {
                    const uint32_t idesc = tc::idesc_bf16(kTileM, p.Npad, false, false);
                    const uint32_t lboA = uint32_t(S) * runBytes;
                    const uint32_t sboB = uint32_t(p.Kpad) * 16u;
                    int i = 0;
                    for(int tile = blockIdx.x; tile < nTiles; tile += gridDim.x, ++i)
                    {
                        const int s = i % NS, n = i / NS;
                        const int a = i & 1, na = i >> 1;
                        if(!tc::mbar_wait(&sFull[s], uint32_t(n) & 1u)
                           || (na >= 1 && !tc::mbar_wait(&sAccEmpty[a], uint32_t(na - 1) & 1u)))
                        {
                            if(p.errorFlag)
                                atomicExch(p.errorFlag, 1);
                            break;
                        }
                        tc::fence_async_smem();
                        tc::fence_after_sync();
                        const uint32_t st = sH + uint32_t(s) * haloBytes;
                        const uint32_t d = tmem + uint32_t(a) * half;
                        // descriptors differ only in their start field (16-byte units), so the
                        // loop adds offsets to two base descriptors
                        const uint64_t aBase = tc::smem_desc(st, lboA, 128u);
                        const uint64_t bBase = tc::smem_desc(sB, 128u, sboB);
                        uint32_t acc = 0;
                        if(cat)
                        {
                            // the chunks in channel order (coarse, then fine), each 128 rows of
                            // cw * 2 bytes with that width's swizzle
                            uint32_t region = st, bOff = 0;
                            for(int part = 0; part < 2; ++part)
                            {
                                const int cw = part == 0 ? rg.cwc : rg.cwf;
                                const int cN = part == 0 ? p.upC : p.Cg - p.upC;
                                const uint32_t rb = uint32_t(cw * 2);
                                const uint64_t swDesc = (tc::smem_desc(0, 16u, 8u * rb) & ~uint64_t(0x3FFF))
                                    | (uint64_t(rb == 32 ? 6 : rb == 64 ? 4 : 2) << 61);
                                for(int c = 0; c < cN; c += cw)
                                {
                                    for(int jp = 0; jp < cw / 16; ++jp)
                                    {
                                        const uint32_t addr = region + uint32_t(jp) * 32u;
                                        tc::mma_bf16(d, swDesc | uint64_t((addr >> 4) & 0x3FFFu), bBase + bOff, idesc, acc);
                                        acc = 1;
                                        bOff += 16u;
                                    }
                                    region += uint32_t(kTileM) * rb;
                                }
                            }
                        }
                        else if(rowB)
                        {
                            // K-major A with the rows' own swizzle (layout 6 / 4 / 2 = 32 / 64 /
                            // 128 bytes), 8-row groups swSpan apart; tap (ty, tx) starts idx0 rows
                            // into run (ty, q) and each K step of 16 channels 32 bytes further.
                            // The swizzle follows the absolute shared-memory address, as the TMA
                            // copy wrote it, so the base-offset field stays 0.
                            const uint64_t swDesc = (tc::smem_desc(0, 16u, swSpan) & ~uint64_t(0x3FFF))
                                | (uint64_t(rowB == 32 ? 6 : rowB == 64 ? 4 : 2) << 61);
                            for(int ty = 0; ty < ks; ++ty)
                                for(int tx = 0; tx < ks; ++tx)
                                {
                                    const int col = p.transposed ? 2 * pad - tx : tx;
                                    const int q = col & (S - 1), idx0 = S == 1 ? col : (col >> 1);
                                    uint32_t addr = st + uint32_t(ty * S + q) * rowPitch + uint32_t(idx0 * rowB);
                                    uint32_t bOff = uint32_t((ty * ks + tx) * p.Cg);
                                    for(int jp = 0; jp < nC / 2; ++jp)
                                    {
                                        tc::mma_bf16(d, swDesc | uint64_t((addr >> 4) & 0x3FFFu), bBase + bOff, idesc, acc);
                                        acc = 1;
                                        addr += 32u;
                                        bOff += 16u;
                                    }
                                }
                        }
                        else
                        for(int ty = 0; ty < ks; ++ty)
                            for(int tx = 0; tx < ks; ++tx)
                            {
                                const int col = p.transposed ? 2 * pad - tx : tx;
                                const int q = col & (S - 1), idx0 = S == 1 ? col : (col >> 1);
                                uint32_t aOff = uint32_t((ty * nC * S + q) * HWp + idx0);
                                uint32_t bOff = uint32_t((ty * ks + tx) * p.Cg);
                                for(int jp = 0; jp < nC / 2; ++jp)
                                {
                                    tc::mma_bf16(d, aBase + aOff, bBase + bOff, idesc, acc);
                                    acc = 1;
                                    aOff += uint32_t(2 * S * HWp);
                                    bOff += 16u;
                                }
                            }
                        tc::mma_commit(&sEmpty[s]);
                        tc::mma_commit(&sAccFull[a]);
                    }
                    // every MMA of this CTA has completed before TMEM is released
                    tc::mma_commit(&sDrain);
                    tc::mbar_wait(&sDrain, 0);
                }
                __syncwarp();
            }
            else
            {
                // epilogue: thread = TMEM lane = pixel of the tile; with TMA two groups of four
                // warps split the accumulator columns
                const uint32_t lane0 = uint32_t(warp & 3) * 32u;
                const int colsPer = TMA ? p.Npad / 2 : p.Npad; // a multiple of 8
                const int cBeg = TMA ? (warp >> 2) * colsPer : 0;
                int i = 0;
                for(int tile = blockIdx.x; tile < nTiles; tile += gridDim.x, ++i)
                {
                    const int a = i & 1;
                    if(!tc::mbar_wait(&sAccFull[a], uint32_t(i >> 1) & 1u))
                    {
                        if(p.errorFlag)
                            atomicExch(p.errorFlag, 1);
                        break;
                    }
                    tc::fence_after_sync();
                    const int xt = tile % tilesPerRow;
                    const int row = tile / tilesPerRow;
                    const int m = tid & 127;
                    const int px = cat ? (m < 64 ? 2 * m : 2 * (m - 64) + 1) : m; // parity-ordered rows
                    row_epilogue(p, tmem + uint32_t(a) * half + (lane0 << 16), xt, row / p.Ho, row % p.Ho, px, cBeg,
                                 colsPer, sBias);
                    tc::fence_before_sync();
                    tc::mbar_arrive(&sAccEmpty[a]);
                }
            }
            tc::fence_before_sync();
            __syncthreads();
            tc::fence_after_sync();
            if(warp == 0)
                tc::tmem_dealloc(tmem, cols);
        }

        // ------------------------------------------------------------------ weight gradient
        __global__ void __launch_bounds__(kThreads, 1) k_conv_wgrad(const __grid_constant__ WgradParams p)
        {
            extern __shared__ unsigned char dsm[];
            __shared__ uint32_t sTmem;
            __shared__ __align__(8) uint64_t sEmpty[kStages];
            __shared__ __align__(8) uint64_t sDone;
            unsigned char* base = dsm + ((128u - (tc::smem_addr(dsm) & 127u)) & 127u);
            const uint32_t stageB = uint32_t(p.Npad) * 128u; // Npad/8 core rows x 8 pixel blocks x 128 B
            const uint32_t stageBytes = uint32_t(kStageBytesA) + stageB;
            const uint32_t s0 = tc::smem_addr(base);
            const int tid = threadIdx.x;
            const uint32_t cols = tmem_columns(p.Npad);
            if(tid < 32)
            {
                tc::tmem_alloc(&sTmem, cols);
                tc::tmem_relinquish();
            }
            if(tid == 0)
            {
                for(int s = 0; s < kStages; ++s)
                    tc::mbar_init(&sEmpty[s], 1);
                tc::mbar_init(&sDone, 1);
                tc::mbar_init_fence();
            }
            bool abortLocal = false, aborted = false;
            tc::fence_before_sync();
            __syncthreads();
            tc::fence_after_sync();
            const uint32_t tmem = sTmem;

            const int P = p.B * p.Ho * p.Wo;
            const int nChunks = (P + kChunkK - 1) / kChunkK;
            const int c0 = blockIdx.y * p.chunksPerSplit;
            const int c1 = min(nChunks, c0 + p.chunksPerSplit);
            const int nk = c1 - c0;
            const int mTile = blockIdx.x;
            const uint32_t idesc = tc::idesc_bf16(kTileM, p.Npad, true, true);
            const int bPieces = (p.Npad / 8) * kChunkK;

            auto load_chunk = [&](int kc, uint32_t G) {
                const uint32_t stA = s0 + (G % kStages) * stageBytes;
                const uint32_t stB = stA + uint32_t(kStageBytesA);
                // A: 16 row blocks (8 channels of one tap) x 64 pixels
#pragma unroll
                for(int q = 0; q < 4; ++q)
                {
                    const int id = q * kThreads + tid;
                    const int px = id & (kChunkK - 1), mb = id >> 6;
                    const int r0 = mTile * kTileM + mb * 8;
                    const int pix = kc * kChunkK + px;
                    const bf16* src = p.x;
                    uint32_t bytes = 0;
                    if(r0 < p.Mtot && pix < P)
                    {
                        const int t = r0 / p.Cin, c = r0 - t * p.Cin;
                        const int ty = t / p.ks, tx = t - ty * p.ks;
                        const int ox = pix % p.Wo, tt = pix / p.Wo;
                        const int oy = tt % p.Ho, b = tt / p.Ho;
                        const int iy = oy * p.stride - p.pad + ty, ix = ox * p.stride - p.pad + tx;
                        if(iy >= 0 && ix >= 0 && iy < p.H && ix < p.W)
                        {
                            src = p.x + ((size_t(b) * p.H + iy) * p.W + ix) * p.Cin + c;
                            bytes = 16;
                        }
                    }
                    tc::cp_async16(stA + uint32_t(mb) * 1024u + uint32_t(px >> 3) * 128u + uint32_t(px & 7) * 16u, src, bytes);
                }
                // B: Npad/8 column blocks x 64 pixels of dY
                for(int id = tid; id < bPieces; id += kThreads)
                {
                    const int px = id & (kChunkK - 1), nb = id >> 6;
                    const int pix = kc * kChunkK + px;
                    const bf16* src = p.dy;
                    uint32_t bytes = 0;
                    if(pix < P && nb * 8 < p.Cout)
                    {
                        src = p.dy + size_t(pix) * p.Cout + nb * 8;
                        bytes = 16;
                    }
                    tc::cp_async16(stB + uint32_t(nb) * 1024u + uint32_t(px >> 3) * 128u + uint32_t(px & 7) * 16u, src, bytes);
                }
            };

            for(int c = 0; c < kStages - 1; ++c)
            {
                if(c < nk)
                    load_chunk(c0 + c, uint32_t(c));
                tc::cp_async_commit();
            }
            for(int kc = 0; kc < nk; ++kc)
            {
                const int kn = kc + kStages - 1;
                if(kn < nk)
                {
                    const uint32_t G = uint32_t(kn);
                    if(G >= kStages && !tc::mbar_wait(&sEmpty[G % kStages], ((G / kStages) - 1) & 1))
                        raise_error(p.errorFlag, abortLocal);
                    load_chunk(c0 + kn, G);
                }
                tc::cp_async_commit();
                tc::cp_async_wait<kStages - 1>();
                tc::fence_async_smem();
                if(__syncthreads_or(abortLocal))
                {
                    aborted = true;
                    break;
                }
                if(tid == 0)
                {
                    tc::fence_after_sync();
                    const uint32_t stA = s0 + (uint32_t(kc) % kStages) * stageBytes;
                    const uint32_t stB = stA + uint32_t(kStageBytesA);
#pragma unroll
                    for(int j = 0; j < kChunkK / 16; ++j)
                    {
                        const uint64_t ad = tc::smem_desc(stA + uint32_t(j) * 256u, 128u, 1024u);
                        const uint64_t bd = tc::smem_desc(stB + uint32_t(j) * 256u, 128u, 1024u);
                        tc::mma_bf16(tmem, ad, bd, idesc, (kc | j) != 0 ? 1u : 0u);
                    }
                    tc::mma_commit(&sEmpty[uint32_t(kc) % kStages]);
                }
            }
            tc::cp_async_wait<0>();
            if(tid == 0)
                tc::mma_commit(&sDone);
            if(!aborted && !tc::mbar_wait(&sDone, 0))
                raise_error(p.errorFlag, abortLocal);
            aborted = __syncthreads_or(abortLocal) != 0;
            tc::fence_after_sync();
            if(aborted)
            {
                // one more bounded wait: the MMAs must be done before TMEM is released
                if(tid == 0)
                    tc::mma_commit(&sDone);
                tc::mbar_wait(&sDone, 1);
            }
            else if(nk > 0)
            {
                const int warp = tid >> 5;
                const uint32_t lane0 = uint32_t(warp & 3) * 32u;
                const int half = warp >> 2;
                const int cpw = p.Npad / 2;
                const int row = mTile * kTileM + (tid & (kTileM - 1));
                for(int cc = half * cpw; cc < (half + 1) * cpw; cc += 8)
                {
                    float v[8];
                    tc::tmem_ld8(tmem + (lane0 << 16) + uint32_t(cc), v);
                    tc::tmem_wait_ld();
                    if(row >= p.Mtot)
                        continue;
#pragma unroll
                    for(int i = 0; i < 8; ++i)
                        if(cc + i < p.Cout)
                            atomicAdd(p.dw + size_t(row) * p.Npad + cc + i, v[i]);
                }
            }
            tc::fence_before_sync();
            __syncthreads();
            if(tid < 32)
                tc::tmem_dealloc(tmem, cols);
        }

        int num_sms()
        {
            static int n = 0;
            if(n == 0)
            {
                int dev = 0;
                cudaGetDevice(&dev);
                cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
                if(n <= 0)
                    n = 148;
            }
            return n;
        }
    } // namespace

    size_t conv_gemm_smem(int Npad, int Kpad)
    {
        return size_t(Npad) * Kpad * 2 + size_t(kStages) * kStageBytesA + 128;
    }
    size_t conv_wgrad_smem(int Npad)
    {
        return size_t(kStages) * (kStageBytesA + size_t(Npad) * 128) + 128;
    }

    bool row_tiles_apply(const ConvGemmParams& p)
    {
        if(p.xUp && (p.ks != 1 || p.stride != 1 || p.upC % 8 != 0 || p.transposed))
            return false;
        return p.Cg % 16 == 0 && p.Npad <= 256
            && ((p.stride == 1 && 2 * p.pad == p.ks - 1) || (p.stride == 2 && !p.transposed && p.ks <= 3 && p.pad <= 1));
    }
    // Swizzled staging for the TMA producer: 16, 32 or 64 channels, each run (an input row,
    // or one parity plane of it at stride 2) one box of Cg * 2-byte pixels, instead of one
    // box per 8-channel chunk (the narrow chunk boxes kept the copy engine busy).  Returns
    // the bytes per staged pixel, 0 where the chunked runs are used.
    inline int swizzle_row_bytes(const ConvGemmParams& p)
    {
        return (p.Cg == 16 || p.Cg == 32 || p.Cg == 64) ? p.Cg * 2 : 0;
    }
    size_t conv_row_smem(const ConvGemmParams& p, int stages, bool tma = false)
    {
        const RowGeom g = row_geom(p.stride, p.ks, p.pad, stages, tma);
        const int rowB = tma ? swizzle_row_bytes(p) : 0;
        if(rowB)
        {
            const size_t span = size_t(8) * rowB, pitch = (size_t(g.HWp) * rowB + span - 1) / span * span;
            return size_t(p.Npad) * p.Kpad * 2 + span + size_t(stages) * p.ks * g.S * pitch + 128;
        }
        return size_t(p.Npad) * p.Kpad * 2 + size_t(stages) * p.ks * (p.Cg / 8) * g.S * g.HWp * 16 + 128;
    }

    namespace
    {
        PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
        {
            static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
            static bool tried = false;
            if(!tried)
            {
                tried = true;
                void* f = nullptr;
                cudaDriverEntryPointQueryResult q{};
                if(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess
                   && q == cudaDriverEntryPointSuccess)
                    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
            }
            return fn;
        }

        // The tensor map of a row-tile convolution's input for the TMA producer (layouts at
        // k_conv_row); false when the input does not fit one (then the cp.async producer runs)
        bool encode_row_map(const ConvGemmParams& p, const RowGeom& g, CUtensorMap& m)
        {
            auto enc = tensor_map_encoder();
            if(!enc || (reinterpret_cast<uintptr_t>(p.x) & 15u) != 0 || p.Cg % 8 != 0)
                return false;
            const cuuint64_t C = cuuint64_t(p.Cg), W = cuuint64_t(p.W), H = cuuint64_t(p.H), B = cuuint64_t(p.B);
            cuuint32_t estr[5] = {1, 1, 1, 1, 1};
            CUresult r;
            if(g.rowB)
            {
                const CUtensorMapSwizzle sw = g.rowB == 32 ? CU_TENSOR_MAP_SWIZZLE_32B
                    : g.rowB == 64                         ? CU_TENSOR_MAP_SWIZZLE_64B
                                                           : CU_TENSOR_MAP_SWIZZLE_128B;
                if(g.S == 1)
                {
                    cuuint64_t dims[4] = {C, W, H, B};
                    cuuint64_t strides[3] = {C * 2, W * C * 2, H * W * C * 2};
                    cuuint32_t box[4] = {cuuint32_t(C), cuuint32_t(g.HWp), 1, 1};
                    r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(p.x), dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
                }
                else
                {
                    if(p.W % 2 != 0)
                        return false; // the parity split views W as (W/2, 2)
                    cuuint64_t dims[5] = {C, 2, W / 2, H, B};
                    cuuint64_t strides[4] = {C * 2, 2 * C * 2, W * C * 2, H * W * C * 2};
                    cuuint32_t box[5] = {cuuint32_t(C), 1, cuuint32_t(g.HWp), 1, 1};
                    r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16*>(p.x), dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
                }
            }
            else if(g.S == 1)
            {
                cuuint64_t dims[4] = {C, W, H, B};
                cuuint64_t strides[3] = {C * 2, W * C * 2, H * W * C * 2};
                cuuint32_t box[4] = {8, cuuint32_t(g.HWn), 1, 1};
                r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(p.x), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            }
            else
            {
                if(p.W % 2 != 0)
                    return false; // the parity split views W as (W/2, 2)
                cuuint64_t dims[5] = {C, 2, W / 2, H, B};
                cuuint64_t strides[4] = {C * 2, 2 * C * 2, W * C * 2, H * W * C * 2};
                cuuint32_t box[5] = {8, 1, cuuint32_t(g.HWn), 1, 1};
                r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16*>(p.x), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            }
            return r == CUDA_SUCCESS;
        }

        inline int chunk_width(int c)
        {
            return c % 64 == 0 ? 64 : c % 32 == 0 ? 32 : c % 16 == 0 ? 16 : 0;
        }
        inline CUtensorMapSwizzle swizzle_of(int rowBytes)
        {
            return rowBytes == 32 ? CU_TENSOR_MAP_SWIZZLE_32B : rowBytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B;
        }

        // The two tensor maps of the implicit concatenation by TMA (layout at k_conv_row):
        // the fine tensor split by column parity, the coarse one plain; false when the layer
        // does not fit (then the cp.async producer gathers it)
        bool encode_cat_maps(const ConvGemmParams& p, RowGeom& g, CUtensorMap& fine, CUtensorMap& coarse)
        {
            auto enc = tensor_map_encoder();
            const int cf = p.Cg - p.upC;
            // columns past the coarse width would read zeros where the gather clamps, so the
            // coarse width must cover W / 2; rows are clamped in the kernel
            if(!enc || !p.xUp || p.ks != 1 || p.stride != 1 || p.pad != 0 || p.transposed || p.W % 2 != 0 || p.Wo != p.W
               || p.Ho != p.H || 2 * p.upInW < p.W || p.upInH < 1 || p.upC <= 0 || cf <= 0 || !chunk_width(p.upC)
               || !chunk_width(cf) || (reinterpret_cast<uintptr_t>(p.x) & 15u) != 0
               || (reinterpret_cast<uintptr_t>(p.xUp) & 15u) != 0)
                return false;
            g.cwc = chunk_width(p.upC);
            g.cwf = chunk_width(cf);
            cuuint32_t estr[5] = {1, 1, 1, 1, 1};
            const cuuint64_t C = cuuint64_t(cf), W = cuuint64_t(p.W), H = cuuint64_t(p.H), B = cuuint64_t(p.B);
            cuuint64_t dims[5] = {C, 2, W / 2, H, B};
            cuuint64_t strides[4] = {C * 2, 2 * C * 2, W * C * 2, H * W * C * 2};
            cuuint32_t box[5] = {cuuint32_t(g.cwf), 1, 64, 1, 1};
            if(enc(&fine, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16*>(p.x), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_of(2 * g.cwf), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)
               != CUDA_SUCCESS)
                return false;
            const cuuint64_t Cc = cuuint64_t(p.upC), Wc = cuuint64_t(p.upInW), Hc = cuuint64_t(p.upInH);
            cuuint64_t dimsC[4] = {Cc, Wc, Hc, B};
            cuuint64_t stridesC[3] = {Cc * 2, Wc * Cc * 2, Hc * Wc * Cc * 2};
            cuuint32_t boxC[4] = {cuuint32_t(g.cwc), 64, 1, 1};
            return enc(&coarse, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(p.xUp), dimsC, stridesC, boxC, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_of(2 * g.cwc), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)
                == CUDA_SUCCESS;
        }

        template<bool TMA>
        void launch_row(const ConvGemmParams& p, int stages, const CUtensorMap& m, cudaStream_t s, int rowB = 0,
                        const CUtensorMap* m2 = nullptr, int cwc = 0, int cwf = 0)
        {
            const size_t smem = conv_row_smem(p, stages, TMA) + (cwc ? 1024 : 0);
            cudaFuncSetAttribute(k_conv_row<TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            cudaFuncSetAttribute(k_conv_row<TMA>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
            const int tiles = p.B * p.Ho * ((p.Wo + kTileM - 1) / kTileM);
            int perSm = ctas_per_sm(k_conv_row<TMA>, row_threads<TMA>(), smem);
            while(perSm > 1 && perSm * 2 * int(tmem_columns(p.Npad)) > 512)
                --perSm;
            const int slots = num_sms() * perSm;
            RowGeom g = row_geom(p.stride, p.ks, p.pad, stages, TMA);
            g.rowB = TMA ? rowB : 0;
            g.cwc = TMA ? cwc : 0;
            g.cwf = TMA ? cwf : 0;
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3(unsigned(tiles < slots ? tiles : slots));
            cfg.blockDim = dim3(unsigned(row_threads<TMA>()));
            cfg.dynamicSmemBytes = smem;
            cfg.stream = s;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attr[0].val.programmaticStreamSerializationAllowed = 1;
            cfg.attrs = attr;
            cfg.numAttrs = p.pdl ? 1 : 0;
            cudaLaunchKernelEx(&cfg, k_conv_row<TMA>, p, g, m, m2 ? *m2 : m);
        }
    } // namespace

    bool g_rowTma = true; // the TMA producer where the input allows it
    bool launch_conv_gemm(const ConvGemmParams& p, cudaStream_t s)
    {
        if(row_tiles_apply(p))
        {
            int stages = 2;
            if(conv_row_smem(p, 2, true) > 227 * 1024)
                stages = 1;
            if(conv_row_smem(p, stages, true) <= 227 * 1024)
            {
                CUtensorMap m{};
                RowGeom g = row_geom(p.stride, p.ks, p.pad, stages, true);
                g.rowB = swizzle_row_bytes(p);
                CUtensorMap m2{};
                if(g_rowTma && p.xUp && conv_row_smem(p, stages, true) + 1024 <= 227 * 1024 && encode_cat_maps(p, g, m, m2))
                    launch_row<true>(p, stages, m, s, 0, &m2, g.cwc, g.cwf);
                else if(g_rowTma && !p.xUp && encode_row_map(p, g, m))
                    launch_row<true>(p, stages, m, s, g.rowB);
                else
                    launch_row<false>(p, stages, m, s);
                return true;
            }
        }
        const size_t smem = conv_gemm_smem(p.Npad, p.Kpad);
        if(smem > 227 * 1024)
            return false;
        cudaFuncSetAttribute(k_conv_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        cudaFuncSetAttribute(k_conv_gemm, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        const int P = p.B * p.Ho * p.Wo;
        const int tiles = (P + kTileM - 1) / kTileM;
        // as many persistent CTAs as fit on an SM (shared memory and TMEM permitting), so one
        // CTA's epilogue and gathers overlap another's MMAs
        int perSm = ctas_per_sm(k_conv_gemm, kThreads, smem);
        while(perSm > 1 && perSm * int(tmem_columns(p.Npad)) > 512)
            --perSm;
        const int slots = num_sms() * perSm;
        const int grid = tiles < slots ? tiles : slots;
        k_conv_gemm<<<grid, kThreads, smem, s>>>(p);
        return true;
    }

    bool launch_conv_wgrad(WgradParams p, cudaStream_t s)
    {
        const size_t smem = conv_wgrad_smem(p.Npad);
        if(smem > 227 * 1024)
            return false;
        cudaFuncSetAttribute(k_conv_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        cudaFuncSetAttribute(k_conv_wgrad, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        const int P = p.B * p.Ho * p.Wo;
        const int nChunks = (P + kChunkK - 1) / kChunkK;
        const int mTiles = (p.Mtot + kTileM - 1) / kTileM;
        // about two CTAs' worth of work per SM in total, at least 4 chunks each
        int splits = (2 * num_sms() + mTiles - 1) / mTiles;
        int per = (nChunks + splits - 1) / splits;
        if(per < 4)
            per = 4;
        splits = (nChunks + per - 1) / per;
        p.chunksPerSplit = per;
        dim3 grid(mTiles, splits);
        k_conv_wgrad<<<grid, kThreads, smem, s>>>(p);
        return true;
    }
} // namespace isaacb

using namespace isaacb;

namespace
{
    int round_up(int v, int m)
    {
        return (v + m - 1) / m * m;
    }

    isaacb_status check_conv(const isaacb_conv_args* a, bool wgrad)
    {
        if(!a)
            return ISAACB_INVALID_ARG;
        if(a->batch == 0 || a->in_h == 0 || a->in_w == 0 || a->out_h == 0 || a->out_w == 0 || a->c_in == 0 || a->c_out == 0)
            return ISAACB_INVALID_ARG;
        if(a->c_in % 8 != 0 || a->c_out % 8 != 0 || a->c_out > 256 || a->ksize < 1 || a->ksize > 7 || a->stride < 1
           || a->stride > 4)
            return ISAACB_INVALID_ARG;
        const uint64_t pin = uint64_t(a->batch) * a->in_h * a->in_w, pout = uint64_t(a->batch) * a->out_h * a->out_w;
        if(pin * a->c_in >= (1ull << 31) || pout * a->c_out >= (1ull << 31))
            return ISAACB_INVALID_ARG;
        if(wgrad ? (!a->x || !a->dy || !a->dw) : (!a->x || !a->w || (!a->y && !a->y_f32)))
            return ISAACB_INVALID_ARG;
        return ISAACB_OK;
    }
} // namespace

extern "C"
{
    isaacb_status isaacb_conv_forward(const isaacb_conv_args* a, void* stream)
    {
        if(check_conv(a, false) != ISAACB_OK)
        {
            set_global_error("isaacb_conv_forward: invalid arguments");
            return ISAACB_INVALID_ARG;
        }
        ConvGemmParams p{};
        p.x = static_cast<const __nv_bfloat16*>(a->x);
        p.w = static_cast<const __nv_bfloat16*>(a->w);
        p.bias = a->bias;
        p.y = static_cast<__nv_bfloat16*>(a->y);
        p.yf = a->y_f32;
        p.mask = static_cast<const __nv_bfloat16*>(a->mask);
        p.B = int(a->batch);
        p.H = int(a->in_h);
        p.W = int(a->in_w);
        p.Cg = int(a->c_in);
        p.Ho = int(a->out_h);
        p.Wo = int(a->out_w);
        p.Cout = int(a->c_out);
        p.Npad = round_up(int(a->c_out), 16);
        p.Kpad = round_up(int(a->ksize * a->ksize * a->c_in), 64);
        p.ks = int(a->ksize);
        p.stride = int(a->stride);
        p.pad = int(a->pad);
        p.transposed = a->transposed ? 1 : 0;
        p.relu = a->relu ? 1 : 0;
        p.accumulate = a->accumulate ? 1 : 0;
        p.errorFlag = a->error_flag;
        p.waitCheckNs = 1000ull * a->wait_check_us;
        if(!launch_conv_gemm(p, (cudaStream_t) stream))
        {
            set_global_error("isaacb_conv_forward: weights do not fit in shared memory");
            return ISAACB_INVALID_ARG;
        }
        const cudaError_t e = cudaGetLastError();
        if(e != cudaSuccess)
        {
            set_global_error(std::string("isaacb_conv_forward: ") + cudaGetErrorString(e));
            return ISAACB_CUDA_ERROR;
        }
        return ISAACB_OK;
    }

    isaacb_status isaacb_conv_set_producer(int32_t tma)
    {
        g_rowTma = tma != 0;
        return ISAACB_OK;
    }

    isaacb_status isaacb_conv_wgrad(const isaacb_conv_args* a, void* stream)
    {
        if(check_conv(a, true) != ISAACB_OK)
        {
            set_global_error("isaacb_conv_wgrad: invalid arguments");
            return ISAACB_INVALID_ARG;
        }
        WgradParams p{};
        p.x = static_cast<const __nv_bfloat16*>(a->x);
        p.dy = static_cast<const __nv_bfloat16*>(a->dy);
        p.dw = a->dw;
        p.B = int(a->batch);
        p.H = int(a->in_h);
        p.W = int(a->in_w);
        p.Cin = int(a->c_in);
        p.Ho = int(a->out_h);
        p.Wo = int(a->out_w);
        p.Cout = int(a->c_out);
        p.Npad = round_up(int(a->c_out), 16);
        p.ks = int(a->ksize);
        p.stride = int(a->stride);
        p.pad = int(a->pad);
        p.Mtot = int(a->ksize * a->ksize * a->c_in);
        p.errorFlag = a->error_flag;
        if(!launch_conv_wgrad(p, (cudaStream_t) stream))
        {
            set_global_error("isaacb_conv_wgrad: tile does not fit in shared memory");
            return ISAACB_INVALID_ARG;
        }
        const cudaError_t e = cudaGetLastError();
        if(e != cudaSuccess)
        {
            set_global_error(std::string("isaacb_conv_wgrad: ") + cudaGetErrorString(e));
            return ISAACB_CUDA_ERROR;
        }
        return ISAACB_OK;
    }
}
