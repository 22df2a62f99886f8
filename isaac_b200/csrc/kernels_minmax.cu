// Min/max of a source after its functor chain: MinMaxKernel / MinMaxParticleKernel
// (lib/isaac/isaac_min_max_kernel.hpp:22-97) followed by the host scan of
// CalcMinMaxIterator (lib/isaac.hpp:372-497).
//
// The reference keeps, per column, the first value in scan order among equal
// candidates (glm::min(a,b) = b<a ? b : a, and a strict '<' in the host scan),
// never lets NaN in, and starts from +/-FLT_MAX.  A single-pass grid reduction
// with the same comparison yields the same value for every input; the only
// values that compare equal yet differ in bits are +0 and -0, so when the
// result is zero a second pass finds which zero comes first in the reference's
// scan order (column x + y*X, then z, then particle index).
#include "isaacb_internal.h"

#include <cfloat>

namespace isaacb
{
    constexpr int kMMThreads = 256;

    __device__ __forceinline__ float mm_value(const MinMaxParams& p, size_t idx)
    {
        float v[4];
        const float* sp = p.src + idx * p.fdim;
        v[0] = __ldg(sp);
        v[1] = p.fdim > 1 ? __ldg(sp + 1) : 0.0f;
        v[2] = p.fdim > 2 ? __ldg(sp + 2) : 0.0f;
        v[3] = p.fdim > 3 ? __ldg(sp + 3) : 0.0f;
        return apply_chain(v, p.fdim, p.chain);
    }
    __device__ __forceinline__ float mm_particle(const MinMaxParams& p, uint32_t k)
    {
        float v[4];
        const float* sp = p.attr + size_t(k) * p.fdim;
        v[0] = __ldg(sp);
        v[1] = p.fdim > 1 ? __ldg(sp + 1) : 0.0f;
        v[2] = p.fdim > 2 ? __ldg(sp + 2) : 0.0f;
        v[3] = p.fdim > 3 ? __ldg(sp + 3) : 0.0f;
        return apply_chain(v, p.fdim, p.chain);
    }

    __device__ __forceinline__ void block_reduce(float& lo, float& hi, float* out)
    {
        __shared__ float sLo[kMMThreads / 32], sHi[kMMThreads / 32];
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
        {
            lo = gmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = gmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        const int w = threadIdx.x >> 5;
        if((threadIdx.x & 31) == 0)
        {
            sLo[w] = lo;
            sHi[w] = hi;
        }
        __syncthreads();
        if(threadIdx.x == 0)
        {
            float a = sLo[0], b = sHi[0];
            for(int i = 1; i < kMMThreads / 32; ++i)
            {
                a = gmin(a, sLo[i]);
                b = gmax(b, sHi[i]);
            }
            out[0] = a;
            out[1] = b;
        }
    }

    __global__ void __launch_bounds__(kMMThreads) k_minmax_partial(const __grid_constant__ MinMaxParams p)
    {
        float lo = FLT_MAX, hi = -FLT_MAX;
        if(!p.particle)
        {
            const size_t n = size_t(p.g.ls[0]) * p.g.ls[1] * p.g.ls[2];
            for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
            {
                const float v = mm_value(p, i);
                lo = gmin(lo, v);
                hi = gmax(hi, v);
            }
        }
        else
        {
            const size_t n = size_t(p.g.lps[0]) * p.g.lps[1] * p.g.lps[2];
            for(size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x)
            {
                for(uint32_t k = __ldg(p.offsets + c); k < __ldg(p.offsets + c + 1); ++k)
                {
                    const float v = mm_particle(p, k);
                    lo = gmin(lo, v);
                    hi = gmax(hi, v);
                }
            }
        }
        block_reduce(lo, hi, p.partial + 2 * blockIdx.x);
    }

    __global__ void __launch_bounds__(kMMThreads) k_minmax_final(const float* __restrict__ partial, int n, float* result)
    {
        float lo = FLT_MAX, hi = -FLT_MAX;
        for(int i = threadIdx.x; i < n; i += blockDim.x)
        {
            lo = gmin(lo, partial[2 * i]);
            hi = gmax(hi, partial[2 * i + 1]);
        }
        block_reduce(lo, hi, result);
    }

    int minmax_blocks(const MinMaxParams& p)
    {
        const size_t n = p.particle ? size_t(p.g.lps[0]) * p.g.lps[1] * p.g.lps[2]
                                    : size_t(p.g.ls[0]) * p.g.ls[1] * p.g.ls[2];
        size_t b = (n + kMMThreads - 1) / kMMThreads;
        const size_t cap = 148 * 8;
        if(b > cap)
            b = cap;
        if(b < 1)
            b = 1;
        return int(b);
    }

    void launch_minmax(const MinMaxParams& p, int blocks, float* result, cudaStream_t s)
    {
        k_minmax_partial<<<blocks, kMMThreads, 0, s>>>(p);
        k_minmax_final<<<1, kMMThreads, 0, s>>>(p.partial, blocks, result);
    }

    // Reference scan-order key of the first +0 and the first -0:
    // keys[0] = first +0, keys[1] = first -0 (64-bit order keys, ULLONG_MAX if none)
    __global__ void __launch_bounds__(kMMThreads) k_minmax_zero_keys(const __grid_constant__ MinMaxParams p)
    {
        if(!p.particle)
        {
            const int LX = p.g.ls[0], LY = p.g.ls[1], LZ = p.g.ls[2];
            const size_t n = size_t(LX) * LY * LZ;
            for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
            {
                const float v = mm_value(p, i);
                if(v == 0.0f)
                {
                    const size_t x = i % LX, y = (i / LX) % LY, z = i / (size_t(LX) * LY);
                    const unsigned long long key = (unsigned long long) ((y * LX + x) * LZ + z);
                    atomicMin(&p.keys[signbit(v) ? 1 : 0], key);
                }
            }
        }
        else
        {
            const int PX = p.g.lps[0], PY = p.g.lps[1], PZ = p.g.lps[2];
            const size_t n = size_t(PX) * PY * PZ;
            for(size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x)
            {
                const uint32_t k0 = __ldg(p.offsets + c), k1 = __ldg(p.offsets + c + 1);
                for(uint32_t k = k0; k < k1; ++k)
                {
                    const float v = mm_particle(p, k);
                    if(v == 0.0f)
                    {
                        const size_t x = c % PX, y = (c / PX) % PY, z = c / (size_t(PX) * PY);
                        // column, then z, then position in the cell (< 2^32 particles per cell)
                        const unsigned long long key
                            = ((unsigned long long) ((y * PX + x) * PZ + z) << 32) | (unsigned long long) (k - k0);
                        atomicMin(&p.keys[signbit(v) ? 1 : 0], key);
                    }
                }
            }
        }
    }

    void launch_minmax_zero_keys(const MinMaxParams& p, cudaStream_t s)
    {
        k_minmax_zero_keys<<<minmax_blocks(p), kMMThreads, 0, s>>>(p);
    }
} // namespace isaacb
