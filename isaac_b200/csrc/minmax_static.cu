// Min/max of one volume source without any device allocation.
//
// Some callers cannot call cudaMalloc: an in-situ simulation that reserves
// nearly all device memory up front for its own heap (as particle-in-cell
// codes do) leaves no room for the library's own buffers, and a solver loop
// that must not synchronise the device cannot afford the implicit
// synchronisation of cudaMalloc/cudaFree.  isaacb_minmax_noalloc serves them:
// it needs no context (a context allocates textures and a G-buffer), the
// caller passes the source and a 2-float device result, and the only scratch
// it uses is the file-scope device array below.
//
// Algorithm: the reference's own two-level scheme (MinMaxKernel,
// lib/isaac/isaac_min_max_kernel.hpp:22-60, then the column scan of
// CalcMinMaxIterator, lib/isaac.hpp:372-434): one thread per (x,y) column
// scans z and writes the column's min/max into the scratch array; one block
// then reduces the columns in column order.  Every combination keeps the
// earlier candidate on ties, so the result is bit-identical to the reference,
// +0/-0 order included, with no second pass.
//
// Scratch contract:
//  * g_columnMinMax holds 2 floats for each of at most kNoAllocMaxColumns
//    columns (2 MiB); every GPU that loads this library keeps it until exit.
//  * A source with more than kNoAllocMaxColumns (x,y) columns is rejected
//    with ISAACB_INVALID_ARG.
//  * Every call looks up the array's device address in the current context
//    (cudaGetSymbolAddress, a host-side lookup).  Nothing is cached, so an
//    address never outlives the context it came from (cudaDeviceReset, or a
//    different driver context made current on the same device).  The first
//    call in a context may load this module's device code there; make it
//    before any stream capture.
//  * Each call overwrites every column entry it later reads, so nothing has to
//    start at zero; the array keeps the last call's contents.
//  * All calls share the one array: calls whose kernels overlap on the GPU
//    (different streams, or different host threads) race on it.  Serialise
//    them on one stream.
#include "../../include/isaac_b200.h"
#include "isaacb_internal.h"

#include <cfloat>
#include <string>

namespace isaacb
{
    void set_global_error(const std::string& msg);

    constexpr uint32_t kNoAllocMaxColumns = 262144; // 2 floats each: 2 MiB
    constexpr uint32_t kNoAllocMaxDepth = 1u << 20; // z planes scanned per column
    __device__ __align__(256) float g_columnMinMax[2 * kNoAllocMaxColumns];

    namespace
    {

        // per (x,y) column: min/max over z in scan order
        __global__ void __launch_bounds__(256) k_column_minmax(
            const float* __restrict__ src,
            int X,
            int Y,
            int Z,
            int fdim,
            const Chain ch,
            float* __restrict__ scratch)
        {
            const int col = blockIdx.x * blockDim.x + threadIdx.x;
            if(col >= X * Y)
                return;
            float lo = FLT_MAX, hi = -FLT_MAX;
            const size_t plane = size_t(X) * Y;
            for(int z = 0; z < Z; ++z)
            {
                const float* p = src + (size_t(z) * plane + col) * fdim;
                float v[4];
                v[0] = __ldg(p);
                v[1] = fdim > 1 ? __ldg(p + 1) : 0.0f;
                v[2] = fdim > 2 ? __ldg(p + 2) : 0.0f;
                v[3] = fdim > 3 ? __ldg(p + 3) : 0.0f;
                const float val = apply_chain(v, fdim, ch);
                lo = gmin(lo, val);
                hi = gmax(hi, val);
            }
            scratch[2 * col] = lo;
            scratch[2 * col + 1] = hi;
        }

        // one block: each thread scans a contiguous run of columns, then an
        // order-preserving tree keeps the earlier candidate on ties
        constexpr int kFinalThreads = 1024;
        __global__ void __launch_bounds__(kFinalThreads)
            k_column_final(const float* __restrict__ scratch, int ncol, float* __restrict__ result)
        {
            __shared__ float sLo[kFinalThreads / 32], sHi[kFinalThreads / 32];
            const int t = threadIdx.x;
            const int chunk = (ncol + kFinalThreads - 1) / kFinalThreads;
            const int c0 = min(ncol, t * chunk), c1 = min(ncol, c0 + chunk);
            float lo = FLT_MAX, hi = -FLT_MAX;
            for(int c = c0; c < c1; ++c)
            {
                lo = gmin(lo, scratch[2 * c]);
                hi = gmax(hi, scratch[2 * c + 1]);
            }
#pragma unroll
            for(int o = 1; o < 32; o <<= 1)
            {
                const float rlo = __shfl_down_sync(0xffffffffu, lo, o);
                const float rhi = __shfl_down_sync(0xffffffffu, hi, o);
                if((t & 31) + o < 32)
                {
                    lo = gmin(lo, rlo);
                    hi = gmax(hi, rhi);
                }
            }
            if((t & 31) == 0)
            {
                sLo[t >> 5] = lo;
                sHi[t >> 5] = hi;
            }
            __syncthreads();
            if(t == 0)
            {
                float a = sLo[0], b = sHi[0];
                for(int w = 1; w < kFinalThreads / 32; ++w)
                {
                    a = gmin(a, sLo[w]);
                    b = gmax(b, sHi[w]);
                }
                result[0] = a;
                result[1] = b;
            }
        }

        // The array's address in the context current on this thread.  Looked up
        // on every call: a cached address would outlive a device reset or point
        // into another context of the same device.
        isaacb_status scratch_for_current_context(float** out)
        {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_columnMinMax);
            if(e != cudaSuccess || !p)
            {
                set_global_error(std::string("isaacb_minmax_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return ISAACB_CUDA_ERROR;
            }
            *out = static_cast<float*>(p);
            return ISAACB_OK;
        }
    } // namespace
} // namespace isaacb

using namespace isaacb;

extern "C" isaacb_status isaacb_minmax_noalloc(
    const float* src,
    const uint32_t size[3],
    uint32_t feature_dim,
    const int32_t bytecode[ISAACB_MAX_FUNCTORS],
    const float params[4 * ISAACB_MAX_FUNCTORS],
    float* result,
    void* stream)
{
    if(!src || !size || !bytecode || !params || !result)
    {
        set_global_error("isaacb_minmax_noalloc: null argument");
        return ISAACB_INVALID_ARG;
    }
    if(size[0] == 0 || size[1] == 0 || size[2] == 0 || feature_dim < 1 || feature_dim > 4)
    {
        set_global_error("isaacb_minmax_noalloc: sizes must be non-zero and feature_dim 1..4");
        return ISAACB_INVALID_ARG;
    }
    const uint64_t columns = uint64_t(size[0]) * size[1];
    if(columns > kNoAllocMaxColumns)
    {
        set_global_error(
            "isaacb_minmax_noalloc: " + std::to_string(columns) + " (x,y) columns exceed the static scratch of "
            + std::to_string(kNoAllocMaxColumns) + " columns");
        return ISAACB_INVALID_ARG;
    }
    if(size[2] > kNoAllocMaxDepth)
    {
        set_global_error(
            "isaacb_minmax_noalloc: depth " + std::to_string(size[2]) + " exceeds the limit of "
            + std::to_string(kNoAllocMaxDepth) + " z planes");
        return ISAACB_INVALID_ARG;
    }
    Chain ch{};
    for(int k = 0; k < kMaxFunctors; ++k)
    {
        if(bytecode[k] < OP_IDEM || bytecode[k] > OP_SUM)
        {
            set_global_error("isaacb_minmax_noalloc: bytecode out of range");
            return ISAACB_INVALID_ARG;
        }
        ch.op[k] = bytecode[k];
    }
    for(int k = 0; k < 4 * kMaxFunctors; ++k)
        ch.p[k] = params[k];
    float* scratch = nullptr;
    const isaacb_status st = scratch_for_current_context(&scratch);
    if(st != ISAACB_OK)
        return st;
    cudaStream_t s = (cudaStream_t) stream;
    const int ncol = int(columns);
    k_column_minmax<<<(ncol + 255) / 256, 256, 0, s>>>(
        src,
        int(size[0]),
        int(size[1]),
        int(size[2]),
        int(feature_dim),
        ch,
        scratch);
    k_column_final<<<1, kFinalThreads, 0, s>>>(scratch, ncol, result);
    const cudaError_t e = cudaGetLastError();
    if(e != cudaSuccess)
    {
        set_global_error(std::string("isaacb_minmax_noalloc: launch: ") + cudaGetErrorString(e));
        return ISAACB_CUDA_ERROR;
    }
    return ISAACB_OK;
}
