// sm_100a building blocks for the tensor-core kernels: tcgen05 (TMEM
// allocation, MMA issue and commit, TMEM loads), shared-memory matrix
// descriptors, mbarriers with bounded waits and cp.async gathers.
//
// Operand layout (no swizzle, "interleaved" canonical form): a core matrix is
// 8 rows of 16 bytes (8 bf16) stored contiguously (128 B).  A descriptor gives
// the start address, the byte distance between core matrices adjacent along
// M/N (SBO) and along K (LBO).  For a K-major operand a core-matrix row runs
// along K; for an MN-major operand it runs along M/N.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

namespace isaacb
{
    namespace tc
    {
        __device__ __forceinline__ uint32_t smem_addr(const void* p)
        {
            return static_cast<uint32_t>(__cvta_generic_to_shared(p));
        }

        // ------------------------------------------------------------ descriptors
        // shared-memory matrix descriptor: start, LBO, SBO in 16-byte units, version 1, no swizzle
        __device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
        {
            uint64_t d = 0;
            d |= uint64_t((addr >> 4) & 0x3FFFu);
            d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
            d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
            d |= uint64_t(1) << 46; // descriptor version for sm_100
            return d;
        }

        // instruction descriptor of kind::f16: BF16 A and B, FP32 accumulator, M x N
        __host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool aMN, bool bMN)
        {
            return (1u << 4) // D = F32
                | (1u << 7) // A = BF16
                | (1u << 10) // B = BF16
                | (uint32_t(aMN ? 1 : 0) << 15) | (uint32_t(bMN ? 1 : 0) << 16) | (uint32_t(N >> 3) << 17)
                | (uint32_t(M >> 4) << 24);
        }

        // ------------------------------------------------------------ programmatic dependent launch
        // Wait until the grids this one depends on have completed and their writes are
        // visible (returns at once for a kernel launched without the programmatic
        // serialization attribute), and let the stream's next kernel start its launch.
        __device__ __forceinline__ void grid_dependency_wait()
        {
            asm volatile("griddepcontrol.wait;" ::: "memory");
        }
        __device__ __forceinline__ void grid_launch_dependents()
        {
            asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
        }

        // ------------------------------------------------------------ TMEM
        __device__ __forceinline__ void tmem_alloc(uint32_t* dstSmem, uint32_t cols)
        {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dstSmem)),
                         "r"(cols)
                         : "memory");
        }
        __device__ __forceinline__ void tmem_relinquish()
        {
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
        __device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols)
        {
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
        }
        __device__ __forceinline__ void fence_before_sync()
        {
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        }
        __device__ __forceinline__ void fence_after_sync()
        {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        }
        // generic-proxy shared-memory writes (st.shared, cp.async) -> visible to the tensor cores
        __device__ __forceinline__ void fence_async_smem()
        {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }

        // D[tmem] (+)= A * B^T, issued by one thread
        __device__ __forceinline__ void mma_bf16(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc, uint32_t accumulate)
        {
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dTmem),
                "l"(aDesc),
                "l"(bDesc),
                "r"(idesc),
                "r"(accumulate)
                : "memory");
        }
        // the mbarrier completes one arrival once every MMA issued so far by this thread has finished
        __device__ __forceinline__ void mma_commit(uint64_t* mbar)
        {
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(mbar))
                         : "memory");
        }

        // 8 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes 32*(w%4)..+31)
        __device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8])
        {
            uint32_t r[8];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                         : "r"(taddr)
                         : "memory");
#pragma unroll
            for(int i = 0; i < 8; ++i)
                v[i] = __uint_as_float(r[i]);
        }
        __device__ __forceinline__ void tmem_wait_ld()
        {
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        }

        // ------------------------------------------------------------ mbarriers
        __device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
        {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
        }
        __device__ __forceinline__ void mbar_init_fence()
        {
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity)
        {
            uint32_t done;
            asm volatile(
                "{\n\t.reg .pred P;\n\tmbarrier.test_wait.parity.shared::cta.b64 P, [%1], %2;\n\tselp.u32 %0, 1, 0, P;\n\t}\n"
                : "=r"(done)
                : "r"(smem_addr(bar)), "r"(parity)
                : "memory");
            return done != 0;
        }
        // one potentially blocking probe: the thread is suspended until the phase completes
        // or a hardware time limit passes, so waiting warps take no issue slots
        __device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity)
        {
            uint32_t done;
            asm volatile(
                "{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\tselp.u32 %0, 1, 0, P;\n\t}\n"
                : "=r"(done)
                : "r"(smem_addr(bar)), "r"(parity)
                : "memory");
            return done != 0;
        }
        __device__ __forceinline__ uint64_t global_ns()
        {
            uint64_t t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            return t;
        }
        // bounded wait for the phase with the given parity to complete: false once `budgetNs`
        // of wall time (about one second by default) has passed (checked between probes,
        // whatever each probe's own suspension limit is) or after 2^26 probes, whichever
        // comes first
        __device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t budgetNs = 1000000000ull)
        {
            if(mbar_try(bar, parity))
                return true;
            const uint64_t t0 = global_ns();
            for(int it = 0; it < (1 << 26); ++it)
            {
                if(mbar_try(bar, parity))
                    return true;
                if(global_ns() - t0 > budgetNs)
                    return false;
            }
            return false;
        }

        // one arrival that also expects `bytes` of asynchronous (TMA) transactions
        __device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
        {
            asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(
                             smem_addr(bar)),
                         "r"(bytes)
                         : "memory");
        }
        // tiled TMA loads of a box at integer coordinates (innermost first) into shared
        // memory, completing `bytes` on the mbarrier; no multicast.  dst 128-byte aligned;
        // the innermost coordinate times the element size a multiple of 16 bytes.
        __device__ __forceinline__ void tma_load_4d(uint32_t dst, const void* tmap, int c0, int c1, int c2, int c3, uint64_t* bar)
        {
            asm volatile(
                "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
                    dst),
                "l"(tmap),
                "r"(c0),
                "r"(c1),
                "r"(c2),
                "r"(c3),
                "r"(smem_addr(bar))
                : "memory");
        }
        __device__ __forceinline__ void tma_load_5d(
            uint32_t dst,
            const void* tmap,
            int c0,
            int c1,
            int c2,
            int c3,
            int c4,
            uint64_t* bar)
        {
            asm volatile(
                "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(
                    dst),
                "l"(tmap),
                "r"(c0),
                "r"(c1),
                "r"(c2),
                "r"(c3),
                "r"(c4),
                "r"(smem_addr(bar))
                : "memory");
        }

        __device__ __forceinline__ void mbar_arrive(uint64_t* bar)
        {
            asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(smem_addr(bar)) : "memory");
        }
        // the barrier receives one arrival once all of this thread's earlier cp.async copies have landed
        __device__ __forceinline__ void cp_async_arrive(uint64_t* bar)
        {
            asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
        }

        // ------------------------------------------------------------ cp.async
        // 16-byte gather; srcBytes = 0 writes zeros (the address is not read)
        __device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t srcBytes)
        {
            asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(srcBytes) : "memory");
        }
        __device__ __forceinline__ void cp_async_commit()
        {
            asm volatile("cp.async.commit_group;" ::: "memory");
        }
        template<int N>
        __device__ __forceinline__ void cp_async_wait()
        {
            asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
        }
    } // namespace tc
} // namespace isaacb
