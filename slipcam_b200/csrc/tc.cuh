// tc.cuh -- the Blackwell tensor-core primitives used by the DFT-GEMM form: TMEM allocation,
// tcgen05.mma (kind::f16, operands in shared memory, FP32 accumulators in TMEM), tcgen05.commit to
// an mbarrier, tcgen05.ld back to registers, and the shared-memory matrix and instruction
// descriptors (no swizzle), written from the PTX ISA's descriptions.
//
// Shared-memory operand layout (no swizzle), in bytes, for a 16-bit element (r, k) of an operand
// with rows r (M for A, N for B) and contraction index k:
//   K-major:  (r / 8) * SBO + (k / 8) * LBO + (r % 8) * 16 + (k % 8) * 2
//   MN-major: (r / 8) * SBO + (k / 8) * LBO + (k % 8) * 16 + (r % 8) * 2
// i.e. 128-byte "core matrices" of 8 x 8 elements; one MMA (K = 16) reads two core-matrix columns
// along k from the descriptor's start address.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace b200 {
namespace tc {

B200_HD uint32_t k_major_offset(int r, int k, uint32_t sbo, uint32_t lbo)
{
    return uint32_t(r / 8) * sbo + uint32_t(k / 8) * lbo + uint32_t(r % 8) * 16u + uint32_t(k % 8) * 2u;
}

B200_HD uint32_t mn_major_offset(int r, int k, uint32_t sbo, uint32_t lbo)
{
    return uint32_t(r / 8) * sbo + uint32_t(k / 8) * lbo + uint32_t(k % 8) * 16u + uint32_t(r % 8) * 2u;
}

// the 64-bit shared-memory matrix descriptor: start address, leading (K) and stride (M/N) byte
// offsets, descriptor version 1, no swizzle
B200_HD uint64_t smem_desc(uint32_t smem_addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= uint64_t((smem_addr >> 4) & 0x3FFFu);
    d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
    d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
    d |= uint64_t(1) << 46;   // version
    return d;                 // base offset 0, layout type 0 (no swizzle)
}

// the 32-bit instruction descriptor of kind::f16: F32 accumulation, F16 A and B
B200_HD uint32_t instr_desc(int M, int N, bool a_mn_major, bool b_mn_major, bool neg_a, bool neg_b)
{
    uint32_t d = 0;
    d |= 1u << 4;                                  // c format F32
    // a, b formats F16 = 0 (bits 7-9, 10-12)
    d |= uint32_t(neg_a) << 13;
    d |= uint32_t(neg_b) << 14;
    d |= uint32_t(a_mn_major) << 15;
    d |= uint32_t(b_mn_major) << 16;
    d |= uint32_t(N >> 3) << 17;
    d |= uint32_t(M >> 4) << 24;
    return d;
}

#ifdef __CUDACC__

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// TMEM: one warp allocates ncols (a power of two, >= 32) and writes the base address to *dst
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// D[tmem] (+)= A * B; accumulate: 0 overwrites D, 1 adds to it
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

// the mbarrier arrives when every MMA issued so far by this thread has completed
__device__ __forceinline__ void mma_commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count));
}

// wait for the phase `parity` of the mbarrier to complete; gives up after max_iter polls and
// returns false (the caller records the timeout)
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint32_t max_iter = 1u << 26)
{
    const uint32_t addr = smem_u32(mbar);
    for (uint32_t it = 0; it < max_iter; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive 32-bit TMEM columns of this thread's lane (32 lanes x 32 bit per warp)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 consecutive columns, without waiting (several loads may be issued before tmem_wait)
__device__ __forceinline__ void tmem_ld32_nowait(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t *r)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// NC (a multiple of 16) consecutive columns of this thread's lane into v, one wait for all
template <int NC>
__device__ __forceinline__ void tmem_ld_cols(uint32_t taddr, float (&v)[NC])
{
    static_assert(NC % 16 == 0, "16-column granules");
    uint32_t r[NC];
#pragma unroll
    for (int c = 0; c + 32 <= NC; c += 32) tmem_ld32_nowait(taddr + uint32_t(c), *reinterpret_cast<uint32_t(*)[32]>(r + c));
    if constexpr (NC % 32) tmem_ld16_nowait(taddr + uint32_t(NC - 16), r + NC - 16);
    tmem_wait();
#pragma unroll
    for (int c = 0; c < NC; ++c) v[c] = __uint_as_float(r[c]);
}

// the mbarrier expects `bytes` more bytes of asynchronous copies in the current phase (one arrival)
__device__ __forceinline__ void mbar_expect_tx(uint64_t *mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes) : "memory");
}

// a 3-D box of a tensor map into shared memory (TMA, no multicast); completion is counted on mbar.
// The innermost coordinate x times the element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_3d(void *dst, const void *tmap, int x, int y, int z, uint64_t *mbar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_u32(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(mbar))
        : "memory");
}

// 4-byte asynchronous copies global -> shared, completed by cp_async_wait_all
__device__ __forceinline__ void cp_async4(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

#endif   // __CUDACC__

}   // namespace tc
}   // namespace b200
