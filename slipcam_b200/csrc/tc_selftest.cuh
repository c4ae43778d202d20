// tc_selftest.cuh -- one CTA computes D (128 x N, FP32) = A (128 x K) * B^T (B given as N x K),
// FP16 operands staged in shared memory in a chosen layout (K-major or MN-major for each), on the
// tensor cores (tcgen05.mma, accumulator in TMEM). It checks the descriptor encodings of tc.cuh
// against a host GEMM before they are trusted in the correlation kernels.
#pragma once

#include <cuda_fp16.h>

#include "tc.cuh"

namespace b200 {

#ifdef __CUDACC__

struct TcSelftestArgs {
    const __half *A;   // 128 x K, row-major
    const __half *B;   // N x K, row-major
    float *D;          // 128 x N, row-major
    int N, K;
    int a_mn, b_mn, neg_b;   // layouts and negation of B
    int *status;
};

__global__ void __launch_bounds__(128) tc_selftest_kernel(TcSelftestArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint32_t tmem_base;
    __shared__ __align__(8) uint64_t mbar;
    const int M = 128, N = a.N, K = a.K;
    unsigned char *sa = smem;
    unsigned char *sb = smem + size_t(M) * K * 2;
    // strides: K-major rows of K elements (SBO = K/8 core matrices); MN-major k-groups of rows
    const uint32_t a_sbo = a.a_mn ? 128u : uint32_t(K / 8) * 128u, a_lbo = a.a_mn ? uint32_t(M / 8) * 128u : 128u;
    const uint32_t b_sbo = a.b_mn ? 128u : uint32_t(K / 8) * 128u, b_lbo = a.b_mn ? uint32_t(N / 8) * 128u : 128u;
    for (int idx = threadIdx.x; idx < M * K; idx += blockDim.x) {
        const int r = idx / K, k = idx % K;
        const uint32_t off = a.a_mn ? tc::mn_major_offset(r, k, a_sbo, a_lbo) : tc::k_major_offset(r, k, a_sbo, a_lbo);
        *reinterpret_cast<__half *>(sa + off) = a.A[idx];
    }
    for (int idx = threadIdx.x; idx < N * K; idx += blockDim.x) {
        const int r = idx / K, k = idx % K;
        const uint32_t off = a.b_mn ? tc::mn_major_offset(r, k, b_sbo, b_lbo) : tc::k_major_offset(r, k, b_sbo, b_lbo);
        *reinterpret_cast<__half *>(sb + off) = a.B[idx];
    }
    tc::fence_smem_async();
    if (threadIdx.x < 32) tc::tmem_alloc(&tmem_base, 256);
    if (threadIdx.x == 0) {
        tc::mbar_init(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t d_tmem = tmem_base;
    if (threadIdx.x == 0) {
        const uint32_t idesc = tc::instr_desc(M, N, a.a_mn, a.b_mn, false, a.neg_b != 0);
        for (int s = 0; s < K / 16; ++s) {
            // one MMA covers k in [16 s, 16 s + 16): two k-groups from the start address
            const uint32_t a_start = tc::smem_u32(sa) + uint32_t(2 * s) * (a.a_mn ? a_lbo : 128u);
            const uint32_t b_start = tc::smem_u32(sb) + uint32_t(2 * s) * (a.b_mn ? b_lbo : 128u);
            tc::mma_f16(d_tmem, tc::smem_desc(a_start, a_lbo, a_sbo), tc::smem_desc(b_start, b_lbo, b_sbo), idesc, s > 0);
        }
        tc::mma_commit(&mbar);
    }
    const bool ok = tc::mbar_wait(&mbar, 0);
    tc::fence_after_sync();
    if (!ok && a.status) atomicExch(a.status, 3);
    // warp w reads TMEM lanes 32 w .. 32 w + 31: row m = threadIdx.x
    const int m = threadIdx.x;
    for (int n0 = 0; n0 < N; n0 += 16) {
        float v[16];
        tc::tmem_ld16(d_tmem + (uint32_t(32 * (threadIdx.x / 32)) << 16) + uint32_t(n0), v);
        for (int j = 0; j < 16 && n0 + j < N; ++j) a.D[size_t(m) * N + n0 + j] = ok ? v[j] : 0.0f;
    }
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) tc::tmem_dealloc(d_tmem, 256);
}

#endif   // __CUDACC__

}   // namespace b200
