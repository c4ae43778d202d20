// corr_tc.cuh -- the tensor-core form: the 2-D DFTs of the correlation as dense DFT-matrix GEMMs
// on tcgen05 (FP16 operands, FP32 accumulation in TMEM), one (window, frame) pair at a time per
// persistent CTA. With D = [w_N^{rc}] (Dr = cos, Di = -sin, N x N, resident in shared memory as
// FP16) every stage is a GEMM whose fixed operand is a block of Dr or Di:
//
//   S1  Y  = X Dr|Di          rows i (chip rows), K = j, N = kappa (Re | Im)     X = chip - round(mean)
//   S2  Z^T = Y^T D            rows kappa, K = (Re|Im, i), N = (Re|Im, ky)        A2 MN-major from S1's rows
//   S3  P = Z conj(R) 2^-s     per thread (one kappa row), R the resident reference spectrum
//   S4  Q^T = P^T conj(D)      rows kappa, K = (Re|Im, ky), N = (Re|Im, u < M)    A4 K-major from S3's rows
//   S5  c^T = [Dr|Di] (w Q)    rows v, K = (Re|Im, kappa), N = u                  B5 MN-major from S4's rows
//
// then the normalization by the variance denominators, the argmax and the FP64 peak epilogue of
// the FP32 form. Each stage writes the next stage's operand straight from its TMEM rows: a thread
// owns one accumulator row and stores it as 16-byte chunks, in the major order the next GEMM reads.
// Power-of-two scales keep every FP16 operand in range: |X| <= 255, |Y| <= 255 N, the reference
// spectrum is scaled by 2^-e with 2^e > W * norm >= max |R|, P by 2^-8 (|P| <= N^2 255 2^-8 < 2^15
// for N <= 160) and w Q by 2^-9. Fixed-size tensor-core tiles: rows beyond the data (chip rows >= N, kappa rows
// >= KP, output rows >= M) read whatever follows in shared memory and their results are ignored.
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>

#include "corr_fft.cuh"
#include "tc.cuh"

namespace b200 {

constexpr uint32_t cmax(uint32_t a, uint32_t b) { return a > b ? a : b; }

// the frequency rows kappa of a real N-point row transform (N / 2 + 1), padded to 16
__host__ __device__ constexpr int tc_kp(int N) { return (N / 2 + 1 + 15) / 16 * 16; }

template <int N>
struct TcGeo {
    static constexpr int NH = N / 2 + 1;                            // frequencies of a real row
    static constexpr int KP = tc_kp(N);                             // kappa rows, padded
    static constexpr int T1 = (N + 127) / 128;                      // row tiles of S1
    static constexpr uint32_t SBO_D = uint32_t(N / 8) * 128u;       // Dr, Di, X: K-major rows of N
    static constexpr uint32_t SBO_A = uint32_t(2 * N / 8) * 128u;   // A2 (MN-major), A4 (K-major): K = 2N
    static constexpr uint32_t SBO_B5 = uint32_t(2 * KP / 8) * 128u; // B5 (MN-major): K = 2 KP
    static constexpr uint32_t A_BYTES = uint32_t(KP / 8) * SBO_A;
    static constexpr uint32_t X_BYTES = cmax(uint32_t(N / 8) * SBO_D, 16u * SBO_B5);
    static constexpr uint32_t D_BYTES = uint32_t(N / 8) * SBO_D;
    static constexpr uint32_t OFF_X = A_BYTES, OFF_DR = OFF_X + X_BYTES, OFF_DI = OFF_DR + D_BYTES;
    static constexpr uint32_t END = OFF_DI + D_BYTES;
    // the furthest byte a full 128-row tile reads
    static constexpr uint32_t READ_END = cmax(cmax(16u * SBO_A, OFF_X + uint32_t(T1) * 16u * SBO_D),
                                              cmax(OFF_DI + 16u * SBO_D, END));
    static constexpr size_t smem_bytes = READ_END;
    static constexpr uint32_t TMEM_COLS = 512;
    static_assert(KP <= 128 && T1 * 2 * KP <= 512 && 2 * N <= 512, "TMEM or tile bounds");
    static_assert(READ_END <= 227 * 1024, "shared memory");
};

#ifdef __CUDACC__

__device__ __forceinline__ uint4 pack8(const float *v, float s)
{
    uint4 r;
    __half2 h0 = __floats2half2_rn(v[0] * s, v[1] * s), h1 = __floats2half2_rn(v[2] * s, v[3] * s);
    __half2 h2 = __floats2half2_rn(v[4] * s, v[5] * s), h3 = __floats2half2_rn(v[6] * s, v[7] * s);
    r.x = *reinterpret_cast<uint32_t *>(&h0);
    r.y = *reinterpret_cast<uint32_t *>(&h1);
    r.z = *reinterpret_cast<uint32_t *>(&h2);
    r.w = *reinterpret_cast<uint32_t *>(&h3);
    return r;
}

__device__ __forceinline__ uint4 pack8(const float *v)
{
    uint4 r;
    __half2 h0 = __floats2half2_rn(v[0], v[1]), h1 = __floats2half2_rn(v[2], v[3]);
    __half2 h2 = __floats2half2_rn(v[4], v[5]), h3 = __floats2half2_rn(v[6], v[7]);
    r.x = *reinterpret_cast<uint32_t *>(&h0);
    r.y = *reinterpret_cast<uint32_t *>(&h1);
    r.z = *reinterpret_cast<uint32_t *>(&h2);
    r.w = *reinterpret_cast<uint32_t *>(&h3);
    return r;
}

// kTcCompute compute warps, kTcParts per TMEM lane quadrant (warps w, w + 4, ... own the same 32
// accumulator rows and split their columns), and a control warp whose first thread issues the MMAs
// and the TMA copies, polls their completion and does the per-pair scalar work, so that no compute
// warp waits behind the tensor core's issue queue
constexpr int kTcCompute = 12;
constexpr int kTcParts = kTcCompute / 4;
constexpr int kTcThreads = 32 * (kTcCompute + 1);
constexpr int kTcCtrl = 32 * kTcCompute;   // the control thread

// the MMAs of the current phase have completed: the control thread polls the mbarrier, the others
// wait at the barrier; false (for all threads) if the poll gave up or any thread passes also_failed
__device__ __forceinline__ bool tc_wait_all(uint64_t *mbar, uint32_t &phase, bool also_failed = false)
{
    bool ok = true;
    if (threadIdx.x == kTcCtrl) ok = tc::mbar_wait(mbar, phase);
    phase ^= 1u;
    const bool failed = __syncthreads_or(!ok || also_failed);
    tc::fence_after_sync();
    return !failed;
}

// 4 pixels (a little-endian word) minus the same offset, as two exact FP16 pairs: a byte b placed
// under the exponent byte 0x64 reads as the half 1024 + b, and 1024 + b - (1024 + m) is exact
__device__ __forceinline__ void bytes_to_half(uint32_t word, __half2 off, uint32_t &lo, uint32_t &hi)
{
    uint32_t a = __byte_perm(word, 0x64646464u, 0x4140);   // (1024 + b0, 1024 + b1)
    uint32_t b = __byte_perm(word, 0x64646464u, 0x4342);   // (1024 + b2, 1024 + b3)
    __half2 ha = __hsub2(*reinterpret_cast<__half2 *>(&a), off);
    __half2 hb = __hsub2(*reinterpret_cast<__half2 *>(&b), off);
    lo = *reinterpret_cast<uint32_t *>(&ha);
    hi = *reinterpret_cast<uint32_t *>(&hb);
}

// shared-memory operands written by this thread become visible to the tensor core
__device__ __forceinline__ void tc_publish()
{
    tc::fence_smem_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
}

// one (window, frame) pair of the tensor-core kernel, as one thread works it out ahead of time
struct PairSetup {
    int64_t q;              // the output index f * nwin + k
    int p, k, f, gy, gx;    // pair, window, frame, gross offset
    int sy, sx, mean;       // the chip's top-left corner and its rounded mean
    float norm;
    bool ok;                // the chip lies inside the frame and the reference window has texture
};


// the rows of the variance-denominator box a TMA copy brings in: x rounded down to 4 floats
// (16 bytes), so BW = M + 3 rounded up to 4 floats per row
__host__ __device__ constexpr int tc_box_width(int M) { return (M + 3 + 3) / 4 * 4; }

// dmap (global memory): the variance denominators of the group as a 3-D tensor (x = column,
// y = row, z = frame), box tc_box_width(M) x M x 1
template <int N>
__global__ void __launch_bounds__(kTcThreads, 1) corr_tc_kernel(CorrArgs a, const uint4 *dtab, int *status,
                                                                  const CUtensorMap *dmap)
{
    using G = TcGeo<N>;
    constexpr int NH = G::NH, KP = G::KP, NT = kTcThreads;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint32_t tmem_base;
    __shared__ __align__(8) uint64_t mbar, tbar;
    __shared__ float s_best[NT / 32];
    __shared__ int s_at[NT / 32];
    __shared__ double s_sq[NT / 32];
    __shared__ float s_fit[9];
    __shared__ int s_peak[3];   // the pending pair's peak: valid, u, v
    __shared__ PairSetup s_next;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int quad = warp & 3, part = warp >> 2;
    const int row = 32 * quad + lane;   // this thread's accumulator row (TMEM lane)
    const bool compute = warp < kTcCompute, ctrl = tid == kTcCtrl;
    unsigned char *A = smem, *X = smem + G::OFF_X;
    float *dvs = reinterpret_cast<float *>(X);         // the variance denominators, from S2 on (X region)
    const uint32_t sA = tc::smem_u32(A), sX = tc::smem_u32(X);
    const uint32_t sDR = tc::smem_u32(smem + G::OFF_DR), sDI = tc::smem_u32(smem + G::OFF_DI);

    // the DFT matrices (already in the K-major layout), once per CTA
    for (int i = tid; i < int(2 * G::D_BYTES / 16); i += NT)
        reinterpret_cast<uint4 *>(smem + G::OFF_DR)[i] = __ldg(dtab + i);
    if (warp == 0) tc::tmem_alloc(&tmem_base, G::TMEM_COLS);
    if (ctrl) {
        tc::mbar_init(&mbar, 1);
        tc::mbar_init(&tbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_publish();
    const uint32_t tmem = tmem_base;
    uint32_t tphase = 0;
    const int BW = tc_box_width(a.M);
    const uint32_t lane_base = uint32_t(32 * quad) << 16;
    // the descriptors at k = 0 (built where they are used); the k-step s starts 256 s bytes on
    // (16 s in the start-address field)
#define B200_TC_DESCS                                                                                  \
    const uint64_t dR0 = tc::smem_desc(sDR, 128, G::SBO_D), dI0 = tc::smem_desc(sDI, 128, G::SBO_D); \
    const uint64_t a0A = tc::smem_desc(sA, 128, G::SBO_A), b0B5 = tc::smem_desc(sA, 128, G::SBO_B5);  \
    (void)dR0; (void)dI0; (void)a0A; (void)b0B5;
    uint32_t phase = 0;
    const int L = a.L, M = a.M, R = a.R, W = a.W;
    const int NO = (M + 15) / 16 * 16;
    const int npairs = a.nwin * a.nf;
    const size_t ss = size_t(a.w) + 1;
    const bool words = ((a.pitch | reinterpret_cast<uintptr_t>(a.frames) | int(a.fstride)) & 3) == 0;

    // the pair whose epilogue is pending: its S5 result in TMEM columns [C5, C5 + NO) while the next
    // pair runs S1 .. S4; its variance denominators come by TMA into the X region after the next
    // pair's S1, the normalization and argmax run during its S2, the SNR patch and the 3 x 3 fit
    // values (read back from TMEM) during its S4, the FP64 peak solve during its S5
    struct Prev {
        int64_t q;
        int f, sy, sx, gy, gx;
        float scale;
        bool live;
    } prev{0, 0, 0, 0, 0, 0, 0.0f, false};
    const uint32_t C5 = uint32_t(G::TMEM_COLS - NO);
    float e_best = -2.0f;   // this thread's running argmax of the pending pair
    int e_at = INT_MAX;
    bool e_valid = false;   // the pending pair's surface has a positive peak
    int e_pu = 0, e_pv = 0;

    // the next pair's window, frame, position and chip mean, worked out by one thread of the last
    // warp while the tensor cores run S1 (global-memory latency off the gather's path)
    auto pair_setup = [&](int p) {
        PairSetup o{};
        o.p = p;
        if (p >= npairs) return o;
        o.k = p / a.nf;
        o.f = p % a.nf;
        o.q = int64_t(o.f) * a.nwin + o.k;
        if (a.gross_mode == 1) {
            o.gy = a.gross[2 * o.f];
            o.gx = a.gross[2 * o.f + 1];
        } else if (a.gross_mode == 2) {
            o.gy = a.gross[2 * o.q];
            o.gx = a.gross[2 * o.q + 1];
        }
        o.sy = a.down[o.k / a.nx] + o.gy - R;
        o.sx = a.across[o.k % a.nx] + o.gx - R;
        o.norm = a.norm[o.k];
        o.ok = o.norm > 0 && o.sy >= 0 && o.sx >= 0 && o.sy + L <= a.h && o.sx + L <= a.w;
        if (o.ok) {
            const uint32_t *sat = a.sat + size_t(o.f) * a.sat_fstride;
            const int sy = o.sy, sx = o.sx;
            const uint32_t box = sat[(sy + L) * ss + sx + L] - sat[sy * ss + sx + L] - sat[(sy + L) * ss + sx] + sat[sy * ss + sx];
            const uint32_t LL = uint32_t(L) * uint32_t(L);
            o.mean = int((box + LL / 2) / LL);
        }
        return o;
    };

    // ---- X = chip - round(mean), FP16, K-major (rows i, columns j), zero outside L x L. Two ways:
    // rows16 (frame rows on 16-byte boundaries and whole 16-byte chunks per row, the width a
    // multiple of 16, so a row's chunks never leave it): aligned 16-byte chunk loads, below; else a
    // warp takes 8 rows x 4 chunks of 8 pixels as 4-byte words, 32-byte pieces of 8 rows from global
    // memory and one contiguous 512-byte store into shared memory. Every load of a thread first.
    const bool rows16 = ((reinterpret_cast<uintptr_t>(a.frames) | uintptr_t(a.pitch) | uintptr_t(a.fstride)) & 15) == 0 &&
                        (a.w & 15) == 0;
    auto gather = [&](const PairSetup &c) {
        if (!compute) return;
        const __half2 off = __float2half2_rn(1024.0f + float(c.mean));
        const uint8_t *chip = a.frames + c.f * a.fstride + int64_t(c.sy) * a.pitch + c.sx;
        if (rows16 && N <= 160) {
            // a warp takes groups of 8 chip rows: lane (r, c) = (lane & 7, lane >> 3) loads the aligned
            // 16-byte chunks c, c + 4, c + 8 of row r (the chip's first byte is byte o of chunk 0, the
            // same o on every row), then writes chip columns 16 q .. 16 q + 15 (q = c + 4 k) from
            // chunks q and q + 1 as two 16-byte FP16 pieces: the 8 lanes of one c fill 128
            // contiguous bytes of a core matrix
            const int o = c.sx & 15, sw = o >> 2, sb = 8 * (o & 3);
            const int r = lane & 7, cg = lane >> 3;
            const int nq = (o + L + 15) >> 4;   // chunks holding chip bytes (they end inside the row)
            const uint4 *rb = reinterpret_cast<const uint4 *>(chip - o);
            const int64_t pq = a.pitch >> 4;    // chunks per frame row
            constexpr int NK = ((N + 30) / 16 + 3) / 4;                  // rounds of 4 chunks (nq <= 4 NK)
            constexpr int NG = N / 8;                                    // groups of 8 rows
            constexpr int GPW = (NG + kTcCompute - 1) / kTcCompute;      // groups per warp
            uint4 all[GPW][NK];   // every load of the warp first: one round trip to memory
#pragma unroll
            for (int t = 0; t < GPW; ++t) {
                const int gi = warp + kTcCompute * t, i = 8 * gi + r;
#pragma unroll
                for (int k = 0; k < NK; ++k) {
                    const int qq = cg + 4 * k;
                    all[t][k] = make_uint4(0u, 0u, 0u, 0u);
                    if (gi < NG && i < L && qq < nq) all[t][k] = __ldg(rb + int64_t(i) * pq + qq);
                }
            }
#pragma unroll
            for (int t = 0; t < GPW; ++t) {
                const int gi = warp + kTcCompute * t, i = 8 * gi + r;
                if (gi >= NG) break;   // warp-uniform
                uint4 raw[NK + 1];
#pragma unroll
                for (int k = 0; k < NK; ++k) raw[k] = all[t][k];
                raw[NK] = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
                for (int k = 0; k < NK; ++k) {
                    // chunk q + 1: lane (r, c + 1) of this round, or lane (r, 0) of the next
                    const int down = (lane + 8) & 31;
                    uint4 nx, nn;
                    nx.x = __shfl_sync(0xffffffffu, raw[k].x, down);
                    nx.y = __shfl_sync(0xffffffffu, raw[k].y, down);
                    nx.z = __shfl_sync(0xffffffffu, raw[k].z, down);
                    nx.w = __shfl_sync(0xffffffffu, raw[k].w, down);
                    nn.x = __shfl_sync(0xffffffffu, raw[k + 1].x, r);
                    nn.y = __shfl_sync(0xffffffffu, raw[k + 1].y, r);
                    nn.z = __shfl_sync(0xffffffffu, raw[k + 1].z, r);
                    nn.w = __shfl_sync(0xffffffffu, raw[k + 1].w, r);
                    if (cg == 3) nx = nn;
                    const int q = cg + 4 * k;
                    if (q >= N / 16) continue;
                    const uint32_t w[8] = {raw[k].x, raw[k].y, raw[k].z, raw[k].w, nx.x, nx.y, nx.z, nx.w};
                    uint32_t b[5];   // bytes 4 sw .. 4 sw + 19 of the 32 (sw is the same on every lane)
                    switch (sw) {
                    case 0: b[0] = w[0]; b[1] = w[1]; b[2] = w[2]; b[3] = w[3]; b[4] = w[4]; break;
                    case 1: b[0] = w[1]; b[1] = w[2]; b[2] = w[3]; b[3] = w[4]; b[4] = w[5]; break;
                    case 2: b[0] = w[2]; b[1] = w[3]; b[2] = w[4]; b[3] = w[5]; b[4] = w[6]; break;
                    default: b[0] = w[3]; b[1] = w[4]; b[2] = w[5]; b[3] = w[6]; b[4] = w[7]; break;
                    }
                    uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = make_uint4(0u, 0u, 0u, 0u);
                    if (i < L) {
                        bytes_to_half(__funnelshift_r(b[0], b[1], sb), off, lo.x, lo.y);
                        bytes_to_half(__funnelshift_r(b[1], b[2], sb), off, lo.z, lo.w);
                        bytes_to_half(__funnelshift_r(b[2], b[3], sb), off, hi.x, hi.y);
                        bytes_to_half(__funnelshift_r(b[3], b[4], sb), off, hi.z, hi.w);
                        const int keep = L - 16 * q;   // chip columns from 16 q on
                        if (keep < 16) {   // the 8 words of the 16 halves: zero past the chip
                            uint32_t hv[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
#pragma unroll
                            for (int e = 0; e < 8; ++e) {
                                if (2 * e >= keep) hv[e] = 0u;
                                else if (2 * e + 1 >= keep) hv[e] &= 0xFFFFu;
                            }
                            lo = make_uint4(hv[0], hv[1], hv[2], hv[3]);
                            hi = make_uint4(hv[4], hv[5], hv[6], hv[7]);
                        }
                    }
                    *reinterpret_cast<uint4 *>(X + tc::k_major_offset(i, 16 * q, G::SBO_D, 128)) = lo;
                    *reinterpret_cast<uint4 *>(X + tc::k_major_offset(i, 16 * q + 8, G::SBO_D, 128)) = hi;
                }
            }
        } else {
                constexpr int NCG = (N / 8 + 3) / 4;               // groups of 4 chunks per row
                constexpr int NB = (N / 8) * NCG;                   // blocks of 8 rows x 4 chunks
                constexpr int PERT = (NB + kTcCompute - 1) / kTcCompute;   // blocks per warp
                constexpr int PERW = (PERT + 1) / 2;                    // in two rounds
    #pragma unroll
                for (int round = 0; round < 2; ++round) {
                uint32_t w0[PERW], w1[PERW], w2[PERW];
    #pragma unroll
                for (int t = 0; t < PERW; ++t) {
                    const int b = warp + kTcCompute * (t + round * PERW);
                    const int i = 8 * (b / NCG) + (lane & 7), j0 = 8 * (4 * (b % NCG) + (lane >> 3));
                    w0[t] = w1[t] = w2[t] = 0u;
                    if (b < NB && t + round * PERW < PERT && i < L && j0 < L && j0 < N) {
                        const uint8_t *src = chip + int64_t(i) * a.pitch + j0;
                        const int left = L - j0;   // chip bytes from src on
                        if (words) {
                            // the aligned words holding the chip bytes among src[0 .. 8)
                            const uintptr_t addr = reinterpret_cast<uintptr_t>(src);
                            const uint32_t *wp = reinterpret_cast<const uint32_t *>(addr & ~uintptr_t(3));
                            const int sh = int(addr & 3);
                            w0[t] = __ldg(wp);
                            if (4 - sh < left) w1[t] = __ldg(wp + 1);
                            if (sh > 0 && 8 - sh < left) w2[t] = __ldg(wp + 2);
                        } else {
                            for (int e = 0; e < 8 && e < left; ++e) {
                                const uint32_t bt = __ldg(src + e);
                                if (e < 4) w0[t] |= bt << (8 * e);
                                else w1[t] |= bt << (8 * (e - 4));
                            }
                        }
                    }
                }
    #pragma unroll
                for (int t = 0; t < PERW; ++t) {
                    const int b = warp + kTcCompute * (t + round * PERW);
                    const int i = 8 * (b / NCG) + (lane & 7), j0 = 8 * (4 * (b % NCG) + (lane >> 3));
                    if (b < NB && t + round * PERW < PERT && j0 < N) {
                        uint4 out = make_uint4(0u, 0u, 0u, 0u);
                        if (i < L && j0 < L) {
                            uint32_t lo = w0[t], hi = w1[t];
                            if (words) {
                                const int sh = int(reinterpret_cast<uintptr_t>(chip + int64_t(i) * a.pitch + j0) & 3);
                                lo = __funnelshift_r(w0[t], w1[t], 8 * sh);
                                hi = __funnelshift_r(w1[t], w2[t], 8 * sh);
                            }
                            bytes_to_half(lo, off, out.x, out.y);
                            bytes_to_half(hi, off, out.z, out.w);
                            if (j0 + 8 > L) {   // the last chunk of a row: zero past the chip
                                const int keep = L - j0;   // 1 .. 7 pixels
                                uint32_t *o = reinterpret_cast<uint32_t *>(&out);
    #pragma unroll
                                for (int e = 0; e < 4; ++e) {
                                    if (2 * e >= keep) o[e] = 0u;
                                    else if (2 * e + 1 >= keep) o[e] &= 0xFFFFu;
                                }
                            }
                        }
                        *reinterpret_cast<uint4 *>(X + tc::k_major_offset(i, j0, G::SBO_D, 128)) = out;
                    }
                }
                }
        }
        tc::fence_smem_async();   // the chip is read by the tensor core
    };

    // ---- the pending pair's epilogue, in three parts (all threads call each)
    // the denominator box (rows sy .. sy + M - 1, columns from sx rounded down to 4) into X
    bool tma_pending = false;   // a denominator box is on its way (waited out before leaving)
    auto epi_fetch = [&]() {
        if (ctrl) {
            tc::mbar_expect_tx(&tbar, uint32_t(BW * M * 4));
            tc::tma_load_3d(dvs, dmap, prev.sx & ~3, prev.sy, prev.f, &tbar);
        }
        tma_pending = true;
    };
    // the normalized surface (thread v holds column v) and this thread's argmax; 16-column chunks
    // of u alternate among the warps of a quadrant. false if the box did not arrive.
    auto epi_normalize = [&]() -> bool {
        const bool ok = tc::mbar_wait(&tbar, tphase);
        tphase ^= 1u;
        tma_pending = !ok;
        e_best = -2.0f;
        e_at = INT_MAX;
        if (compute && 32 * quad < M) {
            const int v = row;
            const bool vin = v < M;
            const float *__restrict__ dv = dvs + (prev.sx & 3) + v;
            float *sv = a.surface ? a.surface + prev.q * M * M + v : nullptr;
            for (int u0 = 16 * part; u0 < NO; u0 += 16 * kTcParts) {   // one 16-column chunk of u per TMEM wait
                uint32_t cr[16];
                tc::tmem_ld16_nowait(tmem + lane_base + C5 + uint32_t(u0), cr);
                const int nu = M - u0 < 16 ? M - u0 : 16;   // rows u of the chunk inside the surface
                float rho[16];
#pragma unroll
                for (int e = 0; e < 16; ++e) rho[e] = vin && e < nu ? dv[(u0 + e) * BW] : 0.0f;
                tc::tmem_wait();
#pragma unroll
                for (int e = 0; e < 16; ++e) rho[e] *= __uint_as_float(cr[e]) * prev.scale;
                if (vin) {
                    if (sv) {
#pragma unroll
                        for (int e = 0; e < 16; ++e)
                            if (e < nu) sv[(u0 + e) * M] = rho[e];
                    }
#pragma unroll
                    for (int e = 0; e < 16; ++e)   // values <= -2 and NaN never win; ties keep the first u
                        if (e < nu && rho[e] > e_best) {
                            e_best = rho[e];
                            e_at = u0 + e;
                        }
                }
            }
            e_at = e_at == INT_MAX ? INT_MAX : e_at * M + v;
        }
        return ok;
    };
    // the surface's argmax (the first in raster order if equal), then the SNR patch's sum of squares
    // and the 3 x 3 fit's values, read back from TMEM with the same arithmetic
    // (the compute warps only, with their own barrier: the control thread may still be issuing)
    auto epi_peak = [&]() {
        float best = e_best;
        int at = e_at;
        for (int o = 16; o > 0; o >>= 1) better(best, at, __shfl_xor_sync(0xffffffffu, best, o), __shfl_xor_sync(0xffffffffu, at, o));
        if (lane == 0) {
            s_best[warp] = best;
            s_at[warp] = at;
        }
        asm volatile("bar.sync 1, %0;" ::"n"(32 * kTcCompute) : "memory");
        best = lane < kTcCompute ? s_best[lane] : -2.0f;
        at = lane < kTcCompute ? s_at[lane] : INT_MAX;
        for (int o = 16; o > 0; o >>= 1) better(best, at, __shfl_xor_sync(0xffffffffu, best, o), __shfl_xor_sync(0xffffffffu, at, o));
        e_valid = best > 0;
        double sq = 0.0;
        if (e_valid) {
            e_pu = at / M;
            e_pv = at % M;
        }
        if (tid == 0) {   // for the control thread's solve
            s_peak[0] = e_valid;
            s_peak[1] = e_pu;
            s_peak[2] = e_pv;
        }
        if (e_valid) {
            int i0, i1, j0, j1;
            snr_patch(M, a.stat, e_pu, e_pv, i0, i1, j0, j1);
            // the warps of a quadrant take alternate 16-row chunks of u from i0
            if (compute && 32 * quad < j1 && 32 * quad + 32 > j0) {   // warp-uniform
                for (int c0 = i0 + 16 * part; c0 < i1; c0 += 16 * kTcParts) {
                    const int cb = c0 + 16 <= NO ? c0 : NO - 16;   // 16 columns inside [0, NO)
                    uint32_t cr[16];
                    tc::tmem_ld16_nowait(tmem + lane_base + C5 + uint32_t(cb), cr);
                    tc::tmem_wait();
                    const int v = row;
                    if (v >= j0 && v < j1) {
                        const float *__restrict__ dv = dvs + (prev.sx & 3) + v;
#pragma unroll
                        for (int e = 0; e < 16; ++e) {
                            const int u = cb + e;
                            if (u < c0 || u >= i1 || u >= c0 + 16) continue;
                            float rho = dv[u * BW];
                            rho *= __uint_as_float(cr[e]) * prev.scale;
                            sq += double(rho) * double(rho);
                            const int du = u - e_pu, dvv = v - e_pv;
                            if (du >= -1 && du <= 1 && dvv >= -1 && dvv <= 1) s_fit[(du + 1) * 3 + dvv + 1] = rho;
                        }
                    }
                }
            }
        }
        for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
        if (lane == 0) s_sq[warp] = sq;
    };
    // the FP64 peak solve and the outputs (one thread), from s_fit and s_sq
    auto epi_finish = [&]() {
        e_valid = s_peak[0] != 0;
        e_pu = s_peak[1];
        e_pv = s_peak[2];
        if (!e_valid) {
            invalid_outputs(prev.q, a.offset, a.peak, a.snr, a.cov);
            if (a.peaks) a.peaks[prev.q].valid = 0;
            return;
        }
        int i0, i1, j0, j1;
        snr_patch(M, a.stat, e_pu, e_pv, i0, i1, j0, j1);
        double sum = 0.0;
        for (int w = 0; w < kTcCompute; ++w) sum += s_sq[w];
        if (a.peaks) {   // for the exact refinement of the peak, which writes the pair's outputs
            PeakInfo &pi = a.peaks[prev.q];
            pi.valid = 1;
            pi.u = e_pu;
            pi.v = e_pv;
            pi.count = (i1 - i0) * (j1 - j0);
            pi.sum = sum;
            for (int t = 0; t < 9; ++t) pi.fit[t] = s_fit[t];
            return;
        }
        peak_outputs(s_fit + 4, 3, M, e_pu, e_pv, R, prev.gy, prev.gx, W * W, sum, (i1 - i0) * (j1 - j0), prev.q,
                     a.offset, a.peak, a.snr, a.cov);
    };
    // the whole epilogue of the pending pair, not overlapped (before a gather that needs X, and at
    // the end); false if a wait gave up
    auto epi_flush = [&]() -> bool {
        if (!prev.live) return true;
        epi_fetch();
        const bool ok = epi_normalize();
        if (compute) epi_peak();
        __syncthreads();
        if (ctrl) epi_finish();
        prev.live = false;
        return !__syncthreads_or(!ok);
    };

    if (ctrl) s_next = pair_setup(blockIdx.x);
    __syncthreads();
    PairSetup cur = s_next;
    if (cur.p < npairs && cur.ok) gather(cur);
    tc_publish();
    bool failed = false;
    while (cur.p < npairs) {
        if (!cur.ok) {   // an invalid pair: its outputs now (the pending epilogue waits)
            if (ctrl) {
                invalid_outputs(cur.q, a.offset, a.peak, a.snr, a.cov);
                if (a.peaks) a.peaks[cur.q].valid = 0;
            }
            if (a.surface)
                for (int i = tid; i < M * M; i += NT) a.surface[cur.q * M * M + i] = 0.0f;
            if (ctrl) s_next = pair_setup(cur.p + gridDim.x);
            __syncthreads();
            cur = s_next;
            __syncthreads();
            if (cur.p < npairs && cur.ok) {
                if (!epi_flush()) {
                    failed = true;
                    break;
                }
                gather(cur);
                tc_publish();
            }
            continue;
        }
        const int k = cur.k;
        const float norm = cur.norm;

        // ---- S1: Y = X [Dr | Di], tile t of 128 chip rows -> TMEM columns [2 KP t, 2 KP (t + 1))
        if (ctrl) {
            B200_TC_DESCS
            const uint32_t id = tc::instr_desc(128, KP, false, false, false, false);
#pragma unroll
            for (int t = 0; t < G::T1; ++t) {
                const uint64_t a0 = tc::smem_desc(sX + uint32_t(t * 16) * G::SBO_D, 128, G::SBO_D);
#pragma unroll 2
                for (int s = 0; s < N / 16; ++s) {
                    tc::mma_f16(tmem + uint32_t(2 * KP * t), a0 + 16u * s, dR0 + 16u * s, id, s > 0);
                    tc::mma_f16(tmem + uint32_t(2 * KP * t + KP), a0 + 16u * s, dI0 + 16u * s, id, s > 0);
                }
            }
            tc::mma_commit(&mbar);
        }
        if (tid == kTcCtrl - 32) s_next = pair_setup(cur.p + gridDim.x);   // a compute warp, idle during S1
        if (!tc_wait_all(&mbar, phase)) {
            failed = true;
            break;
        }
        // the pending pair's denominators into X (free: S1 has read the chip), under the S1 drain
        if (prev.live) epi_fetch();
        // S1 -> A2 (MN-major: m = kappa, k = part * N + i); the warps of a quadrant take the
        // (Re or Im, column block) units in turn
        for (int t = 0; t < G::T1; ++t) {
            if (!compute || 128 * t + 32 * quad >= N) continue;   // warp-uniform
            const int i = 128 * t + row;
            constexpr int NC = KP % 32 ? 16 : 32;   // columns per wait
            constexpr int NCH = KP / NC;
            for (int un = part; un < 2 * NCH; un += kTcParts) {
                const int ri = un / NCH, cb = NC * (un - ri * NCH);
                float v[NC];
                tc::tmem_ld_cols<NC>(tmem + lane_base + uint32_t(2 * KP * t + ri * KP + cb), v);
                if (i < N) {
#pragma unroll
                    for (int c0 = 0; c0 < NC; c0 += 8)
                        *reinterpret_cast<uint4 *>(A + tc::mn_major_offset(cb + c0, ri * N + i, G::SBO_A, 128)) = pack8(v + c0);
                }
            }
        }
        tc_publish();

        // ---- S2: Z^T = Y^T D: Zr in TMEM columns [0, N), Zi in [N, 2N)
        if (ctrl) {
            B200_TC_DESCS
            const uint32_t id = tc::instr_desc(128, N, true, false, false, false);
            const uint32_t idn = tc::instr_desc(128, N, true, false, false, true);
#pragma unroll 2
            for (int s = 0; s < N / 16; ++s) {
                const uint64_t ar = a0A + 16u * s, ai = a0A + uint32_t(N + 16 * s);   // Yr: k = i, Yi: k = N + i
                tc::mma_f16(tmem, ar, dR0 + 16u * s, id, s > 0);        // Zr += Yr Dr
                tc::mma_f16(tmem, ai, dI0 + 16u * s, idn, 1);           // Zr -= Yi Di
                tc::mma_f16(tmem + N, ar, dI0 + 16u * s, id, s > 0);    // Zi += Yr Di
                tc::mma_f16(tmem + N, ai, dR0 + 16u * s, id, 1);        // Zi += Yi Dr
            }
            tc::mma_commit(&mbar);
        }
        // the next pair's chip and reference spectrum into L2 while the tensor cores run S2 (its
        // gather comes during this pair's S5, its S3 one pair later): a few prefetches per thread,
        // every line holding bytes of the chip (inside the frame) or of the window's spectrum
        if (compute) {
            const PairSetup &nx = s_next;
            if (nx.p < npairs && nx.ok) {
                const uint8_t *chip = a.frames + nx.f * a.fstride + int64_t(nx.sy) * a.pitch + nx.sx;
                for (int e = tid; e < 3 * L; e += 32 * kTcCompute) {   // a row of L <= 256 bytes spans <= 3 lines
                    const int i = e / 3, l = e - 3 * i;
                    const uintptr_t first = reinterpret_cast<uintptr_t>(chip + int64_t(i) * a.pitch);
                    const uintptr_t line = (first & ~uintptr_t(127)) + 128 * uintptr_t(l);
                    if (line <= first + uintptr_t(L - 1)) asm volatile("prefetch.global.L2 [%0];" ::"l"(line));
                }
                if (nx.k != k) {
                    const char *r = reinterpret_cast<const char *>(a.spec_tc + size_t(nx.k) * (N / 2) * KP);
                    constexpr int RL = (N / 2) * KP * 16 / 128;   // whole lines: KP is a multiple of 16
                    for (int e = tid; e < RL; e += 32 * kTcCompute)
                        asm volatile("prefetch.global.L2 [%0];" ::"l"(r + 128 * size_t(e)));
                }
            }
        }
        // this thread's row of the reference spectrum (S3): frequency pairs (ky, ky + 1) of the
        // rows kappa side by side, KP float4 per pair (rows NH .. KP - 1 zero)
        int eR = 0;
        frexpf(float(W) * norm, &eR);   // W * norm < 2^eR, and max |R| <= W * norm
        const int kap = row;
        const float4 *rrow = a.spec_tc + size_t(k) * (N / 2) * KP + (kap < KP ? kap : 0);
        const bool tma_ok = prev.live ? epi_normalize() : true;   // while the tensor cores run S2
        if (!tc_wait_all(&mbar, phase, !tma_ok)) {
            failed = true;
            break;
        }

        // ---- S3: P = Z conj(R) 2^-(eR + 8) -> A4 (K-major: row kappa, k = part * N + ky); the
        // 16-column chunks of ky alternate among the warps of a quadrant
        if (compute && 32 * quad < KP) {
            const float sc = ldexpf(1.0f, -(eR + 8));
            for (int c0 = 16 * part; c0 < N; c0 += 16 * kTcParts) {
                uint32_t zr[16], zi[16];
                tc::tmem_ld16_nowait(tmem + lane_base + uint32_t(c0), zr);
                tc::tmem_ld16_nowait(tmem + lane_base + uint32_t(N + c0), zi);
                float4 rc[8];   // the spectrum's 16 frequencies of the chunk (the other warps of the quadrant hide the wait)
#pragma unroll
                for (int e = 0; e < 8; ++e) rc[e] = kap < KP ? __ldg(rrow + (c0 / 2 + e) * KP) : make_float4(0.f, 0.f, 0.f, 0.f);
                tc::tmem_wait();
                if (kap < KP) {
#pragma unroll
                    for (int hh = 0; hh < 2; ++hh) {   // 8 frequencies at a time
                        float pr[8], pi[8];
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const float4 r = rc[4 * hh + e];
                            const int z = 8 * hh + 2 * e;
                            const float ar = __uint_as_float(zr[z]), ai = __uint_as_float(zi[z]);
                            const float br = __uint_as_float(zr[z + 1]), bi = __uint_as_float(zi[z + 1]);
                            pr[2 * e] = (ar * r.x + ai * r.y) * sc;
                            pi[2 * e] = (ai * r.x - ar * r.y) * sc;
                            pr[2 * e + 1] = (br * r.z + bi * r.w) * sc;
                            pi[2 * e + 1] = (bi * r.z - br * r.w) * sc;
                        }
                        *reinterpret_cast<uint4 *>(A + tc::k_major_offset(kap, c0 + 8 * hh, G::SBO_A, 128)) = pack8(pr);
                        *reinterpret_cast<uint4 *>(A + tc::k_major_offset(kap, N + c0 + 8 * hh, G::SBO_A, 128)) = pack8(pi);
                    }
                }
            }
        }
        tc_publish();

        // ---- S4: Q^T = P^T conj(D) for u < NO: Qr in TMEM columns [0, NO), Qi in [NO, 2 NO)
        if (ctrl) {
            B200_TC_DESCS
            const uint32_t id = tc::instr_desc(128, NO, false, false, false, false);
            const uint32_t idn = tc::instr_desc(128, NO, false, false, false, true);
#pragma unroll 2
            for (int s = 0; s < N / 16; ++s) {
                const uint64_t ar = a0A + 16u * s, ai = a0A + uint32_t(N + 16 * s);   // Pr, Pi
                tc::mma_f16(tmem, ar, dR0 + 16u * s, id, s > 0);                 // Qr += Pr Dr
                tc::mma_f16(tmem, ai, dI0 + 16u * s, id, 1);                     // Qr += Pi Di
                tc::mma_f16(tmem + uint32_t(NO), ar, dI0 + 16u * s, idn, s > 0); // Qi -= Pr Di
                tc::mma_f16(tmem + uint32_t(NO), ai, dR0 + 16u * s, id, 1);      // Qi += Pi Dr
            }
            tc::mma_commit(&mbar);
        }
        if (prev.live && compute) epi_peak();   // while the tensor cores run S4
        if (!tc_wait_all(&mbar, phase)) {
            failed = true;
            break;
        }
        // S4 -> B5 in the A region (MN-major: n = u, k = part * KP + kappa), with the Hermitian
        // weights and 2^-9; the warps of a quadrant take the (Qr or Qi, 32-column block) units in turn
        if (compute && 32 * quad < KP) {
            const int kap = row;
            const float wgt = kap >= NH ? 0.0f : ((kap == 0 || 2 * kap == N) ? 1.0f : 2.0f) * (1.0f / 512.0f);
            const int nch = (NO + 31) / 32;
            for (int un = part; un < 2 * nch; un += kTcParts) {
                const int reim = un / nch, c0 = 32 * (un - reim * nch);
                uint32_t r[32];
                tc::tmem_ld16_nowait(tmem + lane_base + uint32_t(reim * NO + c0), r);
                if (c0 + 16 < NO) tc::tmem_ld16_nowait(tmem + lane_base + uint32_t(reim * NO + c0 + 16), r + 16);
                tc::tmem_wait();
                if (kap < KP) {
                    float v[32];
#pragma unroll
                    for (int e = 0; e < 32; ++e) v[e] = __uint_as_float(r[e]);
#pragma unroll
                    for (int h = 0; h < 4; ++h)
                        if (c0 + 8 * h < NO)
                            *reinterpret_cast<uint4 *>(A + tc::mn_major_offset(c0 + 8 * h, reim * KP + kap, G::SBO_B5, 128)) =
                                pack8(v + 8 * h, wgt);
                }
            }
        }
        tc_publish();

        // ---- S5: c^T[v][u] = sum_kappa Dr[v][kappa] B5re[kappa][u] + Di[v][kappa] B5im[kappa][u], into
        // TMEM columns [C5, C5 + NO), which no other stage writes: the epilogue reads it during the next pair
        if (ctrl) {
            B200_TC_DESCS
            const uint32_t id = tc::instr_desc(128, NO, false, true, false, false);
#pragma unroll 2
            for (int s = 0; s < KP / 16; ++s) {
                tc::mma_f16(tmem + C5, dR0 + 16u * s, b0B5 + 16u * s, id, s > 0);
                tc::mma_f16(tmem + C5, dI0 + 16u * s, b0B5 + uint32_t(KP + 16 * s), id, 1);
            }
            tc::mma_commit(&mbar);
        }
        if (prev.live && ctrl) epi_finish();   // while the tensor cores run S5
        const PairSetup next = s_next;
        if (next.p < npairs && next.ok) gather(next);    // X is free: the pending epilogue is done
        if (!tc_wait_all(&mbar, phase)) {
            failed = true;
            break;
        }
        prev = {cur.q, cur.f, cur.sy, cur.sx, cur.gy, cur.gx, ldexpf(1.0f, eR + 17) / (float(N) * float(N) * norm), true};
        cur = next;
    }
    if (!failed && !epi_flush()) failed = true;
    if (failed && ctrl && status) atomicExch(status, 3);
    if (tma_pending) tc::mbar_wait(&tbar, tphase);   // no copy into this CTA's memory may outlive it
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, G::TMEM_COLS);
#undef B200_TC_DESCS
}

// the reference spectra in the order S3 of the tensor-core form reads them: for window k and the
// frequency pair (ky, ky + 1) = (2 p, 2 p + 1), the rows kappa < KP side by side, one float4
// (R[kappa][2 p], R[kappa][2 p + 1]) each, rows NH .. KP - 1 zero. spec holds nwin x NH x N.
__global__ void spec_tc_kernel(const float2 *__restrict__ spec, float4 *__restrict__ out, int N, int nwin)
{
    const int NH = N / 2 + 1, KP = tc_kp(N);
    const int64_t total = int64_t(nwin) * (N / 2) * KP;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const int kap = int(i % KP);
        const int64_t kp = i / KP;
        const int pr = int(kp % (N / 2));
        const int64_t k = kp / (N / 2);
        float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
        if (kap < NH) {
            const float2 *r = spec + (k * NH + kap) * N + 2 * pr;
            o = make_float4(r[0].x, r[0].y, r[1].x, r[1].y);
        }
        out[i] = o;
    }
}

#endif   // __CUDACC__

// the DFT matrices of the tensor-core form as the kernel keeps them in shared memory: Dr then Di,
// each K-major (rows r, columns c, both in [0, N)), FP16 bits; out holds 2 * N * N halves
void tc_dft_table(int N, uint16_t *out);

}   // namespace b200
